"""Generate the Rys quadrature tables (roots and weights for n = 1..9) as CUDA C.

The Rys quadrature of order n for parameter X has nodes x_i = t_i^2 in (0,1) and weights W_i
with sum_i W_i x_i^k = F_k(X) (the Boys function) for k = 0..2n-1.  The reference computes
them for n <= 5 from fitted polynomials (Root1..Root5, src/Rys.jl:176-1478); here they are
computed from the moments, for n <= 9, by published methods:

  * the modified Chebyshev algorithm (Gautschi) turns the moments F_k(X) into the
    three-term recurrence of the orthogonal polynomials (done at 60 significant digits in
    mpmath, so the ill-conditioning of the moment map is harmless);
  * Golub-Welsch: nodes are the eigenvalues of the Jacobi matrix, weights F_0(X) times the
    squared first components of its eigenvectors;
  * for 0 <= X < 100 each node and weight is fitted on unit intervals of X by a Chebyshev
    series of degree 15 (interpolation at Chebyshev points); for X >= 100 the measure's
    moments equal the half-range Gaussian's closely enough (checked: relative error of the
    rule below 1e-16 for n <= 9), so x_i = h_i^2 / X and
    W_i = g_i / sqrt(X) with h_i, g_i the positive nodes and weights of the 2n-point
    Gauss-Hermite rule.

Output: generated/rys_tables.cu (device arrays + an address lookup).  The fit is checked
against fresh high-precision solves at random X and the worst relative errors are printed.

    python gen_rys_tables.py [-j JOBS]
"""
from __future__ import annotations

import argparse
import math
import random
import sys
from multiprocessing import get_context
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "generated" / "rys_tables.cu"

NMAX = 9
XMAX = 100         # Chebyshev fits cover [0, XMAX); asymptotic Hermite form above
NCHEB = 16         # points / coefficients per interval (degree 15)
DPS = 60


def _mp():
    import mpmath
    mpmath.mp.dps = DPS
    return mpmath


def boys(mp, k, X):
    if X == 0:
        return mp.mpf(1) / (2 * k + 1)
    a = mp.mpf(k) + mp.mpf(1) / 2
    return mp.gammainc(a, 0, X) / (2 * X ** a)


def rys_nodes(n, X):
    """Nodes x_i (ascending) and weights W_i of the n-point Rys rule at X, as mpf lists."""
    mp = _mp()
    X = mp.mpf(X)
    mu = [boys(mp, k, X) for k in range(2 * n)]
    sig2 = [mp.mpf(0)] * (2 * n)
    sig1 = mu[:]
    alpha, beta = [mu[1] / mu[0]], [mu[0]]
    for k in range(1, n):
        sig = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            sig[l] = sig1[l + 1] - alpha[k - 1] * sig1[l] - beta[k - 1] * sig2[l]
        alpha.append(sig[k + 1] / sig[k] - sig1[k] / sig1[k - 1])
        beta.append(sig[k] / sig1[k - 1])
        sig2, sig1 = sig1, sig
    J = mp.zeros(n, n)
    for i in range(n):
        J[i, i] = alpha[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(beta[i + 1])
    E, Q = mp.eigsy(J)
    idx = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in idx], [beta[0] * Q[0, i] ** 2 for i in idx]


def cheb_points():
    return [math.cos(math.pi * (k + 0.5) / NCHEB) for k in range(NCHEB)]


def fit_interval(args):
    """Chebyshev coefficients of the 2n functions (nodes then weights) on [j, j+1)."""
    n, j = args
    mp = _mp()
    vals = []
    for s in cheb_points():
        X = mp.mpf(j) + (mp.mpf(s) + 1) / 2
        x, w = rys_nodes(n, X)
        vals.append(x + w)
    coefs = []
    for f in range(2 * n):
        cf = []
        for m in range(NCHEB):
            acc = mp.mpf(0)
            for k in range(NCHEB):
                acc += vals[k][f] * mp.cos(mp.pi * m * (k + mp.mpf(1) / 2) / NCHEB)
            c = 2 * acc / NCHEB
            if m == 0:
                c /= 2
            cf.append(float(c))
        coefs.append(cf)
    return n, j, coefs


def clenshaw(cf, s):
    b1 = b2 = 0.0
    for c in reversed(cf[1:]):
        b1, b2 = 2 * s * b1 - b2 + c, b1
    return s * b1 - b2 + cf[0]


def hermite_half(n):
    """Positive nodes h_i and weights g_i of the 2n-point Gauss-Hermite rule (ascending)."""
    mp = _mp()
    # Golub-Welsch for Hermite: alpha_k = 0, beta_k = k/2, mu_0 = sqrt(pi)
    m = 2 * n
    J = mp.zeros(m, m)
    for i in range(m - 1):
        J[i, i + 1] = J[i + 1, i] = mp.sqrt(mp.mpf(i + 1) / 2)
    E, Q = mp.eigsy(J)
    pts = [(E[i], mp.sqrt(mp.pi) * Q[0, i] ** 2) for i in range(m)]
    pos = sorted([(h, g) for h, g in pts if h > 0], key=lambda t: t[0])
    return [h for h, _ in pos], [g for _, g in pos]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    jobs = [(n, j) for n in range(1, NMAX + 1) for j in range(XMAX)]
    with get_context("spawn").Pool(a.j) as pool:
        res = pool.map(fit_interval, jobs, chunksize=4)
    table = {(n, j): c for n, j, c in res}
    # accuracy check at random X against fresh solves
    rng = random.Random(7)
    worst = {}
    for n in range(1, NMAX + 1):
        w = 0.0
        for _ in range(40):
            X = rng.uniform(0, XMAX)
            j = int(X)
            s = 2 * (X - j) - 1
            x, wt = rys_nodes(n, X)
            for f, exact in enumerate(x + wt):
                approx = clenshaw(table[(n, j)][f], s)
                w = max(w, abs(approx - float(exact)) / abs(float(exact)))
        worst[n] = w
        print(f"n={n}: worst relative error of the fit {w:.2e}", file=sys.stderr)
    herm = {n: hermite_half(n) for n in range(1, NMAX + 1)}
    # check the asymptotic form at X = XMAX
    for n in range(1, NMAX + 1):
        x, wt = rys_nodes(n, XMAX)
        h, g = herm[n]
        mp = _mp()
        e = max(max(abs(h[i] ** 2 / XMAX - x[i]) / x[i] for i in range(n)),
                max(abs(g[i] / mp.sqrt(XMAX) - wt[i]) / wt[i] for i in range(n)))
        print(f"n={n}: asymptotic form at X={XMAX}: relative error {float(e):.2e}", file=sys.stderr)
    # emit
    offs, flat = [], []
    for n in range(1, NMAX + 1):
        offs.append(len(flat))
        for j in range(XMAX):
            for f in range(2 * n):
                flat.extend(table[(n, j)][f])
    hx, hw = [], []
    for n in range(1, NMAX + 1):
        hx.extend(float(v) ** 2 for v in herm[n][0])
        hw.extend(float(v) for v in herm[n][1])

    def arr(vals, per=4):
        lines = []
        for i in range(0, len(vals), per):
            lines.append("    " + ", ".join(float(v).hex() for v in vals[i:i + per]) + ",")
        return "\n".join(lines)

    src = f"""// Generated by gen_rys_tables.py -- Rys quadrature tables.  Do not edit.
// kRysCheb: for n = 1..{NMAX}, X intervals [j, j+1) j < {XMAX}, functions (nodes x_1..x_n, then
// weights W_1..W_n), {NCHEB} Chebyshev coefficients each (argument s = 2(X - j) - 1).
// kRysHerm: for X >= {XMAX}, x_i = kRysHermX2[i] / X and W_i = kRysHermW[i] / sqrt(X) (the
// 2n-point Gauss-Hermite rule's positive nodes squared and their weights), n at kRysHermOff.
// Worst relative fit error at 40 random X per n: {", ".join(f"n{n} {worst[n]:.1e}" for n in worst)}.
#include <cuda_runtime.h>
#include "../eri_common.cuh"

namespace molints {{

__device__ __align__(16) const double kRysCheb[{len(flat)}] = {{
{arr(flat)}
}};
__device__ const double kRysHermX2[{len(hx)}] = {{
{arr(hx)}
}};
__device__ const double kRysHermW[{len(hw)}] = {{
{arr(hw)}
}};

// Device addresses of the tables on the current device (cudaGetSymbolAddress).
int rys_tables(RysTab *t) {{
    void *a = nullptr, *b = nullptr, *c = nullptr;
    if (cudaGetSymbolAddress(&a, kRysCheb) != cudaSuccess) return -1;
    if (cudaGetSymbolAddress(&b, kRysHermX2) != cudaSuccess) return -1;
    if (cudaGetSymbolAddress(&c, kRysHermW) != cudaSuccess) return -1;
    t->cheb = static_cast<const double *>(a);
    t->herm_x2 = static_cast<const double *>(b);
    t->herm_w = static_cast<const double *>(c);
    return 0;
}}

}}  // namespace molints
"""
    OUT.parent.mkdir(exist_ok=True)
    OUT.write_text(src)
    print(f"wrote {OUT} ({len(flat)} coefficients)", file=sys.stderr)


if __name__ == "__main__":
    main()

"""CPU oracle for the ERI path -- TEST INFRASTRUCTURE ONLY.

Only tests, ``__graft_entry__.smoke()`` (as the checker) and ``bench.py``'s CPU-baseline and
reference arms may import this module.  The product (``molecularintegrals.jl_b200``) never
does.  It wraps ``molints_oracle.c``, a plain-C FP64 restatement of the reference Julia
HGP / Boys / Huzinaga code of MolecularIntegrals.jl (file:line citations are in that file),
and adds an mpmath Boys function used to pin the C series.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD_DIR = HERE / "_build"
LIB_PATH = BUILD_DIR / "libmolints_oracle.so"
SRC = HERE / "molints_oracle.c"

_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p


def build(force: bool = False) -> Path:
    """Compile the oracle with gcc (-O3, OpenMP) into oracle/_build/."""
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB_PATH
    BUILD_DIR.mkdir(exist_ok=True)
    tmp = LIB_PATH.with_suffix(f".{os.getpid()}.tmp.so")
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-Wall",
           "-o", str(tmp), str(SRC), "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.oracle_boys.restype = _D
        L.oracle_boys.argtypes = [_I, _D]
        L.oracle_boys_asymp.restype = _D
        L.oracle_boys_asymp.argtypes = [_I, _D]
        L.oracle_farray.argtypes = [_I, _D, _P]
        L.oracle_vrr.argtypes = [_I, _I, _D, _D, _D, _D, _P, _P, _P, _P, _I, _P]
        L.oracle_hrr.argtypes = [_I, _I, _I, _I, _D, _D, _D, _D, _P, _P, _P, _P, _I, _P]
        L.oracle_hrr_size.restype = ctypes.c_size_t
        L.oracle_hrr_size.argtypes = [_I, _I, _I, _I]
        L.oracle_nao.restype = _I
        L.oracle_nao.argtypes = [_I]
        L.oracle_ao_index.restype = _I
        L.oracle_ao_index.argtypes = [_I, _I, _I]
        L.oracle_ao2m.argtypes = [_I, _P]
        L.oracle_pgbf_norm.restype = _D
        L.oracle_pgbf_norm.argtypes = [_D, _I, _I, _I]
        L.oracle_cgbf_norm.restype = _D
        L.oracle_cgbf_norm.argtypes = [_I, _I, _P, _P]
        L.oracle_iindex.restype = ctypes.c_int64
        L.oracle_iindex.argtypes = [ctypes.c_int64] * 4
        L.oracle_npacked.restype = ctypes.c_int64
        L.oracle_npacked.argtypes = [ctypes.c_int64]
        drv = [_I, _P, _P, _P, _P, _P, _P, _P, _I]
        L.oracle_eri_packed_hgp.restype = _I
        L.oracle_eri_packed_hgp.argtypes = drv
        L.oracle_eri_packed_huzinaga.restype = _I
        L.oracle_eri_packed_huzinaga.argtypes = drv
        L.oracle_shell_quartet.restype = _I
        L.oracle_shell_quartet.argtypes = [_I, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P]
        L.oracle_coulomb_prim.restype = _D
        L.oracle_coulomb_prim.argtypes = ([_D, _D, _D, _D, _I, _I, _I] * 4)
        L.oracle_eri_packed_hgp_ld.restype = _I
        L.oracle_eri_packed_hgp_ld.argtypes = drv
        L.oracle_eri_packed_hgp_sample.restype = ctypes.c_int64
        L.oracle_eri_packed_hgp_sample.argtypes = drv + [ctypes.c_int64]
        L.oracle_rys_roots.restype = _I
        L.oracle_rys_roots.argtypes = [_I, _D, _P, _P]
        L.oracle_eri_packed_rys.restype = _I
        L.oracle_eri_packed_rys.argtypes = drv
        L.oracle_coulomb_rys_prim.restype = _D
        L.oracle_coulomb_rys_prim.argtypes = [_D, _P, _P, _D, _P, _P, _D, _P, _P, _D, _P, _P]
        L.oracle_set_orientation.argtypes = [_I]
        L.oracle_get_orientation.restype = _I
        L.oracle_set_boys_tmax.argtypes = [_D]
        L.oracle_get_boys_tmax.restype = _D
        L.oracle_init()
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ------------------------------------------------------------------ Boys
def boys(m: int, T: float) -> float:
    """Fm(m,T) (src/Boys.jl:29-34)."""
    return lib().oracle_boys(m, T)


def farray(mmax: int, T: float) -> np.ndarray:
    """farray(mmax,T) (src/Boys.jl:19-27): F_0..F_{mmax-1}."""
    out = np.zeros(mmax)
    lib().oracle_farray(mmax, T, _ptr(out))
    return out


def set_boys_tmax(tmax: float = 30.0) -> None:
    """Move farray's switch to the asymptotic form (30 in src/Boys.jl:19)."""
    lib().oracle_set_boys_tmax(tmax)


class exact_boys:
    """Context manager: the oracle uses the exact F_m(T) at every T (no asymptotic branch)."""

    def __enter__(self):
        self._old = lib().oracle_get_boys_tmax()
        set_boys_tmax(1e300)

    def __exit__(self, *exc):
        set_boys_tmax(self._old)


class engine_orientation:
    """Context manager: the HGP driver orients each quartet as the engine does (larger L
    first in each pair, higher class as bra) instead of by shell index as the reference."""

    def __enter__(self):
        self._old = lib().oracle_get_orientation()
        lib().oracle_set_orientation(1)

    def __exit__(self, *exc):
        lib().oracle_set_orientation(self._old)


class stable_orientation:
    """Context manager: the HGP driver orients each pair as the engine does now (larger L
    first; for equal L and for an f-d pair the tighter shell first), the orientation in
    which the HRR does not cancel.  The long-double oracle in this mode is the near-exact
    reference for bases with tight and diffuse shells of the same L."""

    def __enter__(self):
        self._old = lib().oracle_get_orientation()
        lib().oracle_set_orientation(2)

    def __exit__(self, *exc):
        lib().oracle_set_orientation(self._old)


def boys_mpmath(m: int, T: float, dps: int = 40) -> float:
    """Exact F_m(T) = 1/2 T^-(m+1/2) gamma_lower(m+1/2, T), in mpmath."""
    import mpmath
    with mpmath.workdps(dps):
        if T == 0:
            return float(mpmath.mpf(1) / (2 * m + 1))
        a = mpmath.mpf(m) + mpmath.mpf(1) / 2
        t = mpmath.mpf(T)
        return float(mpmath.gammainc(a, 0, t) / (2 * t ** a))


# ------------------------------------------------------------------ tables
def nao(l: int) -> int:
    return lib().oracle_nao(l)


def ao_index(i: int, j: int, k: int) -> int:
    """0-based m2ao (src/Basis.jl:295-316)."""
    return lib().oracle_ao_index(i, j, k)


# ------------------------------------------------------------------ primitive VRR/HRR
def vrr(amax, cmax, aexp, bexp, cexp, dexp, A, B, C, D, prefactor_mode=0) -> np.ndarray:
    """vrr(amax,cmax,...) (src/HGP.jl:371-376): array [mmax, nao(amax), nao(cmax)]."""
    mmax = amax + cmax + 1
    out = np.zeros((mmax, nao(amax), nao(cmax)))
    cs = [np.ascontiguousarray(x, dtype=np.float64) for x in (A, B, C, D)]
    lib().oracle_vrr(amax, cmax, aexp, bexp, cexp, dexp, *[_ptr(c) for c in cs],
                     prefactor_mode, _ptr(out))
    return out


def hrr(la, lb, lc, ld, aexp, bexp, cexp, dexp, A, B, C, D, prefactor_mode=0) -> np.ndarray:
    """hrr(...) (src/HGP.jl:392-424): [nao(la+lb), nao(lb), nao(lc+ld), nao(ld)]."""
    out = np.zeros((nao(la + lb), nao(lb), nao(lc + ld), nao(ld)))
    cs = [np.ascontiguousarray(x, dtype=np.float64) for x in (A, B, C, D)]
    lib().oracle_hrr(la, lb, lc, ld, aexp, bexp, cexp, dexp, *[_ptr(c) for c in cs],
                     prefactor_mode, _ptr(out))
    return out


def coulomb_prim(a, b, c, d) -> float:
    """Raw primitive Huzinaga coulomb (src/ERI.jl:15-46); each arg (expn, (x,y,z), (I,J,K))."""
    args = []
    for expn, xyz, ijk in (a, b, c, d):
        args += [float(expn), *map(float, xyz), *map(int, ijk)]
    return lib().oracle_coulomb_prim(*args)


def pgbf_norm(expn, I, J, K) -> float:
    return lib().oracle_pgbf_norm(expn, I, J, K)


# ------------------------------------------------------------------ whole basis
def _shell_arrays(shells):
    xyz = np.ascontiguousarray(shells.xyz, dtype=np.float64)
    L = np.ascontiguousarray(shells.L, dtype=np.int32)
    nprim = np.ascontiguousarray(shells.nprim, dtype=np.int32)
    poff = np.ascontiguousarray(shells.prim_off, dtype=np.int32)
    expn = np.ascontiguousarray(shells.expn, dtype=np.float64)
    coef = np.ascontiguousarray(shells.coef, dtype=np.float64)
    return xyz, L, nprim, poff, expn, coef


def eri_packed_hgp(shells, nthreads: int = 1) -> np.ndarray:
    """all_twoe_ints_chrr with D1-D3, D5 fixed: the normalised packed iindex vector."""
    arrs = _shell_arrays(shells)
    n = shells.nbf
    out = np.zeros(n * (n + 1) * (n * n + n + 2) // 8)
    rc = lib().oracle_eri_packed_hgp(len(arrs[1]), *[_ptr(a) for a in arrs], _ptr(out), nthreads)
    if rc != 0:
        raise ValueError("oracle_eri_packed_hgp: unsupported shell")
    return out


def eri_packed_hgp_ld(shells, nthreads: int = 1) -> np.ndarray:
    """The same restated HGP driver evaluated in long double (64-bit mantissa): a near-exact
    reference for FP64 parity, rounded to double at the end.  nthreads 0 uses every core."""
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    arrs = _shell_arrays(shells)
    n = shells.nbf
    out = np.zeros(n * (n + 1) * (n * n + n + 2) // 8)
    rc = lib().oracle_eri_packed_hgp_ld(len(arrs[1]), *[_ptr(a) for a in arrs], _ptr(out), nthreads)
    if rc != 0:
        raise ValueError("oracle_eri_packed_hgp_ld: unsupported shell")
    return out


def eri_packed_hgp_sample(shells, nthreads: int, stride: int, out: np.ndarray | None = None) -> int:
    """The HGP driver over every stride-th shell quartet; returns the integrals written."""
    arrs = _shell_arrays(shells)
    if out is None:
        out = np.zeros(shells.npacked)
    n = lib().oracle_eri_packed_hgp_sample(len(arrs[1]), *[_ptr(a) for a in arrs], _ptr(out),
                                           nthreads, stride)
    if n < 0:
        raise ValueError("oracle_eri_packed_hgp_sample: unsupported shell")
    return int(n)


def eri_packed_huzinaga(shells, nthreads: int = 1) -> np.ndarray:
    """all_twoe_ints(bfs, coulomb) (src/ERI.jl:104-112): normalised packed iindex vector."""
    arrs = _shell_arrays(shells)
    n = shells.nbf
    out = np.zeros(n * (n + 1) * (n * n + n + 2) // 8)
    rc = lib().oracle_eri_packed_huzinaga(len(arrs[1]), *[_ptr(a) for a in arrs], _ptr(out),
                                          nthreads)
    if rc != 0:
        raise ValueError("oracle_eri_packed_huzinaga: unsupported shell")
    return out


def shell_quartet(shells, sa, sb, sc, sd) -> np.ndarray:
    """Normalised contracted (ab|cd) block [na, nb, nc, nd] for four shells."""
    arrs = _shell_arrays(shells)
    nc = [(int(shells.L[s]) + 1) * (int(shells.L[s]) + 2) // 2 for s in (sa, sb, sc, sd)]
    out = np.zeros(nc)
    lib().oracle_shell_quartet(len(arrs[1]), *[_ptr(a) for a in arrs], sa, sb, sc, sd, _ptr(out))
    return out


def iindex(i, j, k, l) -> int:
    """0-based iindex (src/Utils.jl:19 minus one)."""
    return lib().oracle_iindex(i, j, k, l)


# ------------------------------------------------------------------ mpmath Huzinaga
def coulomb_mpmath(a, b, c, d, dps: int = 40):
    """Primitive Huzinaga coulomb (src/ERI.jl:15-94) in mpmath at `dps` digits; each argument
    is (expn, (x,y,z), (I,J,K)).  Returns an mpf."""
    import mpmath
    with mpmath.workdps(dps):
        mpf = mpmath.mpf
        F = mpmath.factorial

        def boys(m, T):
            if T == 0:
                return mpf(1) / (2 * m + 1)
            am = mpf(m) + mpf(1) / 2
            return mpmath.gammainc(am, 0, T) / (2 * T ** am)

        def binom(n, k):
            return mpmath.binomial(n, k) if 0 <= k <= n else mpf(0)

        def bp(s_, ia, ib, xpa, xpb):
            return sum((binom(ia, s_ - t) * xpa ** (ia - s_ + t) * binom(ib, t) * xpb ** (ib - t)
                        for t in range(s_ + 1) if s_ - ia <= t <= ib), mpf(0))

        def fr2(x, y):
            return F(x) / F(y) / F(x - 2 * y)

        def fB(i, l1, l2, pp, aa, bb, r, g):
            return bp(i, l1, l2, pp - aa, pp - bb) * fr2(i, r) * (4 * g) ** (r - i)

        def barray(l1, l2, l3, l4, pp, aa, bb, qq, cc, dd, g1, g2, delta):
            B = [mpf(0)] * (l1 + l2 + l3 + l4 + 1)
            for i1 in range(l1 + l2 + 1):
                for i2 in range(l3 + l4 + 1):
                    for r1 in range(i1 // 2 + 1):
                        for r2 in range(i2 // 2 + 1):
                            for u in range((i1 + i2) // 2 - r1 - r2 + 1):
                                e = i1 + i2 - 2 * (r1 + r2)
                                B[e - u] += (fB(i1, l1, l2, pp, aa, bb, r1, g1) * (-1) ** i2 *
                                             fB(i2, l3, l4, qq, cc, dd, r2, g2) * (-1) ** u *
                                             fr2(e, u) * (qq - pp) ** (e - 2 * u) / delta ** (e - u))
            return B

        (ea, A, ia), (eb, Bc, ib), (ec, C, ic), (ed, D, id_) = a, b, c, d
        ea, eb, ec, ed = (mpf(float(x)) for x in (ea, eb, ec, ed))
        A, Bc, C, D = ([mpf(float(t)) for t in v] for v in (A, Bc, C, D))
        g1, g2 = ea + eb, ec + ed
        P = [(ea * A[t] + eb * Bc[t]) / g1 for t in range(3)]
        Q = [(ec * C[t] + ed * D[t]) / g2 for t in range(3)]
        rab2 = sum((A[t] - Bc[t]) ** 2 for t in range(3))
        rcd2 = sum((C[t] - D[t]) ** 2 for t in range(3))
        rpq2 = sum((P[t] - Q[t]) ** 2 for t in range(3))
        delta = (1 / g1 + 1 / g2) / 4
        Bs = [barray(ia[t], ib[t], ic[t], id_[t], P[t], A[t], Bc[t], Q[t], C[t], D[t], g1, g2, delta)
              for t in range(3)]
        x = rpq2 / (4 * delta)
        tot = mpf(0)
        for I in range(len(Bs[0])):
            for J in range(len(Bs[1])):
                for K in range(len(Bs[2])):
                    tot += Bs[0][I] * Bs[1][J] * Bs[2][K] * boys(I + J + K, x)
        return (2 * mpmath.pi ** mpf(2.5) / (g1 * g2 * mpmath.sqrt(g1 + g2)) *
                mpmath.exp(-ea * eb * rab2 / g1) * mpmath.exp(-ec * ed * rcd2 / g2) * tot)


def contracted_mpmath(shells, funcs, dps: int = 40) -> float:
    """Normalised contracted integral of four functions given as (shell index, (I,J,K)),
    in mpmath (contract and normalize!, src/Basis.jl:42-98)."""
    import mpmath
    with mpmath.workdps(dps):
        mpf = mpmath.mpf
        terms, gfac = [], mpf(1)
        for s, ijk in funcs:
            L = int(shells.L[s])
            p0, K = int(shells.prim_off[s]), int(shells.nprim[s])
            ex = [mpf(float(x)) for x in shells.expn[p0:p0 + K]]
            co = [mpf(float(x)) for x in shells.coef[p0:p0 + K]]
            S = sum(co[i] * co[j] * (2 * mpmath.sqrt(ex[i] * ex[j]) / (ex[i] + ex[j])) ** (L + mpf(3) / 2)
                    for i in range(K) for j in range(K))
            cn = 1 / mpmath.sqrt(S)
            nc = [co[i] * cn * (2 * ex[i] / mpmath.pi) ** (mpf(3) / 4) * (4 * ex[i]) ** (mpf(L) / 2)
                  for i in range(K)]
            terms.append((s, ijk, ex, nc))
            d2 = 1
            for p in ijk:
                n = 2 * p - 1
                while n > 1:
                    d2 *= n
                    n -= 2
            gfac /= mpmath.sqrt(d2)
        tot = mpf(0)
        import itertools
        for idx in itertools.product(*[range(len(t[2])) for t in terms]):
            args, cf = [], mpf(1)
            for (s, ijk, ex, nc), k in zip(terms, idx):
                args.append((ex[k], shells.xyz[s], ijk))
                cf *= nc[k]
            tot += cf * coulomb_mpmath(*args, dps=dps)
        return float(tot * gfac)


# ------------------------------------------------------------------ Rys
def rys_roots(n: int, X: float):
    """Nodes x_i = t_i^2 and weights of the n-point Rys rule (long-double discretised
    Stieltjes; the reference's Roots for n <= 5, src/Rys.jl:161-174)."""
    r = np.zeros(n)
    w = np.zeros(n)
    if lib().oracle_rys_roots(n, X, _ptr(r), _ptr(w)) != 0:
        raise ValueError("oracle_rys_roots: bad n or X")
    return r, w


def rys_roots_mpmath(n: int, X: float, dps: int = 50):
    """The same rule from the moments F_k(X) at `dps` digits (modified Chebyshev algorithm +
    Golub-Welsch), for pinning."""
    import mpmath
    with mpmath.workdps(dps):
        Xm = mpmath.mpf(X)

        def boys(k):
            if Xm == 0:
                return mpmath.mpf(1) / (2 * k + 1)
            a = mpmath.mpf(k) + mpmath.mpf(1) / 2
            return mpmath.gammainc(a, 0, Xm) / (2 * Xm ** a)
        mu = [boys(k) for k in range(2 * n)]
        s2, s1 = [mpmath.mpf(0)] * (2 * n), mu[:]
        al, be = [mu[1] / mu[0]], [mu[0]]
        for k in range(1, n):
            sg = [mpmath.mpf(0)] * (2 * n)
            for l in range(k, 2 * n - k):
                sg[l] = s1[l + 1] - al[k - 1] * s1[l] - be[k - 1] * s2[l]
            al.append(sg[k + 1] / sg[k] - s1[k] / s1[k - 1])
            be.append(sg[k] / s1[k - 1])
            s2, s1 = s1, sg
        J = mpmath.zeros(n, n)
        for i in range(n):
            J[i, i] = al[i]
            if i + 1 < n:
                J[i, i + 1] = J[i + 1, i] = mpmath.sqrt(be[i + 1])
        E, Q = mpmath.eigsy(J)
        idx = sorted(range(n), key=lambda i: E[i])
        return (np.array([float(E[i]) for i in idx]),
                np.array([float(be[0] * Q[0, i] ** 2) for i in idx]))


def coulomb_rys_prim(a, b, c, d) -> float:
    """coulomb_rys on raw primitives (src/Rys.jl:59-83); args (expn, xyz, ijk)."""
    args = []
    keep = []
    for expn, xyz, ijk in (a, b, c, d):
        X = np.ascontiguousarray(xyz, dtype=np.float64)
        I = np.ascontiguousarray(ijk, dtype=np.int32)
        keep += [X, I]
        args += [float(expn), _ptr(X), _ptr(I)]
    return lib().oracle_coulomb_rys_prim(*args)


def eri_packed_rys(shells, nthreads: int = 1) -> np.ndarray:
    """all_twoe_ints_rys (src/Rys.jl:16-43) with the CGBF norms applied (D4)."""
    arrs = _shell_arrays(shells)
    n = shells.nbf
    out = np.zeros(n * (n + 1) * (n * n + n + 2) // 8)
    rc = lib().oracle_eri_packed_rys(len(arrs[1]), *[_ptr(a) for a in arrs], _ptr(out), nthreads)
    if rc != 0:
        raise ValueError("oracle_eri_packed_rys: unsupported shell")
    return out


# ------------------------------------------------------------------ J/K
def make2JmK(D: np.ndarray, ints: np.ndarray) -> np.ndarray:
    """make2JmK(D, Ints) of src/ERI.jl:114-128 on a packed vector (0-based iindex):
    G_ij = sum_kl D_kl (2 (ij|kl) - (ik|jl)).  Returns (G, J, K)."""
    n = D.shape[0]
    i, j, k, l = np.meshgrid(*[np.arange(n)] * 4, indexing="ij")
    def tri(x):
        return x * (x + 1) // 2
    ij = np.where(i >= j, tri(i) + j, tri(j) + i)
    kl = np.where(k >= l, tri(k) + l, tri(l) + k)
    full = ints[np.where(ij >= kl, tri(ij) + kl, tri(kl) + ij)]
    J = np.einsum("ijkl,kl->ij", full, D)
    K = np.einsum("ikjl,kl->ij", full, D)
    return 2 * J - K, J, K


# ------------------------------------------------------------------ one-electron integrals
def _fact2(n: int) -> float:
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return float(r)


def _binomial_prefactor(s, ia, ib, xpa, xpb):
    """binomial_prefactor of src/OneInts.jl:94-95."""
    from math import comb
    tot = 0.0
    for t in range(s + 1):
        if s - ia <= t <= ib:
            tot += comb(ia, s - t) * xpa ** (ia - s + t) * comb(ib, t) * xpb ** (ib - t)
    return tot


def _overlap1d(la, lb, ax, bx, g):
    """overlap1d, src/OneInts.jl:86-92."""
    return sum(_binomial_prefactor(2 * i, la, lb, ax, bx) * _fact2(2 * i - 1) / (2 * g) ** i
               for i in range((la + lb) // 2 + 1)) if la >= 0 and lb >= 0 else 0.0


def overlap_prim(a, A, ia, b, B, ib) -> float:
    """overlap(aexpn,axyz,aI,aJ,aK,bexpn,bxyz,bI,bJ,bK), src/OneInts.jl:41-52 (no norms)."""
    A, B = np.asarray(A, float), np.asarray(B, float)
    g = a + b
    P = (a * A + b * B) / g
    pre = (np.pi / g) ** 1.5 * np.exp(-a * b * np.sum((A - B) ** 2) / g)
    return pre * np.prod([_overlap1d(ia[t], ib[t], P[t] - A[t], P[t] - B[t], g) for t in range(3)])


def kinetic_prim(a, A, ia, b, B, ib) -> float:
    """kinetic(...) of src/OneInts.jl:124-135 (no norms)."""
    def ov(db):
        return overlap_prim(a, A, ia, b, B, [ib[t] + db[t] for t in range(3)])
    t0 = b * (2 * sum(ib) + 3) * ov((0, 0, 0))
    t1 = -2 * b * b * (ov((2, 0, 0)) + ov((0, 2, 0)) + ov((0, 0, 2)))
    t2 = -0.5 * sum(ib[t] * (ib[t] - 1) * ov(tuple(-2 if u == t else 0 for u in range(3))) for t in range(3))
    return t0 + t1 + t2


def nuclear_prim(a, A, ia, b, B, ib, C) -> float:
    """nuclear_attraction(...) of src/OneInts.jl:208-227 via Aarray (:143-165), exact Boys
    function for Fgamma (no norms, unit charge)."""
    from math import factorial
    A, B, C = (np.asarray(v, float) for v in (A, B, C))
    g = a + b
    P = (a * A + b * B) / g
    PA, PB, PC = P - A, P - B, P - C

    def aarray(l1, l2, pa, pb, pc):
        out = np.zeros(l1 + l2 + 1)
        for i in range(l1 + l2 + 1):
            for r in range(i // 2 + 1):
                for u in range((i - 2 * r) // 2 + 1):
                    I = i - 2 * r - u
                    out[I] += ((-1) ** i * _binomial_prefactor(i, l1, l2, pa, pb) * (-1) ** u * factorial(i)
                               * pc ** (i - 2 * r - 2 * u) * (0.25 / g) ** (r + u)
                               / (factorial(r) * factorial(u) * factorial(i - 2 * r - 2 * u)))
        return out
    Ax, Ay, Az = (aarray(ia[t], ib[t], PA[t], PB[t], PC[t]) for t in range(3))
    T = g * float(PC @ PC)
    tot = 0.0
    for I in range(len(Ax)):
        for J in range(len(Ay)):
            for K in range(len(Az)):
                tot += Ax[I] * Ay[J] * Az[K] * boys(I + J + K, T)
    return -2 * np.pi * np.exp(-a * b * np.sum((A - B) ** 2) / g) * tot / g


def all_1e_ints(shells, atom_xyz, atom_charge):
    """all_1e_ints(bfs, mol), src/OneInts.jl:267-290, for normalised contracted functions:
    (S, T, V), V summed over point charges."""
    from molints_b200 import basis as B_
    n = shells.nbf
    funcs = []  # (centre, ijk, [(expn, normalised coefficient)])
    for s in range(shells.nshell):
        l = int(shells.L[s])
        p0, k = int(shells.prim_off[s]), int(shells.nprim[s])
        ex, co = shells.expn[p0:p0 + k], shells.coef[p0:p0 + k]
        S0 = sum(co[i] * co[j] * (2 * np.sqrt(ex[i] * ex[j]) / (ex[i] + ex[j])) ** (l + 1.5)
                 for i in range(k) for j in range(k))
        for c in B_.shell_components(l):
            g = 1 / np.sqrt(_fact2(2 * c[0] - 1) * _fact2(2 * c[1] - 1) * _fact2(2 * c[2] - 1))
            prims = [(e, cf / np.sqrt(S0) * (2 * e / np.pi) ** 0.75 * (4 * e) ** (l / 2) * g)
                     for e, cf in zip(ex, co)]
            funcs.append((shells.xyz[s], c, prims))
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    atoms = list(zip(np.asarray(atom_xyz, float).reshape(-1, 3), np.asarray(atom_charge, float)))
    for i in range(n):
        for j in range(i + 1):
            A, ia, pa = funcs[i]
            Bc, ib, pb = funcs[j]
            s = t = v = 0.0
            for a, ca in pa:
                for b, cb in pb:
                    s += ca * cb * overlap_prim(a, A, ia, b, Bc, ib)
                    t += ca * cb * kinetic_prim(a, A, ia, b, Bc, ib)
                    v += ca * cb * sum(z * nuclear_prim(a, A, ia, b, Bc, ib, C) for C, z in atoms)
            S[i, j] = S[j, i] = s
            T[i, j] = T[j, i] = t
            V[i, j] = V[j, i] = v
    return S, T, V

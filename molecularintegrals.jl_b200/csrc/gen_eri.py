"""Generate the per-class ERI kernels (CUDA C for sm_100a).

This is the engine's counterpart of the reference's ``vrr_autogen`` (src/HGP.jl:432-534),
which emits unrolled, branch-free Julia VRR code per (amax, cmax).  Here one kernel is
emitted per class pair (la lb | lc ld) with la >= lb, lc >= ld and the bra class at or
above the ket class.  Each kernel evaluates one contracted shell quartet per thread:

  * the HGP vertical recurrence of src/HGP.jl:135-242 -- the a-build (eq. 6a with c = 0,
    :180-197) and the c-build (eq. 6d, :204-240) -- unrolled and pruned to the
    [a0|c0]^(m) entries the class needs, in registers (FP64, or FP32 for MIXED quartets);
  * contraction over the primitive quartets in FP64 after the VRR (cvrr, :50-68);
  * the horizontal recurrences of chrr (:87-114) on the contracted block, bra then ket;
  * the component norms 1/sqrt((2I-1)!!(2J-1)!!(2K-1)!!) and the packed iindex store of
    the quartet's unique integrals.

Run ``python gen_eri.py`` to (re)write ``generated/``; the build does it automatically.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "generated"


def _load_gen_rys():
    import importlib.util
    if "gen_rys" in sys.modules:
        return sys.modules["gen_rys"]
    spec = importlib.util.spec_from_file_location("gen_rys", HERE / "gen_rys.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gen_rys"] = mod
    spec.loader.exec_module(mod)
    return mod


gen_rys = _load_gen_rys()
LMAX = 3            # shell angular momentum of the classes considered
LMAX_ALL_HGP = 2    # every class pair of shells up to d has an HGP kernel
LTAB = 2 * LMAX     # AO tables must reach la + lb
# Class pairs with an f shell get an HGP kernel when their VRR has at most this many entries
# (the low-L partners of f, e.g. (fs|ss), (fp|ps)); the rest run only the Rys kernels.
HGP_MAX_VRR = 500
# Classes whose VRR has fewer entries than this get no FP32 variant: their primitive
# quartet is dominated by the FP64 prefactors and Boys function, so an FP32 VRR would only
# add registers and divergence.  MIXED plans run them in FP64.
MIXED_MIN_VRR = 40
# Two-phase stores: classes with at most this many outputs per quartet have their HRR write the
# chunk's blocks into dynamic shared memory (4 warps x 32 blocks x 8 B each: up to 162 KB) and
# the warp copies them to the scratch as one contiguous run
STAGE_MAX_OUT = 162


# ------------------------------------------------------------------ AO tables
def shell_components(l):
    """src/Basis.jl:269-279 order (x-power descending, then y), l=3 with xzz before xyz."""
    comps = [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]
    if l == 3:
        comps[4], comps[5] = comps[5], comps[4]
    return comps


AO = []           # cumulative AO list (ao2m, src/Basis.jl:306-314), 0-based
NAO = []          # cumulative counts (nao, src/Basis.jl:320-321)
for _l in range(LTAB + 1):
    AO.extend(shell_components(_l))
    NAO.append(len(AO))
AO_INDEX = {c: i for i, c in enumerate(AO)}


def lof(a):
    return sum(AO[a])


def shell_range(l):
    return range(NAO[l - 1] if l > 0 else 0, NAO[l])


def shift_dir(a):
    """First argmax of the powers (shift_direction, src/Basis.jl:346-354)."""
    m = AO[a]
    return max(range(3), key=lambda i: (m[i], -i))


def shift_minus(a, i):
    m = list(AO[a])
    if m[i] == 0:
        return -1
    m[i] -= 1
    return AO_INDEX[tuple(m)]


def shift_plus(a, i):
    m = list(AO[a])
    m[i] += 1
    return AO_INDEX[tuple(m)]


def dfact2(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def comp_norm(a):
    I, J, K = AO[a]
    return 1.0 / math.sqrt(dfact2(2 * I - 1) * dfact2(2 * J - 1) * dfact2(2 * K - 1))


XYZ = "xyz"


# ------------------------------------------------------------------ classes
def pair_classes(lmax=LMAX):
    """Shell-pair classes (la, lb), la >= lb, ordered by la+lb then la."""
    cls = [(la, lb) for la in range(lmax + 1) for lb in range(la + 1)]
    return sorted(cls, key=lambda c: (c[0] + c[1], c[0]))


def class_pairs(lmax=LMAX):
    """Class pairs (X|Y), X at or above Y, that get an HGP kernel."""
    cls = pair_classes(lmax)
    out = []
    for i, X in enumerate(cls):
        for j in range(i + 1):
            Y = cls[j]
            if max(X + Y) > LMAX_ALL_HGP and \
                    len(vrr_entries(X[0], X[0] + X[1], Y[0], Y[0] + Y[1])) > HGP_MAX_VRR:
                continue
            out.append((X, Y))
    return out


def tag_of(X, Y):
    L = "spdfg"
    return f"{L[X[0]]}{L[X[1]]}{L[Y[0]]}{L[Y[1]]}"


# ------------------------------------------------------------------ VRR plan
def vrr_entries(e_lo, e_hi, f_lo, f_hi):
    """Needed [a0|c0]^(m) entries, in an order where every entry follows its inputs."""
    need = set()
    stack = [(a, c, 0) for a in range(NAO[e_lo - 1] if e_lo else 0, NAO[e_hi])
             for c in range(NAO[f_lo - 1] if f_lo else 0, NAO[f_hi])]
    while stack:
        key = stack.pop()
        if key in need:
            continue
        need.add(key)
        stack.extend(vrr_deps(*key))
    return sorted(need, key=lambda k: (k[1], k[0], k[2]))


def vrr_deps(a, c, m):
    if c == 0:
        if a == 0:
            return []
        i = shift_dir(a)
        am = shift_minus(a, i)
        amm = shift_minus(am, i)
        d = [(am, 0, m), (am, 0, m + 1)]
        if amm >= 0:
            d += [(amm, 0, m), (amm, 0, m + 1)]
        return d
    i = shift_dir(c)
    cm = shift_minus(c, i)
    cmm = shift_minus(cm, i)
    am = shift_minus(a, i)
    d = [(a, cm, m), (a, cm, m + 1)]
    if am >= 0:
        d.append((am, cm, m + 1))
    if cmm >= 0:
        d += [(a, cmm, m), (a, cmm, m + 1)]
    return d


def vname(a, c, m):
    return f"v{a}_{c}_{m}"


def vrr_line(a, c, m):
    """The recurrence of src/HGP.jl:189-190 / :218-236 for one entry."""
    if c == 0:
        if a == 0:
            return f"const VT {vname(0, 0, m)} = (VT)(pref * F[{m}]);"
        i = shift_dir(a)
        am = shift_minus(a, i)
        amm = shift_minus(am, i)
        x = XYZ[i]
        s = f"PA{x} * {vname(am, 0, m)} + WP{x} * {vname(am, 0, m + 1)}"
        if amm >= 0:
            k = AO[am][i]
            s += (f" + (VT){k}.0 * oo2z * ({vname(amm, 0, m)} - rho_z * "
                  f"{vname(amm, 0, m + 1)})")
        return f"const VT {vname(a, 0, m)} = {s};"
    i = shift_dir(c)
    cm = shift_minus(c, i)
    cmm = shift_minus(cm, i)
    am = shift_minus(a, i)
    x = XYZ[i]
    s = f"QC{x} * {vname(a, cm, m)} + WQ{x} * {vname(a, cm, m + 1)}"
    if am >= 0:
        s += f" + (VT){AO[a][i]}.0 * oo2ze * {vname(am, cm, m + 1)}"
    if cmm >= 0:
        k = AO[cm][i]
        s += f" + (VT){k}.0 * oo2e * ({vname(a, cmm, m)} - rho_e * {vname(a, cmm, m + 1)})"
    return f"const VT {vname(a, c, m)} = {s};"


# ------------------------------------------------------------------ HRR plan
class HrrPlan:
    """(ab|cd) from the contracted [a0|c0] block: bra HRR then ket HRR (src/HGP.jl:92-114)."""

    def __init__(self, la, lb, lc, ld):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.lines = []
        self.done = {}
        e, f = la + lb, lc + ld
        self.acc_a = [a for l in range(la, e + 1) for a in shell_range(l)]
        self.acc_c = [c for l in range(lc, f + 1) for c in shell_range(l)]
        self.acc_index = {(a, c): i * len(self.acc_c) + j
                          for i, a in enumerate(self.acc_a) for j, c in enumerate(self.acc_c)}
        self.targets = []
        for a in shell_range(la):
            for b in shell_range(lb):
                for c in shell_range(lc):
                    for d in shell_range(ld):
                        self.targets.append((a, b, c, d, self.ket(a, b, c, d)))

    def bra(self, a, b, c):
        if b == 0:
            return f"acc[{self.acc_index[(a, c)]}]"
        key = ("h", a, b, c)
        if key in self.done:
            return self.done[key]
        j = shift_dir(b)
        bm = shift_minus(b, j)
        t1 = self.bra(shift_plus(a, j), bm, c)
        t2 = self.bra(a, bm, c)
        name = f"h{a}_{b}_{c}"
        self.lines.append(f"const double {name} = {t1} + AB{XYZ[j]} * {t2};")
        self.done[key] = name
        return name

    def ket(self, a, b, c, d):
        if d == 0:
            return self.bra(a, b, c)
        key = ("k", a, b, c, d)
        if key in self.done:
            return self.done[key]
        j = shift_dir(d)
        dm = shift_minus(d, j)
        t1 = self.ket(a, b, shift_plus(c, j), dm)
        t2 = self.ket(a, b, c, dm)
        name = f"k{a}_{b}_{c}_{d}"
        self.lines.append(f"const double {name} = {t1} + CD{XYZ[j]} * {t2};")
        self.done[key] = name
        return name


# ------------------------------------------------------------------ emit
def emit_class_pair(X, Y):
    (la, lb), (lc, ld) = X, Y
    tag = tag_of(X, Y)
    e, f = la + lb, lc + ld
    M = e + f
    entries = vrr_entries(la, e, lc, f)
    hp = HrrPlan(la, lb, lc, ld)
    nacc = len(hp.acc_a) * len(hp.acc_c)
    na, nb, nc, nd = [len(shell_range(l)) for l in (la, lb, lc, ld)]
    nout = na * nb * nc * nd
    ind = "        "
    vrr_code = "\n".join(ind + "    " + vrr_line(*k) for k in entries)
    acc_code = "\n".join(
        f"{ind}    acc[{hp.acc_index[(a, c)]}] += (double){vname(a, c, 0)};"
        for a in hp.acc_a for c in hp.acc_c)
    hrr_code = "\n".join("    " + ln for ln in hp.lines)
    out_code = []
    for x, (a, b, c, d, expr) in enumerate(hp.targets):
        g = comp_norm(a) * comp_norm(b) * comp_norm(c) * comp_norm(d)
        if abs(g - 1.0) < 1e-15:
            out_code.append(f"    res[{x}] = {expr};")
        else:
            out_code.append(f"    res[{x}] = {expr} * {g!r};")
    out_code = "\n".join(out_code)
    stores = []
    for ia in range(na):
        for ib in range(nb):
            for ic in range(nc):
                for id_ in range(nd):
                    x = ((ia * nb + ib) * nc + ic) * nd + id_
                    conds = []
                    if la == lb:
                        conds.append(f"(!dab || {ia} >= {ib})")
                    if lc == ld:
                        conds.append(f"(!dcd || {ic} >= {id_})")
                    cond = " && ".join(conds) if conds else "true"
                    stores.append(
                        f"    {{ const long long ij = ij_{ia}_{ib}, kl = kl_{ic}_{id_};\n"
                        f"      if ({cond} && (!same || ij >= kl)) "
                        f"out[packed_index(ij, kl)] = res[{x}]; }}")
    ij_code = "\n".join(f"    const long long ij_{ia}_{ib} = pair_index(ib_.z + {ia}, ib_.w + {ib});"
                        for ia in range(na) for ib in range(nb))
    kl_code = "\n".join(f"    const long long kl_{ic}_{id_} = pair_index(ik_.z + {ic}, ik_.w + {id_});"
                        for ic in range(nc) for id_ in range(nd))
    store_code = "\n".join(stores)
    schwarz = ""
    if X == Y:
        diag = []
        for ia in range(na):
            for ib in range(nb):
                x = ((ia * nb + ib) * nc + ia) * nd + ib
                diag.append(f"    m = fmax(m, fabs(res[{x}]));")
        diag = "\n".join(diag)
        accdiag = "\n".join(f"        w = fmax(w, fabs(acc[{hp.acc_index[(a, a)]}]));" for a in hp.acc_a)
        schwarz = f"""
// Bounds of the pairs of one class.
// full == 0 (plan set-up): for every primitive pair k of pair p, from the diagonal primitive
//   quartet (a_k b_k | a_k b_k):
//     pbound[k].x = b_k = sqrt(max over components |(a_k b_k|a_k b_k)|)
//     pbound[k].y = w_k = sqrt(max over the VRR block |[e0|e0]_kk|), e = la..la+lb
//   By the Schwarz inequality b_k b_l bounds |(a_k b_k|c_l d_l)| and w_k w_l bounds every
//   entry of the VRR output block [e0|f0] that the HRR combines.
// full != 0: the contracted bound Q_p = sqrt(max |(ab|ab)|) into qout[p].
__global__ void __launch_bounds__(128) schwarz_kernel_{tag}(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[{nout}];
    if (full) {{
        quartet_{tag}<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
{diag}
        qout[p] = sqrt(m);
        return;
    }}
    double acc[{nacc}];
    for (int k = 0; k < in.y; ++k) {{
        quartet_{tag}<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
{diag}
{accdiag}
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }}
}}

void launch_schwarz_{tag}(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {{
    if (np <= 0) return;
    schwarz_kernel_{tag}<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}}
"""
    if nout <= STAGE_MAX_OUT:
        sbytes = 4 * 32 * nout * 8
        mixed_attr = (f"        cudaFuncSetAttribute(eri_queue_{tag}<1, 0>, "
                      f"cudaFuncAttributeMaxDynamicSharedMemorySize, {sbytes});\n"
                      if len(entries) >= MIXED_MIN_VRR else "")
        stage_fn = (f"""
// The dynamic shared memory of the two-phase staging ({sbytes} bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_{tag}() {{
    static bool done[64] = {{false}};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {{
        cudaFuncSetAttribute(eri_queue_{tag}<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, {sbytes});
{mixed_attr}        done[dev] = true;
    }}
}}
""" if sbytes > 48 * 1024 else "")
        stage_prep = (f"    // two-phase plans stage the chunk's blocks in {sbytes} bytes of dynamic shared memory\n"
                      f"    const size_t smem = Q.scratch && !Q.jk.J ? {sbytes} : 0;" +
                      (f"\n    if (smem) eri_prepare_{tag}();" if sbytes > 48 * 1024 else ""))
        occ_prep = f"    eri_prepare_{tag}();" if sbytes > 48 * 1024 else ""
    else:
        stage_fn, occ_prep = "", ""
        stage_prep = "    constexpr size_t smem = 0;"
    if nout <= STAGE_MAX_OUT:
        scratch_store = f"""            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * {nout} doubles (launch_eri_{tag})
            double *sb = stg + (threadIdx.x >> 5) * (32 * {nout});
            if (lead) hrr_{tag}(Q.pairs, p, q, acc, sb + kq * {nout});
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long){nout};
            for (int t = lane; t < nlive * {nout}; t += 32) dst[t] = sb[t];
            __syncwarp();"""
    else:
        scratch_store = f"""            // two-phase: each leader stores its quartet's whole block at its slot
            if (lead) {{
                double res[{nout}];
                hrr_{tag}(Q.pairs, p, q, acc, res);
                double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                    (__ldg(&Q.chunk_slot[c]) + base + kq) * (long long){nout};
#pragma unroll
                for (int x = 0; x < {nout}; ++x) dst[x] = res[x];
            }}"""
    if len(entries) >= MIXED_MIN_VRR:
        mixed_dispatch = ("    const bool jk = Q.jk.J != nullptr;\n"
                          "    if (mixed) {{ if (jk) eri_queue_{t}<1, 1><<<grid, 128, 0, s>>>(Q); "
                          "else eri_queue_{t}<1, 0><<<grid, 128, smem, s>>>(Q); }}\n"
                          "    else if (jk) eri_queue_{t}<0, 1><<<grid, 128, 0, s>>>(Q);\n"
                          "    else eri_queue_{t}<0, 0><<<grid, 128, smem, s>>>(Q);").format(t=tag)
        occ_dispatch = ("    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_{t}<1, 0>, 128, 0);\n"
                        "    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_{t}<0, 0>, 128, 0);").format(t=tag)
    else:
        mixed_dispatch = ("    (void)mixed;  // no FP32 variant for this class (MIXED_MIN_VRR)\n"
                          "    if (Q.jk.J) eri_queue_{t}<0, 1><<<grid, 128, 0, s>>>(Q);\n"
                          "    else eri_queue_{t}<0, 0><<<grid, 128, smem, s>>>(Q);").format(t=tag)
        occ_dispatch = ("    (void)mixed;\n"
                        "    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_{t}<0, 0>, 128, 0);").format(t=tag)
    return f"""// Generated by gen_eri.py -- class ({'spdfg'[la]}{'spdfg'[lb]}|{'spdfg'[lc]}{'spdfg'[ld]}).  Do not edit.
// VRR entries: {len(entries)}, contracted block: {nacc}, HRR lines: {len(hp.lines)}, outputs: {nout}.
#include "../eri_common.cuh"

namespace molints {{

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[{nacc}], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_{tag}(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {{
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < {nacc}; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {{
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {{
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[{M + 1}];
            boys_fm<{M}>(T, B, F);
            const VT PAx = (VT)bra.pax, PAy = (VT)bra.pay, PAz = (VT)bra.paz;
            const VT QCx = (VT)ket.pax, QCy = (VT)ket.pay, QCz = (VT)ket.paz;
            const double ez = ket.zeta * r2, zz = bra.zeta * r2;
            const VT WPx = (VT)(-ez * PQx), WPy = (VT)(-ez * PQy), WPz = (VT)(-ez * PQz);
            const VT WQx = (VT)(zz * PQx), WQy = (VT)(zz * PQy), WQz = (VT)(zz * PQz);
            const VT oo2z = (VT)bra.oo2z, oo2e = (VT)ket.oo2z, oo2ze = (VT)(0.5 * r2);
            const VT rho_z = (VT)ez, rho_e = (VT)zz;
            (void)PAx; (void)PAy; (void)PAz; (void)QCx; (void)QCy; (void)QCz;
            (void)WPx; (void)WPy; (void)WPz; (void)WQx; (void)WQy; (void)WQz;
            (void)oo2z; (void)oo2e; (void)oo2ze; (void)rho_z; (void)rho_e;
{vrr_code}
{acc_code}
        }}
    }}
}}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[{nout}] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_{tag}(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {{
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
{hrr_code}
{out_code}
}}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[{nout}]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_{tag}(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {{
    double acc[{nacc}];
    vrr_{tag}<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {{
#pragma unroll
        for (int x = 0; x < {nacc}; ++x) acc_out[x] = acc[x];
    }}
    hrr_{tag}(P, p, q, acc, res);
}}

__device__ __forceinline__ void store_{tag}(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {{
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
{ij_code}
{kl_code}
{store_code}
}}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_{tag}(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {{
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < {nout}; ++x) {{
        const int ia = x / {nb * nc * nd}, ibb = (x / {nc * nd}) % {nb}, ic = (x / {nd}) % {nc}, id = x % {nd};
        if ((dab && ia < ibb) || (dcd && ic < id)) continue;
        const int i = ib_.z + ia, j = ib_.w + ibb, k = ik_.z + ic, l = ik_.w + id;
        if (same && pair_index(i, j) < pair_index(k, l)) continue;
        jk_add(jk, i, j, k, l, res[x]);
    }}
}}

// Persistent work-queue kernel: each warp takes chunks (one bra pair, a run of consecutive
// ket pairs of one molecule) from a shared counter until the chunk list, ordered by
// decreasing estimated cost, is exhausted.  A chunk's count field carries the split in bits
// 16+: lg = log2 S (bits 16-18) and lgj = log2 Sj (bits 20-22).  S lanes share each quartet:
// lane l takes ket pair q0 + l % (32/S) (+ 32/S per round); its group rank s = l / (32/S)
// takes every Sj-th ket primitive from s % Sj and every (S/Sj)-th bra primitive from s / Sj.
// The S partial blocks are summed by a fixed butterfly (the result depends on the split
// alone, not on the chunk), and the group's first lane runs the HRR and stores.  Heavy
// quartets are split so that no single lane's serial primitive loop sets the kernel time.
// JK: digest into J and K (molints_plan_jk) instead of storing the packed integrals; a separate
// instantiation, so that the store kernels carry none of the digestion code.
template <int MIXED, int JK>
__global__ void __launch_bounds__(128) eri_queue_{tag}(const EriQueue Q) {{
    const int lane = threadIdx.x & 31;
    for (;;) {{
        int c = 0;
        if (lane == 0) c = atomicAdd(Q.counter, 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= Q.nchunks) return;
        const int4 ch = __ldg(&Q.chunks[c]);
        const int p = ch.x, cnt = ch.z & 0xffff, lg = (ch.z >> 16) & 7, lgj = (ch.z >> 20) & 7;
        const int W = 32 >> lg, kq = lane & (W - 1), s = lane >> (5 - lg);
        const int js = s & ((1 << lgj) - 1), is = s >> lgj;
        for (int base = 0; base < cnt; base += W) {{
        const int q = ch.y + base + kq;
        const bool live = base + kq < cnt;
        double acc[{nacc}];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {{
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }}
        if (!live || bp.x * bq.x < Q.screen_cut) {{
#pragma unroll
            for (int x = 0; x < {nacc}; ++x) acc[x] = 0.0;
        }} else {{
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_{tag}<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_{tag}<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }}
        if (lg) {{
            for (int off = W; off < 32; off <<= 1) {{
#pragma unroll
                for (int x = 0; x < {nacc}; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }}
        }}
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {{
{scratch_store}
        }} else if (lead) {{
            double res[{nout}];
            hrr_{tag}(Q.pairs, p, q, acc, res);
            if constexpr (JK) {{
                jk_{tag}(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            }} else {{
                store_{tag}(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }}
        }}
        }}
    }}
}}

{stage_fn}
void launch_eri_{tag}(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {{
    if (Q.nchunks <= 0 || grid <= 0) return;
{stage_prep}
{mixed_dispatch}
}}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_{tag}(int mixed) {{
{occ_prep}
    int n = 0;
{occ_dispatch}
    return n;
}}
{schwarz}
}}  // namespace molints
"""


def emit_dispatch(pairs):
    """eri_dispatch.h: launch tables over all pair classes up to f (gen_rys.LMAX).  HGP kernels
    exist for the class pairs of shells up to d; Rys kernels for every class pair."""
    cls = gen_rys.pair_classes()
    hgp = set(pairs)
    lines = ["// Generated by gen_eri.py.  Do not edit.", "#pragma once",
             '#include "eri_common.cuh"', "namespace molints {"]
    for X, Y in pairs:
        t = tag_of(X, Y)
        lines.append(f"void launch_eri_{t}(const EriQueue &Q, int mixed, int grid, cudaStream_t s);")
        lines.append(f"int occupancy_eri_{t}(int mixed);")
        if X == Y:
            lines.append(f"void launch_schwarz_{t}(const PairTab &P, const BoysTab &B, int p0, "
                         f"int np, double2 *pbound, double *qout, int full, cudaStream_t s);")
    for X, Y in gen_rys.class_pairs():
        t = tag_of(X, Y)
        lines.append(f"void launch_rys_{t}(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);")
        lines.append(f"int occupancy_rys_{t}(int mixed);")
        if X == Y:
            lines.append(f"void launch_rys_bound_{t}(const PairTab &P, const RysTab &R, int p0, int np, "
                         f"double2 *pbound, double *qout, int full, cudaStream_t s);")
    lines.append("typedef void (*EriLauncher)(const EriQueue &, int, int, cudaStream_t);")
    lines.append("typedef int (*EriOccupancy)(int);")
    lines.append("typedef void (*SchwarzLauncher)(const PairTab &, const BoysTab &, int, int, "
                 "double2 *, double *, int, cudaStream_t);")
    lines.append("typedef void (*RysLauncher)(const EriQueue &, const RysTab &, int, int, cudaStream_t);")
    lines.append("typedef int (*RysOccupancy)(int);")
    lines.append("typedef void (*RysBoundLauncher)(const PairTab &, const RysTab &, int, int, "
                 "double2 *, double *, int, cudaStream_t);")
    lines.append(f"constexpr int kLmax = {gen_rys.LMAX};      // shells up to f (Rys)")
    lines.append(f"constexpr int kLmaxHgp = {LMAX_ALL_HGP};   // every class pair up to d has an HGP kernel")
    lines.append(f"constexpr int kNumPairClasses = {len(cls)};")
    lines.append("// pair class c = (kPairClassLa[c], kPairClassLb[c]), ordered by la+lb then la")
    lines.append("constexpr int kPairClassLa[] = {" + ", ".join(str(c[0]) for c in cls) + "};")
    lines.append("constexpr int kPairClassLb[] = {" + ", ".join(str(c[1]) for c in cls) + "};")
    n = len(cls)

    def table(ctype, name, fmt, cond=lambda X, Y: True):
        lines.append(f"static const {ctype} {name}[{n}][{n}] = {{")
        for i, X in enumerate(cls):
            row = [fmt(X, Y) if (j <= i and cond(X, Y)) else "nullptr" for j, Y in enumerate(cls)]
            lines.append("    {" + ", ".join(row) + "},")
        lines.append("};")

    lines.append("// [x][y], x >= y (bra class x, ket class y); nullptr where no HGP kernel exists")
    table("EriLauncher", "kEriLaunchers", lambda X, Y: f"launch_eri_{tag_of(X, Y)}", lambda X, Y: (X, Y) in hgp)
    table("EriOccupancy", "kEriOccupancy", lambda X, Y: f"occupancy_eri_{tag_of(X, Y)}", lambda X, Y: (X, Y) in hgp)
    table("char *const", "kEriNames", lambda X, Y: f'"eri_{tag_of(X, Y)}"', lambda X, Y: (X, Y) in hgp)
    lines.append("// relative cost of one primitive quartet of the HGP kernel, 1 + VRR entries / 4 (the")
    lines.append("// (ss|ss) quartet ~ 1); sizes the lane split of heavy quartets; 0 where no HGP kernel")
    lines.append(f"static const float kEriPrimCost[{n}][{n}] = {{")
    for i, X in enumerate(cls):
        row = []
        for j, Y in enumerate(cls):
            if j <= i and (X, Y) in hgp:
                (la, lb), (lc, ld) = X, Y
                row.append(f"{1.0 + len(vrr_entries(la, la + lb, lc, lc + ld)) / 4.0!r}f")
            else:
                row.append("0.0f")
        lines.append("    {" + ", ".join(row) + "},")
    lines.append("};")
    lines.append("// 1 where the class pair's kernel has an FP32 variant for MIXED quartets (HGP: at least")
    lines.append(f"// {MIXED_MIN_VRR} VRR entries; Rys: gen_rys's MIXED_MIN_NBLK / MIXED_MAX_ACC rule), else 0")
    for name, has in (("kEriHasFp32", lambda X, Y: (X, Y) in hgp and
                       len(vrr_entries(X[0], X[0] + X[1], Y[0], Y[0] + Y[1])) >= MIXED_MIN_VRR),
                      ("kRysHasFp32", lambda X, Y: gen_rys.class_tables(X, Y)["mixed"])):
        lines.append(f"static const unsigned char {name}[{n}][{n}] = {{")
        for i, X in enumerate(cls):
            lines.append("    {" + ", ".join("1" if (j <= i and has(X, Y)) else "0"
                                             for j, Y in enumerate(cls)) + "},")
        lines.append("};")
    table("RysLauncher", "kRysLaunchers", lambda X, Y: f"launch_rys_{tag_of(X, Y)}")
    table("RysOccupancy", "kRysOccupancy", lambda X, Y: f"occupancy_rys_{tag_of(X, Y)}")
    table("char *const", "kRysNames", lambda X, Y: f'"rys_{tag_of(X, Y)}"')
    lines.append(f"static const char *const kSchwarzNames[{n}] = {{")
    lines.append("    " + ", ".join(f'"schwarz_{tag_of(X, X)[:2]}"' for X in cls))
    lines.append("};")
    lines.append(f"static const SchwarzLauncher kSchwarzLaunchers[{n}] = {{")
    lines.append("    " + ", ".join(f"launch_schwarz_{tag_of(X, X)}" if (X, X) in hgp else "nullptr"
                                   for X in cls))
    lines.append("};")
    lines.append(f"static const RysBoundLauncher kRysBoundLaunchers[{n}] = {{")
    lines.append("    " + ", ".join(f"launch_rys_bound_{tag_of(X, X)}" for X in cls))
    lines.append("};")
    lines.append("}  // namespace molints")
    return "\n".join(lines) + "\n"


def emit_class_table(path: Path):
    """class_table.h: the default per-class-pair method table of MOLINTS_METHOD_AUTO, from the
    class tuner's result kept in data/class_table_<gpu>.json (the classes it found faster with
    Rys, and those whose FP32 variant it found faster than FP64)."""
    import json
    d = json.loads(path.read_text())
    cls = gen_rys.pair_classes()
    lv = {"s": 0, "p": 1, "d": 2, "f": 3}

    def idx(t):
        return cls.index((lv[t[0]], lv[t[1]])), cls.index((lv[t[2]], lv[t[3]]))
    n = len(cls)
    tab = [[0] * n for _ in range(n)]
    for x in range(n):
        for y in range(x + 1):
            tab[x][y] = 1 | 4  # MOLINTS_METHOD_HGP | MOLINTS_CLASS_NO_FP32
    for t in d["rys"]:
        x, y = idx(t)
        tab[x][y] = 2 | (tab[x][y] & 4)
    for t in d["fp32"]:
        x, y = idx(t)
        tab[x][y] &= 3
    lines = [f"// Generated by gen_eri.py from data/{path.name}.  Do not edit.",
             "// Default MOLINTS_METHOD_AUTO table of contexts on the device named below:",
             f"// {d['source']}.",
             "// Entries: 1 HGP, 2 Rys, | 4 (MOLINTS_CLASS_NO_FP32) where MIXED runs the FP64 kernel.",
             "#pragma once", "#include <stdint.h>", "namespace molints {",
             f'constexpr const char *kTunedDevice = "{d["device"]}";',
             f"static const int32_t kTunedClassMethods[{n}][{n}] = {{"]
    for x in range(n):
        lines.append("    {" + ", ".join(str(v) for v in tab[x]) + "},")
    # work-queue schedule (molints_schedule: lane_cost, hgp_widen, rys_chunks, rys_max_width,
    # gather_blocks), the built-in values where the tuner's result has none
    sc = dict({"lane_cost": 80.0, "hgp_widen": 1, "rys_chunks": 4096, "rys_max_width": 8, "gather_blocks": 5},
              **d.get("schedule", {}))
    keys = ("lane_cost", "hgp_widen", "rys_chunks", "rys_max_width", "gather_blocks")
    lines += ["};",
              "// work-queue schedule: " + ", ".join(keys)
              + (f" ({d['schedule_source']})" if "schedule_source" in d else " (built-in values)"),
              f"static const double kTunedSchedule[{len(keys)}] = {{" +
              ", ".join(repr(float(sc[k])) for k in keys) + "};",
              "}  // namespace molints", ""]
    return "\n".join(lines)


def generate(out_dir: Path = OUT_DIR):
    out_dir.mkdir(parents=True, exist_ok=True)
    pairs = class_pairs()
    written = []
    for X, Y in pairs:
        p = out_dir / f"eri_{tag_of(X, Y)}.cu"
        src = emit_class_pair(X, Y)
        if not p.exists() or p.read_text() != src:
            p.write_text(src)
        written.append(p)
    written += gen_rys.generate(out_dir)
    d = HERE / "eri_dispatch.h"
    src = emit_dispatch(pairs)
    if not d.exists() or d.read_text() != src:
        d.write_text(src)
    t = HERE / "class_table.h"
    src = emit_class_table(HERE.parent / "data" / "class_table_b200.json")
    if not t.exists() or t.read_text() != src:
        t.write_text(src)
    return written


if __name__ == "__main__":
    files = generate()
    print(f"{len(files)} class-pair kernels in {OUT_DIR}", file=sys.stderr)

"""Generate the Rys-quadrature class kernels (CUDA C for sm_100a).

This is the engine's counterpart of the reference's Rys driver (coulomb_rys and Int1d,
src/Rys.jl:27-156), reorganised for the GPU as Rys VRR + HGP HRR:

  * per primitive quartet and root t_r^2 = u_r of the NR = (e+f)/2 + 1 point Rys rule
    (nodes and weights from the tables of gen_rys_tables.py), the 2-D integrals
    I_x(a, c), I_y, I_z for a <= e = la+lb, c <= f = lc+ld by the Rys recurrences
        I(a+1, c) = C00 I(a, c) + a B10 I(a-1, c) + c B00 I(a, c-1)
        I(a, c+1) = D00 I(a, c) + c B01 I(a, c-1) + a B00 I(a-1, c)
    (C00 = PA + (W-P) u, D00 = QC + (W-Q) u, B10 = (1 - eta u/(zeta+eta)) / 2 zeta,
    B01 = (1 - zeta u/(zeta+eta)) / 2 eta, B00 = u / 2(zeta+eta)), the same recurrences as
    Recur (src/Rys.jl:86-120) written in u instead of t^2/(1-t^2);
  * the [e0|f0] block of the class (rows: the cartesian components of l = la..e, columns:
    l = lc..f) as sum_r W_r I_x I_y I_z, contracted over the primitive quartets in FP64;
  * the horizontal recurrence on the contracted block in closed form (the binomial
    transfer of Shift, src/Rys.jl:122-135, applied once per side after contraction):
        (a b| = sum_{k <= b} C(b_x,k_x) C(b_y,k_y) C(b_z,k_z) AB^(b-k) (a+k, 0|
    bra side first, then ket side;
  * component norms and the packed iindex store, as in the HGP kernels.

A group of G threads (32, 64 or 128; a block of 128 threads holds 128/G groups) owns one
contracted shell quartet at a time.  Stage 1 of a primitive batch: one thread per
(primitive quartet, root) evaluates the root and builds the three 2-D tables into shared
memory; stage 2: every thread accumulates its own entries of the [e0|f0] block in registers
(small blocks: NSLOT threads per entry, each over every NSLOT-th quartet of the batch).
After the primitive loop the block goes to shared memory for the two HRR passes.

The class-specific data (block entry -> table offsets, HRR term lists, norms) are emitted as
device arrays; the kernel body is the template in rys_common.cuh.
"""
from __future__ import annotations

import math
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "generated"
LMAX = 3             # shells up to f
NMONO = 20           # monomials AB^(px,py,pz), px+py+pz <= 3
# Classes with at least this many block entries and at most MIXED_MAX_ACC accumulators per
# thread get an FP32 variant for MIXED quartets (stage-2 products summed in FP32 per batch).
MIXED_MIN_NBLK = 32
MIXED_MAX_ACC = 24
COL_MIN_NC = 16
COL_MAX_NA = 48


def shell_components(l):
    """src/Basis.jl:269-279 order (x-power descending, then y), l=3 with xzz before xyz."""
    comps = [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]
    if l == 3:
        comps[4], comps[5] = comps[5], comps[4]
    return comps


def ncart(l):
    return (l + 1) * (l + 2) // 2


# Mirrored pair classes (la < lb): a pair (f, d) whose d shell is the tighter one is computed
# as (d f|, so that the HRR moves angular momentum away from the tight shell (P near A); the
# other orientation loses up to 1e-11 Eh to cancellation.  (For lb <= 1 the loss stays at
# rounding level, and equal-L pairs are reoriented within their class.)
MIRRORED = [(2, 3)]


def pair_classes(lmax=LMAX):
    """Shell-pair classes (la, lb): la >= lb, plus MIRRORED; ordered by la+lb then la."""
    cls = [(la, lb) for la in range(lmax + 1) for lb in range(la + 1)]
    cls += [c for c in MIRRORED if max(c) <= lmax]
    return sorted(cls, key=lambda c: (c[0] + c[1], c[0]))


def class_pairs(lmax=LMAX):
    cls = pair_classes(lmax)
    return [(X, cls[j]) for i, X in enumerate(cls) for j in range(i + 1)]


def tag_of(X, Y):
    L = "spdfg"
    return f"{L[X[0]]}{L[X[1]]}{L[Y[0]]}{L[Y[1]]}"


MONOS = [(px, py, d - px - py) for d in range(4) for px in range(d, -1, -1) for py in range(d - px, -1, -1)]
MONO_INDEX = {m: i for i, m in enumerate(MONOS)}
assert len(MONOS) == NMONO


def dfact2(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def comp_norm(c):
    return 1.0 / math.sqrt(dfact2(2 * c[0] - 1) * dfact2(2 * c[1] - 1) * dfact2(2 * c[2] - 1))


def block_components(l0, l1):
    """Components of the block rows (or columns): l = l0..l1, each shell in reference order."""
    out = []
    for l in range(l0, l1 + 1):
        out.extend(shell_components(l))
    return out


def hrr_terms(lx, ly, rows_index):
    """Closed-form HRR (a b| = sum_k C(b,k) AB^(b-k) (a+k, 0| for a in shell lx, b in shell ly.
    Returns per output r = ia * ncart(ly) + ib the list of (block index, monomial, binomial)."""
    out = []
    for a in shell_components(lx):
        for b in shell_components(ly):
            terms = []
            for kx in range(b[0] + 1):
                for ky in range(b[1] + 1):
                    for kz in range(b[2] + 1):
                        src = rows_index[(a[0] + kx, a[1] + ky, a[2] + kz)]
                        mono = MONO_INDEX[(b[0] - kx, b[1] - ky, b[2] - kz)]
                        binom = math.comb(b[0], kx) * math.comb(b[1], ky) * math.comb(b[2], kz)
                        terms.append((src, mono, binom))
            out.append(terms)
    return out


def class_tables(X, Y):
    """Everything the kernel of class pair (X|Y) needs, as Python data."""
    (la, lb), (lc, ld) = X, Y
    e, f = la + lb, lc + ld
    nr = (e + f) // 2 + 1
    rows = block_components(la, e)
    cols = block_components(lc, f)
    rows_index = {c: i for i, c in enumerate(rows)}
    cols_index = {c: i for i, c in enumerate(cols)}
    S = (e + 1) * (f + 1)
    blk = []
    for a in rows:
        for c in cols:
            offs = [a[t] * (f + 1) + c[t] for t in range(3)]
            blk.append(offs)
    bra = hrr_terms(la, lb, rows_index)
    ket = hrr_terms(lc, ld, cols_index)
    norm_ab = [comp_norm(a) * comp_norm(b) for a in shell_components(la) for b in shell_components(lb)]
    norm_cd = [comp_norm(c) * comp_norm(d) for c in shell_components(lc) for d in shell_components(ld)]
    na, nc = len(rows), len(cols)
    nblk = na * nc
    nab, ncd = ncart(la) * ncart(lb), ncart(lc) * ncart(ld)
    # column mode: one stage-2 thread per block column holds that column's three 2-D table
    # columns and all NA row accumulators in registers (3(E+1) shared loads per root instead
    # of 3 per entry); for blocks with at least COL_MIN_NC columns and at most COL_MAX_NA rows
    col = nc >= COL_MIN_NC and na <= COL_MAX_NA
    if col:
        G = 32 * ((nc + 31) // 32)
    elif nblk <= 128:
        G = 32
    elif nblk <= 1024:
        G = 64
    else:
        G = 128
    # primitive quartets per batch: one stage-1 thread per (quartet, root); the batch's 2-D
    # tables may use the HRR buffers' room (at least 6144 doubles)
    hrr_room = max(nblk + nab * nc, 6144)
    npb = max(1, min(G // nr, hrr_room // (3 * nr * S)))
    # stage-2 slots: a small block is accumulated by NSLOT threads per entry, each taking every
    # NSLOT-th quartet of a batch, and the slots are summed after the primitive loop
    nslot = max(1, min(npb, G // nblk)) if (2 * nblk <= G and not col) else 1
    acc = 1 if (nslot > 1 or col) else (nblk + G - 1) // G
    smem_group = 2 * NMONO + max(npb * nr * 3 * S, nblk + nab * nc, nslot * nblk)
    mixed = nblk >= MIXED_MIN_NBLK and (acc <= MIXED_MAX_ACC or col)
    return dict(la=la, lb=lb, lc=lc, ld=ld, e=e, f=f, nr=nr, rows=rows, cols=cols, S=S,
                blk=blk, bra=bra, ket=ket, norm_ab=norm_ab, norm_cd=norm_cd, na=na, nc=nc,
                nblk=nblk, nab=nab, ncd=ncd, G=G, npb=npb, nslot=nslot, acc=acc,
                smem_group=smem_group, mixed=mixed, col=col)


def _flat_terms(lists):
    off, flat = [0], []
    for terms in lists:
        for src, mono, binom in terms:
            flat.append(src | (mono << 8) | (binom << 16))
        off.append(len(flat))
    return off, flat


def _arr(vals, fmt=str, per=12):
    vals = list(vals)
    lines = []
    for i in range(0, len(vals), per):
        lines.append("    " + ", ".join(fmt(v) for v in vals[i:i + per]) + ",")
    return "\n".join(lines) if lines else "    0,"


def emit_class_pair(X, Y):
    t = class_tables(X, Y)
    tag = tag_of(X, Y)
    blk = [o[0] | (o[1] << 8) | (o[2] << 16) for o in t["blk"]]
    boff, bterm = _flat_terms(t["bra"])
    koff, kterm = _flat_terms(t["ket"])
    smem_block = (128 // t["G"]) * t["smem_group"] * 8
    assert smem_block <= 227 * 1024, (tag, smem_block)
    diag = X == Y
    bound_kernel = bound_launch = ""
    if diag:
        bound_kernel = f"""
__global__ void __launch_bounds__(128) rys_bound_kernel_{tag}(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {{
    rys_bound_body<C_{tag}>(P, R, tabs_{tag}(), p0, np, pbound, qout, full);
}}
"""
        bound_launch = f"""
void launch_rys_bound_{tag}(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {{
    if (np <= 0) return;
    rys_prepare_{tag}();
    constexpr int ng = 128 / C_{tag}::G;
    rys_bound_kernel_{tag}<<<(np + ng - 1) / ng, 128, {smem_block}, s>>>(P, R, p0, np, pbound, qout, full);
}}
"""
    if t["mixed"]:
        mixed_dispatch = (f"    if (mixed) rys_queue_{tag}<1><<<grid, 128, {smem_block}, s>>>(Q, R);\n"
                          f"    else rys_queue_{tag}<0><<<grid, 128, {smem_block}, s>>>(Q, R);")
        occ_dispatch = (f"    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_{tag}<1>, 128, {smem_block});\n"
                        f"    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_{tag}<0>, 128, {smem_block});")
    else:
        mixed_dispatch = (f"    (void)mixed;  // no FP32 variant for this class\n"
                          f"    rys_queue_{tag}<0><<<grid, 128, {smem_block}, s>>>(Q, R);")
        occ_dispatch = (f"    (void)mixed;\n"
                        f"    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_{tag}<0>, 128, {smem_block});")
    if t["col"]:
        F1 = t["f"] + 1
        lines = []
        for ia, a in enumerate(t["rows"]):
            lines.append(f"        acc[{ia}] = fma(x[{a[0]}] * y[{a[1]}], z[{a[2]}], acc[{ia}]);")
        col_code = ("    // stage 2, column mode: acc[row] += x[ax] y[ay] z[az] for the column's table columns\n"
                    "    template <typename T, typename A>\n"
                    "    __device__ __forceinline__ static void col_update(const T *x, const T *y, const T *z, A *acc) {\n"
                    + "\n".join(lines) + "\n    }")
        colpow = ", ".join(str(c[0] | (c[1] << 4) | (c[2] << 8)) for c in t["cols"])
        col_code += f"\n    static constexpr int NCOLS = {t['nc']};"
        col_tab = f"\n// column components cx | cy << 4 | cz << 8\n__device__ const uint16_t kCol_{tag}[{t['nc']}] = {{ {colpow} }};\n"
    else:
        col_code = "    template <typename T, typename A>\n    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}"
        col_tab = ""
    return f"""// Generated by gen_rys.py -- Rys class ({tag[0]}{tag[1]}|{tag[2]}{tag[3]}).  Do not edit.
// roots {t['nr']}, block {t['na']} x {t['nc']}, outputs {t['nab']} x {t['ncd']}, group {t['G']} threads,
// {t['npb']} primitive quartets per batch, {t['nslot']} slot(s), {t['acc']} accumulators per thread, {smem_block} B shared per block{", column mode" if t["col"] else ""}.
#include "../rys_common.cuh"

namespace molints {{

struct C_{tag} {{
    static constexpr int LA = {t['la']}, LB = {t['lb']}, LC = {t['lc']}, LD = {t['ld']};
    static constexpr int E = {t['e']}, F = {t['f']}, NR = {t['nr']};
    static constexpr int NA = {t['na']}, NC = {t['nc']}, NBLK = {t['nblk']};
    static constexpr int NB = {ncart(t['lb'])}, ND = {ncart(t['ld'])};
    static constexpr int NAB = {t['nab']}, NCD = {t['ncd']};
    static constexpr int G = {t['G']}, NPB = {t['npb']}, NSLOT = {t['nslot']}, ACC = {t['acc']};
    static constexpr int S = {t['S']};
    static constexpr int SMEM_GROUP = {t['smem_group']};
    static constexpr bool COL = {'true' if t['col'] else 'false'};
{col_code}
}};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_{tag}[{len(blk)}] = {{
{_arr(blk)}
}};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_{tag}[{len(boff)}] = {{
{_arr(boff)}
}};
__device__ const uint32_t kBraTerm_{tag}[{len(bterm)}] = {{
{_arr(bterm)}
}};
__device__ const uint16_t kKetOff_{tag}[{len(koff)}] = {{
{_arr(koff)}
}};
__device__ const uint32_t kKetTerm_{tag}[{len(kterm)}] = {{
{_arr(kterm)}
}};
__device__ const double kNormAB_{tag}[{len(t['norm_ab'])}] = {{
{_arr(t['norm_ab'], repr, 4)}
}};
__device__ const double kNormCD_{tag}[{len(t['norm_cd'])}] = {{
{_arr(t['norm_cd'], repr, 4)}
}};

{col_tab}
__device__ __forceinline__ RysClassTabs tabs_{tag}() {{
    return RysClassTabs{{kBlk_{tag}, kBraOff_{tag}, kBraTerm_{tag}, kKetOff_{tag}, kKetTerm_{tag},
                        kNormAB_{tag}, kNormCD_{tag}, {"kCol_" + tag if t["col"] else "nullptr"}}};
}}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_{tag}(const EriQueue Q, const RysTab R) {{
    rys_queue_body<C_{tag}, MIXED>(Q, R, tabs_{tag}());
}}
{bound_kernel}
static void rys_prepare_{tag}() {{
    static bool done[64] = {{false}};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {{
        cudaFuncSetAttribute(rys_queue_{tag}<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, {smem_block});
{"        cudaFuncSetAttribute(rys_queue_" + tag + "<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, " + str(smem_block) + ");" if t["mixed"] else ""}
{"        cudaFuncSetAttribute(rys_bound_kernel_" + tag + ", cudaFuncAttributeMaxDynamicSharedMemorySize, " + str(smem_block) + ");" if diag else ""}
        done[dev] = true;
    }}
}}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_{tag}(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {{
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_{tag}();
    constexpr int ng = 128 / C_{tag}::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
{mixed_dispatch}
}}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_{tag}(int mixed) {{
    rys_prepare_{tag}();
    int n = 0;
{occ_dispatch}
    return n;
}}
{bound_launch}
}}  // namespace molints
"""


def generate(out_dir: Path = OUT_DIR):
    out_dir.mkdir(parents=True, exist_ok=True)
    written = []
    for X, Y in class_pairs():
        p = out_dir / f"rys_{tag_of(X, Y)}.cu"
        src = emit_class_pair(X, Y)
        if not p.exists() or p.read_text() != src:
            p.write_text(src)
        written.append(p)
    return written

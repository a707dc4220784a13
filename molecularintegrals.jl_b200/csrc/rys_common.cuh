// rys_common.cuh -- device templates of the Rys class kernels (generated/rys_*.cu).
//
// One group of C::G threads owns one contracted shell quartet (ab|cd) at a time:
//   1. rys_contract: the primitive quartets in batches of C::NPB.  Stage 1, one thread per
//      (primitive quartet, root): the Rys node u and weight W of that root, then the three
//      2-D tables I(a, c), a <= E, c <= F (the x table carries the prefactor and W) into
//      shared memory.  Stage 2, every thread: its own entries of the [e0|f0] block, sum over
//      the batch and the roots of I_x I_y I_z, accumulated in registers in FP64 (blocks of
//      at most G/2 entries: C::NSLOT threads per entry, summed at the end).  The contracted
//      block ends in shared memory.
//   2. rys_hrr: bra HRR into a (ab|f0) buffer, then ket HRR, both in the closed binomial form,
//      times the component norms; a sink stores (or reduces) each (ab|cd).
// Recurrences: Rys, Dupuis and King's 2-D integrals in the Head-Gordon/Pople variables, with
// u = t^2 the root (see gen_rys.py); MolecularIntegrals.jl states the same method in
// src/Rys.jl:59-156.
#pragma once
#include <algorithm>
#include <type_traits>

#include "eri_common.cuh"

namespace molints {

constexpr int kRysXmax = 100;   // Chebyshev fits on [0, 100); Gauss-Hermite limit above
constexpr int kRysNcheb = 16;
constexpr int kRysNmono = 20;   // AB^(px,py,pz), px+py+pz <= 3

// Class tables emitted by gen_rys.py.
struct RysClassTabs {
    const uint32_t *blk;       // [NBLK] block entry -> table offsets x | y << 8 | z << 16
    const uint16_t *bra_off;   // [NAB+1] term ranges of the bra outputs
    const uint32_t *bra_term;  // block row | monomial << 8 | binomial << 16
    const uint16_t *ket_off;   // [NCD+1]
    const uint32_t *ket_term;  // block column | monomial << 8 | binomial << 16
    const double *norm_ab;     // [NAB] component norms of a and b
    const double *norm_cd;     // [NCD]
    const uint16_t *col;       // column mode: [NC] column components cx | cy << 4 | cz << 8
};

// (px, py, pz) of monomial m, packed px | py << 2 | pz << 4, in gen_rys.MONOS order.
static __device__ const unsigned char kRysMonoPow[kRysNmono] = {
    0x00, 0x01, 0x04, 0x10, 0x02, 0x05, 0x11, 0x08, 0x14, 0x20,
    0x03, 0x06, 0x12, 0x09, 0x15, 0x21, 0x0c, 0x18, 0x24, 0x30};

__device__ __forceinline__ double rys_monomial(int m, double x, double y, double z) {
    const unsigned p = kRysMonoPow[m];
    double v = 1.0;
    for (unsigned i = 0; i < (p & 3u); ++i) v *= x;
    for (unsigned i = 0; i < ((p >> 2) & 3u); ++i) v *= y;
    for (unsigned i = 0; i < ((p >> 4) & 3u); ++i) v *= z;
    return v;
}

// sum_k c_k T_k(s) for 16 coefficients by Clenshaw's recurrence.
__device__ __forceinline__ double clenshaw16(const double *__restrict__ c, double s) {
    const double2 *v = reinterpret_cast<const double2 *>(c);
    double2 q[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) q[k] = __ldg(v + k);
    const double s2 = 2.0 * s;
    double b1 = 0.0, b2 = 0.0;
#pragma unroll
    for (int k = 15; k >= 1; --k) {
        const double ck = (k & 1) ? q[k >> 1].y : q[k >> 1].x;
        const double t = fma(s2, b1, ck - b2);
        b2 = b1;
        b1 = t;
    }
    return fma(s, b1, q[0].x - b2);
}

// Node u_r = t_r^2 and weight W_r of the NR-point Rys rule at X >= 0:
// sum_r W_r u_r^m = F_m(X) for m < 2 NR.
template <int NR>
__device__ __forceinline__ void rys_root(const RysTab &R, double X, int r, double &u, double &w) {
    if (X < (double)kRysXmax) {
        const int j = (int)X;
        const double s = 2.0 * (X - (double)j) - 1.0;
        const double *c = R.cheb + (size_t)kRysXmax * kRysNcheb * NR * (NR - 1) +
                          ((size_t)j * 2 * NR + r) * kRysNcheb;
        u = clenshaw16(c, s);
        w = clenshaw16(c + NR * kRysNcheb, s);
    } else {
        const int o = NR * (NR - 1) / 2 + r;
        const double ox = 1.0 / X;
        u = __ldg(R.herm_x2 + o) * ox;
        w = __ldg(R.herm_w + o) * sqrt(ox);
    }
}

// Barrier over the G threads of group gid (named barrier gid+1 for 64-thread groups).
template <int G>
__device__ __forceinline__ void group_sync(int gid) {
    if constexpr (G == 32) {
        __syncwarp();
    } else if constexpr (G >= 128) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(gid + 1), "r"(G) : "memory");
    }
}

template <int G>
__device__ __forceinline__ double group_max(double v, double *red, int gid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if constexpr (G == 32) {
        return v;
    } else {
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        group_sync<G>(gid);
        double r = 0.0;
#pragma unroll
        for (int w = 0; w < G / 32; ++w) r = fmax(r, red[gid * (G / 32) + w]);
        group_sync<G>(gid);
        return r;
    }
}

// Stage 1 of a primitive batch: thread tb*NR + tr (tb < nb) evaluates root tr of primitive
// quartet g0 + tb and writes the three 2-D tables of that root into tabs.
template <class C, typename TT>
__device__ __forceinline__ void rys_stage1(const PairTab &P, const RysTab &R, const int4 ib, const int4 ik,
                                           int i0, int j0, int nbp, int g0, int nb, int tb, int tr,
                                           TT *__restrict__ tabs) {
    constexpr int S = C::S, F1 = C::F + 1, NR = C::NR, E = C::E, F = C::F;
    if (tb < nb) {
        const int g = g0 + tb;
        const int gj = g / nbp;
        const PrimPair bra = load_pp(P.pp, ib.x + i0 + (g - gj * nbp));
        const PrimPair ket = load_pp(P.pp, ik.x + j0 + gj);
        const double rz = rsqrt(bra.zeta + ket.zeta);
        const double r2 = rz * rz;
        const double PQv[3] = {bra.px - ket.px, bra.py - ket.py, bra.pz - ket.pz};
        const double X = bra.zeta * ket.zeta * r2 * (PQv[0] * PQv[0] + PQv[1] * PQv[1] + PQv[2] * PQv[2]);
        double u, w;
        rys_root<NR>(R, X, tr, u, w);
        const double ez = ket.zeta * r2, zz = bra.zeta * r2;
        const double PAv[3] = {bra.pax, bra.pay, bra.paz}, QCv[3] = {ket.pax, ket.pay, ket.paz};
        const double b10 = bra.oo2z * fma(-ez, u, 1.0);
        const double b01 = ket.oo2z * fma(-zz, u, 1.0);
        const double b00 = 0.5 * r2 * u;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const double c00 = fma(-ez * PQv[ax], u, PAv[ax]);
            const double d00 = fma(zz * PQv[ax], u, QCv[ax]);
            TT *tab = tabs + ((tb * NR + tr) * 3 + ax) * S;
            // column c = 0 by the a-recurrence, then column c+1 from columns c and c-1
            double cur[E + 1], prev[E + 1];
            cur[0] = ax == 0 ? bra.kab * ket.kab * rz * w : 1.0;
            if (E > 0) cur[1] = c00 * cur[0];
#pragma unroll
            for (int a = 1; a < E; ++a) cur[a + 1] = fma(c00, cur[a], (double)a * b10 * cur[a - 1]);
#pragma unroll
            for (int a = 0; a <= E; ++a) {
                tab[a * F1] = (TT)cur[a];
                prev[a] = 0.0;
            }
#pragma unroll
            for (int c = 0; c < F; ++c) {
                double nxt[E + 1];
#pragma unroll
                for (int a = 0; a <= E; ++a) {
                    double v = d00 * cur[a];
                    if (c > 0) v = fma((double)c * b01, prev[a], v);
                    if (a > 0) v = fma((double)a * b00, cur[a - 1], v);
                    nxt[a] = v;
                }
#pragma unroll
                for (int a = 0; a <= E; ++a) {
                    prev[a] = cur[a];
                    cur[a] = nxt[a];
                    tab[a * F1 + c + 1] = (TT)nxt[a];
                }
            }
        }
    }
}

// Column mode of rys_contract (classes with C::COL): stage-2 thread `lane` < NC owns block
// column lane; per primitive quartet and root it loads the column's three 2-D table columns
// (3 (E+1) values) into registers and updates all NA row accumulators of the column
// (C::col_update, generated with literal indices), so shared memory is read 3(E+1) times per
// root instead of 3 times per block entry.
template <class C, bool F32>
__device__ __forceinline__ void rys_contract_col(const PairTab &P, const RysTab &R, const int4 ib,
                                                 const int4 ik, int i0, int i1, int j0, int j1,
                                                 double *__restrict__ work, const uint16_t *__restrict__ colpow,
                                                 int lane, int gid) {
    constexpr int S = C::S, F1 = C::F + 1, NR = C::NR, E = C::E, NA = C::NA, NC = C::NC;
    using TT = typename std::conditional<F32, float, double>::type;
    TT *__restrict__ tabs = reinterpret_cast<TT *>(work);
    double acc[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) acc[a] = 0.0;
    int cx = 0, cy = 0, cz = 0;
    if (lane < NC) {
        const unsigned cp = __ldg(&colpow[lane]);
        cx = cp & 15u;
        cy = (cp >> 4) & 15u;
        cz = cp >> 8;
    }
    const int nbp = i1 - i0, nq = nbp * (j1 - j0);
    const int tb = lane / NR, tr = lane - tb * NR;
    for (int g0 = 0; g0 < nq; g0 += C::NPB) {
        const int nb = min(C::NPB, nq - g0);
        rys_stage1<C, TT>(P, R, ib, ik, i0, j0, nbp, g0, nb, tb, tr, tabs);
        group_sync<C::G>(gid);
        if (lane < NC) {
            TT bacc[F32 ? NA : 1];
            if constexpr (F32) {
#pragma unroll
                for (int a = 0; a < NA; ++a) bacc[a] = (TT)0;
            }
            for (int b = 0; b < nb; ++b) {
#pragma unroll 1
                for (int r = 0; r < NR; ++r) {
                    const TT *__restrict__ t0 = tabs + (b * NR + r) * 3 * S;
                    TT x[E + 1], y[E + 1], z[E + 1];
#pragma unroll
                    for (int a = 0; a <= E; ++a) {
                        x[a] = t0[a * F1 + cx];
                        y[a] = t0[S + a * F1 + cy];
                        z[a] = t0[2 * S + a * F1 + cz];
                    }
                    if constexpr (F32) C::col_update(x, y, z, bacc);
                    else C::col_update(x, y, z, acc);
                }
            }
            if constexpr (F32) {
#pragma unroll
                for (int a = 0; a < NA; ++a) acc[a] += (double)bacc[a];
            }
        }
        group_sync<C::G>(gid);
    }
    if (lane < NC) {
#pragma unroll
        for (int a = 0; a < NA; ++a) work[a * NC + lane] = acc[a];
    }
    group_sync<C::G>(gid);
}

// The contracted [e0|f0] block of bra pair ib (primitive pairs [i0, i1)) and ket pair ik
// ([j0, j1)) into work[0 .. NBLK).  All G threads of the group call it; it ends with a barrier.
// F32 (MIXED quartets below the FP32 cutoff): the 2-D tables are stored in FP32 and a batch's
// products are summed in FP32, then added to the FP64 accumulators (roots, weights and the
// recurrences stay FP64).
template <class C, bool F32 = false>
__device__ __forceinline__ void rys_contract(const PairTab &P, const RysTab &R, const RysClassTabs &T,
                                             const int4 ib, const int4 ik, int i0, int i1, int j0,
                                             int j1, double *__restrict__ work, int lane, int gid) {
    constexpr int S = C::S, F1 = C::F + 1, NR = C::NR, E = C::E, F = C::F;
    constexpr int NSLOT = C::NSLOT;
    using TT = typename std::conditional<F32, float, double>::type;
    TT *__restrict__ tabs = reinterpret_cast<TT *>(work);
    if constexpr (C::COL) {
        rys_contract_col<C, F32>(P, R, ib, ik, i0, i1, j0, j1, work, T.col, lane, gid);
        return;
    }
    double acc[C::ACC];
    uint32_t off[C::ACC];
    // slot layout (NSLOT > 1): thread = slot * NBLK + entry, ACC == 1
    const int slot = NSLOT > 1 ? lane / C::NBLK : 0;
#pragma unroll
    for (int k = 0; k < C::ACC; ++k) {
        acc[k] = 0.0;
        const int e = NSLOT > 1 ? lane - slot * C::NBLK : lane + k * C::G;
        off[k] = (e < C::NBLK && slot < NSLOT) ? __ldg(&T.blk[e]) : 0u;
    }
    const int nbp = i1 - i0, nq = nbp * (j1 - j0);
    const int tb = lane / NR, tr = lane - tb * NR;
    for (int g0 = 0; g0 < nq; g0 += C::NPB) {
        const int nb = min(C::NPB, nq - g0);
        rys_stage1<C, TT>(P, R, ib, ik, i0, j0, nbp, g0, nb, tb, tr, tabs);
        group_sync<C::G>(gid);
        if (slot < NSLOT) {
            if constexpr (F32) {
                // the batch's products summed in FP32, then added to the FP64 accumulators
                float bacc[C::ACC];
#pragma unroll
                for (int k = 0; k < C::ACC; ++k) bacc[k] = 0.0f;
                for (int b = slot; b < nb; b += NSLOT) {
#pragma unroll 1
                    for (int r = 0; r < NR; ++r) {
                        const TT *__restrict__ tx = tabs + (b * NR + r) * 3 * S;
#pragma unroll
                        for (int k = 0; k < C::ACC; ++k) {
                            const uint32_t o = off[k];
                            bacc[k] = fmaf(tx[o & 255u] * tx[S + ((o >> 8) & 255u)], tx[2 * S + (o >> 16)], bacc[k]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < C::ACC; ++k) acc[k] += (double)bacc[k];
            } else {
                for (int b = slot; b < nb; b += NSLOT) {
#pragma unroll 1
                    for (int r = 0; r < NR; ++r) {
                        const TT *__restrict__ tx = tabs + (b * NR + r) * 3 * S;
#pragma unroll
                        for (int k = 0; k < C::ACC; ++k) {
                            const uint32_t o = off[k];
                            acc[k] = fma(tx[o & 255u] * tx[S + ((o >> 8) & 255u)], tx[2 * S + (o >> 16)], acc[k]);
                        }
                    }
                }
            }
        }
        group_sync<C::G>(gid);
    }
    if constexpr (NSLOT > 1) {
        if (slot < NSLOT) work[lane] = acc[0];  // work[slot * NBLK + entry]
        group_sync<C::G>(gid);
        if (lane < C::NBLK) {
            double v = work[lane];
#pragma unroll
            for (int s2 = 1; s2 < NSLOT; ++s2) v += work[s2 * C::NBLK + lane];
            work[lane] = v;
        }
    } else {
#pragma unroll
        for (int k = 0; k < C::ACC; ++k) {
            const int e = lane + k * C::G;
            if (e < C::NBLK) work[e] = acc[k];
        }
    }
    group_sync<C::G>(gid);
}

// HRR of the contracted block blk[NA][NC] (shared) into the normalised (ab|cd): bra pass into
// mid[NAB][NC], barrier, ket pass; sink(r, s, value) gets output (r = ia*NB + ib,
// s = ic*ND + id).  DIAG: only the outputs s == r (the bound kernels, bra pair == ket pair).
template <class C, bool DIAG, class Sink>
__device__ __forceinline__ void rys_hrr(const RysClassTabs &T, const double *__restrict__ blk,
                                        double *__restrict__ mid, const double *__restrict__ mono,
                                        int lane, int gid, Sink &&sink) {
    for (int w = lane; w < C::NAB * C::NC; w += C::G) {
        const int r = w / C::NC, c = w - r * C::NC;
        const int t1 = __ldg(&T.bra_off[r + 1]);
        double v = 0.0;
        for (int t = __ldg(&T.bra_off[r]); t < t1; ++t) {
            const uint32_t x = __ldg(&T.bra_term[t]);
            v = fma((double)(x >> 16) * mono[(x >> 8) & 255u], blk[(x & 255u) * C::NC + c], v);
        }
        mid[w] = v;
    }
    group_sync<C::G>(gid);
    const double *__restrict__ mcd = mono + kRysNmono;
    if constexpr (DIAG) {
        for (int r = lane; r < C::NAB; r += C::G) {
            const int t1 = __ldg(&T.ket_off[r + 1]);
            double v = 0.0;
            for (int t = __ldg(&T.ket_off[r]); t < t1; ++t) {
                const uint32_t x = __ldg(&T.ket_term[t]);
                v = fma((double)(x >> 16) * mcd[(x >> 8) & 255u], mid[r * C::NC + (x & 255u)], v);
            }
            sink(r, r, v * __ldg(&T.norm_ab[r]) * __ldg(&T.norm_cd[r]));
        }
    } else {
        for (int w = lane; w < C::NAB * C::NCD; w += C::G) {
            const int s = w / C::NAB, r = w - s * C::NAB;
            const int t1 = __ldg(&T.ket_off[s + 1]);
            double v = 0.0;
            for (int t = __ldg(&T.ket_off[s]); t < t1; ++t) {
                const uint32_t x = __ldg(&T.ket_term[t]);
                v = fma((double)(x >> 16) * mcd[(x >> 8) & 255u], mid[r * C::NC + (x & 255u)], v);
            }
            sink(r, s, v * __ldg(&T.norm_ab[r]) * __ldg(&T.norm_cd[s]));
        }
    }
}

// Persistent work-queue kernel body: each group takes chunks (one bra pair, a run of ket pairs
// of one molecule) from the class pair's counter and computes their quartets one by one.
template <class C, int MIXED = 0>
__device__ __forceinline__ void rys_queue_body(const EriQueue &Q, const RysTab &R, const RysClassTabs &T) {
    extern __shared__ __align__(16) double rys_smem[];
    __shared__ int s_chunk[128 / C::G];
    const int gid = threadIdx.x / C::G, lane = threadIdx.x - gid * C::G;
    double *mono = rys_smem + gid * C::SMEM_GROUP;
    double *work = mono + 2 * kRysNmono;
    for (;;) {
        if (lane == 0) s_chunk[gid] = atomicAdd(Q.counter, 1);
        group_sync<C::G>(gid);
        const int c = s_chunk[gid];
        group_sync<C::G>(gid);
        if (c >= Q.nchunks) return;
        const int4 ch = __ldg(&Q.chunks[c]);
        double *__restrict__ out = Q.out + __ldg(&Q.mol_out[ch.w]);
        const int p = ch.x;
        const int4 ib = __ldg(&Q.pairs.info[p]);
        const double2 bp = __ldg(&Q.pairs.bnd[p]);
        const double4 gb = ldg4(&Q.pairs.geo[p]);
        for (int q = ch.y; q < ch.y + ch.z; ++q) {
            const int4 ik = __ldg(&Q.pairs.info[q]);
            const double2 bq = __ldg(&Q.pairs.bnd[q]);
            const int nbp = (bp.x * bq.x < Q.screen_cut) ? 0 : ib.y;  // screened: written as 0
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                rys_contract<C, true>(Q.pairs, R, T, ib, ik, 0, nbp, 0, ik.y, work, lane, gid);
            else
                rys_contract<C, false>(Q.pairs, R, T, ib, ik, 0, nbp, 0, ik.y, work, lane, gid);
            const double4 gk = ldg4(&Q.pairs.geo[q]);
            for (int m = lane; m < 2 * kRysNmono; m += C::G)
                mono[m] = m < kRysNmono ? rys_monomial(m, gb.x, gb.y, gb.z)
                                        : rys_monomial(m - kRysNmono, gk.x, gk.y, gk.z);
            group_sync<C::G>(gid);
            const bool dab = ib.z == ib.w, dcd = ik.z == ik.w, same = p == q;
            // two-phase output: the quartet's whole block, (bra component, ket component) row-major
            double *__restrict__ blk = (Q.scratch && !Q.jk.J)
                ? Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                      (__ldg(&Q.chunk_slot[c]) + (q - ch.y)) * (long long)(C::NAB * C::NCD)
                : nullptr;
            rys_hrr<C, false>(T, work, work + C::NBLK, mono, lane, gid, [&](int r, int s, double v) {
                if (blk) { blk[r * C::NCD + s] = v; return; }
                const int ia = r / C::NB, jb = r - ia * C::NB, ic = s / C::ND, jd = s - ic * C::ND;
                if ((dab && ia < jb) || (dcd && ic < jd)) return;
                const long long ij = pair_index(ib.z + ia, ib.w + jb), kl = pair_index(ik.z + ic, ik.w + jd);
                if (same && ij < kl) return;
                if (Q.jk.J) jk_add(Q.jk, ib.z + ia, ib.w + jb, ik.z + ic, ik.w + jd, v);
                else out[packed_index(ij, kl)] = v;
            });
            group_sync<C::G>(gid);
        }
    }
}

// Bounds of the pairs [p0, p0+np) of a pair class (bra class == ket class), one group per pair:
// full == 0: for every primitive pair k, from the diagonal primitive quartet,
//   pbound[k] = {sqrt(max |(a_k b_k|a_k b_k)|), sqrt(max |[e0|e0]_kk|)};
// full != 0: the contracted Q_p = sqrt(max |(ab|ab)|) into qout[p].
template <class C>
__device__ __forceinline__ void rys_bound_body(const PairTab &P, const RysTab &R, const RysClassTabs &T,
                                               int p0, int np, double2 *pbound, double *qout, int full) {
    extern __shared__ __align__(16) double rys_smem[];
    __shared__ double s_red[4];
    constexpr int NG = 128 / C::G;
    const int gid = threadIdx.x / C::G, lane = threadIdx.x - gid * C::G;
    const int t = blockIdx.x * NG + gid;
    if (t >= np) return;
    double *mono = rys_smem + gid * C::SMEM_GROUP;
    double *work = mono + 2 * kRysNmono;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    const double4 g = ldg4(&P.geo[p]);
    for (int m = lane; m < 2 * kRysNmono; m += C::G) mono[m] = rys_monomial(m % kRysNmono, g.x, g.y, g.z);
    const int nk = full ? 1 : in.y;
    for (int k = 0; k < nk; ++k) {
        const int i0 = full ? 0 : k, i1 = full ? in.y : k + 1;
        rys_contract<C>(P, R, T, in, in, i0, i1, i0, i1, work, lane, gid);
        double wmax = 0.0, m = 0.0;
        for (int a = lane; a < C::NA; a += C::G) wmax = fmax(wmax, fabs(work[a * C::NC + a]));
        rys_hrr<C, true>(T, work, work + C::NBLK, mono, lane, gid,
                         [&](int, int, double v) { m = fmax(m, fabs(v)); });
        m = group_max<C::G>(m, s_red, gid);
        wmax = group_max<C::G>(wmax, s_red, gid);
        if (lane == 0) {
            if (full) qout[p] = sqrt(m);
            else pbound[in.x + k] = make_double2(sqrt(m), sqrt(wmax));
        }
        group_sync<C::G>(gid);
    }
}

}  // namespace molints

// Generated by gen_eri.py -- class (ss|ss).  Do not edit.
// VRR entries: 1, contracted block: 1, HRR lines: 0, outputs: 1.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[1], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_ssss(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 1; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[1];
            boys_fm<0>(T, B, F);
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
            const VT v0_0_0 = (VT)(pref * F[0]);
            acc[0] += (double)v0_0_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[1] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_ssss(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;

    res[0] = acc[0];
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[1]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_ssss(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[1];
    vrr_ssss<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 1; ++x) acc_out[x] = acc[x];
    }
    hrr_ssss(P, p, q, acc, res);
}

__device__ __forceinline__ void store_ssss(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
    const long long ij_0_0 = pair_index(ib_.z + 0, ib_.w + 0);
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_ssss(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 1; ++x) {
        const int ia = x / 1, ibb = (x / 1) % 1, ic = (x / 1) % 1, id = x % 1;
        if ((dab && ia < ibb) || (dcd && ic < id)) continue;
        const int i = ib_.z + ia, j = ib_.w + ibb, k = ik_.z + ic, l = ik_.w + id;
        if (same && pair_index(i, j) < pair_index(k, l)) continue;
        jk_add(jk, i, j, k, l, res[x]);
    }
}

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
__global__ void __launch_bounds__(128) eri_queue_ssss(const EriQueue Q) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int c = 0;
        if (lane == 0) c = atomicAdd(Q.counter, 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= Q.nchunks) return;
        const int4 ch = __ldg(&Q.chunks[c]);
        const int p = ch.x, cnt = ch.z & 0xffff, lg = (ch.z >> 16) & 7, lgj = (ch.z >> 20) & 7;
        const int W = 32 >> lg, kq = lane & (W - 1), s = lane >> (5 - lg);
        const int js = s & ((1 << lgj) - 1), is = s >> lgj;
        for (int base = 0; base < cnt; base += W) {
        const int q = ch.y + base + kq;
        const bool live = base + kq < cnt;
        double acc[1];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 1; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_ssss<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_ssss<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 1; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 1 doubles (launch_eri_ssss)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 1);
            if (lead) hrr_ssss(Q.pairs, p, q, acc, sb + kq * 1);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)1;
            for (int t = lane; t < nlive * 1; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[1];
            hrr_ssss(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_ssss(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_ssss(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_ssss(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 1024 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 1024 : 0;
    (void)mixed;  // no FP32 variant for this class (MIXED_MIN_VRR)
    if (Q.jk.J) eri_queue_ssss<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_ssss<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_ssss(int mixed) {

    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_ssss<0, 0>, 128, 0);
    return n;
}

// Bounds of the pairs of one class.
// full == 0 (plan set-up): for every primitive pair k of pair p, from the diagonal primitive
//   quartet (a_k b_k | a_k b_k):
//     pbound[k].x = b_k = sqrt(max over components |(a_k b_k|a_k b_k)|)
//     pbound[k].y = w_k = sqrt(max over the VRR block |[e0|e0]_kk|), e = la..la+lb
//   By the Schwarz inequality b_k b_l bounds |(a_k b_k|c_l d_l)| and w_k w_l bounds every
//   entry of the VRR output block [e0|f0] that the HRR combines.
// full != 0: the contracted bound Q_p = sqrt(max |(ab|ab)|) into qout[p].
__global__ void __launch_bounds__(128) schwarz_kernel_ssss(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[1];
    if (full) {
        quartet_ssss<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
    m = fmax(m, fabs(res[0]));
        qout[p] = sqrt(m);
        return;
    }
    double acc[1];
    for (int k = 0; k < in.y; ++k) {
        quartet_ssss<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
    m = fmax(m, fabs(res[0]));
        w = fmax(w, fabs(acc[0]));
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }
}

void launch_schwarz_ssss(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    schwarz_kernel_ssss<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}

}  // namespace molints

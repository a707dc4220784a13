// eri_generic.cu -- the shell quartets with a g shell (l = 4): one thread block per contracted
// quartet, Rys quadrature with up to nine roots, any angular momentum up to (gg|gg).
//
// The generated class kernels cover every class pair up to (ff|ff).  The reference's tables stop
// at l = 4 (shell_indices, src/Basis.jl:269-279) and its Huzinaga driver, all_twoe_ints
// (src/ERI.jl:15-112), accepts such shells; this kernel is their drop-in.  It follows
// coulomb_rys (src/Rys.jl:46-83) per primitive quartet -- roots and weights at X = rho |PQ|^2,
// the 1-D integrals of Int1d/Recur (src/Rys.jl:86-125) and the binomial transfer of Shift
// (src/Rys.jl:128-135) -- with the contracted-function norms applied (the reference driver
// leaves them out), and the outputs accumulated over primitive quartets in FP64:
//
//   G(i, k) per axis and root, i <= la+lb, k <= lc+ld, from G(0,0) = 1 and
//     G(i+1, k) = C00 G(i, k) + i B10 G(i-1, k) + k B00 G(i, k-1)
//     G(i, k+1) = D00 G(i, k) + k B01 G(i, k-1) + i B00 G(i-1, k)
//   with u the root (t^2), B00 = u / 2(z+e), B10 = (1 - e u/(z+e)) / 2z,
//   B01 = (1 - z u/(z+e)) / 2e, C00 = PA + e (Q-P) u/(z+e), D00 = QC + z (P-Q) u/(z+e);
//   H(ia, ib, k) = sum_s C(ib, s) AB^(ib-s) G(ia+s, k)   (bra transfer, AB = A - B);
//   I(ia, ib, ic, id) = sum_t C(id, t) CD^(id-t) H(ia, ib, ic+t);
//   (ab|cd) += c_a c_b c_c c_d 2 pi^(5/2) / (z e sqrt(z+e)) exp(-ab/z AB^2 - cd/e CD^2)
//              sum_r W_r Ix Iy Iz.
//
// The block walks its outputs in tiles of kGenTile (a register accumulator per thread and output
// of the tile) and, per tile, every primitive quartet.  Quartets with a g shell are rare in the
// basis sets the engine serves; this kernel is written for generality, not speed.
#include <cuda_runtime.h>

#include "../../include/molints.h"
#include "eri_common.cuh"

namespace molints {

constexpr int kGenThreads = 256;
constexpr int kGenAcc = 4;                        // outputs per thread and tile
constexpr int kGenTile = kGenThreads * kGenAcc;   // outputs per tile
constexpr int kGenL = 4;                          // highest shell angular momentum
constexpr int kGenE = 2 * kGenL;                  // la + lb
constexpr int kGenNr = 2 * kGenL + 1;             // roots: (4 kGenL) / 2 + 1
constexpr int kGenRysXmax = 100;
constexpr int kGenNcheb = 16;

// Cartesian components of l = 0..4 in the reference's shell_indices order, flat (35 entries):
// x | y << 4 | z << 8, those of shell l starting at c_gen_comp_off[l].
__constant__ unsigned short c_gen_comp[35] = {0x0, 0x1, 0x10, 0x100, 0x2, 0x11, 0x101, 0x20, 0x110, 0x200, 0x3, 0x12, 0x102, 0x21, 0x201, 0x111, 0x30, 0x120, 0x210, 0x300, 0x4, 0x13, 0x103, 0x22, 0x112, 0x202, 0x31, 0x121, 0x211, 0x301, 0x40, 0x130, 0x220, 0x310, 0x400};
// 1/sqrt((2I-1)!!(2J-1)!!(2K-1)!!) of each component
__constant__ double c_gen_norm[35] = {0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.279a74590331dp-1, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.279a74590331dp-1, 0x1.0000000000000p+0, 0x1.279a74590331dp-1, 0x1.08654a2d4f6dap-2, 0x1.279a74590331dp-1, 0x1.279a74590331dp-1, 0x1.279a74590331dp-1, 0x1.279a74590331dp-1, 0x1.0000000000000p+0, 0x1.08654a2d4f6dap-2, 0x1.279a74590331dp-1, 0x1.279a74590331dp-1, 0x1.08654a2d4f6dap-2, 0x1.8fba8a1bf6f97p-4, 0x1.08654a2d4f6dap-2, 0x1.08654a2d4f6dap-2, 0x1.5555555555555p-2, 0x1.279a74590331dp-1, 0x1.5555555555555p-2, 0x1.08654a2d4f6dap-2, 0x1.279a74590331dp-1, 0x1.279a74590331dp-1, 0x1.08654a2d4f6dap-2, 0x1.8fba8a1bf6f97p-4, 0x1.08654a2d4f6dap-2, 0x1.5555555555555p-2, 0x1.08654a2d4f6dap-2, 0x1.8fba8a1bf6f97p-4};
__constant__ int c_gen_comp_off[kGenL + 2] = {0, 1, 4, 10, 20, 35};

// The per-quartet work of the generic kernel.
struct GenQuartets {
    const int4 *quartet;          // global shells (I, J, K, L), reference order
    const int *mol;               // molecule of each quartet
    long long n;
    const double *xyz;            // shells: centre
    const int *L, *nprim, *poff, *fn_off;  // angular momentum, primitives, first function in molecule
    const double *expn, *ncoef;   // primitive exponents, normalised coefficients
    const long long *mol_out;     // packed offset of each molecule
    double *out;
    RysTab rys;
};

// Node u_r and weight W_r of the n-point Rys rule at X (the tables of rys_root<NR> in
// rys_common.cuh, n a run-time value).
__device__ __forceinline__ double gen_clenshaw(const double *__restrict__ c, double s) {
    double b1 = 0.0, b2 = 0.0;
    for (int k = kGenNcheb - 1; k >= 1; --k) {
        const double t = fma(2.0 * s, b1, __ldg(c + k) - b2);
        b2 = b1;
        b1 = t;
    }
    return fma(s, b1, __ldg(c) - b2);
}

__device__ void gen_root(const RysTab &R, int n, double X, int r, double &u, double &w) {
    if (X < (double)kGenRysXmax) {
        const int j = (int)X;
        const double s = 2.0 * (X - (double)j) - 1.0;
        const double *c = R.cheb + (size_t)kGenRysXmax * kGenNcheb * n * (n - 1) +
                          ((size_t)j * 2 * n + r) * kGenNcheb;
        u = gen_clenshaw(c, s);
        w = gen_clenshaw(c + (size_t)n * kGenNcheb, s);
    } else {
        const int o = n * (n - 1) / 2 + r;
        const double ox = 1.0 / X;
        u = __ldg(R.herm_x2 + o) * ox;
        w = __ldg(R.herm_w + o) * sqrt(ox);
    }
}

__device__ __forceinline__ double gen_binom(int n, int k) {
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (double)(n - k + i) / (double)i;
    return r;
}

__global__ void __launch_bounds__(kGenThreads) eri_generic_kernel(const GenQuartets Gq) {
    // one root at a time, per axis: G[(E+1)(F+1)] then H[(la+1)(lb+1)(F+1)]
    __shared__ double sG[3][(kGenE + 1) * (kGenE + 1)];
    __shared__ double sH[3][(kGenL + 1) * (kGenL + 1) * (kGenE + 1)];
    __shared__ double sRoot[kGenNr], sW[kGenNr];
    __shared__ double sPar[16];
    const int tid = threadIdx.x;
    for (long long qi = blockIdx.x; qi < Gq.n; qi += gridDim.x) {
        const int4 q = __ldg(&Gq.quartet[qi]);
        const int sh[4] = {q.x, q.y, q.z, q.w};
        int l[4], np[4], po[4], fo[4];
        double X0[4][3];
        for (int t = 0; t < 4; ++t) {
            l[t] = __ldg(&Gq.L[sh[t]]);
            np[t] = __ldg(&Gq.nprim[sh[t]]);
            po[t] = __ldg(&Gq.poff[sh[t]]);
            fo[t] = __ldg(&Gq.fn_off[sh[t]]);
            for (int k = 0; k < 3; ++k) X0[t][k] = __ldg(&Gq.xyz[3 * sh[t] + k]);
        }
        const int nc[4] = {(l[0] + 1) * (l[0] + 2) / 2, (l[1] + 1) * (l[1] + 2) / 2,
                           (l[2] + 1) * (l[2] + 2) / 2, (l[3] + 1) * (l[3] + 2) / 2};
        const int E = l[0] + l[1], F = l[2] + l[3], nr = (E + F) / 2 + 1;
        const int nout = nc[0] * nc[1] * nc[2] * nc[3];
        const int F1 = F + 1, HS = (l[0] + 1) * (l[1] + 1) * F1;
        double AB[3], CD[3], ab2 = 0.0, cd2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            AB[k] = X0[0][k] - X0[1][k];
            CD[k] = X0[2][k] - X0[3][k];
            ab2 += AB[k] * AB[k];
            cd2 += CD[k] * CD[k];
        }
        const bool same_ab = q.x == q.y, same_cd = q.z == q.w, same_pq = q.x == q.z && q.y == q.w;
        const long long obase = __ldg(&Gq.mol_out[__ldg(&Gq.mol[qi])]);
        for (int t0 = 0; t0 < nout; t0 += kGenTile) {
            double acc[kGenAcc];
            for (int j = 0; j < kGenAcc; ++j) acc[j] = 0.0;
            for (int pa = 0; pa < np[0]; ++pa)
                for (int pb = 0; pb < np[1]; ++pb)
                    for (int pc = 0; pc < np[2]; ++pc)
                        for (int pd = 0; pd < np[3]; ++pd) {
                            __syncthreads();  // the previous primitive quartet's readers are done
                            if (tid == 0) {
                                const double a = __ldg(&Gq.expn[po[0] + pa]), b = __ldg(&Gq.expn[po[1] + pb]);
                                const double c = __ldg(&Gq.expn[po[2] + pc]), d = __ldg(&Gq.expn[po[3] + pd]);
                                const double z = a + b, e = c + d, ze = z + e;
                                double P[3], Q[3], pq2 = 0.0;
                                for (int k = 0; k < 3; ++k) {
                                    P[k] = (a * X0[0][k] + b * X0[1][k]) / z;
                                    Q[k] = (c * X0[2][k] + d * X0[3][k]) / e;
                                    pq2 += (P[k] - Q[k]) * (P[k] - Q[k]);
                                }
                                const double coef = __ldg(&Gq.ncoef[po[0] + pa]) * __ldg(&Gq.ncoef[po[1] + pb]) *
                                                    __ldg(&Gq.ncoef[po[2] + pc]) * __ldg(&Gq.ncoef[po[3] + pd]);
                                sPar[0] = 2.0 * 17.493418327624862 /* pi^2.5 */ / (z * e * sqrt(ze)) *
                                          exp(-a * b / z * ab2 - c * d / e * cd2) * coef;
                                sPar[1] = z * e / ze * pq2;  // X
                                sPar[2] = z;
                                sPar[3] = e;
                                for (int k = 0; k < 3; ++k) {
                                    sPar[4 + k] = P[k] - X0[0][k];      // PA
                                    sPar[7 + k] = Q[k] - X0[2][k];      // QC
                                    sPar[10 + k] = Q[k] - P[k];         // Q - P
                                }
                            }
                            __syncthreads();
                            if (tid < nr) gen_root(Gq.rys, nr, sPar[1], tid, sRoot[tid], sW[tid]);
                            __syncthreads();
                            const double pref = sPar[0];
                            for (int r = 0; r < nr; ++r) {
                                __syncthreads();  // the previous root's readers are done
                                if (tid < 3) {
                                    // G table of root r on axis tid, serially
                                    const int k = tid;
                                    const double u = sRoot[r], z = sPar[2], e = sPar[3], ze = z + e;
                                    const double B00 = 0.5 * u / ze, B10 = (1.0 - e * u / ze) / (2.0 * z),
                                                 B01 = (1.0 - z * u / ze) / (2.0 * e);
                                    const double C00 = sPar[4 + k] + e * sPar[10 + k] * u / ze;
                                    const double D00 = sPar[7 + k] - z * sPar[10 + k] * u / ze;
                                    double *g = sG[k];
                                    g[0] = 1.0;
                                    for (int i = 1; i <= E; ++i)
                                        g[i * F1] = C00 * g[(i - 1) * F1] + (i > 1 ? (i - 1) * B10 * g[(i - 2) * F1] : 0.0);
                                    for (int kk = 1; kk <= F; ++kk)
                                        for (int i = 0; i <= E; ++i) {
                                            double v = D00 * g[i * F1 + kk - 1];
                                            if (kk > 1) v += (kk - 1) * B01 * g[i * F1 + kk - 2];
                                            if (i > 0) v += i * B00 * g[(i - 1) * F1 + kk - 1];
                                            g[i * F1 + kk] = v;
                                        }
                                }
                                __syncthreads();
                                // bra transfer H(ia, ib, k) on every axis
                                for (int x = tid; x < 3 * HS; x += kGenThreads) {
                                    const int k = x / HS, h = x - k * HS;
                                    const int ia = h / ((l[1] + 1) * F1), rem = h - ia * (l[1] + 1) * F1;
                                    const int ib = rem / F1, kk = rem - ib * F1;
                                    double v = 0.0, p = 1.0;
                                    for (int s = ib; s >= 0; --s) {  // C(ib, s) AB^(ib - s) G(ia + s, kk)
                                        v += gen_binom(ib, s) * p * sG[k][(ia + s) * F1 + kk];
                                        p *= AB[k];
                                    }
                                    sH[k][h] = v;
                                }
                                __syncthreads();
                                const double wr = pref * sW[r];
                                for (int j = 0; j < kGenAcc; ++j) {
                                    const int o = t0 + j * kGenThreads + tid;
                                    if (o >= nout) break;
                                    const int id = o % nc[3], ic = (o / nc[3]) % nc[2],
                                              ib = (o / (nc[3] * nc[2])) % nc[1], ia = o / (nc[3] * nc[2] * nc[1]);
                                    const unsigned ca = c_gen_comp[c_gen_comp_off[l[0]] + ia],
                                                   cb = c_gen_comp[c_gen_comp_off[l[1]] + ib],
                                                   cc = c_gen_comp[c_gen_comp_off[l[2]] + ic],
                                                   cd = c_gen_comp[c_gen_comp_off[l[3]] + id];
                                    double prod = wr;
                                    for (int k = 0; k < 3; ++k) {
                                        const int ax = (ca >> (4 * k)) & 15, bx = (cb >> (4 * k)) & 15,
                                                  cx = (cc >> (4 * k)) & 15, dx = (cd >> (4 * k)) & 15;
                                        const double *h = sH[k] + (ax * (l[1] + 1) + bx) * F1;
                                        double v = 0.0, p = 1.0;
                                        for (int t = dx; t >= 0; --t) {  // C(dx, t) CD^(dx - t) H(.., cx + t)
                                            v += gen_binom(dx, t) * p * h[cx + t];
                                            p *= CD[k];
                                        }
                                        prod *= v;
                                    }
                                    acc[j] += prod;
                                }
                            }
                        }
            // the tile's unique integrals, normalised, at their iindex positions
            for (int j = 0; j < kGenAcc; ++j) {
                const int o = t0 + j * kGenThreads + tid;
                if (o >= nout) break;
                const int id = o % nc[3], ic = (o / nc[3]) % nc[2], ib = (o / (nc[3] * nc[2])) % nc[1],
                          ia = o / (nc[3] * nc[2] * nc[1]);
                const int i = fo[0] + ia, jj = fo[1] + ib, k = fo[2] + ic, ll = fo[3] + id;
                if ((same_ab && i < jj) || (same_cd && k < ll)) continue;
                const long long ij = pair_index(i, jj), kl = pair_index(k, ll);
                if (same_pq && ij < kl) continue;
                const double nrm = c_gen_norm[c_gen_comp_off[l[0]] + ia] * c_gen_norm[c_gen_comp_off[l[1]] + ib] *
                                   c_gen_norm[c_gen_comp_off[l[2]] + ic] * c_gen_norm[c_gen_comp_off[l[3]] + id];
                Gq.out[obase + packed_index(ij, kl)] = acc[j] * nrm;
            }
        }
    }
}

void launch_eri_generic(const GenQuartets &G, int grid, cudaStream_t s) {
    if (G.n <= 0 || grid <= 0) return;
    eri_generic_kernel<<<grid, kGenThreads, 0, s>>>(G);
}

}  // namespace molints

// eri_common.cuh -- device data layout and shared device functions of the ERI engine.
//
// Layout in HBM (all arrays are owned by a plan, see molints.cu):
//   * shell pairs, canonical orientation (L_A >= L_B), sorted by pair class and then by
//     contraction length; structure of arrays:
//       info[p] = {first primitive pair, number of primitive pairs, first function of A,
//                  first function of B}                      (int4, 16 B)
//       geo[p]  = {A-B (x,y,z), unused}                    (double4, 32 B)
//       bnd[p]  = {Qabs_p, R_p}: bounds for screening and for FP32 quartets (double2)
//   * primitive pairs, 80 B each (5 x 16 B vector loads): PrimPair below;
//   * the Boys table (T = 0..40 step 1/16, F_0..F_22 and e^-T per row);
//   * the packed output vector, 0-based iindex order (src/Utils.jl:14-19).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace molints {

constexpr int kBoysRows = 641;            // T_n = n/16, n = 0..640 (T up to 40)
constexpr int kBoysCols = 24;             // F_0..F_22 at T_n, then e^-T_n
constexpr int kBoysTaylor = 8;            // Taylor terms about T_n; |T - T_n| <= 1/32
constexpr double kBoysStepInv = 16.0;
constexpr double kBoysStep = 0.0625;
constexpr double kBoysTableMax = 40.0;    // exact-mode switch to the asymptotic form
constexpr int kBoysMaxM1 = 16;            // scaled tables exist for M = 0..15
constexpr int kBoysScaledCols = 10;       // F_{M+k}(T_n)/k! for k < 8, e^-T_n, pad (80 B)
constexpr double kBoysReferenceSwitch = 30.0;  // farray's Tmax, src/Boys.jl:19

// Record of one primitive pair (a, b) of a canonical shell pair (A, B):
//   zeta = a + b
//   kab  = sqrt(2) pi^(5/4) c_a c_b exp(-a b |A-B|^2 / zeta) / zeta, with c_a, c_b the
//          fully normalised contraction coefficients (radial primitive norm x CGBF norm)
//   oo2z = 1 / (2 zeta)
//   P    = (a A + b B) / zeta (gaussian_product_center, src/OneInts.jl:78-83)
//   PA   = P - A
//   b    = sqrt(max |(ab|ab)|) of this primitive pair (its Schwarz bound; 0 before the plan's
//          bound pass)
// so that kab_bra * kab_ket / sqrt(zeta+eta) is the [00|00] prefactor of HGP eq. 12,
// 2 pi^(5/2) / (zeta eta sqrt(zeta+eta)) x exp(...) x coefficients.
struct PrimPair {
    double zeta, kab, oo2z, px, py, pz, pax, pay, paz, b;
};
static_assert(sizeof(PrimPair) == 80, "PrimPair is 5 x 16 bytes");

struct PairTab {
    const int4 *info;
    const double4 *geo;   // A - B (w unused)
    const PrimPair *pp;
    const double2 *bnd;   // x: Qabs_p = sum_k b_k, y: R_p = (1+|AB|)^lb sum_k w_k (kept prims)
};

struct BoysTab {
    const double *tab;     // [kBoysRows][kBoysCols]: F_0..F_22, e^-T_n
    const double *scaled;  // [kBoysMaxM1][kBoysRows][kBoysScaledCols]
    double t_switch;       // asymptotic form at T >= t_switch
};

// Rys quadrature tables (generated/rys_tables.cu): for n = 1..7 roots, Chebyshev series of
// the nodes u_i = t_i^2 and weights W_i on unit intervals of X < 100, and the Gauss-Hermite
// limits x_i = h_i^2 / X, W_i = g_i / sqrt(X) above.
struct RysTab {
    const double *cheb;     // [n][interval j < 100][2n functions][16 coefficients]
    const double *herm_x2;  // h_i^2 of the 2n-point Gauss-Hermite rule, n at n(n-1)/2
    const double *herm_w;   // g_i, same layout
};
int rys_tables(RysTab *t);  // device addresses on the current device; 0 on success

// Coulomb and exchange digestion (molints_plan_jk): J_pq = sum_rs D_rs (pq|rs) and
// K_pr = sum_qs D_qs (pq|rs), full n x n row-major, accumulated with FP64 atomics.
struct JKOut {
    const double *D;   // symmetric density, n x n
    double *J, *K;     // zeroed before the execute
    int n;
};

// The chunk queue of one class pair: chunk c = {bra pair, first ket pair, ket count |
// split << 16, molecule}.  HGP: split = lg | lgj << 4, S = 2^lg lanes share each quartet and
// lane l of the warp that takes the chunk computes its share of (bra | first + l % (32/S) +
// (32/S) i), the ket primitives split over 2^lgj lanes and the bra primitives over the rest
// (split 0: one lane per quartet).  Rys chunks have split 0.  Chunks never cross a bra pair, a
// molecule or, when bra and ket class coincide, the triangle q <= p.
struct EriQueue {
    PairTab pairs;
    BoysTab boys;
    JKOut jk;                     // jk.J != nullptr: digest into J and K instead of storing
    double *out;                  // packed outputs of all molecules (device)
    const long long *mol_out;     // offset of each molecule's packed vector in out
    const int4 *chunks;
    int nchunks;
    int *counter;                 // next chunk; zero at launch
    double screen_cut;            // Qabs_p Qabs_q below this: written as 0
    double fp32_cut;              // R_p R_q below this (MIXED kernels): FP32 VRR
    // two-phase output (scratch != nullptr): quartet (p, q0 + t) of chunk c (molecule m = its
    // w field) has slot u = chunk_slot[c] + t of its class pair's region for molecule m,
    // region[m * kRegionFields ..] = {offset, first bra, first ket, kets}: its whole block
    // (ma, mb, mc, md row-major) goes to scratch[offset + u * block size].  A gather pass
    // writes the packed vector from the scratch afterwards.
    double *scratch;
    const long long *chunk_slot;
    const long long *region;
};
constexpr int kRegionFields = 4;

__device__ __forceinline__ PrimPair load_pp(const PrimPair *__restrict__ base, int k) {
    const double2 *v = reinterpret_cast<const double2 *>(base + k);
    const double2 a = __ldg(v), b = __ldg(v + 1), c = __ldg(v + 2), d = __ldg(v + 3),
                  e = __ldg(v + 4);
    PrimPair r;
    r.zeta = a.x; r.kab = a.y; r.oo2z = b.x; r.px = b.y; r.py = c.x; r.pz = c.y;
    r.pax = d.x; r.pay = d.y; r.paz = e.x; r.b = e.y;
    return r;
}

// F_0..F_M at T: the farray structure of src/Boys.jl:19-27.
//   T <  t_switch: F_M by an 8-term Taylor expansion about the nearest table point,
//                  F_M(T_n - d) = sum_k [F_{M+k}(T_n)/k!] d^k (the table row of M holds the
//                  bracketed coefficients, so this is 7 FMAs), e^-T = e^-T_n e^d, then the
//                  downward recursion F_m = (2T F_{m+1} + e^-T) / (2m+1).
//   T >= t_switch: the asymptotic family F_m = (2m-1)!! / (2T)^m * sqrt(pi/T)/2, the values
//                  farray's Fm_asymp top order and e^-T-free recursion produce.
// The table index is rounded with the 1.5*2^52 trick: T*16 + 1.5*2^52 holds round(T*16) in
// its low mantissa bits, and subtracting the constant back gives T_n*16 exactly.
template <int M>
__device__ __forceinline__ void boys_fm(double T, const BoysTab &bt, double *F) {
    static_assert(M < kBoysMaxM1, "Boys order beyond the scaled tables");
    if (T < bt.t_switch) {
        constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52
        const double t16 = fma(T, kBoysStepInv, kMagic);
        const int n = __double2loint(t16);
        const double d = fma(t16 - kMagic, kBoysStep, -T);
        const double2 *__restrict__ r2 = reinterpret_cast<const double2 *>(
            bt.scaled + ((size_t)M * kBoysRows + n) * kBoysScaledCols);
        const double2 c01 = __ldg(r2), c23 = __ldg(r2 + 1), c45 = __ldg(r2 + 2), c67 = __ldg(r2 + 3);
        double f = fma(c67.y, d, c67.x);
        f = fma(f, d, c45.y);
        f = fma(f, d, c45.x);
        f = fma(f, d, c23.y);
        f = fma(f, d, c23.x);
        f = fma(f, d, c01.y);
        f = fma(f, d, c01.x);
        F[M] = f;
        if (M > 0) {
            const double emtn = __ldg(r2 + 4).x;
            // e^d for |d| <= 1/32 by its Taylor polynomial to d^7
            double ed = fma(d, 1.0 / 5040, 1.0 / 720);
            ed = fma(ed, d, 1.0 / 120);
            ed = fma(ed, d, 1.0 / 24);
            ed = fma(ed, d, 1.0 / 6);
            ed = fma(ed, d, 0.5);
            ed = fma(ed, d, 1.0);
            ed = fma(ed, d, 1.0);
            const double emt = emtn * ed;
            const double t2 = 2.0 * T;
#pragma unroll
            for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], emt) * (1.0 / (2 * m + 1));
        }
    } else {
        const double r = rsqrt(T);
        F[0] = 0.88622692545275801365 * r;  // sqrt(pi)/2
        const double oo2t = 0.5 * r * r;
#pragma unroll
        for (int m = 1; m <= M; ++m) F[m] = F[m - 1] * ((2 * m - 1) * oo2t);
    }
}

__device__ __forceinline__ double4 ldg4(const double4 *p) {
    const double2 *v = reinterpret_cast<const double2 *>(p);
    const double2 a = __ldg(v), b = __ldg(v + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ long long tri_ll(long long i) { return i * (i + 1) / 2; }

// One unique integral v = (ij|kl) into J and K: every distinct index permutation (pq|rs) of
// the 8-fold symmetry adds D_rs v to J_pq and D_qs v to K_pr (the Fock-build contraction that
// make2JmK, src/ERI.jl:114-128, performs on the packed vector).  J and K are symmetric, so only
// the targets on or below the diagonal are accumulated (half the atomics); molints_plan_jk
// mirrors the lower triangles afterwards.
__device__ __forceinline__ void jk_add(const JKOut &jk, int i, int j, int k, int l, double v) {
    if (v == 0.0) return;
    if (i < j) { const int t = i; i = j; j = t; }
    if (k < l) { const int t = k; k = l; l = t; }
    const long long n = jk.n;
    const bool dij = i != j, dkl = k != l;
    const bool dbk = (tri_ll(i) + j) != (tri_ll(k) + l);
    const double *__restrict__ D = jk.D;
    // J: J_ij += (1 + [k != l]) D_kl v (i >= j); J_kl += (1 + [i != j]) D_ij v (k >= l)
    atomicAdd(&jk.J[i * n + j], (dkl ? 2.0 : 1.0) * __ldg(&D[k * n + l]) * v);
    if (dbk) atomicAdd(&jk.J[k * n + l], (dij ? 2.0 : 1.0) * __ldg(&D[i * n + j]) * v);
    // K: (pq|rs) -> K_pr += D_qs v over the distinct permutations, targets with p >= r only
    const int pq[2][2] = {{i, j}, {j, i}}, rs[2][2] = {{k, l}, {l, k}};
    for (int a = 0; a < (dij ? 2 : 1); ++a)
        for (int b = 0; b < (dkl ? 2 : 1); ++b) {
            const int p0 = pq[a][0], q0 = pq[a][1], r0 = rs[b][0], s0 = rs[b][1];
            if (p0 >= r0) atomicAdd(&jk.K[p0 * n + r0], __ldg(&D[q0 * n + s0]) * v);
            if (dbk && r0 >= p0) atomicAdd(&jk.K[r0 * n + p0], __ldg(&D[s0 * n + q0]) * v);
        }
}

// 0-based packed index of the function-pair indices ij, kl (iindex, src/Utils.jl:19).
__device__ __forceinline__ long long packed_index(long long ij, long long kl) {
    return ij >= kl ? tri_ll(ij) + kl : tri_ll(kl) + ij;
}
__device__ __forceinline__ long long pair_index(int i, int j) {
    return i >= j ? tri_ll(i) + j : tri_ll(j) + i;
}

}  // namespace molints

// Generated by gen_eri.py -- class (ds|ds).  Do not edit.
// VRR entries: 116, contracted block: 36, HRR lines: 0, outputs: 36.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[36], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_dsds(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 36; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[5];
            boys_fm<4>(T, B, F);
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
            const VT v0_0_1 = (VT)(pref * F[1]);
            const VT v0_0_2 = (VT)(pref * F[2]);
            const VT v0_0_3 = (VT)(pref * F[3]);
            const VT v0_0_4 = (VT)(pref * F[4]);
            const VT v1_0_0 = PAx * v0_0_0 + WPx * v0_0_1;
            const VT v1_0_1 = PAx * v0_0_1 + WPx * v0_0_2;
            const VT v1_0_2 = PAx * v0_0_2 + WPx * v0_0_3;
            const VT v1_0_3 = PAx * v0_0_3 + WPx * v0_0_4;
            const VT v2_0_0 = PAy * v0_0_0 + WPy * v0_0_1;
            const VT v2_0_1 = PAy * v0_0_1 + WPy * v0_0_2;
            const VT v2_0_2 = PAy * v0_0_2 + WPy * v0_0_3;
            const VT v2_0_3 = PAy * v0_0_3 + WPy * v0_0_4;
            const VT v3_0_0 = PAz * v0_0_0 + WPz * v0_0_1;
            const VT v3_0_1 = PAz * v0_0_1 + WPz * v0_0_2;
            const VT v3_0_2 = PAz * v0_0_2 + WPz * v0_0_3;
            const VT v3_0_3 = PAz * v0_0_3 + WPz * v0_0_4;
            const VT v4_0_0 = PAx * v1_0_0 + WPx * v1_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v4_0_1 = PAx * v1_0_1 + WPx * v1_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v4_0_2 = PAx * v1_0_2 + WPx * v1_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v5_0_0 = PAx * v2_0_0 + WPx * v2_0_1;
            const VT v5_0_1 = PAx * v2_0_1 + WPx * v2_0_2;
            const VT v5_0_2 = PAx * v2_0_2 + WPx * v2_0_3;
            const VT v6_0_0 = PAx * v3_0_0 + WPx * v3_0_1;
            const VT v6_0_1 = PAx * v3_0_1 + WPx * v3_0_2;
            const VT v6_0_2 = PAx * v3_0_2 + WPx * v3_0_3;
            const VT v7_0_0 = PAy * v2_0_0 + WPy * v2_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v7_0_1 = PAy * v2_0_1 + WPy * v2_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v7_0_2 = PAy * v2_0_2 + WPy * v2_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v8_0_0 = PAy * v3_0_0 + WPy * v3_0_1;
            const VT v8_0_1 = PAy * v3_0_1 + WPy * v3_0_2;
            const VT v8_0_2 = PAy * v3_0_2 + WPy * v3_0_3;
            const VT v9_0_0 = PAz * v3_0_0 + WPz * v3_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v9_0_1 = PAz * v3_0_1 + WPz * v3_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v9_0_2 = PAz * v3_0_2 + WPz * v3_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v1_1_1 = QCx * v1_0_1 + WQx * v1_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v2_1_1 = QCx * v2_0_1 + WQx * v2_0_2;
            const VT v3_1_1 = QCx * v3_0_1 + WQx * v3_0_2;
            const VT v4_1_0 = QCx * v4_0_0 + WQx * v4_0_1 + (VT)2.0 * oo2ze * v1_0_1;
            const VT v4_1_1 = QCx * v4_0_1 + WQx * v4_0_2 + (VT)2.0 * oo2ze * v1_0_2;
            const VT v5_1_0 = QCx * v5_0_0 + WQx * v5_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v5_1_1 = QCx * v5_0_1 + WQx * v5_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v6_1_0 = QCx * v6_0_0 + WQx * v6_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v6_1_1 = QCx * v6_0_1 + WQx * v6_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v7_1_0 = QCx * v7_0_0 + WQx * v7_0_1;
            const VT v7_1_1 = QCx * v7_0_1 + WQx * v7_0_2;
            const VT v8_1_0 = QCx * v8_0_0 + WQx * v8_0_1;
            const VT v8_1_1 = QCx * v8_0_1 + WQx * v8_0_2;
            const VT v9_1_0 = QCx * v9_0_0 + WQx * v9_0_1;
            const VT v9_1_1 = QCx * v9_0_1 + WQx * v9_0_2;
            const VT v1_2_1 = QCy * v1_0_1 + WQy * v1_0_2;
            const VT v2_2_1 = QCy * v2_0_1 + WQy * v2_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v3_2_1 = QCy * v3_0_1 + WQy * v3_0_2;
            const VT v4_2_0 = QCy * v4_0_0 + WQy * v4_0_1;
            const VT v4_2_1 = QCy * v4_0_1 + WQy * v4_0_2;
            const VT v5_2_0 = QCy * v5_0_0 + WQy * v5_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v5_2_1 = QCy * v5_0_1 + WQy * v5_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v6_2_0 = QCy * v6_0_0 + WQy * v6_0_1;
            const VT v6_2_1 = QCy * v6_0_1 + WQy * v6_0_2;
            const VT v7_2_0 = QCy * v7_0_0 + WQy * v7_0_1 + (VT)2.0 * oo2ze * v2_0_1;
            const VT v7_2_1 = QCy * v7_0_1 + WQy * v7_0_2 + (VT)2.0 * oo2ze * v2_0_2;
            const VT v8_2_0 = QCy * v8_0_0 + WQy * v8_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v8_2_1 = QCy * v8_0_1 + WQy * v8_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v9_2_0 = QCy * v9_0_0 + WQy * v9_0_1;
            const VT v9_2_1 = QCy * v9_0_1 + WQy * v9_0_2;
            const VT v1_3_1 = QCz * v1_0_1 + WQz * v1_0_2;
            const VT v2_3_1 = QCz * v2_0_1 + WQz * v2_0_2;
            const VT v3_3_1 = QCz * v3_0_1 + WQz * v3_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v4_3_0 = QCz * v4_0_0 + WQz * v4_0_1;
            const VT v4_3_1 = QCz * v4_0_1 + WQz * v4_0_2;
            const VT v5_3_0 = QCz * v5_0_0 + WQz * v5_0_1;
            const VT v5_3_1 = QCz * v5_0_1 + WQz * v5_0_2;
            const VT v6_3_0 = QCz * v6_0_0 + WQz * v6_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v6_3_1 = QCz * v6_0_1 + WQz * v6_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v7_3_0 = QCz * v7_0_0 + WQz * v7_0_1;
            const VT v7_3_1 = QCz * v7_0_1 + WQz * v7_0_2;
            const VT v8_3_0 = QCz * v8_0_0 + WQz * v8_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v8_3_1 = QCz * v8_0_1 + WQz * v8_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v9_3_0 = QCz * v9_0_0 + WQz * v9_0_1 + (VT)2.0 * oo2ze * v3_0_1;
            const VT v9_3_1 = QCz * v9_0_1 + WQz * v9_0_2 + (VT)2.0 * oo2ze * v3_0_2;
            const VT v4_4_0 = QCx * v4_1_0 + WQx * v4_1_1 + (VT)2.0 * oo2ze * v1_1_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v5_4_0 = QCx * v5_1_0 + WQx * v5_1_1 + (VT)1.0 * oo2ze * v2_1_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v6_4_0 = QCx * v6_1_0 + WQx * v6_1_1 + (VT)1.0 * oo2ze * v3_1_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v7_4_0 = QCx * v7_1_0 + WQx * v7_1_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v8_4_0 = QCx * v8_1_0 + WQx * v8_1_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v9_4_0 = QCx * v9_1_0 + WQx * v9_1_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v4_5_0 = QCx * v4_2_0 + WQx * v4_2_1 + (VT)2.0 * oo2ze * v1_2_1;
            const VT v5_5_0 = QCx * v5_2_0 + WQx * v5_2_1 + (VT)1.0 * oo2ze * v2_2_1;
            const VT v6_5_0 = QCx * v6_2_0 + WQx * v6_2_1 + (VT)1.0 * oo2ze * v3_2_1;
            const VT v7_5_0 = QCx * v7_2_0 + WQx * v7_2_1;
            const VT v8_5_0 = QCx * v8_2_0 + WQx * v8_2_1;
            const VT v9_5_0 = QCx * v9_2_0 + WQx * v9_2_1;
            const VT v4_6_0 = QCx * v4_3_0 + WQx * v4_3_1 + (VT)2.0 * oo2ze * v1_3_1;
            const VT v5_6_0 = QCx * v5_3_0 + WQx * v5_3_1 + (VT)1.0 * oo2ze * v2_3_1;
            const VT v6_6_0 = QCx * v6_3_0 + WQx * v6_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v7_6_0 = QCx * v7_3_0 + WQx * v7_3_1;
            const VT v8_6_0 = QCx * v8_3_0 + WQx * v8_3_1;
            const VT v9_6_0 = QCx * v9_3_0 + WQx * v9_3_1;
            const VT v4_7_0 = QCy * v4_2_0 + WQy * v4_2_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v5_7_0 = QCy * v5_2_0 + WQy * v5_2_1 + (VT)1.0 * oo2ze * v1_2_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v6_7_0 = QCy * v6_2_0 + WQy * v6_2_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v7_7_0 = QCy * v7_2_0 + WQy * v7_2_1 + (VT)2.0 * oo2ze * v2_2_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v8_7_0 = QCy * v8_2_0 + WQy * v8_2_1 + (VT)1.0 * oo2ze * v3_2_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v9_7_0 = QCy * v9_2_0 + WQy * v9_2_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v4_8_0 = QCy * v4_3_0 + WQy * v4_3_1;
            const VT v5_8_0 = QCy * v5_3_0 + WQy * v5_3_1 + (VT)1.0 * oo2ze * v1_3_1;
            const VT v6_8_0 = QCy * v6_3_0 + WQy * v6_3_1;
            const VT v7_8_0 = QCy * v7_3_0 + WQy * v7_3_1 + (VT)2.0 * oo2ze * v2_3_1;
            const VT v8_8_0 = QCy * v8_3_0 + WQy * v8_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v9_8_0 = QCy * v9_3_0 + WQy * v9_3_1;
            const VT v4_9_0 = QCz * v4_3_0 + WQz * v4_3_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v5_9_0 = QCz * v5_3_0 + WQz * v5_3_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v6_9_0 = QCz * v6_3_0 + WQz * v6_3_1 + (VT)1.0 * oo2ze * v1_3_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v7_9_0 = QCz * v7_3_0 + WQz * v7_3_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v8_9_0 = QCz * v8_3_0 + WQz * v8_3_1 + (VT)1.0 * oo2ze * v2_3_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v9_9_0 = QCz * v9_3_0 + WQz * v9_3_1 + (VT)2.0 * oo2ze * v3_3_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            acc[0] += (double)v4_4_0;
            acc[1] += (double)v4_5_0;
            acc[2] += (double)v4_6_0;
            acc[3] += (double)v4_7_0;
            acc[4] += (double)v4_8_0;
            acc[5] += (double)v4_9_0;
            acc[6] += (double)v5_4_0;
            acc[7] += (double)v5_5_0;
            acc[8] += (double)v5_6_0;
            acc[9] += (double)v5_7_0;
            acc[10] += (double)v5_8_0;
            acc[11] += (double)v5_9_0;
            acc[12] += (double)v6_4_0;
            acc[13] += (double)v6_5_0;
            acc[14] += (double)v6_6_0;
            acc[15] += (double)v6_7_0;
            acc[16] += (double)v6_8_0;
            acc[17] += (double)v6_9_0;
            acc[18] += (double)v7_4_0;
            acc[19] += (double)v7_5_0;
            acc[20] += (double)v7_6_0;
            acc[21] += (double)v7_7_0;
            acc[22] += (double)v7_8_0;
            acc[23] += (double)v7_9_0;
            acc[24] += (double)v8_4_0;
            acc[25] += (double)v8_5_0;
            acc[26] += (double)v8_6_0;
            acc[27] += (double)v8_7_0;
            acc[28] += (double)v8_8_0;
            acc[29] += (double)v8_9_0;
            acc[30] += (double)v9_4_0;
            acc[31] += (double)v9_5_0;
            acc[32] += (double)v9_6_0;
            acc[33] += (double)v9_7_0;
            acc[34] += (double)v9_8_0;
            acc[35] += (double)v9_9_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[36] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_dsds(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;

    res[0] = acc[0] * 0.3333333333333334;
    res[1] = acc[1] * 0.5773502691896258;
    res[2] = acc[2] * 0.5773502691896258;
    res[3] = acc[3] * 0.3333333333333334;
    res[4] = acc[4] * 0.5773502691896258;
    res[5] = acc[5] * 0.3333333333333334;
    res[6] = acc[6] * 0.5773502691896258;
    res[7] = acc[7];
    res[8] = acc[8];
    res[9] = acc[9] * 0.5773502691896258;
    res[10] = acc[10];
    res[11] = acc[11] * 0.5773502691896258;
    res[12] = acc[12] * 0.5773502691896258;
    res[13] = acc[13];
    res[14] = acc[14];
    res[15] = acc[15] * 0.5773502691896258;
    res[16] = acc[16];
    res[17] = acc[17] * 0.5773502691896258;
    res[18] = acc[18] * 0.3333333333333334;
    res[19] = acc[19] * 0.5773502691896258;
    res[20] = acc[20] * 0.5773502691896258;
    res[21] = acc[21] * 0.3333333333333334;
    res[22] = acc[22] * 0.5773502691896258;
    res[23] = acc[23] * 0.3333333333333334;
    res[24] = acc[24] * 0.5773502691896258;
    res[25] = acc[25];
    res[26] = acc[26];
    res[27] = acc[27] * 0.5773502691896258;
    res[28] = acc[28];
    res[29] = acc[29] * 0.5773502691896258;
    res[30] = acc[30] * 0.3333333333333334;
    res[31] = acc[31] * 0.5773502691896258;
    res[32] = acc[32] * 0.5773502691896258;
    res[33] = acc[33] * 0.3333333333333334;
    res[34] = acc[34] * 0.5773502691896258;
    res[35] = acc[35] * 0.3333333333333334;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[36]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_dsds(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[36];
    vrr_dsds<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 36; ++x) acc_out[x] = acc[x];
    }
    hrr_dsds(P, p, q, acc, res);
}

__device__ __forceinline__ void store_dsds(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
    const long long ij_0_0 = pair_index(ib_.z + 0, ib_.w + 0);
    const long long ij_1_0 = pair_index(ib_.z + 1, ib_.w + 0);
    const long long ij_2_0 = pair_index(ib_.z + 2, ib_.w + 0);
    const long long ij_3_0 = pair_index(ib_.z + 3, ib_.w + 0);
    const long long ij_4_0 = pair_index(ib_.z + 4, ib_.w + 0);
    const long long ij_5_0 = pair_index(ib_.z + 5, ib_.w + 0);
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    const long long kl_1_0 = pair_index(ik_.z + 1, ik_.w + 0);
    const long long kl_2_0 = pair_index(ik_.z + 2, ik_.w + 0);
    const long long kl_3_0 = pair_index(ik_.z + 3, ik_.w + 0);
    const long long kl_4_0 = pair_index(ik_.z + 4, ik_.w + 0);
    const long long kl_5_0 = pair_index(ik_.z + 5, ik_.w + 0);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_1_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_1_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_1_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_2_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_2_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_2_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_3_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_3_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_3_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_4_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_4_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_4_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_5_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_5_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_5_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_dsds(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 36; ++x) {
        const int ia = x / 6, ibb = (x / 6) % 1, ic = (x / 1) % 6, id = x % 1;
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
__global__ void __launch_bounds__(128) eri_queue_dsds(const EriQueue Q) {
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
        double acc[36];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 36; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_dsds<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_dsds<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 36; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 36 doubles (launch_eri_dsds)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 36);
            if (lead) hrr_dsds(Q.pairs, p, q, acc, sb + kq * 36);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)36;
            for (int t = lane; t < nlive * 36; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[36];
            hrr_dsds(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_dsds(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_dsds(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_dsds(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 36864 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 36864 : 0;
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_dsds<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_dsds<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_dsds<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_dsds<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_dsds(int mixed) {

    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dsds<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dsds<0, 0>, 128, 0);
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
__global__ void __launch_bounds__(128) schwarz_kernel_dsds(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[36];
    if (full) {
        quartet_dsds<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[7]));
    m = fmax(m, fabs(res[14]));
    m = fmax(m, fabs(res[21]));
    m = fmax(m, fabs(res[28]));
    m = fmax(m, fabs(res[35]));
        qout[p] = sqrt(m);
        return;
    }
    double acc[36];
    for (int k = 0; k < in.y; ++k) {
        quartet_dsds<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[7]));
    m = fmax(m, fabs(res[14]));
    m = fmax(m, fabs(res[21]));
    m = fmax(m, fabs(res[28]));
    m = fmax(m, fabs(res[35]));
        w = fmax(w, fabs(acc[0]));
        w = fmax(w, fabs(acc[7]));
        w = fmax(w, fabs(acc[14]));
        w = fmax(w, fabs(acc[21]));
        w = fmax(w, fabs(acc[28]));
        w = fmax(w, fabs(acc[35]));
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }
}

void launch_schwarz_dsds(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    schwarz_kernel_dsds<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}

}  // namespace molints

// Generated by gen_eri.py -- class (ff|ss).  Do not edit.
// VRR entries: 210, contracted block: 74, HRR lines: 351, outputs: 100.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[74], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_ffss(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 74; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[7];
            boys_fm<6>(T, B, F);
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
            const VT v0_0_5 = (VT)(pref * F[5]);
            const VT v0_0_6 = (VT)(pref * F[6]);
            const VT v1_0_0 = PAx * v0_0_0 + WPx * v0_0_1;
            const VT v1_0_1 = PAx * v0_0_1 + WPx * v0_0_2;
            const VT v1_0_2 = PAx * v0_0_2 + WPx * v0_0_3;
            const VT v1_0_3 = PAx * v0_0_3 + WPx * v0_0_4;
            const VT v1_0_4 = PAx * v0_0_4 + WPx * v0_0_5;
            const VT v1_0_5 = PAx * v0_0_5 + WPx * v0_0_6;
            const VT v2_0_0 = PAy * v0_0_0 + WPy * v0_0_1;
            const VT v2_0_1 = PAy * v0_0_1 + WPy * v0_0_2;
            const VT v2_0_2 = PAy * v0_0_2 + WPy * v0_0_3;
            const VT v2_0_3 = PAy * v0_0_3 + WPy * v0_0_4;
            const VT v2_0_4 = PAy * v0_0_4 + WPy * v0_0_5;
            const VT v2_0_5 = PAy * v0_0_5 + WPy * v0_0_6;
            const VT v3_0_0 = PAz * v0_0_0 + WPz * v0_0_1;
            const VT v3_0_1 = PAz * v0_0_1 + WPz * v0_0_2;
            const VT v3_0_2 = PAz * v0_0_2 + WPz * v0_0_3;
            const VT v3_0_3 = PAz * v0_0_3 + WPz * v0_0_4;
            const VT v3_0_4 = PAz * v0_0_4 + WPz * v0_0_5;
            const VT v3_0_5 = PAz * v0_0_5 + WPz * v0_0_6;
            const VT v4_0_0 = PAx * v1_0_0 + WPx * v1_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v4_0_1 = PAx * v1_0_1 + WPx * v1_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v4_0_2 = PAx * v1_0_2 + WPx * v1_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v4_0_3 = PAx * v1_0_3 + WPx * v1_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v4_0_4 = PAx * v1_0_4 + WPx * v1_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v5_0_0 = PAx * v2_0_0 + WPx * v2_0_1;
            const VT v5_0_1 = PAx * v2_0_1 + WPx * v2_0_2;
            const VT v5_0_2 = PAx * v2_0_2 + WPx * v2_0_3;
            const VT v5_0_3 = PAx * v2_0_3 + WPx * v2_0_4;
            const VT v5_0_4 = PAx * v2_0_4 + WPx * v2_0_5;
            const VT v6_0_0 = PAx * v3_0_0 + WPx * v3_0_1;
            const VT v6_0_1 = PAx * v3_0_1 + WPx * v3_0_2;
            const VT v6_0_2 = PAx * v3_0_2 + WPx * v3_0_3;
            const VT v6_0_3 = PAx * v3_0_3 + WPx * v3_0_4;
            const VT v6_0_4 = PAx * v3_0_4 + WPx * v3_0_5;
            const VT v7_0_0 = PAy * v2_0_0 + WPy * v2_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v7_0_1 = PAy * v2_0_1 + WPy * v2_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v7_0_2 = PAy * v2_0_2 + WPy * v2_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v7_0_3 = PAy * v2_0_3 + WPy * v2_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v7_0_4 = PAy * v2_0_4 + WPy * v2_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v8_0_0 = PAy * v3_0_0 + WPy * v3_0_1;
            const VT v8_0_1 = PAy * v3_0_1 + WPy * v3_0_2;
            const VT v8_0_2 = PAy * v3_0_2 + WPy * v3_0_3;
            const VT v8_0_3 = PAy * v3_0_3 + WPy * v3_0_4;
            const VT v8_0_4 = PAy * v3_0_4 + WPy * v3_0_5;
            const VT v9_0_0 = PAz * v3_0_0 + WPz * v3_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v9_0_1 = PAz * v3_0_1 + WPz * v3_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v9_0_2 = PAz * v3_0_2 + WPz * v3_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v9_0_3 = PAz * v3_0_3 + WPz * v3_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v9_0_4 = PAz * v3_0_4 + WPz * v3_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v10_0_0 = PAx * v4_0_0 + WPx * v4_0_1 + (VT)2.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v10_0_1 = PAx * v4_0_1 + WPx * v4_0_2 + (VT)2.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v10_0_2 = PAx * v4_0_2 + WPx * v4_0_3 + (VT)2.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v10_0_3 = PAx * v4_0_3 + WPx * v4_0_4 + (VT)2.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v11_0_0 = PAx * v5_0_0 + WPx * v5_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v11_0_1 = PAx * v5_0_1 + WPx * v5_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v11_0_2 = PAx * v5_0_2 + WPx * v5_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v11_0_3 = PAx * v5_0_3 + WPx * v5_0_4 + (VT)1.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v12_0_0 = PAx * v6_0_0 + WPx * v6_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v12_0_1 = PAx * v6_0_1 + WPx * v6_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v12_0_2 = PAx * v6_0_2 + WPx * v6_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v12_0_3 = PAx * v6_0_3 + WPx * v6_0_4 + (VT)1.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v13_0_0 = PAy * v5_0_0 + WPy * v5_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v13_0_1 = PAy * v5_0_1 + WPy * v5_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v13_0_2 = PAy * v5_0_2 + WPy * v5_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v13_0_3 = PAy * v5_0_3 + WPy * v5_0_4 + (VT)1.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v14_0_0 = PAz * v6_0_0 + WPz * v6_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v14_0_1 = PAz * v6_0_1 + WPz * v6_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v14_0_2 = PAz * v6_0_2 + WPz * v6_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v14_0_3 = PAz * v6_0_3 + WPz * v6_0_4 + (VT)1.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v15_0_0 = PAx * v8_0_0 + WPx * v8_0_1;
            const VT v15_0_1 = PAx * v8_0_1 + WPx * v8_0_2;
            const VT v15_0_2 = PAx * v8_0_2 + WPx * v8_0_3;
            const VT v15_0_3 = PAx * v8_0_3 + WPx * v8_0_4;
            const VT v16_0_0 = PAy * v7_0_0 + WPy * v7_0_1 + (VT)2.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v16_0_1 = PAy * v7_0_1 + WPy * v7_0_2 + (VT)2.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v16_0_2 = PAy * v7_0_2 + WPy * v7_0_3 + (VT)2.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v16_0_3 = PAy * v7_0_3 + WPy * v7_0_4 + (VT)2.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v17_0_0 = PAy * v8_0_0 + WPy * v8_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v17_0_1 = PAy * v8_0_1 + WPy * v8_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v17_0_2 = PAy * v8_0_2 + WPy * v8_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v17_0_3 = PAy * v8_0_3 + WPy * v8_0_4 + (VT)1.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v18_0_0 = PAz * v8_0_0 + WPz * v8_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v18_0_1 = PAz * v8_0_1 + WPz * v8_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v18_0_2 = PAz * v8_0_2 + WPz * v8_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v18_0_3 = PAz * v8_0_3 + WPz * v8_0_4 + (VT)1.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v19_0_0 = PAz * v9_0_0 + WPz * v9_0_1 + (VT)2.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v19_0_1 = PAz * v9_0_1 + WPz * v9_0_2 + (VT)2.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v19_0_2 = PAz * v9_0_2 + WPz * v9_0_3 + (VT)2.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v19_0_3 = PAz * v9_0_3 + WPz * v9_0_4 + (VT)2.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v20_0_0 = PAx * v10_0_0 + WPx * v10_0_1 + (VT)3.0 * oo2z * (v4_0_0 - rho_z * v4_0_1);
            const VT v20_0_1 = PAx * v10_0_1 + WPx * v10_0_2 + (VT)3.0 * oo2z * (v4_0_1 - rho_z * v4_0_2);
            const VT v20_0_2 = PAx * v10_0_2 + WPx * v10_0_3 + (VT)3.0 * oo2z * (v4_0_2 - rho_z * v4_0_3);
            const VT v21_0_0 = PAx * v11_0_0 + WPx * v11_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v21_0_1 = PAx * v11_0_1 + WPx * v11_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v21_0_2 = PAx * v11_0_2 + WPx * v11_0_3 + (VT)2.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v22_0_0 = PAx * v12_0_0 + WPx * v12_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v22_0_1 = PAx * v12_0_1 + WPx * v12_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v22_0_2 = PAx * v12_0_2 + WPx * v12_0_3 + (VT)2.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v23_0_0 = PAx * v13_0_0 + WPx * v13_0_1 + (VT)1.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v23_0_1 = PAx * v13_0_1 + WPx * v13_0_2 + (VT)1.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v23_0_2 = PAx * v13_0_2 + WPx * v13_0_3 + (VT)1.0 * oo2z * (v7_0_2 - rho_z * v7_0_3);
            const VT v24_0_0 = PAx * v15_0_0 + WPx * v15_0_1 + (VT)1.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v24_0_1 = PAx * v15_0_1 + WPx * v15_0_2 + (VT)1.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v24_0_2 = PAx * v15_0_2 + WPx * v15_0_3 + (VT)1.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v25_0_0 = PAx * v14_0_0 + WPx * v14_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v25_0_1 = PAx * v14_0_1 + WPx * v14_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v25_0_2 = PAx * v14_0_2 + WPx * v14_0_3 + (VT)1.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v26_0_0 = PAy * v13_0_0 + WPy * v13_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v26_0_1 = PAy * v13_0_1 + WPy * v13_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v26_0_2 = PAy * v13_0_2 + WPy * v13_0_3 + (VT)2.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v27_0_0 = PAy * v15_0_0 + WPy * v15_0_1 + (VT)1.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v27_0_1 = PAy * v15_0_1 + WPy * v15_0_2 + (VT)1.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v27_0_2 = PAy * v15_0_2 + WPy * v15_0_3 + (VT)1.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v28_0_0 = PAz * v15_0_0 + WPz * v15_0_1 + (VT)1.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v28_0_1 = PAz * v15_0_1 + WPz * v15_0_2 + (VT)1.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v28_0_2 = PAz * v15_0_2 + WPz * v15_0_3 + (VT)1.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v29_0_0 = PAz * v14_0_0 + WPz * v14_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v29_0_1 = PAz * v14_0_1 + WPz * v14_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v29_0_2 = PAz * v14_0_2 + WPz * v14_0_3 + (VT)2.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v30_0_0 = PAy * v16_0_0 + WPy * v16_0_1 + (VT)3.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v30_0_1 = PAy * v16_0_1 + WPy * v16_0_2 + (VT)3.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v30_0_2 = PAy * v16_0_2 + WPy * v16_0_3 + (VT)3.0 * oo2z * (v7_0_2 - rho_z * v7_0_3);
            const VT v31_0_0 = PAy * v17_0_0 + WPy * v17_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v31_0_1 = PAy * v17_0_1 + WPy * v17_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v31_0_2 = PAy * v17_0_2 + WPy * v17_0_3 + (VT)2.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v32_0_0 = PAy * v18_0_0 + WPy * v18_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v32_0_1 = PAy * v18_0_1 + WPy * v18_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v32_0_2 = PAy * v18_0_2 + WPy * v18_0_3 + (VT)1.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v33_0_0 = PAz * v18_0_0 + WPz * v18_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v33_0_1 = PAz * v18_0_1 + WPz * v18_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v33_0_2 = PAz * v18_0_2 + WPz * v18_0_3 + (VT)2.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v34_0_0 = PAz * v19_0_0 + WPz * v19_0_1 + (VT)3.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v34_0_1 = PAz * v19_0_1 + WPz * v19_0_2 + (VT)3.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v34_0_2 = PAz * v19_0_2 + WPz * v19_0_3 + (VT)3.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v35_0_0 = PAx * v20_0_0 + WPx * v20_0_1 + (VT)4.0 * oo2z * (v10_0_0 - rho_z * v10_0_1);
            const VT v35_0_1 = PAx * v20_0_1 + WPx * v20_0_2 + (VT)4.0 * oo2z * (v10_0_1 - rho_z * v10_0_2);
            const VT v36_0_0 = PAx * v21_0_0 + WPx * v21_0_1 + (VT)3.0 * oo2z * (v11_0_0 - rho_z * v11_0_1);
            const VT v36_0_1 = PAx * v21_0_1 + WPx * v21_0_2 + (VT)3.0 * oo2z * (v11_0_1 - rho_z * v11_0_2);
            const VT v37_0_0 = PAx * v22_0_0 + WPx * v22_0_1 + (VT)3.0 * oo2z * (v12_0_0 - rho_z * v12_0_1);
            const VT v37_0_1 = PAx * v22_0_1 + WPx * v22_0_2 + (VT)3.0 * oo2z * (v12_0_1 - rho_z * v12_0_2);
            const VT v38_0_0 = PAx * v23_0_0 + WPx * v23_0_1 + (VT)2.0 * oo2z * (v13_0_0 - rho_z * v13_0_1);
            const VT v38_0_1 = PAx * v23_0_1 + WPx * v23_0_2 + (VT)2.0 * oo2z * (v13_0_1 - rho_z * v13_0_2);
            const VT v39_0_0 = PAx * v24_0_0 + WPx * v24_0_1 + (VT)2.0 * oo2z * (v15_0_0 - rho_z * v15_0_1);
            const VT v39_0_1 = PAx * v24_0_1 + WPx * v24_0_2 + (VT)2.0 * oo2z * (v15_0_1 - rho_z * v15_0_2);
            const VT v40_0_0 = PAx * v25_0_0 + WPx * v25_0_1 + (VT)2.0 * oo2z * (v14_0_0 - rho_z * v14_0_1);
            const VT v40_0_1 = PAx * v25_0_1 + WPx * v25_0_2 + (VT)2.0 * oo2z * (v14_0_1 - rho_z * v14_0_2);
            const VT v41_0_0 = PAy * v23_0_0 + WPy * v23_0_1 + (VT)2.0 * oo2z * (v11_0_0 - rho_z * v11_0_1);
            const VT v41_0_1 = PAy * v23_0_1 + WPy * v23_0_2 + (VT)2.0 * oo2z * (v11_0_1 - rho_z * v11_0_2);
            const VT v42_0_0 = PAx * v27_0_0 + WPx * v27_0_1 + (VT)1.0 * oo2z * (v17_0_0 - rho_z * v17_0_1);
            const VT v42_0_1 = PAx * v27_0_1 + WPx * v27_0_2 + (VT)1.0 * oo2z * (v17_0_1 - rho_z * v17_0_2);
            const VT v43_0_0 = PAx * v28_0_0 + WPx * v28_0_1 + (VT)1.0 * oo2z * (v18_0_0 - rho_z * v18_0_1);
            const VT v43_0_1 = PAx * v28_0_1 + WPx * v28_0_2 + (VT)1.0 * oo2z * (v18_0_1 - rho_z * v18_0_2);
            const VT v44_0_0 = PAz * v25_0_0 + WPz * v25_0_1 + (VT)2.0 * oo2z * (v12_0_0 - rho_z * v12_0_1);
            const VT v44_0_1 = PAz * v25_0_1 + WPz * v25_0_2 + (VT)2.0 * oo2z * (v12_0_1 - rho_z * v12_0_2);
            const VT v45_0_0 = PAy * v26_0_0 + WPy * v26_0_1 + (VT)3.0 * oo2z * (v13_0_0 - rho_z * v13_0_1);
            const VT v45_0_1 = PAy * v26_0_1 + WPy * v26_0_2 + (VT)3.0 * oo2z * (v13_0_1 - rho_z * v13_0_2);
            const VT v46_0_0 = PAy * v27_0_0 + WPy * v27_0_1 + (VT)2.0 * oo2z * (v15_0_0 - rho_z * v15_0_1);
            const VT v46_0_1 = PAy * v27_0_1 + WPy * v27_0_2 + (VT)2.0 * oo2z * (v15_0_1 - rho_z * v15_0_2);
            const VT v47_0_0 = PAy * v28_0_0 + WPy * v28_0_1 + (VT)1.0 * oo2z * (v14_0_0 - rho_z * v14_0_1);
            const VT v47_0_1 = PAy * v28_0_1 + WPy * v28_0_2 + (VT)1.0 * oo2z * (v14_0_1 - rho_z * v14_0_2);
            const VT v48_0_0 = PAz * v28_0_0 + WPz * v28_0_1 + (VT)2.0 * oo2z * (v15_0_0 - rho_z * v15_0_1);
            const VT v48_0_1 = PAz * v28_0_1 + WPz * v28_0_2 + (VT)2.0 * oo2z * (v15_0_1 - rho_z * v15_0_2);
            const VT v49_0_0 = PAz * v29_0_0 + WPz * v29_0_1 + (VT)3.0 * oo2z * (v14_0_0 - rho_z * v14_0_1);
            const VT v49_0_1 = PAz * v29_0_1 + WPz * v29_0_2 + (VT)3.0 * oo2z * (v14_0_1 - rho_z * v14_0_2);
            const VT v50_0_0 = PAy * v30_0_0 + WPy * v30_0_1 + (VT)4.0 * oo2z * (v16_0_0 - rho_z * v16_0_1);
            const VT v50_0_1 = PAy * v30_0_1 + WPy * v30_0_2 + (VT)4.0 * oo2z * (v16_0_1 - rho_z * v16_0_2);
            const VT v51_0_0 = PAy * v31_0_0 + WPy * v31_0_1 + (VT)3.0 * oo2z * (v17_0_0 - rho_z * v17_0_1);
            const VT v51_0_1 = PAy * v31_0_1 + WPy * v31_0_2 + (VT)3.0 * oo2z * (v17_0_1 - rho_z * v17_0_2);
            const VT v52_0_0 = PAy * v32_0_0 + WPy * v32_0_1 + (VT)2.0 * oo2z * (v18_0_0 - rho_z * v18_0_1);
            const VT v52_0_1 = PAy * v32_0_1 + WPy * v32_0_2 + (VT)2.0 * oo2z * (v18_0_1 - rho_z * v18_0_2);
            const VT v53_0_0 = PAz * v32_0_0 + WPz * v32_0_1 + (VT)2.0 * oo2z * (v17_0_0 - rho_z * v17_0_1);
            const VT v53_0_1 = PAz * v32_0_1 + WPz * v32_0_2 + (VT)2.0 * oo2z * (v17_0_1 - rho_z * v17_0_2);
            const VT v54_0_0 = PAz * v33_0_0 + WPz * v33_0_1 + (VT)3.0 * oo2z * (v18_0_0 - rho_z * v18_0_1);
            const VT v54_0_1 = PAz * v33_0_1 + WPz * v33_0_2 + (VT)3.0 * oo2z * (v18_0_1 - rho_z * v18_0_2);
            const VT v55_0_0 = PAz * v34_0_0 + WPz * v34_0_1 + (VT)4.0 * oo2z * (v19_0_0 - rho_z * v19_0_1);
            const VT v55_0_1 = PAz * v34_0_1 + WPz * v34_0_2 + (VT)4.0 * oo2z * (v19_0_1 - rho_z * v19_0_2);
            const VT v56_0_0 = PAx * v35_0_0 + WPx * v35_0_1 + (VT)5.0 * oo2z * (v20_0_0 - rho_z * v20_0_1);
            const VT v57_0_0 = PAx * v36_0_0 + WPx * v36_0_1 + (VT)4.0 * oo2z * (v21_0_0 - rho_z * v21_0_1);
            const VT v58_0_0 = PAx * v37_0_0 + WPx * v37_0_1 + (VT)4.0 * oo2z * (v22_0_0 - rho_z * v22_0_1);
            const VT v59_0_0 = PAx * v38_0_0 + WPx * v38_0_1 + (VT)3.0 * oo2z * (v23_0_0 - rho_z * v23_0_1);
            const VT v60_0_0 = PAx * v39_0_0 + WPx * v39_0_1 + (VT)3.0 * oo2z * (v24_0_0 - rho_z * v24_0_1);
            const VT v61_0_0 = PAx * v40_0_0 + WPx * v40_0_1 + (VT)3.0 * oo2z * (v25_0_0 - rho_z * v25_0_1);
            const VT v62_0_0 = PAx * v41_0_0 + WPx * v41_0_1 + (VT)2.0 * oo2z * (v26_0_0 - rho_z * v26_0_1);
            const VT v63_0_0 = PAx * v42_0_0 + WPx * v42_0_1 + (VT)2.0 * oo2z * (v27_0_0 - rho_z * v27_0_1);
            const VT v64_0_0 = PAx * v43_0_0 + WPx * v43_0_1 + (VT)2.0 * oo2z * (v28_0_0 - rho_z * v28_0_1);
            const VT v65_0_0 = PAx * v44_0_0 + WPx * v44_0_1 + (VT)2.0 * oo2z * (v29_0_0 - rho_z * v29_0_1);
            const VT v66_0_0 = PAy * v41_0_0 + WPy * v41_0_1 + (VT)3.0 * oo2z * (v23_0_0 - rho_z * v23_0_1);
            const VT v67_0_0 = PAy * v42_0_0 + WPy * v42_0_1 + (VT)2.0 * oo2z * (v24_0_0 - rho_z * v24_0_1);
            const VT v68_0_0 = PAx * v47_0_0 + WPx * v47_0_1 + (VT)1.0 * oo2z * (v32_0_0 - rho_z * v32_0_1);
            const VT v69_0_0 = PAz * v43_0_0 + WPz * v43_0_1 + (VT)2.0 * oo2z * (v24_0_0 - rho_z * v24_0_1);
            const VT v70_0_0 = PAz * v44_0_0 + WPz * v44_0_1 + (VT)3.0 * oo2z * (v25_0_0 - rho_z * v25_0_1);
            const VT v71_0_0 = PAy * v45_0_0 + WPy * v45_0_1 + (VT)4.0 * oo2z * (v26_0_0 - rho_z * v26_0_1);
            const VT v72_0_0 = PAy * v46_0_0 + WPy * v46_0_1 + (VT)3.0 * oo2z * (v27_0_0 - rho_z * v27_0_1);
            const VT v73_0_0 = PAy * v47_0_0 + WPy * v47_0_1 + (VT)2.0 * oo2z * (v28_0_0 - rho_z * v28_0_1);
            const VT v74_0_0 = PAz * v47_0_0 + WPz * v47_0_1 + (VT)2.0 * oo2z * (v27_0_0 - rho_z * v27_0_1);
            const VT v75_0_0 = PAz * v48_0_0 + WPz * v48_0_1 + (VT)3.0 * oo2z * (v28_0_0 - rho_z * v28_0_1);
            const VT v76_0_0 = PAz * v49_0_0 + WPz * v49_0_1 + (VT)4.0 * oo2z * (v29_0_0 - rho_z * v29_0_1);
            const VT v77_0_0 = PAy * v50_0_0 + WPy * v50_0_1 + (VT)5.0 * oo2z * (v30_0_0 - rho_z * v30_0_1);
            const VT v78_0_0 = PAy * v51_0_0 + WPy * v51_0_1 + (VT)4.0 * oo2z * (v31_0_0 - rho_z * v31_0_1);
            const VT v79_0_0 = PAy * v52_0_0 + WPy * v52_0_1 + (VT)3.0 * oo2z * (v32_0_0 - rho_z * v32_0_1);
            const VT v80_0_0 = PAy * v53_0_0 + WPy * v53_0_1 + (VT)2.0 * oo2z * (v33_0_0 - rho_z * v33_0_1);
            const VT v81_0_0 = PAz * v53_0_0 + WPz * v53_0_1 + (VT)3.0 * oo2z * (v32_0_0 - rho_z * v32_0_1);
            const VT v82_0_0 = PAz * v54_0_0 + WPz * v54_0_1 + (VT)4.0 * oo2z * (v33_0_0 - rho_z * v33_0_1);
            const VT v83_0_0 = PAz * v55_0_0 + WPz * v55_0_1 + (VT)5.0 * oo2z * (v34_0_0 - rho_z * v34_0_1);
            acc[0] += (double)v10_0_0;
            acc[1] += (double)v11_0_0;
            acc[2] += (double)v12_0_0;
            acc[3] += (double)v13_0_0;
            acc[4] += (double)v14_0_0;
            acc[5] += (double)v15_0_0;
            acc[6] += (double)v16_0_0;
            acc[7] += (double)v17_0_0;
            acc[8] += (double)v18_0_0;
            acc[9] += (double)v19_0_0;
            acc[10] += (double)v20_0_0;
            acc[11] += (double)v21_0_0;
            acc[12] += (double)v22_0_0;
            acc[13] += (double)v23_0_0;
            acc[14] += (double)v24_0_0;
            acc[15] += (double)v25_0_0;
            acc[16] += (double)v26_0_0;
            acc[17] += (double)v27_0_0;
            acc[18] += (double)v28_0_0;
            acc[19] += (double)v29_0_0;
            acc[20] += (double)v30_0_0;
            acc[21] += (double)v31_0_0;
            acc[22] += (double)v32_0_0;
            acc[23] += (double)v33_0_0;
            acc[24] += (double)v34_0_0;
            acc[25] += (double)v35_0_0;
            acc[26] += (double)v36_0_0;
            acc[27] += (double)v37_0_0;
            acc[28] += (double)v38_0_0;
            acc[29] += (double)v39_0_0;
            acc[30] += (double)v40_0_0;
            acc[31] += (double)v41_0_0;
            acc[32] += (double)v42_0_0;
            acc[33] += (double)v43_0_0;
            acc[34] += (double)v44_0_0;
            acc[35] += (double)v45_0_0;
            acc[36] += (double)v46_0_0;
            acc[37] += (double)v47_0_0;
            acc[38] += (double)v48_0_0;
            acc[39] += (double)v49_0_0;
            acc[40] += (double)v50_0_0;
            acc[41] += (double)v51_0_0;
            acc[42] += (double)v52_0_0;
            acc[43] += (double)v53_0_0;
            acc[44] += (double)v54_0_0;
            acc[45] += (double)v55_0_0;
            acc[46] += (double)v56_0_0;
            acc[47] += (double)v57_0_0;
            acc[48] += (double)v58_0_0;
            acc[49] += (double)v59_0_0;
            acc[50] += (double)v60_0_0;
            acc[51] += (double)v61_0_0;
            acc[52] += (double)v62_0_0;
            acc[53] += (double)v63_0_0;
            acc[54] += (double)v64_0_0;
            acc[55] += (double)v65_0_0;
            acc[56] += (double)v66_0_0;
            acc[57] += (double)v67_0_0;
            acc[58] += (double)v68_0_0;
            acc[59] += (double)v69_0_0;
            acc[60] += (double)v70_0_0;
            acc[61] += (double)v71_0_0;
            acc[62] += (double)v72_0_0;
            acc[63] += (double)v73_0_0;
            acc[64] += (double)v74_0_0;
            acc[65] += (double)v75_0_0;
            acc[66] += (double)v76_0_0;
            acc[67] += (double)v77_0_0;
            acc[68] += (double)v78_0_0;
            acc[69] += (double)v79_0_0;
            acc[70] += (double)v80_0_0;
            acc[71] += (double)v81_0_0;
            acc[72] += (double)v82_0_0;
            acc[73] += (double)v83_0_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[100] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_ffss(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h35_1_0 = acc[46] + ABx * acc[25];
    const double h20_1_0 = acc[25] + ABx * acc[10];
    const double h20_4_0 = h35_1_0 + ABx * h20_1_0;
    const double h10_1_0 = acc[10] + ABx * acc[0];
    const double h10_4_0 = h20_1_0 + ABx * h10_1_0;
    const double h10_10_0 = h20_4_0 + ABx * h10_4_0;
    const double h35_2_0 = acc[47] + ABy * acc[25];
    const double h20_2_0 = acc[26] + ABy * acc[10];
    const double h20_5_0 = h35_2_0 + ABx * h20_2_0;
    const double h10_2_0 = acc[11] + ABy * acc[0];
    const double h10_5_0 = h20_2_0 + ABx * h10_2_0;
    const double h10_11_0 = h20_5_0 + ABx * h10_5_0;
    const double h35_3_0 = acc[48] + ABz * acc[25];
    const double h20_3_0 = acc[27] + ABz * acc[10];
    const double h20_6_0 = h35_3_0 + ABx * h20_3_0;
    const double h10_3_0 = acc[12] + ABz * acc[0];
    const double h10_6_0 = h20_3_0 + ABx * h10_3_0;
    const double h10_12_0 = h20_6_0 + ABx * h10_6_0;
    const double h36_2_0 = acc[49] + ABy * acc[26];
    const double h21_2_0 = acc[28] + ABy * acc[11];
    const double h21_5_0 = h36_2_0 + ABx * h21_2_0;
    const double h10_13_0 = h21_5_0 + ABy * h10_5_0;
    const double h37_3_0 = acc[51] + ABz * acc[27];
    const double h22_3_0 = acc[30] + ABz * acc[12];
    const double h22_6_0 = h37_3_0 + ABx * h22_3_0;
    const double h10_14_0 = h22_6_0 + ABz * h10_6_0;
    const double h36_3_0 = acc[50] + ABz * acc[26];
    const double h20_8_0 = h36_3_0 + ABy * h20_3_0;
    const double h21_3_0 = acc[29] + ABz * acc[11];
    const double h10_8_0 = h21_3_0 + ABy * h10_3_0;
    const double h10_15_0 = h20_8_0 + ABx * h10_8_0;
    const double h38_2_0 = acc[52] + ABy * acc[28];
    const double h21_7_0 = h38_2_0 + ABy * h21_2_0;
    const double h10_7_0 = h21_2_0 + ABy * h10_2_0;
    const double h10_16_0 = h21_7_0 + ABy * h10_7_0;
    const double h38_3_0 = acc[53] + ABz * acc[28];
    const double h21_8_0 = h38_3_0 + ABy * h21_3_0;
    const double h10_17_0 = h21_8_0 + ABy * h10_8_0;
    const double h39_3_0 = acc[54] + ABz * acc[29];
    const double h22_8_0 = h39_3_0 + ABy * h22_3_0;
    const double h10_18_0 = h22_8_0 + ABz * h10_8_0;
    const double h40_3_0 = acc[55] + ABz * acc[30];
    const double h22_9_0 = h40_3_0 + ABz * h22_3_0;
    const double h10_9_0 = h22_3_0 + ABz * h10_3_0;
    const double h10_19_0 = h22_9_0 + ABz * h10_9_0;
    const double h36_1_0 = acc[47] + ABx * acc[26];
    const double h21_1_0 = acc[26] + ABx * acc[11];
    const double h21_4_0 = h36_1_0 + ABx * h21_1_0;
    const double h11_1_0 = acc[11] + ABx * acc[1];
    const double h11_4_0 = h21_1_0 + ABx * h11_1_0;
    const double h11_10_0 = h21_4_0 + ABx * h11_4_0;
    const double h11_2_0 = acc[13] + ABy * acc[1];
    const double h11_5_0 = h21_2_0 + ABx * h11_2_0;
    const double h11_11_0 = h21_5_0 + ABx * h11_5_0;
    const double h21_6_0 = h36_3_0 + ABx * h21_3_0;
    const double h11_3_0 = acc[14] + ABz * acc[1];
    const double h11_6_0 = h21_3_0 + ABx * h11_3_0;
    const double h11_12_0 = h21_6_0 + ABx * h11_6_0;
    const double h23_2_0 = acc[31] + ABy * acc[13];
    const double h23_5_0 = h38_2_0 + ABx * h23_2_0;
    const double h11_13_0 = h23_5_0 + ABy * h11_5_0;
    const double h24_3_0 = acc[33] + ABz * acc[14];
    const double h24_6_0 = h39_3_0 + ABx * h24_3_0;
    const double h11_14_0 = h24_6_0 + ABz * h11_6_0;
    const double h23_3_0 = acc[32] + ABz * acc[13];
    const double h11_8_0 = h23_3_0 + ABy * h11_3_0;
    const double h11_15_0 = h21_8_0 + ABx * h11_8_0;
    const double h41_2_0 = acc[56] + ABy * acc[31];
    const double h23_7_0 = h41_2_0 + ABy * h23_2_0;
    const double h11_7_0 = h23_2_0 + ABy * h11_2_0;
    const double h11_16_0 = h23_7_0 + ABy * h11_7_0;
    const double h41_3_0 = acc[57] + ABz * acc[31];
    const double h23_8_0 = h41_3_0 + ABy * h23_3_0;
    const double h11_17_0 = h23_8_0 + ABy * h11_8_0;
    const double h42_3_0 = acc[58] + ABz * acc[32];
    const double h24_8_0 = h42_3_0 + ABy * h24_3_0;
    const double h11_18_0 = h24_8_0 + ABz * h11_8_0;
    const double h43_3_0 = acc[59] + ABz * acc[33];
    const double h24_9_0 = h43_3_0 + ABz * h24_3_0;
    const double h11_9_0 = h24_3_0 + ABz * h11_3_0;
    const double h11_19_0 = h24_9_0 + ABz * h11_9_0;
    const double h37_1_0 = acc[48] + ABx * acc[27];
    const double h22_1_0 = acc[27] + ABx * acc[12];
    const double h22_4_0 = h37_1_0 + ABx * h22_1_0;
    const double h12_1_0 = acc[12] + ABx * acc[2];
    const double h12_4_0 = h22_1_0 + ABx * h12_1_0;
    const double h12_10_0 = h22_4_0 + ABx * h12_4_0;
    const double h37_2_0 = acc[50] + ABy * acc[27];
    const double h22_2_0 = acc[29] + ABy * acc[12];
    const double h22_5_0 = h37_2_0 + ABx * h22_2_0;
    const double h12_2_0 = acc[14] + ABy * acc[2];
    const double h12_5_0 = h22_2_0 + ABx * h12_2_0;
    const double h12_11_0 = h22_5_0 + ABx * h12_5_0;
    const double h12_3_0 = acc[15] + ABz * acc[2];
    const double h12_6_0 = h22_3_0 + ABx * h12_3_0;
    const double h12_12_0 = h22_6_0 + ABx * h12_6_0;
    const double h39_2_0 = acc[53] + ABy * acc[29];
    const double h24_2_0 = acc[32] + ABy * acc[14];
    const double h24_5_0 = h39_2_0 + ABx * h24_2_0;
    const double h12_13_0 = h24_5_0 + ABy * h12_5_0;
    const double h25_3_0 = acc[34] + ABz * acc[15];
    const double h25_6_0 = h40_3_0 + ABx * h25_3_0;
    const double h12_14_0 = h25_6_0 + ABz * h12_6_0;
    const double h12_8_0 = h24_3_0 + ABy * h12_3_0;
    const double h12_15_0 = h22_8_0 + ABx * h12_8_0;
    const double h42_2_0 = acc[57] + ABy * acc[32];
    const double h24_7_0 = h42_2_0 + ABy * h24_2_0;
    const double h12_7_0 = h24_2_0 + ABy * h12_2_0;
    const double h12_16_0 = h24_7_0 + ABy * h12_7_0;
    const double h12_17_0 = h24_8_0 + ABy * h12_8_0;
    const double h25_8_0 = h43_3_0 + ABy * h25_3_0;
    const double h12_18_0 = h25_8_0 + ABz * h12_8_0;
    const double h44_3_0 = acc[60] + ABz * acc[34];
    const double h25_9_0 = h44_3_0 + ABz * h25_3_0;
    const double h12_9_0 = h25_3_0 + ABz * h12_3_0;
    const double h12_19_0 = h25_9_0 + ABz * h12_9_0;
    const double h38_1_0 = acc[49] + ABx * acc[28];
    const double h23_1_0 = acc[28] + ABx * acc[13];
    const double h23_4_0 = h38_1_0 + ABx * h23_1_0;
    const double h13_1_0 = acc[13] + ABx * acc[3];
    const double h13_4_0 = h23_1_0 + ABx * h13_1_0;
    const double h13_10_0 = h23_4_0 + ABx * h13_4_0;
    const double h13_2_0 = acc[16] + ABy * acc[3];
    const double h13_5_0 = h23_2_0 + ABx * h13_2_0;
    const double h13_11_0 = h23_5_0 + ABx * h13_5_0;
    const double h23_6_0 = h38_3_0 + ABx * h23_3_0;
    const double h13_3_0 = acc[17] + ABz * acc[3];
    const double h13_6_0 = h23_3_0 + ABx * h13_3_0;
    const double h13_12_0 = h23_6_0 + ABx * h13_6_0;
    const double h26_2_0 = acc[35] + ABy * acc[16];
    const double h26_5_0 = h41_2_0 + ABx * h26_2_0;
    const double h13_13_0 = h26_5_0 + ABy * h13_5_0;
    const double h27_3_0 = acc[37] + ABz * acc[17];
    const double h27_6_0 = h42_3_0 + ABx * h27_3_0;
    const double h13_14_0 = h27_6_0 + ABz * h13_6_0;
    const double h26_3_0 = acc[36] + ABz * acc[16];
    const double h13_8_0 = h26_3_0 + ABy * h13_3_0;
    const double h13_15_0 = h23_8_0 + ABx * h13_8_0;
    const double h45_2_0 = acc[61] + ABy * acc[35];
    const double h26_7_0 = h45_2_0 + ABy * h26_2_0;
    const double h13_7_0 = h26_2_0 + ABy * h13_2_0;
    const double h13_16_0 = h26_7_0 + ABy * h13_7_0;
    const double h45_3_0 = acc[62] + ABz * acc[35];
    const double h26_8_0 = h45_3_0 + ABy * h26_3_0;
    const double h13_17_0 = h26_8_0 + ABy * h13_8_0;
    const double h46_3_0 = acc[63] + ABz * acc[36];
    const double h27_8_0 = h46_3_0 + ABy * h27_3_0;
    const double h13_18_0 = h27_8_0 + ABz * h13_8_0;
    const double h47_3_0 = acc[64] + ABz * acc[37];
    const double h27_9_0 = h47_3_0 + ABz * h27_3_0;
    const double h13_9_0 = h27_3_0 + ABz * h13_3_0;
    const double h13_19_0 = h27_9_0 + ABz * h13_9_0;
    const double h40_1_0 = acc[51] + ABx * acc[30];
    const double h25_1_0 = acc[30] + ABx * acc[15];
    const double h25_4_0 = h40_1_0 + ABx * h25_1_0;
    const double h14_1_0 = acc[15] + ABx * acc[4];
    const double h14_4_0 = h25_1_0 + ABx * h14_1_0;
    const double h14_10_0 = h25_4_0 + ABx * h14_4_0;
    const double h40_2_0 = acc[54] + ABy * acc[30];
    const double h25_2_0 = acc[33] + ABy * acc[15];
    const double h25_5_0 = h40_2_0 + ABx * h25_2_0;
    const double h14_2_0 = acc[18] + ABy * acc[4];
    const double h14_5_0 = h25_2_0 + ABx * h14_2_0;
    const double h14_11_0 = h25_5_0 + ABx * h14_5_0;
    const double h14_3_0 = acc[19] + ABz * acc[4];
    const double h14_6_0 = h25_3_0 + ABx * h14_3_0;
    const double h14_12_0 = h25_6_0 + ABx * h14_6_0;
    const double h43_2_0 = acc[58] + ABy * acc[33];
    const double h28_2_0 = acc[37] + ABy * acc[18];
    const double h28_5_0 = h43_2_0 + ABx * h28_2_0;
    const double h14_13_0 = h28_5_0 + ABy * h14_5_0;
    const double h29_3_0 = acc[39] + ABz * acc[19];
    const double h29_6_0 = h44_3_0 + ABx * h29_3_0;
    const double h14_14_0 = h29_6_0 + ABz * h14_6_0;
    const double h28_3_0 = acc[38] + ABz * acc[18];
    const double h14_8_0 = h28_3_0 + ABy * h14_3_0;
    const double h14_15_0 = h25_8_0 + ABx * h14_8_0;
    const double h47_2_0 = acc[63] + ABy * acc[37];
    const double h28_7_0 = h47_2_0 + ABy * h28_2_0;
    const double h14_7_0 = h28_2_0 + ABy * h14_2_0;
    const double h14_16_0 = h28_7_0 + ABy * h14_7_0;
    const double h28_8_0 = h47_3_0 + ABy * h28_3_0;
    const double h14_17_0 = h28_8_0 + ABy * h14_8_0;
    const double h48_3_0 = acc[65] + ABz * acc[38];
    const double h29_8_0 = h48_3_0 + ABy * h29_3_0;
    const double h14_18_0 = h29_8_0 + ABz * h14_8_0;
    const double h49_3_0 = acc[66] + ABz * acc[39];
    const double h29_9_0 = h49_3_0 + ABz * h29_3_0;
    const double h14_9_0 = h29_3_0 + ABz * h14_3_0;
    const double h14_19_0 = h29_9_0 + ABz * h14_9_0;
    const double h39_1_0 = acc[50] + ABx * acc[29];
    const double h24_1_0 = acc[29] + ABx * acc[14];
    const double h24_4_0 = h39_1_0 + ABx * h24_1_0;
    const double h15_1_0 = acc[14] + ABx * acc[5];
    const double h15_4_0 = h24_1_0 + ABx * h15_1_0;
    const double h15_10_0 = h24_4_0 + ABx * h15_4_0;
    const double h15_2_0 = acc[17] + ABy * acc[5];
    const double h15_5_0 = h24_2_0 + ABx * h15_2_0;
    const double h15_11_0 = h24_5_0 + ABx * h15_5_0;
    const double h15_3_0 = acc[18] + ABz * acc[5];
    const double h15_6_0 = h24_3_0 + ABx * h15_3_0;
    const double h15_12_0 = h24_6_0 + ABx * h15_6_0;
    const double h27_2_0 = acc[36] + ABy * acc[17];
    const double h27_5_0 = h42_2_0 + ABx * h27_2_0;
    const double h15_13_0 = h27_5_0 + ABy * h15_5_0;
    const double h28_6_0 = h43_3_0 + ABx * h28_3_0;
    const double h15_14_0 = h28_6_0 + ABz * h15_6_0;
    const double h15_8_0 = h27_3_0 + ABy * h15_3_0;
    const double h15_15_0 = h24_8_0 + ABx * h15_8_0;
    const double h46_2_0 = acc[62] + ABy * acc[36];
    const double h27_7_0 = h46_2_0 + ABy * h27_2_0;
    const double h15_7_0 = h27_2_0 + ABy * h15_2_0;
    const double h15_16_0 = h27_7_0 + ABy * h15_7_0;
    const double h15_17_0 = h27_8_0 + ABy * h15_8_0;
    const double h15_18_0 = h28_8_0 + ABz * h15_8_0;
    const double h28_9_0 = h48_3_0 + ABz * h28_3_0;
    const double h15_9_0 = h28_3_0 + ABz * h15_3_0;
    const double h15_19_0 = h28_9_0 + ABz * h15_9_0;
    const double h41_1_0 = acc[52] + ABx * acc[31];
    const double h26_1_0 = acc[31] + ABx * acc[16];
    const double h26_4_0 = h41_1_0 + ABx * h26_1_0;
    const double h16_1_0 = acc[16] + ABx * acc[6];
    const double h16_4_0 = h26_1_0 + ABx * h16_1_0;
    const double h16_10_0 = h26_4_0 + ABx * h16_4_0;
    const double h16_2_0 = acc[20] + ABy * acc[6];
    const double h16_5_0 = h26_2_0 + ABx * h16_2_0;
    const double h16_11_0 = h26_5_0 + ABx * h16_5_0;
    const double h26_6_0 = h41_3_0 + ABx * h26_3_0;
    const double h16_3_0 = acc[21] + ABz * acc[6];
    const double h16_6_0 = h26_3_0 + ABx * h16_3_0;
    const double h16_12_0 = h26_6_0 + ABx * h16_6_0;
    const double h30_2_0 = acc[40] + ABy * acc[20];
    const double h30_5_0 = h45_2_0 + ABx * h30_2_0;
    const double h16_13_0 = h30_5_0 + ABy * h16_5_0;
    const double h31_3_0 = acc[42] + ABz * acc[21];
    const double h31_6_0 = h46_3_0 + ABx * h31_3_0;
    const double h16_14_0 = h31_6_0 + ABz * h16_6_0;
    const double h30_3_0 = acc[41] + ABz * acc[20];
    const double h16_8_0 = h30_3_0 + ABy * h16_3_0;
    const double h16_15_0 = h26_8_0 + ABx * h16_8_0;
    const double h50_2_0 = acc[67] + ABy * acc[40];
    const double h30_7_0 = h50_2_0 + ABy * h30_2_0;
    const double h16_7_0 = h30_2_0 + ABy * h16_2_0;
    const double h16_16_0 = h30_7_0 + ABy * h16_7_0;
    const double h50_3_0 = acc[68] + ABz * acc[40];
    const double h30_8_0 = h50_3_0 + ABy * h30_3_0;
    const double h16_17_0 = h30_8_0 + ABy * h16_8_0;
    const double h51_3_0 = acc[69] + ABz * acc[41];
    const double h31_8_0 = h51_3_0 + ABy * h31_3_0;
    const double h16_18_0 = h31_8_0 + ABz * h16_8_0;
    const double h52_3_0 = acc[70] + ABz * acc[42];
    const double h31_9_0 = h52_3_0 + ABz * h31_3_0;
    const double h16_9_0 = h31_3_0 + ABz * h16_3_0;
    const double h16_19_0 = h31_9_0 + ABz * h16_9_0;
    const double h42_1_0 = acc[53] + ABx * acc[32];
    const double h27_1_0 = acc[32] + ABx * acc[17];
    const double h27_4_0 = h42_1_0 + ABx * h27_1_0;
    const double h17_1_0 = acc[17] + ABx * acc[7];
    const double h17_4_0 = h27_1_0 + ABx * h17_1_0;
    const double h17_10_0 = h27_4_0 + ABx * h17_4_0;
    const double h17_2_0 = acc[21] + ABy * acc[7];
    const double h17_5_0 = h27_2_0 + ABx * h17_2_0;
    const double h17_11_0 = h27_5_0 + ABx * h17_5_0;
    const double h17_3_0 = acc[22] + ABz * acc[7];
    const double h17_6_0 = h27_3_0 + ABx * h17_3_0;
    const double h17_12_0 = h27_6_0 + ABx * h17_6_0;
    const double h31_2_0 = acc[41] + ABy * acc[21];
    const double h31_5_0 = h46_2_0 + ABx * h31_2_0;
    const double h17_13_0 = h31_5_0 + ABy * h17_5_0;
    const double h32_3_0 = acc[43] + ABz * acc[22];
    const double h32_6_0 = h47_3_0 + ABx * h32_3_0;
    const double h17_14_0 = h32_6_0 + ABz * h17_6_0;
    const double h17_8_0 = h31_3_0 + ABy * h17_3_0;
    const double h17_15_0 = h27_8_0 + ABx * h17_8_0;
    const double h51_2_0 = acc[68] + ABy * acc[41];
    const double h31_7_0 = h51_2_0 + ABy * h31_2_0;
    const double h17_7_0 = h31_2_0 + ABy * h17_2_0;
    const double h17_16_0 = h31_7_0 + ABy * h17_7_0;
    const double h17_17_0 = h31_8_0 + ABy * h17_8_0;
    const double h32_8_0 = h52_3_0 + ABy * h32_3_0;
    const double h17_18_0 = h32_8_0 + ABz * h17_8_0;
    const double h53_3_0 = acc[71] + ABz * acc[43];
    const double h32_9_0 = h53_3_0 + ABz * h32_3_0;
    const double h17_9_0 = h32_3_0 + ABz * h17_3_0;
    const double h17_19_0 = h32_9_0 + ABz * h17_9_0;
    const double h43_1_0 = acc[54] + ABx * acc[33];
    const double h28_1_0 = acc[33] + ABx * acc[18];
    const double h28_4_0 = h43_1_0 + ABx * h28_1_0;
    const double h18_1_0 = acc[18] + ABx * acc[8];
    const double h18_4_0 = h28_1_0 + ABx * h18_1_0;
    const double h18_10_0 = h28_4_0 + ABx * h18_4_0;
    const double h18_2_0 = acc[22] + ABy * acc[8];
    const double h18_5_0 = h28_2_0 + ABx * h18_2_0;
    const double h18_11_0 = h28_5_0 + ABx * h18_5_0;
    const double h18_3_0 = acc[23] + ABz * acc[8];
    const double h18_6_0 = h28_3_0 + ABx * h18_3_0;
    const double h18_12_0 = h28_6_0 + ABx * h18_6_0;
    const double h32_2_0 = acc[42] + ABy * acc[22];
    const double h32_5_0 = h47_2_0 + ABx * h32_2_0;
    const double h18_13_0 = h32_5_0 + ABy * h18_5_0;
    const double h33_3_0 = acc[44] + ABz * acc[23];
    const double h33_6_0 = h48_3_0 + ABx * h33_3_0;
    const double h18_14_0 = h33_6_0 + ABz * h18_6_0;
    const double h18_8_0 = h32_3_0 + ABy * h18_3_0;
    const double h18_15_0 = h28_8_0 + ABx * h18_8_0;
    const double h52_2_0 = acc[69] + ABy * acc[42];
    const double h32_7_0 = h52_2_0 + ABy * h32_2_0;
    const double h18_7_0 = h32_2_0 + ABy * h18_2_0;
    const double h18_16_0 = h32_7_0 + ABy * h18_7_0;
    const double h18_17_0 = h32_8_0 + ABy * h18_8_0;
    const double h33_8_0 = h53_3_0 + ABy * h33_3_0;
    const double h18_18_0 = h33_8_0 + ABz * h18_8_0;
    const double h54_3_0 = acc[72] + ABz * acc[44];
    const double h33_9_0 = h54_3_0 + ABz * h33_3_0;
    const double h18_9_0 = h33_3_0 + ABz * h18_3_0;
    const double h18_19_0 = h33_9_0 + ABz * h18_9_0;
    const double h44_1_0 = acc[55] + ABx * acc[34];
    const double h29_1_0 = acc[34] + ABx * acc[19];
    const double h29_4_0 = h44_1_0 + ABx * h29_1_0;
    const double h19_1_0 = acc[19] + ABx * acc[9];
    const double h19_4_0 = h29_1_0 + ABx * h19_1_0;
    const double h19_10_0 = h29_4_0 + ABx * h19_4_0;
    const double h44_2_0 = acc[59] + ABy * acc[34];
    const double h29_2_0 = acc[38] + ABy * acc[19];
    const double h29_5_0 = h44_2_0 + ABx * h29_2_0;
    const double h19_2_0 = acc[23] + ABy * acc[9];
    const double h19_5_0 = h29_2_0 + ABx * h19_2_0;
    const double h19_11_0 = h29_5_0 + ABx * h19_5_0;
    const double h19_3_0 = acc[24] + ABz * acc[9];
    const double h19_6_0 = h29_3_0 + ABx * h19_3_0;
    const double h19_12_0 = h29_6_0 + ABx * h19_6_0;
    const double h48_2_0 = acc[64] + ABy * acc[38];
    const double h33_2_0 = acc[43] + ABy * acc[23];
    const double h33_5_0 = h48_2_0 + ABx * h33_2_0;
    const double h19_13_0 = h33_5_0 + ABy * h19_5_0;
    const double h34_3_0 = acc[45] + ABz * acc[24];
    const double h34_6_0 = h49_3_0 + ABx * h34_3_0;
    const double h19_14_0 = h34_6_0 + ABz * h19_6_0;
    const double h19_8_0 = h33_3_0 + ABy * h19_3_0;
    const double h19_15_0 = h29_8_0 + ABx * h19_8_0;
    const double h53_2_0 = acc[70] + ABy * acc[43];
    const double h33_7_0 = h53_2_0 + ABy * h33_2_0;
    const double h19_7_0 = h33_2_0 + ABy * h19_2_0;
    const double h19_16_0 = h33_7_0 + ABy * h19_7_0;
    const double h19_17_0 = h33_8_0 + ABy * h19_8_0;
    const double h34_8_0 = h54_3_0 + ABy * h34_3_0;
    const double h19_18_0 = h34_8_0 + ABz * h19_8_0;
    const double h55_3_0 = acc[73] + ABz * acc[45];
    const double h34_9_0 = h55_3_0 + ABz * h34_3_0;
    const double h19_9_0 = h34_3_0 + ABz * h19_3_0;
    const double h19_19_0 = h34_9_0 + ABz * h19_9_0;
    res[0] = h10_10_0 * 0.06666666666666665;
    res[1] = h10_11_0 * 0.14907119849998599;
    res[2] = h10_12_0 * 0.14907119849998599;
    res[3] = h10_13_0 * 0.14907119849998599;
    res[4] = h10_14_0 * 0.14907119849998599;
    res[5] = h10_15_0 * 0.2581988897471611;
    res[6] = h10_16_0 * 0.06666666666666665;
    res[7] = h10_17_0 * 0.14907119849998599;
    res[8] = h10_18_0 * 0.14907119849998599;
    res[9] = h10_19_0 * 0.06666666666666665;
    res[10] = h11_10_0 * 0.14907119849998599;
    res[11] = h11_11_0 * 0.3333333333333334;
    res[12] = h11_12_0 * 0.3333333333333334;
    res[13] = h11_13_0 * 0.3333333333333334;
    res[14] = h11_14_0 * 0.3333333333333334;
    res[15] = h11_15_0 * 0.5773502691896258;
    res[16] = h11_16_0 * 0.14907119849998599;
    res[17] = h11_17_0 * 0.3333333333333334;
    res[18] = h11_18_0 * 0.3333333333333334;
    res[19] = h11_19_0 * 0.14907119849998599;
    res[20] = h12_10_0 * 0.14907119849998599;
    res[21] = h12_11_0 * 0.3333333333333334;
    res[22] = h12_12_0 * 0.3333333333333334;
    res[23] = h12_13_0 * 0.3333333333333334;
    res[24] = h12_14_0 * 0.3333333333333334;
    res[25] = h12_15_0 * 0.5773502691896258;
    res[26] = h12_16_0 * 0.14907119849998599;
    res[27] = h12_17_0 * 0.3333333333333334;
    res[28] = h12_18_0 * 0.3333333333333334;
    res[29] = h12_19_0 * 0.14907119849998599;
    res[30] = h13_10_0 * 0.14907119849998599;
    res[31] = h13_11_0 * 0.3333333333333334;
    res[32] = h13_12_0 * 0.3333333333333334;
    res[33] = h13_13_0 * 0.3333333333333334;
    res[34] = h13_14_0 * 0.3333333333333334;
    res[35] = h13_15_0 * 0.5773502691896258;
    res[36] = h13_16_0 * 0.14907119849998599;
    res[37] = h13_17_0 * 0.3333333333333334;
    res[38] = h13_18_0 * 0.3333333333333334;
    res[39] = h13_19_0 * 0.14907119849998599;
    res[40] = h14_10_0 * 0.14907119849998599;
    res[41] = h14_11_0 * 0.3333333333333334;
    res[42] = h14_12_0 * 0.3333333333333334;
    res[43] = h14_13_0 * 0.3333333333333334;
    res[44] = h14_14_0 * 0.3333333333333334;
    res[45] = h14_15_0 * 0.5773502691896258;
    res[46] = h14_16_0 * 0.14907119849998599;
    res[47] = h14_17_0 * 0.3333333333333334;
    res[48] = h14_18_0 * 0.3333333333333334;
    res[49] = h14_19_0 * 0.14907119849998599;
    res[50] = h15_10_0 * 0.2581988897471611;
    res[51] = h15_11_0 * 0.5773502691896258;
    res[52] = h15_12_0 * 0.5773502691896258;
    res[53] = h15_13_0 * 0.5773502691896258;
    res[54] = h15_14_0 * 0.5773502691896258;
    res[55] = h15_15_0;
    res[56] = h15_16_0 * 0.2581988897471611;
    res[57] = h15_17_0 * 0.5773502691896258;
    res[58] = h15_18_0 * 0.5773502691896258;
    res[59] = h15_19_0 * 0.2581988897471611;
    res[60] = h16_10_0 * 0.06666666666666665;
    res[61] = h16_11_0 * 0.14907119849998599;
    res[62] = h16_12_0 * 0.14907119849998599;
    res[63] = h16_13_0 * 0.14907119849998599;
    res[64] = h16_14_0 * 0.14907119849998599;
    res[65] = h16_15_0 * 0.2581988897471611;
    res[66] = h16_16_0 * 0.06666666666666665;
    res[67] = h16_17_0 * 0.14907119849998599;
    res[68] = h16_18_0 * 0.14907119849998599;
    res[69] = h16_19_0 * 0.06666666666666665;
    res[70] = h17_10_0 * 0.14907119849998599;
    res[71] = h17_11_0 * 0.3333333333333334;
    res[72] = h17_12_0 * 0.3333333333333334;
    res[73] = h17_13_0 * 0.3333333333333334;
    res[74] = h17_14_0 * 0.3333333333333334;
    res[75] = h17_15_0 * 0.5773502691896258;
    res[76] = h17_16_0 * 0.14907119849998599;
    res[77] = h17_17_0 * 0.3333333333333334;
    res[78] = h17_18_0 * 0.3333333333333334;
    res[79] = h17_19_0 * 0.14907119849998599;
    res[80] = h18_10_0 * 0.14907119849998599;
    res[81] = h18_11_0 * 0.3333333333333334;
    res[82] = h18_12_0 * 0.3333333333333334;
    res[83] = h18_13_0 * 0.3333333333333334;
    res[84] = h18_14_0 * 0.3333333333333334;
    res[85] = h18_15_0 * 0.5773502691896258;
    res[86] = h18_16_0 * 0.14907119849998599;
    res[87] = h18_17_0 * 0.3333333333333334;
    res[88] = h18_18_0 * 0.3333333333333334;
    res[89] = h18_19_0 * 0.14907119849998599;
    res[90] = h19_10_0 * 0.06666666666666665;
    res[91] = h19_11_0 * 0.14907119849998599;
    res[92] = h19_12_0 * 0.14907119849998599;
    res[93] = h19_13_0 * 0.14907119849998599;
    res[94] = h19_14_0 * 0.14907119849998599;
    res[95] = h19_15_0 * 0.2581988897471611;
    res[96] = h19_16_0 * 0.06666666666666665;
    res[97] = h19_17_0 * 0.14907119849998599;
    res[98] = h19_18_0 * 0.14907119849998599;
    res[99] = h19_19_0 * 0.06666666666666665;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[100]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_ffss(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[74];
    vrr_ffss<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 74; ++x) acc_out[x] = acc[x];
    }
    hrr_ffss(P, p, q, acc, res);
}

__device__ __forceinline__ void store_ffss(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
    const long long ij_0_0 = pair_index(ib_.z + 0, ib_.w + 0);
    const long long ij_0_1 = pair_index(ib_.z + 0, ib_.w + 1);
    const long long ij_0_2 = pair_index(ib_.z + 0, ib_.w + 2);
    const long long ij_0_3 = pair_index(ib_.z + 0, ib_.w + 3);
    const long long ij_0_4 = pair_index(ib_.z + 0, ib_.w + 4);
    const long long ij_0_5 = pair_index(ib_.z + 0, ib_.w + 5);
    const long long ij_0_6 = pair_index(ib_.z + 0, ib_.w + 6);
    const long long ij_0_7 = pair_index(ib_.z + 0, ib_.w + 7);
    const long long ij_0_8 = pair_index(ib_.z + 0, ib_.w + 8);
    const long long ij_0_9 = pair_index(ib_.z + 0, ib_.w + 9);
    const long long ij_1_0 = pair_index(ib_.z + 1, ib_.w + 0);
    const long long ij_1_1 = pair_index(ib_.z + 1, ib_.w + 1);
    const long long ij_1_2 = pair_index(ib_.z + 1, ib_.w + 2);
    const long long ij_1_3 = pair_index(ib_.z + 1, ib_.w + 3);
    const long long ij_1_4 = pair_index(ib_.z + 1, ib_.w + 4);
    const long long ij_1_5 = pair_index(ib_.z + 1, ib_.w + 5);
    const long long ij_1_6 = pair_index(ib_.z + 1, ib_.w + 6);
    const long long ij_1_7 = pair_index(ib_.z + 1, ib_.w + 7);
    const long long ij_1_8 = pair_index(ib_.z + 1, ib_.w + 8);
    const long long ij_1_9 = pair_index(ib_.z + 1, ib_.w + 9);
    const long long ij_2_0 = pair_index(ib_.z + 2, ib_.w + 0);
    const long long ij_2_1 = pair_index(ib_.z + 2, ib_.w + 1);
    const long long ij_2_2 = pair_index(ib_.z + 2, ib_.w + 2);
    const long long ij_2_3 = pair_index(ib_.z + 2, ib_.w + 3);
    const long long ij_2_4 = pair_index(ib_.z + 2, ib_.w + 4);
    const long long ij_2_5 = pair_index(ib_.z + 2, ib_.w + 5);
    const long long ij_2_6 = pair_index(ib_.z + 2, ib_.w + 6);
    const long long ij_2_7 = pair_index(ib_.z + 2, ib_.w + 7);
    const long long ij_2_8 = pair_index(ib_.z + 2, ib_.w + 8);
    const long long ij_2_9 = pair_index(ib_.z + 2, ib_.w + 9);
    const long long ij_3_0 = pair_index(ib_.z + 3, ib_.w + 0);
    const long long ij_3_1 = pair_index(ib_.z + 3, ib_.w + 1);
    const long long ij_3_2 = pair_index(ib_.z + 3, ib_.w + 2);
    const long long ij_3_3 = pair_index(ib_.z + 3, ib_.w + 3);
    const long long ij_3_4 = pair_index(ib_.z + 3, ib_.w + 4);
    const long long ij_3_5 = pair_index(ib_.z + 3, ib_.w + 5);
    const long long ij_3_6 = pair_index(ib_.z + 3, ib_.w + 6);
    const long long ij_3_7 = pair_index(ib_.z + 3, ib_.w + 7);
    const long long ij_3_8 = pair_index(ib_.z + 3, ib_.w + 8);
    const long long ij_3_9 = pair_index(ib_.z + 3, ib_.w + 9);
    const long long ij_4_0 = pair_index(ib_.z + 4, ib_.w + 0);
    const long long ij_4_1 = pair_index(ib_.z + 4, ib_.w + 1);
    const long long ij_4_2 = pair_index(ib_.z + 4, ib_.w + 2);
    const long long ij_4_3 = pair_index(ib_.z + 4, ib_.w + 3);
    const long long ij_4_4 = pair_index(ib_.z + 4, ib_.w + 4);
    const long long ij_4_5 = pair_index(ib_.z + 4, ib_.w + 5);
    const long long ij_4_6 = pair_index(ib_.z + 4, ib_.w + 6);
    const long long ij_4_7 = pair_index(ib_.z + 4, ib_.w + 7);
    const long long ij_4_8 = pair_index(ib_.z + 4, ib_.w + 8);
    const long long ij_4_9 = pair_index(ib_.z + 4, ib_.w + 9);
    const long long ij_5_0 = pair_index(ib_.z + 5, ib_.w + 0);
    const long long ij_5_1 = pair_index(ib_.z + 5, ib_.w + 1);
    const long long ij_5_2 = pair_index(ib_.z + 5, ib_.w + 2);
    const long long ij_5_3 = pair_index(ib_.z + 5, ib_.w + 3);
    const long long ij_5_4 = pair_index(ib_.z + 5, ib_.w + 4);
    const long long ij_5_5 = pair_index(ib_.z + 5, ib_.w + 5);
    const long long ij_5_6 = pair_index(ib_.z + 5, ib_.w + 6);
    const long long ij_5_7 = pair_index(ib_.z + 5, ib_.w + 7);
    const long long ij_5_8 = pair_index(ib_.z + 5, ib_.w + 8);
    const long long ij_5_9 = pair_index(ib_.z + 5, ib_.w + 9);
    const long long ij_6_0 = pair_index(ib_.z + 6, ib_.w + 0);
    const long long ij_6_1 = pair_index(ib_.z + 6, ib_.w + 1);
    const long long ij_6_2 = pair_index(ib_.z + 6, ib_.w + 2);
    const long long ij_6_3 = pair_index(ib_.z + 6, ib_.w + 3);
    const long long ij_6_4 = pair_index(ib_.z + 6, ib_.w + 4);
    const long long ij_6_5 = pair_index(ib_.z + 6, ib_.w + 5);
    const long long ij_6_6 = pair_index(ib_.z + 6, ib_.w + 6);
    const long long ij_6_7 = pair_index(ib_.z + 6, ib_.w + 7);
    const long long ij_6_8 = pair_index(ib_.z + 6, ib_.w + 8);
    const long long ij_6_9 = pair_index(ib_.z + 6, ib_.w + 9);
    const long long ij_7_0 = pair_index(ib_.z + 7, ib_.w + 0);
    const long long ij_7_1 = pair_index(ib_.z + 7, ib_.w + 1);
    const long long ij_7_2 = pair_index(ib_.z + 7, ib_.w + 2);
    const long long ij_7_3 = pair_index(ib_.z + 7, ib_.w + 3);
    const long long ij_7_4 = pair_index(ib_.z + 7, ib_.w + 4);
    const long long ij_7_5 = pair_index(ib_.z + 7, ib_.w + 5);
    const long long ij_7_6 = pair_index(ib_.z + 7, ib_.w + 6);
    const long long ij_7_7 = pair_index(ib_.z + 7, ib_.w + 7);
    const long long ij_7_8 = pair_index(ib_.z + 7, ib_.w + 8);
    const long long ij_7_9 = pair_index(ib_.z + 7, ib_.w + 9);
    const long long ij_8_0 = pair_index(ib_.z + 8, ib_.w + 0);
    const long long ij_8_1 = pair_index(ib_.z + 8, ib_.w + 1);
    const long long ij_8_2 = pair_index(ib_.z + 8, ib_.w + 2);
    const long long ij_8_3 = pair_index(ib_.z + 8, ib_.w + 3);
    const long long ij_8_4 = pair_index(ib_.z + 8, ib_.w + 4);
    const long long ij_8_5 = pair_index(ib_.z + 8, ib_.w + 5);
    const long long ij_8_6 = pair_index(ib_.z + 8, ib_.w + 6);
    const long long ij_8_7 = pair_index(ib_.z + 8, ib_.w + 7);
    const long long ij_8_8 = pair_index(ib_.z + 8, ib_.w + 8);
    const long long ij_8_9 = pair_index(ib_.z + 8, ib_.w + 9);
    const long long ij_9_0 = pair_index(ib_.z + 9, ib_.w + 0);
    const long long ij_9_1 = pair_index(ib_.z + 9, ib_.w + 1);
    const long long ij_9_2 = pair_index(ib_.z + 9, ib_.w + 2);
    const long long ij_9_3 = pair_index(ib_.z + 9, ib_.w + 3);
    const long long ij_9_4 = pair_index(ib_.z + 9, ib_.w + 4);
    const long long ij_9_5 = pair_index(ib_.z + 9, ib_.w + 5);
    const long long ij_9_6 = pair_index(ib_.z + 9, ib_.w + 6);
    const long long ij_9_7 = pair_index(ib_.z + 9, ib_.w + 7);
    const long long ij_9_8 = pair_index(ib_.z + 9, ib_.w + 8);
    const long long ij_9_9 = pair_index(ib_.z + 9, ib_.w + 9);
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_3, kl = kl_0_0;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_4, kl = kl_0_0;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_5, kl = kl_0_0;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_6, kl = kl_0_0;
      if ((!dab || 0 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_7, kl = kl_0_0;
      if ((!dab || 0 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_8, kl = kl_0_0;
      if ((!dab || 0 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_0_9, kl = kl_0_0;
      if ((!dab || 0 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_1_3, kl = kl_0_0;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_1_4, kl = kl_0_0;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_1_5, kl = kl_0_0;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_1_6, kl = kl_0_0;
      if ((!dab || 1 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_1_7, kl = kl_0_0;
      if ((!dab || 1 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_1_8, kl = kl_0_0;
      if ((!dab || 1 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_1_9, kl = kl_0_0;
      if ((!dab || 1 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_2_3, kl = kl_0_0;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_2_4, kl = kl_0_0;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_2_5, kl = kl_0_0;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_2_6, kl = kl_0_0;
      if ((!dab || 2 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_2_7, kl = kl_0_0;
      if ((!dab || 2 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_2_8, kl = kl_0_0;
      if ((!dab || 2 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_2_9, kl = kl_0_0;
      if ((!dab || 2 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_3_3, kl = kl_0_0;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_3_4, kl = kl_0_0;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_3_5, kl = kl_0_0;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_3_6, kl = kl_0_0;
      if ((!dab || 3 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_3_7, kl = kl_0_0;
      if ((!dab || 3 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_3_8, kl = kl_0_0;
      if ((!dab || 3 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_3_9, kl = kl_0_0;
      if ((!dab || 3 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_4_3, kl = kl_0_0;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_4_4, kl = kl_0_0;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_4_5, kl = kl_0_0;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_4_6, kl = kl_0_0;
      if ((!dab || 4 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_4_7, kl = kl_0_0;
      if ((!dab || 4 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_4_8, kl = kl_0_0;
      if ((!dab || 4 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_4_9, kl = kl_0_0;
      if ((!dab || 4 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_5_3, kl = kl_0_0;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_5_4, kl = kl_0_0;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_5_5, kl = kl_0_0;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_5_6, kl = kl_0_0;
      if ((!dab || 5 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_5_7, kl = kl_0_0;
      if ((!dab || 5 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_5_8, kl = kl_0_0;
      if ((!dab || 5 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_5_9, kl = kl_0_0;
      if ((!dab || 5 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if ((!dab || 6 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_6_1, kl = kl_0_0;
      if ((!dab || 6 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_6_2, kl = kl_0_0;
      if ((!dab || 6 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_6_3, kl = kl_0_0;
      if ((!dab || 6 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_6_4, kl = kl_0_0;
      if ((!dab || 6 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_6_5, kl = kl_0_0;
      if ((!dab || 6 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_6_6, kl = kl_0_0;
      if ((!dab || 6 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_6_7, kl = kl_0_0;
      if ((!dab || 6 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_6_8, kl = kl_0_0;
      if ((!dab || 6 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_6_9, kl = kl_0_0;
      if ((!dab || 6 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if ((!dab || 7 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_7_1, kl = kl_0_0;
      if ((!dab || 7 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_7_2, kl = kl_0_0;
      if ((!dab || 7 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_7_3, kl = kl_0_0;
      if ((!dab || 7 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_7_4, kl = kl_0_0;
      if ((!dab || 7 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_7_5, kl = kl_0_0;
      if ((!dab || 7 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_7_6, kl = kl_0_0;
      if ((!dab || 7 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_7_7, kl = kl_0_0;
      if ((!dab || 7 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_7_8, kl = kl_0_0;
      if ((!dab || 7 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_7_9, kl = kl_0_0;
      if ((!dab || 7 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if ((!dab || 8 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_8_1, kl = kl_0_0;
      if ((!dab || 8 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_8_2, kl = kl_0_0;
      if ((!dab || 8 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_8_3, kl = kl_0_0;
      if ((!dab || 8 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_8_4, kl = kl_0_0;
      if ((!dab || 8 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_8_5, kl = kl_0_0;
      if ((!dab || 8 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_8_6, kl = kl_0_0;
      if ((!dab || 8 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_8_7, kl = kl_0_0;
      if ((!dab || 8 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_8_8, kl = kl_0_0;
      if ((!dab || 8 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_8_9, kl = kl_0_0;
      if ((!dab || 8 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if ((!dab || 9 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_9_1, kl = kl_0_0;
      if ((!dab || 9 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_9_2, kl = kl_0_0;
      if ((!dab || 9 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_9_3, kl = kl_0_0;
      if ((!dab || 9 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_9_4, kl = kl_0_0;
      if ((!dab || 9 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_9_5, kl = kl_0_0;
      if ((!dab || 9 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_9_6, kl = kl_0_0;
      if ((!dab || 9 >= 6) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_9_7, kl = kl_0_0;
      if ((!dab || 9 >= 7) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_9_8, kl = kl_0_0;
      if ((!dab || 9 >= 8) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_9_9, kl = kl_0_0;
      if ((!dab || 9 >= 9) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_ffss(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 100; ++x) {
        const int ia = x / 10, ibb = (x / 1) % 10, ic = (x / 1) % 1, id = x % 1;
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
__global__ void __launch_bounds__(128) eri_queue_ffss(const EriQueue Q) {
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
        double acc[74];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 74; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_ffss<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_ffss<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 74; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 100 doubles (launch_eri_ffss)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 100);
            if (lead) hrr_ffss(Q.pairs, p, q, acc, sb + kq * 100);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)100;
            for (int t = lane; t < nlive * 100; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[100];
            hrr_ffss(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_ffss(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_ffss(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (102400 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_ffss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_ffss<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 102400);
        cudaFuncSetAttribute(eri_queue_ffss<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 102400);
        done[dev] = true;
    }
}

void launch_eri_ffss(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 102400 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 102400 : 0;
    if (smem) eri_prepare_ffss();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_ffss<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_ffss<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_ffss<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_ffss<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_ffss(int mixed) {
    eri_prepare_ffss();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_ffss<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_ffss<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

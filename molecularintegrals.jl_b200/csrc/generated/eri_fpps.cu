// Generated by gen_eri.py -- class (fp|ps).  Do not edit.
// VRR entries: 180, contracted block: 75, HRR lines: 90, outputs: 90.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[75], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_fpps(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 75; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[6];
            boys_fm<5>(T, B, F);
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
            const VT v1_0_0 = PAx * v0_0_0 + WPx * v0_0_1;
            const VT v1_0_1 = PAx * v0_0_1 + WPx * v0_0_2;
            const VT v1_0_2 = PAx * v0_0_2 + WPx * v0_0_3;
            const VT v1_0_3 = PAx * v0_0_3 + WPx * v0_0_4;
            const VT v1_0_4 = PAx * v0_0_4 + WPx * v0_0_5;
            const VT v2_0_0 = PAy * v0_0_0 + WPy * v0_0_1;
            const VT v2_0_1 = PAy * v0_0_1 + WPy * v0_0_2;
            const VT v2_0_2 = PAy * v0_0_2 + WPy * v0_0_3;
            const VT v2_0_3 = PAy * v0_0_3 + WPy * v0_0_4;
            const VT v2_0_4 = PAy * v0_0_4 + WPy * v0_0_5;
            const VT v3_0_0 = PAz * v0_0_0 + WPz * v0_0_1;
            const VT v3_0_1 = PAz * v0_0_1 + WPz * v0_0_2;
            const VT v3_0_2 = PAz * v0_0_2 + WPz * v0_0_3;
            const VT v3_0_3 = PAz * v0_0_3 + WPz * v0_0_4;
            const VT v3_0_4 = PAz * v0_0_4 + WPz * v0_0_5;
            const VT v4_0_0 = PAx * v1_0_0 + WPx * v1_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v4_0_1 = PAx * v1_0_1 + WPx * v1_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v4_0_2 = PAx * v1_0_2 + WPx * v1_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v4_0_3 = PAx * v1_0_3 + WPx * v1_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v5_0_0 = PAx * v2_0_0 + WPx * v2_0_1;
            const VT v5_0_1 = PAx * v2_0_1 + WPx * v2_0_2;
            const VT v5_0_2 = PAx * v2_0_2 + WPx * v2_0_3;
            const VT v5_0_3 = PAx * v2_0_3 + WPx * v2_0_4;
            const VT v6_0_0 = PAx * v3_0_0 + WPx * v3_0_1;
            const VT v6_0_1 = PAx * v3_0_1 + WPx * v3_0_2;
            const VT v6_0_2 = PAx * v3_0_2 + WPx * v3_0_3;
            const VT v6_0_3 = PAx * v3_0_3 + WPx * v3_0_4;
            const VT v7_0_0 = PAy * v2_0_0 + WPy * v2_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v7_0_1 = PAy * v2_0_1 + WPy * v2_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v7_0_2 = PAy * v2_0_2 + WPy * v2_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v7_0_3 = PAy * v2_0_3 + WPy * v2_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v8_0_0 = PAy * v3_0_0 + WPy * v3_0_1;
            const VT v8_0_1 = PAy * v3_0_1 + WPy * v3_0_2;
            const VT v8_0_2 = PAy * v3_0_2 + WPy * v3_0_3;
            const VT v8_0_3 = PAy * v3_0_3 + WPy * v3_0_4;
            const VT v9_0_0 = PAz * v3_0_0 + WPz * v3_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v9_0_1 = PAz * v3_0_1 + WPz * v3_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v9_0_2 = PAz * v3_0_2 + WPz * v3_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v9_0_3 = PAz * v3_0_3 + WPz * v3_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v10_0_0 = PAx * v4_0_0 + WPx * v4_0_1 + (VT)2.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v10_0_1 = PAx * v4_0_1 + WPx * v4_0_2 + (VT)2.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v10_0_2 = PAx * v4_0_2 + WPx * v4_0_3 + (VT)2.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v11_0_0 = PAx * v5_0_0 + WPx * v5_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v11_0_1 = PAx * v5_0_1 + WPx * v5_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v11_0_2 = PAx * v5_0_2 + WPx * v5_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v12_0_0 = PAx * v6_0_0 + WPx * v6_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v12_0_1 = PAx * v6_0_1 + WPx * v6_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v12_0_2 = PAx * v6_0_2 + WPx * v6_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v13_0_0 = PAy * v5_0_0 + WPy * v5_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v13_0_1 = PAy * v5_0_1 + WPy * v5_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v13_0_2 = PAy * v5_0_2 + WPy * v5_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v14_0_0 = PAz * v6_0_0 + WPz * v6_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v14_0_1 = PAz * v6_0_1 + WPz * v6_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v14_0_2 = PAz * v6_0_2 + WPz * v6_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v15_0_0 = PAx * v8_0_0 + WPx * v8_0_1;
            const VT v15_0_1 = PAx * v8_0_1 + WPx * v8_0_2;
            const VT v15_0_2 = PAx * v8_0_2 + WPx * v8_0_3;
            const VT v16_0_0 = PAy * v7_0_0 + WPy * v7_0_1 + (VT)2.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v16_0_1 = PAy * v7_0_1 + WPy * v7_0_2 + (VT)2.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v16_0_2 = PAy * v7_0_2 + WPy * v7_0_3 + (VT)2.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v17_0_0 = PAy * v8_0_0 + WPy * v8_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v17_0_1 = PAy * v8_0_1 + WPy * v8_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v17_0_2 = PAy * v8_0_2 + WPy * v8_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v18_0_0 = PAz * v8_0_0 + WPz * v8_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v18_0_1 = PAz * v8_0_1 + WPz * v8_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v18_0_2 = PAz * v8_0_2 + WPz * v8_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v19_0_0 = PAz * v9_0_0 + WPz * v9_0_1 + (VT)2.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v19_0_1 = PAz * v9_0_1 + WPz * v9_0_2 + (VT)2.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v19_0_2 = PAz * v9_0_2 + WPz * v9_0_3 + (VT)2.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v20_0_0 = PAx * v10_0_0 + WPx * v10_0_1 + (VT)3.0 * oo2z * (v4_0_0 - rho_z * v4_0_1);
            const VT v20_0_1 = PAx * v10_0_1 + WPx * v10_0_2 + (VT)3.0 * oo2z * (v4_0_1 - rho_z * v4_0_2);
            const VT v21_0_0 = PAx * v11_0_0 + WPx * v11_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v21_0_1 = PAx * v11_0_1 + WPx * v11_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v22_0_0 = PAx * v12_0_0 + WPx * v12_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v22_0_1 = PAx * v12_0_1 + WPx * v12_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v23_0_0 = PAx * v13_0_0 + WPx * v13_0_1 + (VT)1.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v23_0_1 = PAx * v13_0_1 + WPx * v13_0_2 + (VT)1.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v24_0_0 = PAx * v15_0_0 + WPx * v15_0_1 + (VT)1.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v24_0_1 = PAx * v15_0_1 + WPx * v15_0_2 + (VT)1.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v25_0_0 = PAx * v14_0_0 + WPx * v14_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v25_0_1 = PAx * v14_0_1 + WPx * v14_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v26_0_0 = PAy * v13_0_0 + WPy * v13_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v26_0_1 = PAy * v13_0_1 + WPy * v13_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v27_0_0 = PAy * v15_0_0 + WPy * v15_0_1 + (VT)1.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v27_0_1 = PAy * v15_0_1 + WPy * v15_0_2 + (VT)1.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v28_0_0 = PAz * v15_0_0 + WPz * v15_0_1 + (VT)1.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v28_0_1 = PAz * v15_0_1 + WPz * v15_0_2 + (VT)1.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v29_0_0 = PAz * v14_0_0 + WPz * v14_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v29_0_1 = PAz * v14_0_1 + WPz * v14_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v30_0_0 = PAy * v16_0_0 + WPy * v16_0_1 + (VT)3.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v30_0_1 = PAy * v16_0_1 + WPy * v16_0_2 + (VT)3.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v31_0_0 = PAy * v17_0_0 + WPy * v17_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v31_0_1 = PAy * v17_0_1 + WPy * v17_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v32_0_0 = PAy * v18_0_0 + WPy * v18_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v32_0_1 = PAy * v18_0_1 + WPy * v18_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v33_0_0 = PAz * v18_0_0 + WPz * v18_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v33_0_1 = PAz * v18_0_1 + WPz * v18_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v34_0_0 = PAz * v19_0_0 + WPz * v19_0_1 + (VT)3.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v34_0_1 = PAz * v19_0_1 + WPz * v19_0_2 + (VT)3.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v10_1_0 = QCx * v10_0_0 + WQx * v10_0_1 + (VT)3.0 * oo2ze * v4_0_1;
            const VT v11_1_0 = QCx * v11_0_0 + WQx * v11_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v12_1_0 = QCx * v12_0_0 + WQx * v12_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v13_1_0 = QCx * v13_0_0 + WQx * v13_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v14_1_0 = QCx * v14_0_0 + WQx * v14_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v15_1_0 = QCx * v15_0_0 + WQx * v15_0_1 + (VT)1.0 * oo2ze * v8_0_1;
            const VT v16_1_0 = QCx * v16_0_0 + WQx * v16_0_1;
            const VT v17_1_0 = QCx * v17_0_0 + WQx * v17_0_1;
            const VT v18_1_0 = QCx * v18_0_0 + WQx * v18_0_1;
            const VT v19_1_0 = QCx * v19_0_0 + WQx * v19_0_1;
            const VT v20_1_0 = QCx * v20_0_0 + WQx * v20_0_1 + (VT)4.0 * oo2ze * v10_0_1;
            const VT v21_1_0 = QCx * v21_0_0 + WQx * v21_0_1 + (VT)3.0 * oo2ze * v11_0_1;
            const VT v22_1_0 = QCx * v22_0_0 + WQx * v22_0_1 + (VT)3.0 * oo2ze * v12_0_1;
            const VT v23_1_0 = QCx * v23_0_0 + WQx * v23_0_1 + (VT)2.0 * oo2ze * v13_0_1;
            const VT v24_1_0 = QCx * v24_0_0 + WQx * v24_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v25_1_0 = QCx * v25_0_0 + WQx * v25_0_1 + (VT)2.0 * oo2ze * v14_0_1;
            const VT v26_1_0 = QCx * v26_0_0 + WQx * v26_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v27_1_0 = QCx * v27_0_0 + WQx * v27_0_1 + (VT)1.0 * oo2ze * v17_0_1;
            const VT v28_1_0 = QCx * v28_0_0 + WQx * v28_0_1 + (VT)1.0 * oo2ze * v18_0_1;
            const VT v29_1_0 = QCx * v29_0_0 + WQx * v29_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v30_1_0 = QCx * v30_0_0 + WQx * v30_0_1;
            const VT v31_1_0 = QCx * v31_0_0 + WQx * v31_0_1;
            const VT v32_1_0 = QCx * v32_0_0 + WQx * v32_0_1;
            const VT v33_1_0 = QCx * v33_0_0 + WQx * v33_0_1;
            const VT v34_1_0 = QCx * v34_0_0 + WQx * v34_0_1;
            const VT v10_2_0 = QCy * v10_0_0 + WQy * v10_0_1;
            const VT v11_2_0 = QCy * v11_0_0 + WQy * v11_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v12_2_0 = QCy * v12_0_0 + WQy * v12_0_1;
            const VT v13_2_0 = QCy * v13_0_0 + WQy * v13_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v14_2_0 = QCy * v14_0_0 + WQy * v14_0_1;
            const VT v15_2_0 = QCy * v15_0_0 + WQy * v15_0_1 + (VT)1.0 * oo2ze * v6_0_1;
            const VT v16_2_0 = QCy * v16_0_0 + WQy * v16_0_1 + (VT)3.0 * oo2ze * v7_0_1;
            const VT v17_2_0 = QCy * v17_0_0 + WQy * v17_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v18_2_0 = QCy * v18_0_0 + WQy * v18_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v19_2_0 = QCy * v19_0_0 + WQy * v19_0_1;
            const VT v20_2_0 = QCy * v20_0_0 + WQy * v20_0_1;
            const VT v21_2_0 = QCy * v21_0_0 + WQy * v21_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v22_2_0 = QCy * v22_0_0 + WQy * v22_0_1;
            const VT v23_2_0 = QCy * v23_0_0 + WQy * v23_0_1 + (VT)2.0 * oo2ze * v11_0_1;
            const VT v24_2_0 = QCy * v24_0_0 + WQy * v24_0_1 + (VT)1.0 * oo2ze * v12_0_1;
            const VT v25_2_0 = QCy * v25_0_0 + WQy * v25_0_1;
            const VT v26_2_0 = QCy * v26_0_0 + WQy * v26_0_1 + (VT)3.0 * oo2ze * v13_0_1;
            const VT v27_2_0 = QCy * v27_0_0 + WQy * v27_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v28_2_0 = QCy * v28_0_0 + WQy * v28_0_1 + (VT)1.0 * oo2ze * v14_0_1;
            const VT v29_2_0 = QCy * v29_0_0 + WQy * v29_0_1;
            const VT v30_2_0 = QCy * v30_0_0 + WQy * v30_0_1 + (VT)4.0 * oo2ze * v16_0_1;
            const VT v31_2_0 = QCy * v31_0_0 + WQy * v31_0_1 + (VT)3.0 * oo2ze * v17_0_1;
            const VT v32_2_0 = QCy * v32_0_0 + WQy * v32_0_1 + (VT)2.0 * oo2ze * v18_0_1;
            const VT v33_2_0 = QCy * v33_0_0 + WQy * v33_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v34_2_0 = QCy * v34_0_0 + WQy * v34_0_1;
            const VT v10_3_0 = QCz * v10_0_0 + WQz * v10_0_1;
            const VT v11_3_0 = QCz * v11_0_0 + WQz * v11_0_1;
            const VT v12_3_0 = QCz * v12_0_0 + WQz * v12_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v13_3_0 = QCz * v13_0_0 + WQz * v13_0_1;
            const VT v14_3_0 = QCz * v14_0_0 + WQz * v14_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v15_3_0 = QCz * v15_0_0 + WQz * v15_0_1 + (VT)1.0 * oo2ze * v5_0_1;
            const VT v16_3_0 = QCz * v16_0_0 + WQz * v16_0_1;
            const VT v17_3_0 = QCz * v17_0_0 + WQz * v17_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v18_3_0 = QCz * v18_0_0 + WQz * v18_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v19_3_0 = QCz * v19_0_0 + WQz * v19_0_1 + (VT)3.0 * oo2ze * v9_0_1;
            const VT v20_3_0 = QCz * v20_0_0 + WQz * v20_0_1;
            const VT v21_3_0 = QCz * v21_0_0 + WQz * v21_0_1;
            const VT v22_3_0 = QCz * v22_0_0 + WQz * v22_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v23_3_0 = QCz * v23_0_0 + WQz * v23_0_1;
            const VT v24_3_0 = QCz * v24_0_0 + WQz * v24_0_1 + (VT)1.0 * oo2ze * v11_0_1;
            const VT v25_3_0 = QCz * v25_0_0 + WQz * v25_0_1 + (VT)2.0 * oo2ze * v12_0_1;
            const VT v26_3_0 = QCz * v26_0_0 + WQz * v26_0_1;
            const VT v27_3_0 = QCz * v27_0_0 + WQz * v27_0_1 + (VT)1.0 * oo2ze * v13_0_1;
            const VT v28_3_0 = QCz * v28_0_0 + WQz * v28_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v29_3_0 = QCz * v29_0_0 + WQz * v29_0_1 + (VT)3.0 * oo2ze * v14_0_1;
            const VT v30_3_0 = QCz * v30_0_0 + WQz * v30_0_1;
            const VT v31_3_0 = QCz * v31_0_0 + WQz * v31_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v32_3_0 = QCz * v32_0_0 + WQz * v32_0_1 + (VT)2.0 * oo2ze * v17_0_1;
            const VT v33_3_0 = QCz * v33_0_0 + WQz * v33_0_1 + (VT)3.0 * oo2ze * v18_0_1;
            const VT v34_3_0 = QCz * v34_0_0 + WQz * v34_0_1 + (VT)4.0 * oo2ze * v19_0_1;
            acc[0] += (double)v10_1_0;
            acc[1] += (double)v10_2_0;
            acc[2] += (double)v10_3_0;
            acc[3] += (double)v11_1_0;
            acc[4] += (double)v11_2_0;
            acc[5] += (double)v11_3_0;
            acc[6] += (double)v12_1_0;
            acc[7] += (double)v12_2_0;
            acc[8] += (double)v12_3_0;
            acc[9] += (double)v13_1_0;
            acc[10] += (double)v13_2_0;
            acc[11] += (double)v13_3_0;
            acc[12] += (double)v14_1_0;
            acc[13] += (double)v14_2_0;
            acc[14] += (double)v14_3_0;
            acc[15] += (double)v15_1_0;
            acc[16] += (double)v15_2_0;
            acc[17] += (double)v15_3_0;
            acc[18] += (double)v16_1_0;
            acc[19] += (double)v16_2_0;
            acc[20] += (double)v16_3_0;
            acc[21] += (double)v17_1_0;
            acc[22] += (double)v17_2_0;
            acc[23] += (double)v17_3_0;
            acc[24] += (double)v18_1_0;
            acc[25] += (double)v18_2_0;
            acc[26] += (double)v18_3_0;
            acc[27] += (double)v19_1_0;
            acc[28] += (double)v19_2_0;
            acc[29] += (double)v19_3_0;
            acc[30] += (double)v20_1_0;
            acc[31] += (double)v20_2_0;
            acc[32] += (double)v20_3_0;
            acc[33] += (double)v21_1_0;
            acc[34] += (double)v21_2_0;
            acc[35] += (double)v21_3_0;
            acc[36] += (double)v22_1_0;
            acc[37] += (double)v22_2_0;
            acc[38] += (double)v22_3_0;
            acc[39] += (double)v23_1_0;
            acc[40] += (double)v23_2_0;
            acc[41] += (double)v23_3_0;
            acc[42] += (double)v24_1_0;
            acc[43] += (double)v24_2_0;
            acc[44] += (double)v24_3_0;
            acc[45] += (double)v25_1_0;
            acc[46] += (double)v25_2_0;
            acc[47] += (double)v25_3_0;
            acc[48] += (double)v26_1_0;
            acc[49] += (double)v26_2_0;
            acc[50] += (double)v26_3_0;
            acc[51] += (double)v27_1_0;
            acc[52] += (double)v27_2_0;
            acc[53] += (double)v27_3_0;
            acc[54] += (double)v28_1_0;
            acc[55] += (double)v28_2_0;
            acc[56] += (double)v28_3_0;
            acc[57] += (double)v29_1_0;
            acc[58] += (double)v29_2_0;
            acc[59] += (double)v29_3_0;
            acc[60] += (double)v30_1_0;
            acc[61] += (double)v30_2_0;
            acc[62] += (double)v30_3_0;
            acc[63] += (double)v31_1_0;
            acc[64] += (double)v31_2_0;
            acc[65] += (double)v31_3_0;
            acc[66] += (double)v32_1_0;
            acc[67] += (double)v32_2_0;
            acc[68] += (double)v32_3_0;
            acc[69] += (double)v33_1_0;
            acc[70] += (double)v33_2_0;
            acc[71] += (double)v33_3_0;
            acc[72] += (double)v34_1_0;
            acc[73] += (double)v34_2_0;
            acc[74] += (double)v34_3_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[90] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_fpps(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h10_1_1 = acc[30] + ABx * acc[0];
    const double h10_1_2 = acc[31] + ABx * acc[1];
    const double h10_1_3 = acc[32] + ABx * acc[2];
    const double h10_2_1 = acc[33] + ABy * acc[0];
    const double h10_2_2 = acc[34] + ABy * acc[1];
    const double h10_2_3 = acc[35] + ABy * acc[2];
    const double h10_3_1 = acc[36] + ABz * acc[0];
    const double h10_3_2 = acc[37] + ABz * acc[1];
    const double h10_3_3 = acc[38] + ABz * acc[2];
    const double h11_1_1 = acc[33] + ABx * acc[3];
    const double h11_1_2 = acc[34] + ABx * acc[4];
    const double h11_1_3 = acc[35] + ABx * acc[5];
    const double h11_2_1 = acc[39] + ABy * acc[3];
    const double h11_2_2 = acc[40] + ABy * acc[4];
    const double h11_2_3 = acc[41] + ABy * acc[5];
    const double h11_3_1 = acc[42] + ABz * acc[3];
    const double h11_3_2 = acc[43] + ABz * acc[4];
    const double h11_3_3 = acc[44] + ABz * acc[5];
    const double h12_1_1 = acc[36] + ABx * acc[6];
    const double h12_1_2 = acc[37] + ABx * acc[7];
    const double h12_1_3 = acc[38] + ABx * acc[8];
    const double h12_2_1 = acc[42] + ABy * acc[6];
    const double h12_2_2 = acc[43] + ABy * acc[7];
    const double h12_2_3 = acc[44] + ABy * acc[8];
    const double h12_3_1 = acc[45] + ABz * acc[6];
    const double h12_3_2 = acc[46] + ABz * acc[7];
    const double h12_3_3 = acc[47] + ABz * acc[8];
    const double h13_1_1 = acc[39] + ABx * acc[9];
    const double h13_1_2 = acc[40] + ABx * acc[10];
    const double h13_1_3 = acc[41] + ABx * acc[11];
    const double h13_2_1 = acc[48] + ABy * acc[9];
    const double h13_2_2 = acc[49] + ABy * acc[10];
    const double h13_2_3 = acc[50] + ABy * acc[11];
    const double h13_3_1 = acc[51] + ABz * acc[9];
    const double h13_3_2 = acc[52] + ABz * acc[10];
    const double h13_3_3 = acc[53] + ABz * acc[11];
    const double h14_1_1 = acc[45] + ABx * acc[12];
    const double h14_1_2 = acc[46] + ABx * acc[13];
    const double h14_1_3 = acc[47] + ABx * acc[14];
    const double h14_2_1 = acc[54] + ABy * acc[12];
    const double h14_2_2 = acc[55] + ABy * acc[13];
    const double h14_2_3 = acc[56] + ABy * acc[14];
    const double h14_3_1 = acc[57] + ABz * acc[12];
    const double h14_3_2 = acc[58] + ABz * acc[13];
    const double h14_3_3 = acc[59] + ABz * acc[14];
    const double h15_1_1 = acc[42] + ABx * acc[15];
    const double h15_1_2 = acc[43] + ABx * acc[16];
    const double h15_1_3 = acc[44] + ABx * acc[17];
    const double h15_2_1 = acc[51] + ABy * acc[15];
    const double h15_2_2 = acc[52] + ABy * acc[16];
    const double h15_2_3 = acc[53] + ABy * acc[17];
    const double h15_3_1 = acc[54] + ABz * acc[15];
    const double h15_3_2 = acc[55] + ABz * acc[16];
    const double h15_3_3 = acc[56] + ABz * acc[17];
    const double h16_1_1 = acc[48] + ABx * acc[18];
    const double h16_1_2 = acc[49] + ABx * acc[19];
    const double h16_1_3 = acc[50] + ABx * acc[20];
    const double h16_2_1 = acc[60] + ABy * acc[18];
    const double h16_2_2 = acc[61] + ABy * acc[19];
    const double h16_2_3 = acc[62] + ABy * acc[20];
    const double h16_3_1 = acc[63] + ABz * acc[18];
    const double h16_3_2 = acc[64] + ABz * acc[19];
    const double h16_3_3 = acc[65] + ABz * acc[20];
    const double h17_1_1 = acc[51] + ABx * acc[21];
    const double h17_1_2 = acc[52] + ABx * acc[22];
    const double h17_1_3 = acc[53] + ABx * acc[23];
    const double h17_2_1 = acc[63] + ABy * acc[21];
    const double h17_2_2 = acc[64] + ABy * acc[22];
    const double h17_2_3 = acc[65] + ABy * acc[23];
    const double h17_3_1 = acc[66] + ABz * acc[21];
    const double h17_3_2 = acc[67] + ABz * acc[22];
    const double h17_3_3 = acc[68] + ABz * acc[23];
    const double h18_1_1 = acc[54] + ABx * acc[24];
    const double h18_1_2 = acc[55] + ABx * acc[25];
    const double h18_1_3 = acc[56] + ABx * acc[26];
    const double h18_2_1 = acc[66] + ABy * acc[24];
    const double h18_2_2 = acc[67] + ABy * acc[25];
    const double h18_2_3 = acc[68] + ABy * acc[26];
    const double h18_3_1 = acc[69] + ABz * acc[24];
    const double h18_3_2 = acc[70] + ABz * acc[25];
    const double h18_3_3 = acc[71] + ABz * acc[26];
    const double h19_1_1 = acc[57] + ABx * acc[27];
    const double h19_1_2 = acc[58] + ABx * acc[28];
    const double h19_1_3 = acc[59] + ABx * acc[29];
    const double h19_2_1 = acc[69] + ABy * acc[27];
    const double h19_2_2 = acc[70] + ABy * acc[28];
    const double h19_2_3 = acc[71] + ABy * acc[29];
    const double h19_3_1 = acc[72] + ABz * acc[27];
    const double h19_3_2 = acc[73] + ABz * acc[28];
    const double h19_3_3 = acc[74] + ABz * acc[29];
    res[0] = h10_1_1 * 0.2581988897471611;
    res[1] = h10_1_2 * 0.2581988897471611;
    res[2] = h10_1_3 * 0.2581988897471611;
    res[3] = h10_2_1 * 0.2581988897471611;
    res[4] = h10_2_2 * 0.2581988897471611;
    res[5] = h10_2_3 * 0.2581988897471611;
    res[6] = h10_3_1 * 0.2581988897471611;
    res[7] = h10_3_2 * 0.2581988897471611;
    res[8] = h10_3_3 * 0.2581988897471611;
    res[9] = h11_1_1 * 0.5773502691896258;
    res[10] = h11_1_2 * 0.5773502691896258;
    res[11] = h11_1_3 * 0.5773502691896258;
    res[12] = h11_2_1 * 0.5773502691896258;
    res[13] = h11_2_2 * 0.5773502691896258;
    res[14] = h11_2_3 * 0.5773502691896258;
    res[15] = h11_3_1 * 0.5773502691896258;
    res[16] = h11_3_2 * 0.5773502691896258;
    res[17] = h11_3_3 * 0.5773502691896258;
    res[18] = h12_1_1 * 0.5773502691896258;
    res[19] = h12_1_2 * 0.5773502691896258;
    res[20] = h12_1_3 * 0.5773502691896258;
    res[21] = h12_2_1 * 0.5773502691896258;
    res[22] = h12_2_2 * 0.5773502691896258;
    res[23] = h12_2_3 * 0.5773502691896258;
    res[24] = h12_3_1 * 0.5773502691896258;
    res[25] = h12_3_2 * 0.5773502691896258;
    res[26] = h12_3_3 * 0.5773502691896258;
    res[27] = h13_1_1 * 0.5773502691896258;
    res[28] = h13_1_2 * 0.5773502691896258;
    res[29] = h13_1_3 * 0.5773502691896258;
    res[30] = h13_2_1 * 0.5773502691896258;
    res[31] = h13_2_2 * 0.5773502691896258;
    res[32] = h13_2_3 * 0.5773502691896258;
    res[33] = h13_3_1 * 0.5773502691896258;
    res[34] = h13_3_2 * 0.5773502691896258;
    res[35] = h13_3_3 * 0.5773502691896258;
    res[36] = h14_1_1 * 0.5773502691896258;
    res[37] = h14_1_2 * 0.5773502691896258;
    res[38] = h14_1_3 * 0.5773502691896258;
    res[39] = h14_2_1 * 0.5773502691896258;
    res[40] = h14_2_2 * 0.5773502691896258;
    res[41] = h14_2_3 * 0.5773502691896258;
    res[42] = h14_3_1 * 0.5773502691896258;
    res[43] = h14_3_2 * 0.5773502691896258;
    res[44] = h14_3_3 * 0.5773502691896258;
    res[45] = h15_1_1;
    res[46] = h15_1_2;
    res[47] = h15_1_3;
    res[48] = h15_2_1;
    res[49] = h15_2_2;
    res[50] = h15_2_3;
    res[51] = h15_3_1;
    res[52] = h15_3_2;
    res[53] = h15_3_3;
    res[54] = h16_1_1 * 0.2581988897471611;
    res[55] = h16_1_2 * 0.2581988897471611;
    res[56] = h16_1_3 * 0.2581988897471611;
    res[57] = h16_2_1 * 0.2581988897471611;
    res[58] = h16_2_2 * 0.2581988897471611;
    res[59] = h16_2_3 * 0.2581988897471611;
    res[60] = h16_3_1 * 0.2581988897471611;
    res[61] = h16_3_2 * 0.2581988897471611;
    res[62] = h16_3_3 * 0.2581988897471611;
    res[63] = h17_1_1 * 0.5773502691896258;
    res[64] = h17_1_2 * 0.5773502691896258;
    res[65] = h17_1_3 * 0.5773502691896258;
    res[66] = h17_2_1 * 0.5773502691896258;
    res[67] = h17_2_2 * 0.5773502691896258;
    res[68] = h17_2_3 * 0.5773502691896258;
    res[69] = h17_3_1 * 0.5773502691896258;
    res[70] = h17_3_2 * 0.5773502691896258;
    res[71] = h17_3_3 * 0.5773502691896258;
    res[72] = h18_1_1 * 0.5773502691896258;
    res[73] = h18_1_2 * 0.5773502691896258;
    res[74] = h18_1_3 * 0.5773502691896258;
    res[75] = h18_2_1 * 0.5773502691896258;
    res[76] = h18_2_2 * 0.5773502691896258;
    res[77] = h18_2_3 * 0.5773502691896258;
    res[78] = h18_3_1 * 0.5773502691896258;
    res[79] = h18_3_2 * 0.5773502691896258;
    res[80] = h18_3_3 * 0.5773502691896258;
    res[81] = h19_1_1 * 0.2581988897471611;
    res[82] = h19_1_2 * 0.2581988897471611;
    res[83] = h19_1_3 * 0.2581988897471611;
    res[84] = h19_2_1 * 0.2581988897471611;
    res[85] = h19_2_2 * 0.2581988897471611;
    res[86] = h19_2_3 * 0.2581988897471611;
    res[87] = h19_3_1 * 0.2581988897471611;
    res[88] = h19_3_2 * 0.2581988897471611;
    res[89] = h19_3_3 * 0.2581988897471611;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[90]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_fpps(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[75];
    vrr_fpps<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 75; ++x) acc_out[x] = acc[x];
    }
    hrr_fpps(P, p, q, acc, res);
}

__device__ __forceinline__ void store_fpps(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
    const long long ij_0_0 = pair_index(ib_.z + 0, ib_.w + 0);
    const long long ij_0_1 = pair_index(ib_.z + 0, ib_.w + 1);
    const long long ij_0_2 = pair_index(ib_.z + 0, ib_.w + 2);
    const long long ij_1_0 = pair_index(ib_.z + 1, ib_.w + 0);
    const long long ij_1_1 = pair_index(ib_.z + 1, ib_.w + 1);
    const long long ij_1_2 = pair_index(ib_.z + 1, ib_.w + 2);
    const long long ij_2_0 = pair_index(ib_.z + 2, ib_.w + 0);
    const long long ij_2_1 = pair_index(ib_.z + 2, ib_.w + 1);
    const long long ij_2_2 = pair_index(ib_.z + 2, ib_.w + 2);
    const long long ij_3_0 = pair_index(ib_.z + 3, ib_.w + 0);
    const long long ij_3_1 = pair_index(ib_.z + 3, ib_.w + 1);
    const long long ij_3_2 = pair_index(ib_.z + 3, ib_.w + 2);
    const long long ij_4_0 = pair_index(ib_.z + 4, ib_.w + 0);
    const long long ij_4_1 = pair_index(ib_.z + 4, ib_.w + 1);
    const long long ij_4_2 = pair_index(ib_.z + 4, ib_.w + 2);
    const long long ij_5_0 = pair_index(ib_.z + 5, ib_.w + 0);
    const long long ij_5_1 = pair_index(ib_.z + 5, ib_.w + 1);
    const long long ij_5_2 = pair_index(ib_.z + 5, ib_.w + 2);
    const long long ij_6_0 = pair_index(ib_.z + 6, ib_.w + 0);
    const long long ij_6_1 = pair_index(ib_.z + 6, ib_.w + 1);
    const long long ij_6_2 = pair_index(ib_.z + 6, ib_.w + 2);
    const long long ij_7_0 = pair_index(ib_.z + 7, ib_.w + 0);
    const long long ij_7_1 = pair_index(ib_.z + 7, ib_.w + 1);
    const long long ij_7_2 = pair_index(ib_.z + 7, ib_.w + 2);
    const long long ij_8_0 = pair_index(ib_.z + 8, ib_.w + 0);
    const long long ij_8_1 = pair_index(ib_.z + 8, ib_.w + 1);
    const long long ij_8_2 = pair_index(ib_.z + 8, ib_.w + 2);
    const long long ij_9_0 = pair_index(ib_.z + 9, ib_.w + 0);
    const long long ij_9_1 = pair_index(ib_.z + 9, ib_.w + 1);
    const long long ij_9_2 = pair_index(ib_.z + 9, ib_.w + 2);
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    const long long kl_1_0 = pair_index(ik_.z + 1, ik_.w + 0);
    const long long kl_2_0 = pair_index(ik_.z + 2, ik_.w + 0);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_3_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_3_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_3_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_3_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_4_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_4_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_4_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_4_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_5_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_5_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_5_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_5_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_6_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_6_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_6_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_6_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_6_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_6_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_6_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_6_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_7_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_7_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_7_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_7_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_7_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_7_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_7_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_7_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_8_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_8_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_8_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_8_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_8_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_8_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_8_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_8_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_9_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_9_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_9_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_9_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_9_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_9_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_9_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_9_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_fpps(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 90; ++x) {
        const int ia = x / 9, ibb = (x / 3) % 3, ic = (x / 1) % 3, id = x % 1;
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
__global__ void __launch_bounds__(128) eri_queue_fpps(const EriQueue Q) {
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
        double acc[75];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 75; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_fpps<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_fpps<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 75; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 90 doubles (launch_eri_fpps)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 90);
            if (lead) hrr_fpps(Q.pairs, p, q, acc, sb + kq * 90);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)90;
            for (int t = lane; t < nlive * 90; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[90];
            hrr_fpps(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_fpps(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_fpps(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (92160 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_fpps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_fpps<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 92160);
        cudaFuncSetAttribute(eri_queue_fpps<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 92160);
        done[dev] = true;
    }
}

void launch_eri_fpps(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 92160 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 92160 : 0;
    if (smem) eri_prepare_fpps();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_fpps<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_fpps<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_fpps<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_fpps<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_fpps(int mixed) {
    eri_prepare_fpps();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fpps<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fpps<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

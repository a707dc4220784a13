// Generated by gen_eri.py -- class (fs|fs).  Do not edit.
// VRR entries: 486, contracted block: 100, HRR lines: 0, outputs: 100.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[100], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_fsfs(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 100; ++x) acc[x] = 0.0;
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
            const VT v1_1_2 = QCx * v1_0_2 + WQx * v1_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v2_1_2 = QCx * v2_0_2 + WQx * v2_0_3;
            const VT v3_1_2 = QCx * v3_0_2 + WQx * v3_0_3;
            const VT v4_1_1 = QCx * v4_0_1 + WQx * v4_0_2 + (VT)2.0 * oo2ze * v1_0_2;
            const VT v4_1_2 = QCx * v4_0_2 + WQx * v4_0_3 + (VT)2.0 * oo2ze * v1_0_3;
            const VT v5_1_1 = QCx * v5_0_1 + WQx * v5_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v5_1_2 = QCx * v5_0_2 + WQx * v5_0_3 + (VT)1.0 * oo2ze * v2_0_3;
            const VT v6_1_1 = QCx * v6_0_1 + WQx * v6_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v6_1_2 = QCx * v6_0_2 + WQx * v6_0_3 + (VT)1.0 * oo2ze * v3_0_3;
            const VT v7_1_1 = QCx * v7_0_1 + WQx * v7_0_2;
            const VT v7_1_2 = QCx * v7_0_2 + WQx * v7_0_3;
            const VT v8_1_1 = QCx * v8_0_1 + WQx * v8_0_2;
            const VT v8_1_2 = QCx * v8_0_2 + WQx * v8_0_3;
            const VT v9_1_1 = QCx * v9_0_1 + WQx * v9_0_2;
            const VT v9_1_2 = QCx * v9_0_2 + WQx * v9_0_3;
            const VT v10_1_0 = QCx * v10_0_0 + WQx * v10_0_1 + (VT)3.0 * oo2ze * v4_0_1;
            const VT v10_1_1 = QCx * v10_0_1 + WQx * v10_0_2 + (VT)3.0 * oo2ze * v4_0_2;
            const VT v10_1_2 = QCx * v10_0_2 + WQx * v10_0_3 + (VT)3.0 * oo2ze * v4_0_3;
            const VT v11_1_0 = QCx * v11_0_0 + WQx * v11_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v11_1_1 = QCx * v11_0_1 + WQx * v11_0_2 + (VT)2.0 * oo2ze * v5_0_2;
            const VT v11_1_2 = QCx * v11_0_2 + WQx * v11_0_3 + (VT)2.0 * oo2ze * v5_0_3;
            const VT v12_1_0 = QCx * v12_0_0 + WQx * v12_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v12_1_1 = QCx * v12_0_1 + WQx * v12_0_2 + (VT)2.0 * oo2ze * v6_0_2;
            const VT v12_1_2 = QCx * v12_0_2 + WQx * v12_0_3 + (VT)2.0 * oo2ze * v6_0_3;
            const VT v13_1_0 = QCx * v13_0_0 + WQx * v13_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v13_1_1 = QCx * v13_0_1 + WQx * v13_0_2 + (VT)1.0 * oo2ze * v7_0_2;
            const VT v13_1_2 = QCx * v13_0_2 + WQx * v13_0_3 + (VT)1.0 * oo2ze * v7_0_3;
            const VT v14_1_0 = QCx * v14_0_0 + WQx * v14_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v14_1_1 = QCx * v14_0_1 + WQx * v14_0_2 + (VT)1.0 * oo2ze * v9_0_2;
            const VT v14_1_2 = QCx * v14_0_2 + WQx * v14_0_3 + (VT)1.0 * oo2ze * v9_0_3;
            const VT v15_1_0 = QCx * v15_0_0 + WQx * v15_0_1 + (VT)1.0 * oo2ze * v8_0_1;
            const VT v15_1_1 = QCx * v15_0_1 + WQx * v15_0_2 + (VT)1.0 * oo2ze * v8_0_2;
            const VT v15_1_2 = QCx * v15_0_2 + WQx * v15_0_3 + (VT)1.0 * oo2ze * v8_0_3;
            const VT v16_1_0 = QCx * v16_0_0 + WQx * v16_0_1;
            const VT v16_1_1 = QCx * v16_0_1 + WQx * v16_0_2;
            const VT v16_1_2 = QCx * v16_0_2 + WQx * v16_0_3;
            const VT v17_1_0 = QCx * v17_0_0 + WQx * v17_0_1;
            const VT v17_1_1 = QCx * v17_0_1 + WQx * v17_0_2;
            const VT v17_1_2 = QCx * v17_0_2 + WQx * v17_0_3;
            const VT v18_1_0 = QCx * v18_0_0 + WQx * v18_0_1;
            const VT v18_1_1 = QCx * v18_0_1 + WQx * v18_0_2;
            const VT v18_1_2 = QCx * v18_0_2 + WQx * v18_0_3;
            const VT v19_1_0 = QCx * v19_0_0 + WQx * v19_0_1;
            const VT v19_1_1 = QCx * v19_0_1 + WQx * v19_0_2;
            const VT v19_1_2 = QCx * v19_0_2 + WQx * v19_0_3;
            const VT v1_2_2 = QCy * v1_0_2 + WQy * v1_0_3;
            const VT v2_2_2 = QCy * v2_0_2 + WQy * v2_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v3_2_2 = QCy * v3_0_2 + WQy * v3_0_3;
            const VT v4_2_1 = QCy * v4_0_1 + WQy * v4_0_2;
            const VT v4_2_2 = QCy * v4_0_2 + WQy * v4_0_3;
            const VT v5_2_1 = QCy * v5_0_1 + WQy * v5_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v5_2_2 = QCy * v5_0_2 + WQy * v5_0_3 + (VT)1.0 * oo2ze * v1_0_3;
            const VT v6_2_1 = QCy * v6_0_1 + WQy * v6_0_2;
            const VT v6_2_2 = QCy * v6_0_2 + WQy * v6_0_3;
            const VT v7_2_1 = QCy * v7_0_1 + WQy * v7_0_2 + (VT)2.0 * oo2ze * v2_0_2;
            const VT v7_2_2 = QCy * v7_0_2 + WQy * v7_0_3 + (VT)2.0 * oo2ze * v2_0_3;
            const VT v8_2_1 = QCy * v8_0_1 + WQy * v8_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v8_2_2 = QCy * v8_0_2 + WQy * v8_0_3 + (VT)1.0 * oo2ze * v3_0_3;
            const VT v9_2_1 = QCy * v9_0_1 + WQy * v9_0_2;
            const VT v9_2_2 = QCy * v9_0_2 + WQy * v9_0_3;
            const VT v10_2_0 = QCy * v10_0_0 + WQy * v10_0_1;
            const VT v10_2_1 = QCy * v10_0_1 + WQy * v10_0_2;
            const VT v10_2_2 = QCy * v10_0_2 + WQy * v10_0_3;
            const VT v11_2_0 = QCy * v11_0_0 + WQy * v11_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v11_2_1 = QCy * v11_0_1 + WQy * v11_0_2 + (VT)1.0 * oo2ze * v4_0_2;
            const VT v11_2_2 = QCy * v11_0_2 + WQy * v11_0_3 + (VT)1.0 * oo2ze * v4_0_3;
            const VT v12_2_0 = QCy * v12_0_0 + WQy * v12_0_1;
            const VT v12_2_1 = QCy * v12_0_1 + WQy * v12_0_2;
            const VT v12_2_2 = QCy * v12_0_2 + WQy * v12_0_3;
            const VT v13_2_0 = QCy * v13_0_0 + WQy * v13_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v13_2_1 = QCy * v13_0_1 + WQy * v13_0_2 + (VT)2.0 * oo2ze * v5_0_2;
            const VT v13_2_2 = QCy * v13_0_2 + WQy * v13_0_3 + (VT)2.0 * oo2ze * v5_0_3;
            const VT v14_2_0 = QCy * v14_0_0 + WQy * v14_0_1;
            const VT v14_2_1 = QCy * v14_0_1 + WQy * v14_0_2;
            const VT v14_2_2 = QCy * v14_0_2 + WQy * v14_0_3;
            const VT v15_2_0 = QCy * v15_0_0 + WQy * v15_0_1 + (VT)1.0 * oo2ze * v6_0_1;
            const VT v15_2_1 = QCy * v15_0_1 + WQy * v15_0_2 + (VT)1.0 * oo2ze * v6_0_2;
            const VT v15_2_2 = QCy * v15_0_2 + WQy * v15_0_3 + (VT)1.0 * oo2ze * v6_0_3;
            const VT v16_2_0 = QCy * v16_0_0 + WQy * v16_0_1 + (VT)3.0 * oo2ze * v7_0_1;
            const VT v16_2_1 = QCy * v16_0_1 + WQy * v16_0_2 + (VT)3.0 * oo2ze * v7_0_2;
            const VT v16_2_2 = QCy * v16_0_2 + WQy * v16_0_3 + (VT)3.0 * oo2ze * v7_0_3;
            const VT v17_2_0 = QCy * v17_0_0 + WQy * v17_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v17_2_1 = QCy * v17_0_1 + WQy * v17_0_2 + (VT)2.0 * oo2ze * v8_0_2;
            const VT v17_2_2 = QCy * v17_0_2 + WQy * v17_0_3 + (VT)2.0 * oo2ze * v8_0_3;
            const VT v18_2_0 = QCy * v18_0_0 + WQy * v18_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v18_2_1 = QCy * v18_0_1 + WQy * v18_0_2 + (VT)1.0 * oo2ze * v9_0_2;
            const VT v18_2_2 = QCy * v18_0_2 + WQy * v18_0_3 + (VT)1.0 * oo2ze * v9_0_3;
            const VT v19_2_0 = QCy * v19_0_0 + WQy * v19_0_1;
            const VT v19_2_1 = QCy * v19_0_1 + WQy * v19_0_2;
            const VT v19_2_2 = QCy * v19_0_2 + WQy * v19_0_3;
            const VT v1_3_2 = QCz * v1_0_2 + WQz * v1_0_3;
            const VT v2_3_2 = QCz * v2_0_2 + WQz * v2_0_3;
            const VT v3_3_2 = QCz * v3_0_2 + WQz * v3_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v4_3_1 = QCz * v4_0_1 + WQz * v4_0_2;
            const VT v4_3_2 = QCz * v4_0_2 + WQz * v4_0_3;
            const VT v5_3_1 = QCz * v5_0_1 + WQz * v5_0_2;
            const VT v5_3_2 = QCz * v5_0_2 + WQz * v5_0_3;
            const VT v6_3_1 = QCz * v6_0_1 + WQz * v6_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v6_3_2 = QCz * v6_0_2 + WQz * v6_0_3 + (VT)1.0 * oo2ze * v1_0_3;
            const VT v7_3_1 = QCz * v7_0_1 + WQz * v7_0_2;
            const VT v7_3_2 = QCz * v7_0_2 + WQz * v7_0_3;
            const VT v8_3_1 = QCz * v8_0_1 + WQz * v8_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v8_3_2 = QCz * v8_0_2 + WQz * v8_0_3 + (VT)1.0 * oo2ze * v2_0_3;
            const VT v9_3_1 = QCz * v9_0_1 + WQz * v9_0_2 + (VT)2.0 * oo2ze * v3_0_2;
            const VT v9_3_2 = QCz * v9_0_2 + WQz * v9_0_3 + (VT)2.0 * oo2ze * v3_0_3;
            const VT v10_3_0 = QCz * v10_0_0 + WQz * v10_0_1;
            const VT v10_3_1 = QCz * v10_0_1 + WQz * v10_0_2;
            const VT v10_3_2 = QCz * v10_0_2 + WQz * v10_0_3;
            const VT v11_3_0 = QCz * v11_0_0 + WQz * v11_0_1;
            const VT v11_3_1 = QCz * v11_0_1 + WQz * v11_0_2;
            const VT v11_3_2 = QCz * v11_0_2 + WQz * v11_0_3;
            const VT v12_3_0 = QCz * v12_0_0 + WQz * v12_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v12_3_1 = QCz * v12_0_1 + WQz * v12_0_2 + (VT)1.0 * oo2ze * v4_0_2;
            const VT v12_3_2 = QCz * v12_0_2 + WQz * v12_0_3 + (VT)1.0 * oo2ze * v4_0_3;
            const VT v13_3_0 = QCz * v13_0_0 + WQz * v13_0_1;
            const VT v13_3_1 = QCz * v13_0_1 + WQz * v13_0_2;
            const VT v13_3_2 = QCz * v13_0_2 + WQz * v13_0_3;
            const VT v14_3_0 = QCz * v14_0_0 + WQz * v14_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v14_3_1 = QCz * v14_0_1 + WQz * v14_0_2 + (VT)2.0 * oo2ze * v6_0_2;
            const VT v14_3_2 = QCz * v14_0_2 + WQz * v14_0_3 + (VT)2.0 * oo2ze * v6_0_3;
            const VT v15_3_0 = QCz * v15_0_0 + WQz * v15_0_1 + (VT)1.0 * oo2ze * v5_0_1;
            const VT v15_3_1 = QCz * v15_0_1 + WQz * v15_0_2 + (VT)1.0 * oo2ze * v5_0_2;
            const VT v15_3_2 = QCz * v15_0_2 + WQz * v15_0_3 + (VT)1.0 * oo2ze * v5_0_3;
            const VT v16_3_0 = QCz * v16_0_0 + WQz * v16_0_1;
            const VT v16_3_1 = QCz * v16_0_1 + WQz * v16_0_2;
            const VT v16_3_2 = QCz * v16_0_2 + WQz * v16_0_3;
            const VT v17_3_0 = QCz * v17_0_0 + WQz * v17_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v17_3_1 = QCz * v17_0_1 + WQz * v17_0_2 + (VT)1.0 * oo2ze * v7_0_2;
            const VT v17_3_2 = QCz * v17_0_2 + WQz * v17_0_3 + (VT)1.0 * oo2ze * v7_0_3;
            const VT v18_3_0 = QCz * v18_0_0 + WQz * v18_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v18_3_1 = QCz * v18_0_1 + WQz * v18_0_2 + (VT)2.0 * oo2ze * v8_0_2;
            const VT v18_3_2 = QCz * v18_0_2 + WQz * v18_0_3 + (VT)2.0 * oo2ze * v8_0_3;
            const VT v19_3_0 = QCz * v19_0_0 + WQz * v19_0_1 + (VT)3.0 * oo2ze * v9_0_1;
            const VT v19_3_1 = QCz * v19_0_1 + WQz * v19_0_2 + (VT)3.0 * oo2ze * v9_0_2;
            const VT v19_3_2 = QCz * v19_0_2 + WQz * v19_0_3 + (VT)3.0 * oo2ze * v9_0_3;
            const VT v4_4_1 = QCx * v4_1_1 + WQx * v4_1_2 + (VT)2.0 * oo2ze * v1_1_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v5_4_1 = QCx * v5_1_1 + WQx * v5_1_2 + (VT)1.0 * oo2ze * v2_1_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v6_4_1 = QCx * v6_1_1 + WQx * v6_1_2 + (VT)1.0 * oo2ze * v3_1_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v7_4_1 = QCx * v7_1_1 + WQx * v7_1_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v8_4_1 = QCx * v8_1_1 + WQx * v8_1_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v9_4_1 = QCx * v9_1_1 + WQx * v9_1_2 + (VT)1.0 * oo2e * (v9_0_1 - rho_e * v9_0_2);
            const VT v10_4_0 = QCx * v10_1_0 + WQx * v10_1_1 + (VT)3.0 * oo2ze * v4_1_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v10_4_1 = QCx * v10_1_1 + WQx * v10_1_2 + (VT)3.0 * oo2ze * v4_1_2 + (VT)1.0 * oo2e * (v10_0_1 - rho_e * v10_0_2);
            const VT v11_4_0 = QCx * v11_1_0 + WQx * v11_1_1 + (VT)2.0 * oo2ze * v5_1_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v11_4_1 = QCx * v11_1_1 + WQx * v11_1_2 + (VT)2.0 * oo2ze * v5_1_2 + (VT)1.0 * oo2e * (v11_0_1 - rho_e * v11_0_2);
            const VT v12_4_0 = QCx * v12_1_0 + WQx * v12_1_1 + (VT)2.0 * oo2ze * v6_1_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v12_4_1 = QCx * v12_1_1 + WQx * v12_1_2 + (VT)2.0 * oo2ze * v6_1_2 + (VT)1.0 * oo2e * (v12_0_1 - rho_e * v12_0_2);
            const VT v13_4_0 = QCx * v13_1_0 + WQx * v13_1_1 + (VT)1.0 * oo2ze * v7_1_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v13_4_1 = QCx * v13_1_1 + WQx * v13_1_2 + (VT)1.0 * oo2ze * v7_1_2 + (VT)1.0 * oo2e * (v13_0_1 - rho_e * v13_0_2);
            const VT v14_4_0 = QCx * v14_1_0 + WQx * v14_1_1 + (VT)1.0 * oo2ze * v9_1_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v14_4_1 = QCx * v14_1_1 + WQx * v14_1_2 + (VT)1.0 * oo2ze * v9_1_2 + (VT)1.0 * oo2e * (v14_0_1 - rho_e * v14_0_2);
            const VT v15_4_0 = QCx * v15_1_0 + WQx * v15_1_1 + (VT)1.0 * oo2ze * v8_1_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v15_4_1 = QCx * v15_1_1 + WQx * v15_1_2 + (VT)1.0 * oo2ze * v8_1_2 + (VT)1.0 * oo2e * (v15_0_1 - rho_e * v15_0_2);
            const VT v16_4_0 = QCx * v16_1_0 + WQx * v16_1_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v16_4_1 = QCx * v16_1_1 + WQx * v16_1_2 + (VT)1.0 * oo2e * (v16_0_1 - rho_e * v16_0_2);
            const VT v17_4_0 = QCx * v17_1_0 + WQx * v17_1_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v17_4_1 = QCx * v17_1_1 + WQx * v17_1_2 + (VT)1.0 * oo2e * (v17_0_1 - rho_e * v17_0_2);
            const VT v18_4_0 = QCx * v18_1_0 + WQx * v18_1_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v18_4_1 = QCx * v18_1_1 + WQx * v18_1_2 + (VT)1.0 * oo2e * (v18_0_1 - rho_e * v18_0_2);
            const VT v19_4_0 = QCx * v19_1_0 + WQx * v19_1_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v19_4_1 = QCx * v19_1_1 + WQx * v19_1_2 + (VT)1.0 * oo2e * (v19_0_1 - rho_e * v19_0_2);
            const VT v4_5_1 = QCx * v4_2_1 + WQx * v4_2_2 + (VT)2.0 * oo2ze * v1_2_2;
            const VT v5_5_1 = QCx * v5_2_1 + WQx * v5_2_2 + (VT)1.0 * oo2ze * v2_2_2;
            const VT v6_5_1 = QCx * v6_2_1 + WQx * v6_2_2 + (VT)1.0 * oo2ze * v3_2_2;
            const VT v7_5_1 = QCx * v7_2_1 + WQx * v7_2_2;
            const VT v8_5_1 = QCx * v8_2_1 + WQx * v8_2_2;
            const VT v9_5_1 = QCx * v9_2_1 + WQx * v9_2_2;
            const VT v10_5_0 = QCx * v10_2_0 + WQx * v10_2_1 + (VT)3.0 * oo2ze * v4_2_1;
            const VT v10_5_1 = QCx * v10_2_1 + WQx * v10_2_2 + (VT)3.0 * oo2ze * v4_2_2;
            const VT v11_5_0 = QCx * v11_2_0 + WQx * v11_2_1 + (VT)2.0 * oo2ze * v5_2_1;
            const VT v11_5_1 = QCx * v11_2_1 + WQx * v11_2_2 + (VT)2.0 * oo2ze * v5_2_2;
            const VT v12_5_0 = QCx * v12_2_0 + WQx * v12_2_1 + (VT)2.0 * oo2ze * v6_2_1;
            const VT v12_5_1 = QCx * v12_2_1 + WQx * v12_2_2 + (VT)2.0 * oo2ze * v6_2_2;
            const VT v13_5_0 = QCx * v13_2_0 + WQx * v13_2_1 + (VT)1.0 * oo2ze * v7_2_1;
            const VT v13_5_1 = QCx * v13_2_1 + WQx * v13_2_2 + (VT)1.0 * oo2ze * v7_2_2;
            const VT v14_5_0 = QCx * v14_2_0 + WQx * v14_2_1 + (VT)1.0 * oo2ze * v9_2_1;
            const VT v14_5_1 = QCx * v14_2_1 + WQx * v14_2_2 + (VT)1.0 * oo2ze * v9_2_2;
            const VT v15_5_0 = QCx * v15_2_0 + WQx * v15_2_1 + (VT)1.0 * oo2ze * v8_2_1;
            const VT v15_5_1 = QCx * v15_2_1 + WQx * v15_2_2 + (VT)1.0 * oo2ze * v8_2_2;
            const VT v16_5_0 = QCx * v16_2_0 + WQx * v16_2_1;
            const VT v16_5_1 = QCx * v16_2_1 + WQx * v16_2_2;
            const VT v17_5_0 = QCx * v17_2_0 + WQx * v17_2_1;
            const VT v17_5_1 = QCx * v17_2_1 + WQx * v17_2_2;
            const VT v18_5_0 = QCx * v18_2_0 + WQx * v18_2_1;
            const VT v18_5_1 = QCx * v18_2_1 + WQx * v18_2_2;
            const VT v19_5_0 = QCx * v19_2_0 + WQx * v19_2_1;
            const VT v19_5_1 = QCx * v19_2_1 + WQx * v19_2_2;
            const VT v4_6_1 = QCx * v4_3_1 + WQx * v4_3_2 + (VT)2.0 * oo2ze * v1_3_2;
            const VT v5_6_1 = QCx * v5_3_1 + WQx * v5_3_2 + (VT)1.0 * oo2ze * v2_3_2;
            const VT v6_6_1 = QCx * v6_3_1 + WQx * v6_3_2 + (VT)1.0 * oo2ze * v3_3_2;
            const VT v7_6_1 = QCx * v7_3_1 + WQx * v7_3_2;
            const VT v8_6_1 = QCx * v8_3_1 + WQx * v8_3_2;
            const VT v9_6_1 = QCx * v9_3_1 + WQx * v9_3_2;
            const VT v10_6_0 = QCx * v10_3_0 + WQx * v10_3_1 + (VT)3.0 * oo2ze * v4_3_1;
            const VT v10_6_1 = QCx * v10_3_1 + WQx * v10_3_2 + (VT)3.0 * oo2ze * v4_3_2;
            const VT v11_6_0 = QCx * v11_3_0 + WQx * v11_3_1 + (VT)2.0 * oo2ze * v5_3_1;
            const VT v11_6_1 = QCx * v11_3_1 + WQx * v11_3_2 + (VT)2.0 * oo2ze * v5_3_2;
            const VT v12_6_0 = QCx * v12_3_0 + WQx * v12_3_1 + (VT)2.0 * oo2ze * v6_3_1;
            const VT v12_6_1 = QCx * v12_3_1 + WQx * v12_3_2 + (VT)2.0 * oo2ze * v6_3_2;
            const VT v13_6_0 = QCx * v13_3_0 + WQx * v13_3_1 + (VT)1.0 * oo2ze * v7_3_1;
            const VT v13_6_1 = QCx * v13_3_1 + WQx * v13_3_2 + (VT)1.0 * oo2ze * v7_3_2;
            const VT v14_6_0 = QCx * v14_3_0 + WQx * v14_3_1 + (VT)1.0 * oo2ze * v9_3_1;
            const VT v14_6_1 = QCx * v14_3_1 + WQx * v14_3_2 + (VT)1.0 * oo2ze * v9_3_2;
            const VT v15_6_0 = QCx * v15_3_0 + WQx * v15_3_1 + (VT)1.0 * oo2ze * v8_3_1;
            const VT v15_6_1 = QCx * v15_3_1 + WQx * v15_3_2 + (VT)1.0 * oo2ze * v8_3_2;
            const VT v16_6_0 = QCx * v16_3_0 + WQx * v16_3_1;
            const VT v16_6_1 = QCx * v16_3_1 + WQx * v16_3_2;
            const VT v17_6_0 = QCx * v17_3_0 + WQx * v17_3_1;
            const VT v17_6_1 = QCx * v17_3_1 + WQx * v17_3_2;
            const VT v18_6_0 = QCx * v18_3_0 + WQx * v18_3_1;
            const VT v18_6_1 = QCx * v18_3_1 + WQx * v18_3_2;
            const VT v19_6_0 = QCx * v19_3_0 + WQx * v19_3_1;
            const VT v19_6_1 = QCx * v19_3_1 + WQx * v19_3_2;
            const VT v4_7_1 = QCy * v4_2_1 + WQy * v4_2_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v5_7_1 = QCy * v5_2_1 + WQy * v5_2_2 + (VT)1.0 * oo2ze * v1_2_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v6_7_1 = QCy * v6_2_1 + WQy * v6_2_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v7_7_1 = QCy * v7_2_1 + WQy * v7_2_2 + (VT)2.0 * oo2ze * v2_2_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v8_7_1 = QCy * v8_2_1 + WQy * v8_2_2 + (VT)1.0 * oo2ze * v3_2_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v9_7_1 = QCy * v9_2_1 + WQy * v9_2_2 + (VT)1.0 * oo2e * (v9_0_1 - rho_e * v9_0_2);
            const VT v10_7_0 = QCy * v10_2_0 + WQy * v10_2_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v10_7_1 = QCy * v10_2_1 + WQy * v10_2_2 + (VT)1.0 * oo2e * (v10_0_1 - rho_e * v10_0_2);
            const VT v11_7_0 = QCy * v11_2_0 + WQy * v11_2_1 + (VT)1.0 * oo2ze * v4_2_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v11_7_1 = QCy * v11_2_1 + WQy * v11_2_2 + (VT)1.0 * oo2ze * v4_2_2 + (VT)1.0 * oo2e * (v11_0_1 - rho_e * v11_0_2);
            const VT v12_7_0 = QCy * v12_2_0 + WQy * v12_2_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v12_7_1 = QCy * v12_2_1 + WQy * v12_2_2 + (VT)1.0 * oo2e * (v12_0_1 - rho_e * v12_0_2);
            const VT v13_7_0 = QCy * v13_2_0 + WQy * v13_2_1 + (VT)2.0 * oo2ze * v5_2_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v13_7_1 = QCy * v13_2_1 + WQy * v13_2_2 + (VT)2.0 * oo2ze * v5_2_2 + (VT)1.0 * oo2e * (v13_0_1 - rho_e * v13_0_2);
            const VT v14_7_0 = QCy * v14_2_0 + WQy * v14_2_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v14_7_1 = QCy * v14_2_1 + WQy * v14_2_2 + (VT)1.0 * oo2e * (v14_0_1 - rho_e * v14_0_2);
            const VT v15_7_0 = QCy * v15_2_0 + WQy * v15_2_1 + (VT)1.0 * oo2ze * v6_2_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v15_7_1 = QCy * v15_2_1 + WQy * v15_2_2 + (VT)1.0 * oo2ze * v6_2_2 + (VT)1.0 * oo2e * (v15_0_1 - rho_e * v15_0_2);
            const VT v16_7_0 = QCy * v16_2_0 + WQy * v16_2_1 + (VT)3.0 * oo2ze * v7_2_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v16_7_1 = QCy * v16_2_1 + WQy * v16_2_2 + (VT)3.0 * oo2ze * v7_2_2 + (VT)1.0 * oo2e * (v16_0_1 - rho_e * v16_0_2);
            const VT v17_7_0 = QCy * v17_2_0 + WQy * v17_2_1 + (VT)2.0 * oo2ze * v8_2_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v17_7_1 = QCy * v17_2_1 + WQy * v17_2_2 + (VT)2.0 * oo2ze * v8_2_2 + (VT)1.0 * oo2e * (v17_0_1 - rho_e * v17_0_2);
            const VT v18_7_0 = QCy * v18_2_0 + WQy * v18_2_1 + (VT)1.0 * oo2ze * v9_2_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v18_7_1 = QCy * v18_2_1 + WQy * v18_2_2 + (VT)1.0 * oo2ze * v9_2_2 + (VT)1.0 * oo2e * (v18_0_1 - rho_e * v18_0_2);
            const VT v19_7_0 = QCy * v19_2_0 + WQy * v19_2_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v19_7_1 = QCy * v19_2_1 + WQy * v19_2_2 + (VT)1.0 * oo2e * (v19_0_1 - rho_e * v19_0_2);
            const VT v4_8_1 = QCy * v4_3_1 + WQy * v4_3_2;
            const VT v5_8_1 = QCy * v5_3_1 + WQy * v5_3_2 + (VT)1.0 * oo2ze * v1_3_2;
            const VT v6_8_1 = QCy * v6_3_1 + WQy * v6_3_2;
            const VT v7_8_1 = QCy * v7_3_1 + WQy * v7_3_2 + (VT)2.0 * oo2ze * v2_3_2;
            const VT v8_8_1 = QCy * v8_3_1 + WQy * v8_3_2 + (VT)1.0 * oo2ze * v3_3_2;
            const VT v9_8_1 = QCy * v9_3_1 + WQy * v9_3_2;
            const VT v10_8_0 = QCy * v10_3_0 + WQy * v10_3_1;
            const VT v10_8_1 = QCy * v10_3_1 + WQy * v10_3_2;
            const VT v11_8_0 = QCy * v11_3_0 + WQy * v11_3_1 + (VT)1.0 * oo2ze * v4_3_1;
            const VT v11_8_1 = QCy * v11_3_1 + WQy * v11_3_2 + (VT)1.0 * oo2ze * v4_3_2;
            const VT v12_8_0 = QCy * v12_3_0 + WQy * v12_3_1;
            const VT v12_8_1 = QCy * v12_3_1 + WQy * v12_3_2;
            const VT v13_8_0 = QCy * v13_3_0 + WQy * v13_3_1 + (VT)2.0 * oo2ze * v5_3_1;
            const VT v13_8_1 = QCy * v13_3_1 + WQy * v13_3_2 + (VT)2.0 * oo2ze * v5_3_2;
            const VT v14_8_0 = QCy * v14_3_0 + WQy * v14_3_1;
            const VT v14_8_1 = QCy * v14_3_1 + WQy * v14_3_2;
            const VT v15_8_0 = QCy * v15_3_0 + WQy * v15_3_1 + (VT)1.0 * oo2ze * v6_3_1;
            const VT v15_8_1 = QCy * v15_3_1 + WQy * v15_3_2 + (VT)1.0 * oo2ze * v6_3_2;
            const VT v16_8_0 = QCy * v16_3_0 + WQy * v16_3_1 + (VT)3.0 * oo2ze * v7_3_1;
            const VT v16_8_1 = QCy * v16_3_1 + WQy * v16_3_2 + (VT)3.0 * oo2ze * v7_3_2;
            const VT v17_8_0 = QCy * v17_3_0 + WQy * v17_3_1 + (VT)2.0 * oo2ze * v8_3_1;
            const VT v17_8_1 = QCy * v17_3_1 + WQy * v17_3_2 + (VT)2.0 * oo2ze * v8_3_2;
            const VT v18_8_0 = QCy * v18_3_0 + WQy * v18_3_1 + (VT)1.0 * oo2ze * v9_3_1;
            const VT v18_8_1 = QCy * v18_3_1 + WQy * v18_3_2 + (VT)1.0 * oo2ze * v9_3_2;
            const VT v19_8_0 = QCy * v19_3_0 + WQy * v19_3_1;
            const VT v19_8_1 = QCy * v19_3_1 + WQy * v19_3_2;
            const VT v4_9_1 = QCz * v4_3_1 + WQz * v4_3_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v5_9_1 = QCz * v5_3_1 + WQz * v5_3_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v6_9_1 = QCz * v6_3_1 + WQz * v6_3_2 + (VT)1.0 * oo2ze * v1_3_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v7_9_1 = QCz * v7_3_1 + WQz * v7_3_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v8_9_1 = QCz * v8_3_1 + WQz * v8_3_2 + (VT)1.0 * oo2ze * v2_3_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v9_9_1 = QCz * v9_3_1 + WQz * v9_3_2 + (VT)2.0 * oo2ze * v3_3_2 + (VT)1.0 * oo2e * (v9_0_1 - rho_e * v9_0_2);
            const VT v10_9_0 = QCz * v10_3_0 + WQz * v10_3_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v10_9_1 = QCz * v10_3_1 + WQz * v10_3_2 + (VT)1.0 * oo2e * (v10_0_1 - rho_e * v10_0_2);
            const VT v11_9_0 = QCz * v11_3_0 + WQz * v11_3_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v11_9_1 = QCz * v11_3_1 + WQz * v11_3_2 + (VT)1.0 * oo2e * (v11_0_1 - rho_e * v11_0_2);
            const VT v12_9_0 = QCz * v12_3_0 + WQz * v12_3_1 + (VT)1.0 * oo2ze * v4_3_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v12_9_1 = QCz * v12_3_1 + WQz * v12_3_2 + (VT)1.0 * oo2ze * v4_3_2 + (VT)1.0 * oo2e * (v12_0_1 - rho_e * v12_0_2);
            const VT v13_9_0 = QCz * v13_3_0 + WQz * v13_3_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v13_9_1 = QCz * v13_3_1 + WQz * v13_3_2 + (VT)1.0 * oo2e * (v13_0_1 - rho_e * v13_0_2);
            const VT v14_9_0 = QCz * v14_3_0 + WQz * v14_3_1 + (VT)2.0 * oo2ze * v6_3_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v14_9_1 = QCz * v14_3_1 + WQz * v14_3_2 + (VT)2.0 * oo2ze * v6_3_2 + (VT)1.0 * oo2e * (v14_0_1 - rho_e * v14_0_2);
            const VT v15_9_0 = QCz * v15_3_0 + WQz * v15_3_1 + (VT)1.0 * oo2ze * v5_3_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v15_9_1 = QCz * v15_3_1 + WQz * v15_3_2 + (VT)1.0 * oo2ze * v5_3_2 + (VT)1.0 * oo2e * (v15_0_1 - rho_e * v15_0_2);
            const VT v16_9_0 = QCz * v16_3_0 + WQz * v16_3_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v16_9_1 = QCz * v16_3_1 + WQz * v16_3_2 + (VT)1.0 * oo2e * (v16_0_1 - rho_e * v16_0_2);
            const VT v17_9_0 = QCz * v17_3_0 + WQz * v17_3_1 + (VT)1.0 * oo2ze * v7_3_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v17_9_1 = QCz * v17_3_1 + WQz * v17_3_2 + (VT)1.0 * oo2ze * v7_3_2 + (VT)1.0 * oo2e * (v17_0_1 - rho_e * v17_0_2);
            const VT v18_9_0 = QCz * v18_3_0 + WQz * v18_3_1 + (VT)2.0 * oo2ze * v8_3_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v18_9_1 = QCz * v18_3_1 + WQz * v18_3_2 + (VT)2.0 * oo2ze * v8_3_2 + (VT)1.0 * oo2e * (v18_0_1 - rho_e * v18_0_2);
            const VT v19_9_0 = QCz * v19_3_0 + WQz * v19_3_1 + (VT)3.0 * oo2ze * v9_3_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v19_9_1 = QCz * v19_3_1 + WQz * v19_3_2 + (VT)3.0 * oo2ze * v9_3_2 + (VT)1.0 * oo2e * (v19_0_1 - rho_e * v19_0_2);
            const VT v10_10_0 = QCx * v10_4_0 + WQx * v10_4_1 + (VT)3.0 * oo2ze * v4_4_1 + (VT)2.0 * oo2e * (v10_1_0 - rho_e * v10_1_1);
            const VT v11_10_0 = QCx * v11_4_0 + WQx * v11_4_1 + (VT)2.0 * oo2ze * v5_4_1 + (VT)2.0 * oo2e * (v11_1_0 - rho_e * v11_1_1);
            const VT v12_10_0 = QCx * v12_4_0 + WQx * v12_4_1 + (VT)2.0 * oo2ze * v6_4_1 + (VT)2.0 * oo2e * (v12_1_0 - rho_e * v12_1_1);
            const VT v13_10_0 = QCx * v13_4_0 + WQx * v13_4_1 + (VT)1.0 * oo2ze * v7_4_1 + (VT)2.0 * oo2e * (v13_1_0 - rho_e * v13_1_1);
            const VT v14_10_0 = QCx * v14_4_0 + WQx * v14_4_1 + (VT)1.0 * oo2ze * v9_4_1 + (VT)2.0 * oo2e * (v14_1_0 - rho_e * v14_1_1);
            const VT v15_10_0 = QCx * v15_4_0 + WQx * v15_4_1 + (VT)1.0 * oo2ze * v8_4_1 + (VT)2.0 * oo2e * (v15_1_0 - rho_e * v15_1_1);
            const VT v16_10_0 = QCx * v16_4_0 + WQx * v16_4_1 + (VT)2.0 * oo2e * (v16_1_0 - rho_e * v16_1_1);
            const VT v17_10_0 = QCx * v17_4_0 + WQx * v17_4_1 + (VT)2.0 * oo2e * (v17_1_0 - rho_e * v17_1_1);
            const VT v18_10_0 = QCx * v18_4_0 + WQx * v18_4_1 + (VT)2.0 * oo2e * (v18_1_0 - rho_e * v18_1_1);
            const VT v19_10_0 = QCx * v19_4_0 + WQx * v19_4_1 + (VT)2.0 * oo2e * (v19_1_0 - rho_e * v19_1_1);
            const VT v10_11_0 = QCx * v10_5_0 + WQx * v10_5_1 + (VT)3.0 * oo2ze * v4_5_1 + (VT)1.0 * oo2e * (v10_2_0 - rho_e * v10_2_1);
            const VT v11_11_0 = QCx * v11_5_0 + WQx * v11_5_1 + (VT)2.0 * oo2ze * v5_5_1 + (VT)1.0 * oo2e * (v11_2_0 - rho_e * v11_2_1);
            const VT v12_11_0 = QCx * v12_5_0 + WQx * v12_5_1 + (VT)2.0 * oo2ze * v6_5_1 + (VT)1.0 * oo2e * (v12_2_0 - rho_e * v12_2_1);
            const VT v13_11_0 = QCx * v13_5_0 + WQx * v13_5_1 + (VT)1.0 * oo2ze * v7_5_1 + (VT)1.0 * oo2e * (v13_2_0 - rho_e * v13_2_1);
            const VT v14_11_0 = QCx * v14_5_0 + WQx * v14_5_1 + (VT)1.0 * oo2ze * v9_5_1 + (VT)1.0 * oo2e * (v14_2_0 - rho_e * v14_2_1);
            const VT v15_11_0 = QCx * v15_5_0 + WQx * v15_5_1 + (VT)1.0 * oo2ze * v8_5_1 + (VT)1.0 * oo2e * (v15_2_0 - rho_e * v15_2_1);
            const VT v16_11_0 = QCx * v16_5_0 + WQx * v16_5_1 + (VT)1.0 * oo2e * (v16_2_0 - rho_e * v16_2_1);
            const VT v17_11_0 = QCx * v17_5_0 + WQx * v17_5_1 + (VT)1.0 * oo2e * (v17_2_0 - rho_e * v17_2_1);
            const VT v18_11_0 = QCx * v18_5_0 + WQx * v18_5_1 + (VT)1.0 * oo2e * (v18_2_0 - rho_e * v18_2_1);
            const VT v19_11_0 = QCx * v19_5_0 + WQx * v19_5_1 + (VT)1.0 * oo2e * (v19_2_0 - rho_e * v19_2_1);
            const VT v10_12_0 = QCx * v10_6_0 + WQx * v10_6_1 + (VT)3.0 * oo2ze * v4_6_1 + (VT)1.0 * oo2e * (v10_3_0 - rho_e * v10_3_1);
            const VT v11_12_0 = QCx * v11_6_0 + WQx * v11_6_1 + (VT)2.0 * oo2ze * v5_6_1 + (VT)1.0 * oo2e * (v11_3_0 - rho_e * v11_3_1);
            const VT v12_12_0 = QCx * v12_6_0 + WQx * v12_6_1 + (VT)2.0 * oo2ze * v6_6_1 + (VT)1.0 * oo2e * (v12_3_0 - rho_e * v12_3_1);
            const VT v13_12_0 = QCx * v13_6_0 + WQx * v13_6_1 + (VT)1.0 * oo2ze * v7_6_1 + (VT)1.0 * oo2e * (v13_3_0 - rho_e * v13_3_1);
            const VT v14_12_0 = QCx * v14_6_0 + WQx * v14_6_1 + (VT)1.0 * oo2ze * v9_6_1 + (VT)1.0 * oo2e * (v14_3_0 - rho_e * v14_3_1);
            const VT v15_12_0 = QCx * v15_6_0 + WQx * v15_6_1 + (VT)1.0 * oo2ze * v8_6_1 + (VT)1.0 * oo2e * (v15_3_0 - rho_e * v15_3_1);
            const VT v16_12_0 = QCx * v16_6_0 + WQx * v16_6_1 + (VT)1.0 * oo2e * (v16_3_0 - rho_e * v16_3_1);
            const VT v17_12_0 = QCx * v17_6_0 + WQx * v17_6_1 + (VT)1.0 * oo2e * (v17_3_0 - rho_e * v17_3_1);
            const VT v18_12_0 = QCx * v18_6_0 + WQx * v18_6_1 + (VT)1.0 * oo2e * (v18_3_0 - rho_e * v18_3_1);
            const VT v19_12_0 = QCx * v19_6_0 + WQx * v19_6_1 + (VT)1.0 * oo2e * (v19_3_0 - rho_e * v19_3_1);
            const VT v10_13_0 = QCy * v10_5_0 + WQy * v10_5_1 + (VT)1.0 * oo2e * (v10_1_0 - rho_e * v10_1_1);
            const VT v11_13_0 = QCy * v11_5_0 + WQy * v11_5_1 + (VT)1.0 * oo2ze * v4_5_1 + (VT)1.0 * oo2e * (v11_1_0 - rho_e * v11_1_1);
            const VT v12_13_0 = QCy * v12_5_0 + WQy * v12_5_1 + (VT)1.0 * oo2e * (v12_1_0 - rho_e * v12_1_1);
            const VT v13_13_0 = QCy * v13_5_0 + WQy * v13_5_1 + (VT)2.0 * oo2ze * v5_5_1 + (VT)1.0 * oo2e * (v13_1_0 - rho_e * v13_1_1);
            const VT v14_13_0 = QCy * v14_5_0 + WQy * v14_5_1 + (VT)1.0 * oo2e * (v14_1_0 - rho_e * v14_1_1);
            const VT v15_13_0 = QCy * v15_5_0 + WQy * v15_5_1 + (VT)1.0 * oo2ze * v6_5_1 + (VT)1.0 * oo2e * (v15_1_0 - rho_e * v15_1_1);
            const VT v16_13_0 = QCy * v16_5_0 + WQy * v16_5_1 + (VT)3.0 * oo2ze * v7_5_1 + (VT)1.0 * oo2e * (v16_1_0 - rho_e * v16_1_1);
            const VT v17_13_0 = QCy * v17_5_0 + WQy * v17_5_1 + (VT)2.0 * oo2ze * v8_5_1 + (VT)1.0 * oo2e * (v17_1_0 - rho_e * v17_1_1);
            const VT v18_13_0 = QCy * v18_5_0 + WQy * v18_5_1 + (VT)1.0 * oo2ze * v9_5_1 + (VT)1.0 * oo2e * (v18_1_0 - rho_e * v18_1_1);
            const VT v19_13_0 = QCy * v19_5_0 + WQy * v19_5_1 + (VT)1.0 * oo2e * (v19_1_0 - rho_e * v19_1_1);
            const VT v10_14_0 = QCz * v10_6_0 + WQz * v10_6_1 + (VT)1.0 * oo2e * (v10_1_0 - rho_e * v10_1_1);
            const VT v11_14_0 = QCz * v11_6_0 + WQz * v11_6_1 + (VT)1.0 * oo2e * (v11_1_0 - rho_e * v11_1_1);
            const VT v12_14_0 = QCz * v12_6_0 + WQz * v12_6_1 + (VT)1.0 * oo2ze * v4_6_1 + (VT)1.0 * oo2e * (v12_1_0 - rho_e * v12_1_1);
            const VT v13_14_0 = QCz * v13_6_0 + WQz * v13_6_1 + (VT)1.0 * oo2e * (v13_1_0 - rho_e * v13_1_1);
            const VT v14_14_0 = QCz * v14_6_0 + WQz * v14_6_1 + (VT)2.0 * oo2ze * v6_6_1 + (VT)1.0 * oo2e * (v14_1_0 - rho_e * v14_1_1);
            const VT v15_14_0 = QCz * v15_6_0 + WQz * v15_6_1 + (VT)1.0 * oo2ze * v5_6_1 + (VT)1.0 * oo2e * (v15_1_0 - rho_e * v15_1_1);
            const VT v16_14_0 = QCz * v16_6_0 + WQz * v16_6_1 + (VT)1.0 * oo2e * (v16_1_0 - rho_e * v16_1_1);
            const VT v17_14_0 = QCz * v17_6_0 + WQz * v17_6_1 + (VT)1.0 * oo2ze * v7_6_1 + (VT)1.0 * oo2e * (v17_1_0 - rho_e * v17_1_1);
            const VT v18_14_0 = QCz * v18_6_0 + WQz * v18_6_1 + (VT)2.0 * oo2ze * v8_6_1 + (VT)1.0 * oo2e * (v18_1_0 - rho_e * v18_1_1);
            const VT v19_14_0 = QCz * v19_6_0 + WQz * v19_6_1 + (VT)3.0 * oo2ze * v9_6_1 + (VT)1.0 * oo2e * (v19_1_0 - rho_e * v19_1_1);
            const VT v10_15_0 = QCx * v10_8_0 + WQx * v10_8_1 + (VT)3.0 * oo2ze * v4_8_1;
            const VT v11_15_0 = QCx * v11_8_0 + WQx * v11_8_1 + (VT)2.0 * oo2ze * v5_8_1;
            const VT v12_15_0 = QCx * v12_8_0 + WQx * v12_8_1 + (VT)2.0 * oo2ze * v6_8_1;
            const VT v13_15_0 = QCx * v13_8_0 + WQx * v13_8_1 + (VT)1.0 * oo2ze * v7_8_1;
            const VT v14_15_0 = QCx * v14_8_0 + WQx * v14_8_1 + (VT)1.0 * oo2ze * v9_8_1;
            const VT v15_15_0 = QCx * v15_8_0 + WQx * v15_8_1 + (VT)1.0 * oo2ze * v8_8_1;
            const VT v16_15_0 = QCx * v16_8_0 + WQx * v16_8_1;
            const VT v17_15_0 = QCx * v17_8_0 + WQx * v17_8_1;
            const VT v18_15_0 = QCx * v18_8_0 + WQx * v18_8_1;
            const VT v19_15_0 = QCx * v19_8_0 + WQx * v19_8_1;
            const VT v10_16_0 = QCy * v10_7_0 + WQy * v10_7_1 + (VT)2.0 * oo2e * (v10_2_0 - rho_e * v10_2_1);
            const VT v11_16_0 = QCy * v11_7_0 + WQy * v11_7_1 + (VT)1.0 * oo2ze * v4_7_1 + (VT)2.0 * oo2e * (v11_2_0 - rho_e * v11_2_1);
            const VT v12_16_0 = QCy * v12_7_0 + WQy * v12_7_1 + (VT)2.0 * oo2e * (v12_2_0 - rho_e * v12_2_1);
            const VT v13_16_0 = QCy * v13_7_0 + WQy * v13_7_1 + (VT)2.0 * oo2ze * v5_7_1 + (VT)2.0 * oo2e * (v13_2_0 - rho_e * v13_2_1);
            const VT v14_16_0 = QCy * v14_7_0 + WQy * v14_7_1 + (VT)2.0 * oo2e * (v14_2_0 - rho_e * v14_2_1);
            const VT v15_16_0 = QCy * v15_7_0 + WQy * v15_7_1 + (VT)1.0 * oo2ze * v6_7_1 + (VT)2.0 * oo2e * (v15_2_0 - rho_e * v15_2_1);
            const VT v16_16_0 = QCy * v16_7_0 + WQy * v16_7_1 + (VT)3.0 * oo2ze * v7_7_1 + (VT)2.0 * oo2e * (v16_2_0 - rho_e * v16_2_1);
            const VT v17_16_0 = QCy * v17_7_0 + WQy * v17_7_1 + (VT)2.0 * oo2ze * v8_7_1 + (VT)2.0 * oo2e * (v17_2_0 - rho_e * v17_2_1);
            const VT v18_16_0 = QCy * v18_7_0 + WQy * v18_7_1 + (VT)1.0 * oo2ze * v9_7_1 + (VT)2.0 * oo2e * (v18_2_0 - rho_e * v18_2_1);
            const VT v19_16_0 = QCy * v19_7_0 + WQy * v19_7_1 + (VT)2.0 * oo2e * (v19_2_0 - rho_e * v19_2_1);
            const VT v10_17_0 = QCy * v10_8_0 + WQy * v10_8_1 + (VT)1.0 * oo2e * (v10_3_0 - rho_e * v10_3_1);
            const VT v11_17_0 = QCy * v11_8_0 + WQy * v11_8_1 + (VT)1.0 * oo2ze * v4_8_1 + (VT)1.0 * oo2e * (v11_3_0 - rho_e * v11_3_1);
            const VT v12_17_0 = QCy * v12_8_0 + WQy * v12_8_1 + (VT)1.0 * oo2e * (v12_3_0 - rho_e * v12_3_1);
            const VT v13_17_0 = QCy * v13_8_0 + WQy * v13_8_1 + (VT)2.0 * oo2ze * v5_8_1 + (VT)1.0 * oo2e * (v13_3_0 - rho_e * v13_3_1);
            const VT v14_17_0 = QCy * v14_8_0 + WQy * v14_8_1 + (VT)1.0 * oo2e * (v14_3_0 - rho_e * v14_3_1);
            const VT v15_17_0 = QCy * v15_8_0 + WQy * v15_8_1 + (VT)1.0 * oo2ze * v6_8_1 + (VT)1.0 * oo2e * (v15_3_0 - rho_e * v15_3_1);
            const VT v16_17_0 = QCy * v16_8_0 + WQy * v16_8_1 + (VT)3.0 * oo2ze * v7_8_1 + (VT)1.0 * oo2e * (v16_3_0 - rho_e * v16_3_1);
            const VT v17_17_0 = QCy * v17_8_0 + WQy * v17_8_1 + (VT)2.0 * oo2ze * v8_8_1 + (VT)1.0 * oo2e * (v17_3_0 - rho_e * v17_3_1);
            const VT v18_17_0 = QCy * v18_8_0 + WQy * v18_8_1 + (VT)1.0 * oo2ze * v9_8_1 + (VT)1.0 * oo2e * (v18_3_0 - rho_e * v18_3_1);
            const VT v19_17_0 = QCy * v19_8_0 + WQy * v19_8_1 + (VT)1.0 * oo2e * (v19_3_0 - rho_e * v19_3_1);
            const VT v10_18_0 = QCz * v10_8_0 + WQz * v10_8_1 + (VT)1.0 * oo2e * (v10_2_0 - rho_e * v10_2_1);
            const VT v11_18_0 = QCz * v11_8_0 + WQz * v11_8_1 + (VT)1.0 * oo2e * (v11_2_0 - rho_e * v11_2_1);
            const VT v12_18_0 = QCz * v12_8_0 + WQz * v12_8_1 + (VT)1.0 * oo2ze * v4_8_1 + (VT)1.0 * oo2e * (v12_2_0 - rho_e * v12_2_1);
            const VT v13_18_0 = QCz * v13_8_0 + WQz * v13_8_1 + (VT)1.0 * oo2e * (v13_2_0 - rho_e * v13_2_1);
            const VT v14_18_0 = QCz * v14_8_0 + WQz * v14_8_1 + (VT)2.0 * oo2ze * v6_8_1 + (VT)1.0 * oo2e * (v14_2_0 - rho_e * v14_2_1);
            const VT v15_18_0 = QCz * v15_8_0 + WQz * v15_8_1 + (VT)1.0 * oo2ze * v5_8_1 + (VT)1.0 * oo2e * (v15_2_0 - rho_e * v15_2_1);
            const VT v16_18_0 = QCz * v16_8_0 + WQz * v16_8_1 + (VT)1.0 * oo2e * (v16_2_0 - rho_e * v16_2_1);
            const VT v17_18_0 = QCz * v17_8_0 + WQz * v17_8_1 + (VT)1.0 * oo2ze * v7_8_1 + (VT)1.0 * oo2e * (v17_2_0 - rho_e * v17_2_1);
            const VT v18_18_0 = QCz * v18_8_0 + WQz * v18_8_1 + (VT)2.0 * oo2ze * v8_8_1 + (VT)1.0 * oo2e * (v18_2_0 - rho_e * v18_2_1);
            const VT v19_18_0 = QCz * v19_8_0 + WQz * v19_8_1 + (VT)3.0 * oo2ze * v9_8_1 + (VT)1.0 * oo2e * (v19_2_0 - rho_e * v19_2_1);
            const VT v10_19_0 = QCz * v10_9_0 + WQz * v10_9_1 + (VT)2.0 * oo2e * (v10_3_0 - rho_e * v10_3_1);
            const VT v11_19_0 = QCz * v11_9_0 + WQz * v11_9_1 + (VT)2.0 * oo2e * (v11_3_0 - rho_e * v11_3_1);
            const VT v12_19_0 = QCz * v12_9_0 + WQz * v12_9_1 + (VT)1.0 * oo2ze * v4_9_1 + (VT)2.0 * oo2e * (v12_3_0 - rho_e * v12_3_1);
            const VT v13_19_0 = QCz * v13_9_0 + WQz * v13_9_1 + (VT)2.0 * oo2e * (v13_3_0 - rho_e * v13_3_1);
            const VT v14_19_0 = QCz * v14_9_0 + WQz * v14_9_1 + (VT)2.0 * oo2ze * v6_9_1 + (VT)2.0 * oo2e * (v14_3_0 - rho_e * v14_3_1);
            const VT v15_19_0 = QCz * v15_9_0 + WQz * v15_9_1 + (VT)1.0 * oo2ze * v5_9_1 + (VT)2.0 * oo2e * (v15_3_0 - rho_e * v15_3_1);
            const VT v16_19_0 = QCz * v16_9_0 + WQz * v16_9_1 + (VT)2.0 * oo2e * (v16_3_0 - rho_e * v16_3_1);
            const VT v17_19_0 = QCz * v17_9_0 + WQz * v17_9_1 + (VT)1.0 * oo2ze * v7_9_1 + (VT)2.0 * oo2e * (v17_3_0 - rho_e * v17_3_1);
            const VT v18_19_0 = QCz * v18_9_0 + WQz * v18_9_1 + (VT)2.0 * oo2ze * v8_9_1 + (VT)2.0 * oo2e * (v18_3_0 - rho_e * v18_3_1);
            const VT v19_19_0 = QCz * v19_9_0 + WQz * v19_9_1 + (VT)3.0 * oo2ze * v9_9_1 + (VT)2.0 * oo2e * (v19_3_0 - rho_e * v19_3_1);
            acc[0] += (double)v10_10_0;
            acc[1] += (double)v10_11_0;
            acc[2] += (double)v10_12_0;
            acc[3] += (double)v10_13_0;
            acc[4] += (double)v10_14_0;
            acc[5] += (double)v10_15_0;
            acc[6] += (double)v10_16_0;
            acc[7] += (double)v10_17_0;
            acc[8] += (double)v10_18_0;
            acc[9] += (double)v10_19_0;
            acc[10] += (double)v11_10_0;
            acc[11] += (double)v11_11_0;
            acc[12] += (double)v11_12_0;
            acc[13] += (double)v11_13_0;
            acc[14] += (double)v11_14_0;
            acc[15] += (double)v11_15_0;
            acc[16] += (double)v11_16_0;
            acc[17] += (double)v11_17_0;
            acc[18] += (double)v11_18_0;
            acc[19] += (double)v11_19_0;
            acc[20] += (double)v12_10_0;
            acc[21] += (double)v12_11_0;
            acc[22] += (double)v12_12_0;
            acc[23] += (double)v12_13_0;
            acc[24] += (double)v12_14_0;
            acc[25] += (double)v12_15_0;
            acc[26] += (double)v12_16_0;
            acc[27] += (double)v12_17_0;
            acc[28] += (double)v12_18_0;
            acc[29] += (double)v12_19_0;
            acc[30] += (double)v13_10_0;
            acc[31] += (double)v13_11_0;
            acc[32] += (double)v13_12_0;
            acc[33] += (double)v13_13_0;
            acc[34] += (double)v13_14_0;
            acc[35] += (double)v13_15_0;
            acc[36] += (double)v13_16_0;
            acc[37] += (double)v13_17_0;
            acc[38] += (double)v13_18_0;
            acc[39] += (double)v13_19_0;
            acc[40] += (double)v14_10_0;
            acc[41] += (double)v14_11_0;
            acc[42] += (double)v14_12_0;
            acc[43] += (double)v14_13_0;
            acc[44] += (double)v14_14_0;
            acc[45] += (double)v14_15_0;
            acc[46] += (double)v14_16_0;
            acc[47] += (double)v14_17_0;
            acc[48] += (double)v14_18_0;
            acc[49] += (double)v14_19_0;
            acc[50] += (double)v15_10_0;
            acc[51] += (double)v15_11_0;
            acc[52] += (double)v15_12_0;
            acc[53] += (double)v15_13_0;
            acc[54] += (double)v15_14_0;
            acc[55] += (double)v15_15_0;
            acc[56] += (double)v15_16_0;
            acc[57] += (double)v15_17_0;
            acc[58] += (double)v15_18_0;
            acc[59] += (double)v15_19_0;
            acc[60] += (double)v16_10_0;
            acc[61] += (double)v16_11_0;
            acc[62] += (double)v16_12_0;
            acc[63] += (double)v16_13_0;
            acc[64] += (double)v16_14_0;
            acc[65] += (double)v16_15_0;
            acc[66] += (double)v16_16_0;
            acc[67] += (double)v16_17_0;
            acc[68] += (double)v16_18_0;
            acc[69] += (double)v16_19_0;
            acc[70] += (double)v17_10_0;
            acc[71] += (double)v17_11_0;
            acc[72] += (double)v17_12_0;
            acc[73] += (double)v17_13_0;
            acc[74] += (double)v17_14_0;
            acc[75] += (double)v17_15_0;
            acc[76] += (double)v17_16_0;
            acc[77] += (double)v17_17_0;
            acc[78] += (double)v17_18_0;
            acc[79] += (double)v17_19_0;
            acc[80] += (double)v18_10_0;
            acc[81] += (double)v18_11_0;
            acc[82] += (double)v18_12_0;
            acc[83] += (double)v18_13_0;
            acc[84] += (double)v18_14_0;
            acc[85] += (double)v18_15_0;
            acc[86] += (double)v18_16_0;
            acc[87] += (double)v18_17_0;
            acc[88] += (double)v18_18_0;
            acc[89] += (double)v18_19_0;
            acc[90] += (double)v19_10_0;
            acc[91] += (double)v19_11_0;
            acc[92] += (double)v19_12_0;
            acc[93] += (double)v19_13_0;
            acc[94] += (double)v19_14_0;
            acc[95] += (double)v19_15_0;
            acc[96] += (double)v19_16_0;
            acc[97] += (double)v19_17_0;
            acc[98] += (double)v19_18_0;
            acc[99] += (double)v19_19_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[100] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_fsfs(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;

    res[0] = acc[0] * 0.06666666666666665;
    res[1] = acc[1] * 0.14907119849998599;
    res[2] = acc[2] * 0.14907119849998599;
    res[3] = acc[3] * 0.14907119849998599;
    res[4] = acc[4] * 0.14907119849998599;
    res[5] = acc[5] * 0.2581988897471611;
    res[6] = acc[6] * 0.06666666666666665;
    res[7] = acc[7] * 0.14907119849998599;
    res[8] = acc[8] * 0.14907119849998599;
    res[9] = acc[9] * 0.06666666666666665;
    res[10] = acc[10] * 0.14907119849998599;
    res[11] = acc[11] * 0.3333333333333334;
    res[12] = acc[12] * 0.3333333333333334;
    res[13] = acc[13] * 0.3333333333333334;
    res[14] = acc[14] * 0.3333333333333334;
    res[15] = acc[15] * 0.5773502691896258;
    res[16] = acc[16] * 0.14907119849998599;
    res[17] = acc[17] * 0.3333333333333334;
    res[18] = acc[18] * 0.3333333333333334;
    res[19] = acc[19] * 0.14907119849998599;
    res[20] = acc[20] * 0.14907119849998599;
    res[21] = acc[21] * 0.3333333333333334;
    res[22] = acc[22] * 0.3333333333333334;
    res[23] = acc[23] * 0.3333333333333334;
    res[24] = acc[24] * 0.3333333333333334;
    res[25] = acc[25] * 0.5773502691896258;
    res[26] = acc[26] * 0.14907119849998599;
    res[27] = acc[27] * 0.3333333333333334;
    res[28] = acc[28] * 0.3333333333333334;
    res[29] = acc[29] * 0.14907119849998599;
    res[30] = acc[30] * 0.14907119849998599;
    res[31] = acc[31] * 0.3333333333333334;
    res[32] = acc[32] * 0.3333333333333334;
    res[33] = acc[33] * 0.3333333333333334;
    res[34] = acc[34] * 0.3333333333333334;
    res[35] = acc[35] * 0.5773502691896258;
    res[36] = acc[36] * 0.14907119849998599;
    res[37] = acc[37] * 0.3333333333333334;
    res[38] = acc[38] * 0.3333333333333334;
    res[39] = acc[39] * 0.14907119849998599;
    res[40] = acc[40] * 0.14907119849998599;
    res[41] = acc[41] * 0.3333333333333334;
    res[42] = acc[42] * 0.3333333333333334;
    res[43] = acc[43] * 0.3333333333333334;
    res[44] = acc[44] * 0.3333333333333334;
    res[45] = acc[45] * 0.5773502691896258;
    res[46] = acc[46] * 0.14907119849998599;
    res[47] = acc[47] * 0.3333333333333334;
    res[48] = acc[48] * 0.3333333333333334;
    res[49] = acc[49] * 0.14907119849998599;
    res[50] = acc[50] * 0.2581988897471611;
    res[51] = acc[51] * 0.5773502691896258;
    res[52] = acc[52] * 0.5773502691896258;
    res[53] = acc[53] * 0.5773502691896258;
    res[54] = acc[54] * 0.5773502691896258;
    res[55] = acc[55];
    res[56] = acc[56] * 0.2581988897471611;
    res[57] = acc[57] * 0.5773502691896258;
    res[58] = acc[58] * 0.5773502691896258;
    res[59] = acc[59] * 0.2581988897471611;
    res[60] = acc[60] * 0.06666666666666665;
    res[61] = acc[61] * 0.14907119849998599;
    res[62] = acc[62] * 0.14907119849998599;
    res[63] = acc[63] * 0.14907119849998599;
    res[64] = acc[64] * 0.14907119849998599;
    res[65] = acc[65] * 0.2581988897471611;
    res[66] = acc[66] * 0.06666666666666665;
    res[67] = acc[67] * 0.14907119849998599;
    res[68] = acc[68] * 0.14907119849998599;
    res[69] = acc[69] * 0.06666666666666665;
    res[70] = acc[70] * 0.14907119849998599;
    res[71] = acc[71] * 0.3333333333333334;
    res[72] = acc[72] * 0.3333333333333334;
    res[73] = acc[73] * 0.3333333333333334;
    res[74] = acc[74] * 0.3333333333333334;
    res[75] = acc[75] * 0.5773502691896258;
    res[76] = acc[76] * 0.14907119849998599;
    res[77] = acc[77] * 0.3333333333333334;
    res[78] = acc[78] * 0.3333333333333334;
    res[79] = acc[79] * 0.14907119849998599;
    res[80] = acc[80] * 0.14907119849998599;
    res[81] = acc[81] * 0.3333333333333334;
    res[82] = acc[82] * 0.3333333333333334;
    res[83] = acc[83] * 0.3333333333333334;
    res[84] = acc[84] * 0.3333333333333334;
    res[85] = acc[85] * 0.5773502691896258;
    res[86] = acc[86] * 0.14907119849998599;
    res[87] = acc[87] * 0.3333333333333334;
    res[88] = acc[88] * 0.3333333333333334;
    res[89] = acc[89] * 0.14907119849998599;
    res[90] = acc[90] * 0.06666666666666665;
    res[91] = acc[91] * 0.14907119849998599;
    res[92] = acc[92] * 0.14907119849998599;
    res[93] = acc[93] * 0.14907119849998599;
    res[94] = acc[94] * 0.14907119849998599;
    res[95] = acc[95] * 0.2581988897471611;
    res[96] = acc[96] * 0.06666666666666665;
    res[97] = acc[97] * 0.14907119849998599;
    res[98] = acc[98] * 0.14907119849998599;
    res[99] = acc[99] * 0.06666666666666665;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[100]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_fsfs(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[100];
    vrr_fsfs<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 100; ++x) acc_out[x] = acc[x];
    }
    hrr_fsfs(P, p, q, acc, res);
}

__device__ __forceinline__ void store_fsfs(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
    const long long ij_0_0 = pair_index(ib_.z + 0, ib_.w + 0);
    const long long ij_1_0 = pair_index(ib_.z + 1, ib_.w + 0);
    const long long ij_2_0 = pair_index(ib_.z + 2, ib_.w + 0);
    const long long ij_3_0 = pair_index(ib_.z + 3, ib_.w + 0);
    const long long ij_4_0 = pair_index(ib_.z + 4, ib_.w + 0);
    const long long ij_5_0 = pair_index(ib_.z + 5, ib_.w + 0);
    const long long ij_6_0 = pair_index(ib_.z + 6, ib_.w + 0);
    const long long ij_7_0 = pair_index(ib_.z + 7, ib_.w + 0);
    const long long ij_8_0 = pair_index(ib_.z + 8, ib_.w + 0);
    const long long ij_9_0 = pair_index(ib_.z + 9, ib_.w + 0);
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    const long long kl_1_0 = pair_index(ik_.z + 1, ik_.w + 0);
    const long long kl_2_0 = pair_index(ik_.z + 2, ik_.w + 0);
    const long long kl_3_0 = pair_index(ik_.z + 3, ik_.w + 0);
    const long long kl_4_0 = pair_index(ik_.z + 4, ik_.w + 0);
    const long long kl_5_0 = pair_index(ik_.z + 5, ik_.w + 0);
    const long long kl_6_0 = pair_index(ik_.z + 6, ik_.w + 0);
    const long long kl_7_0 = pair_index(ik_.z + 7, ik_.w + 0);
    const long long kl_8_0 = pair_index(ik_.z + 8, ik_.w + 0);
    const long long kl_9_0 = pair_index(ik_.z + 9, ik_.w + 0);
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
    { const long long ij = ij_0_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_0_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_1_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_1_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_1_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_1_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_1_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_1_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_1_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_2_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_2_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_2_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_2_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_2_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_2_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_2_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_3_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_3_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_3_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_3_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_3_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_3_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_3_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_4_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_4_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_4_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_4_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_4_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_4_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_4_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_5_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_5_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_5_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_5_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_5_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_5_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_5_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_6_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_6_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_6_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_6_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_6_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_6_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_6_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_6_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_6_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_7_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_7_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_7_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_7_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_7_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_7_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_7_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_7_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_7_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_8_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_8_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_8_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_8_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_8_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_8_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_8_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_8_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_8_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_9_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_9_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_9_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_9_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_9_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_9_0, kl = kl_6_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_9_0, kl = kl_7_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_9_0, kl = kl_8_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_9_0, kl = kl_9_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_fsfs(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 100; ++x) {
        const int ia = x / 10, ibb = (x / 10) % 1, ic = (x / 1) % 10, id = x % 1;
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
__global__ void __launch_bounds__(128) eri_queue_fsfs(const EriQueue Q) {
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
        double acc[100];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 100; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_fsfs<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_fsfs<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 100; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 100 doubles (launch_eri_fsfs)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 100);
            if (lead) hrr_fsfs(Q.pairs, p, q, acc, sb + kq * 100);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)100;
            for (int t = lane; t < nlive * 100; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[100];
            hrr_fsfs(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_fsfs(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_fsfs(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (102400 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_fsfs() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_fsfs<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 102400);
        cudaFuncSetAttribute(eri_queue_fsfs<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 102400);
        done[dev] = true;
    }
}

void launch_eri_fsfs(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 102400 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 102400 : 0;
    if (smem) eri_prepare_fsfs();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_fsfs<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_fsfs<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_fsfs<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_fsfs<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_fsfs(int mixed) {
    eri_prepare_fsfs();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fsfs<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fsfs<0, 0>, 128, 0);
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
__global__ void __launch_bounds__(128) schwarz_kernel_fsfs(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[100];
    if (full) {
        quartet_fsfs<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[11]));
    m = fmax(m, fabs(res[22]));
    m = fmax(m, fabs(res[33]));
    m = fmax(m, fabs(res[44]));
    m = fmax(m, fabs(res[55]));
    m = fmax(m, fabs(res[66]));
    m = fmax(m, fabs(res[77]));
    m = fmax(m, fabs(res[88]));
    m = fmax(m, fabs(res[99]));
        qout[p] = sqrt(m);
        return;
    }
    double acc[100];
    for (int k = 0; k < in.y; ++k) {
        quartet_fsfs<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[11]));
    m = fmax(m, fabs(res[22]));
    m = fmax(m, fabs(res[33]));
    m = fmax(m, fabs(res[44]));
    m = fmax(m, fabs(res[55]));
    m = fmax(m, fabs(res[66]));
    m = fmax(m, fabs(res[77]));
    m = fmax(m, fabs(res[88]));
    m = fmax(m, fabs(res[99]));
        w = fmax(w, fabs(acc[0]));
        w = fmax(w, fabs(acc[11]));
        w = fmax(w, fabs(acc[22]));
        w = fmax(w, fabs(acc[33]));
        w = fmax(w, fabs(acc[44]));
        w = fmax(w, fabs(acc[55]));
        w = fmax(w, fabs(acc[66]));
        w = fmax(w, fabs(acc[77]));
        w = fmax(w, fabs(acc[88]));
        w = fmax(w, fabs(acc[99]));
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }
}

void launch_schwarz_fsfs(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    schwarz_kernel_fsfs<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}

}  // namespace molints

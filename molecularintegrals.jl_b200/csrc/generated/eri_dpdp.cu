// Generated by gen_eri.py -- class (dp|dp).  Do not edit.
// VRR entries: 630, contracted block: 256, HRR lines: 612, outputs: 324.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[256], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_dpdp(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 256; ++x) acc[x] = 0.0;
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
            const VT v0_1_2 = QCx * v0_0_2 + WQx * v0_0_3;
            const VT v1_1_1 = QCx * v1_0_1 + WQx * v1_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v1_1_2 = QCx * v1_0_2 + WQx * v1_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v2_1_1 = QCx * v2_0_1 + WQx * v2_0_2;
            const VT v2_1_2 = QCx * v2_0_2 + WQx * v2_0_3;
            const VT v3_1_1 = QCx * v3_0_1 + WQx * v3_0_2;
            const VT v3_1_2 = QCx * v3_0_2 + WQx * v3_0_3;
            const VT v4_1_0 = QCx * v4_0_0 + WQx * v4_0_1 + (VT)2.0 * oo2ze * v1_0_1;
            const VT v4_1_1 = QCx * v4_0_1 + WQx * v4_0_2 + (VT)2.0 * oo2ze * v1_0_2;
            const VT v4_1_2 = QCx * v4_0_2 + WQx * v4_0_3 + (VT)2.0 * oo2ze * v1_0_3;
            const VT v5_1_0 = QCx * v5_0_0 + WQx * v5_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v5_1_1 = QCx * v5_0_1 + WQx * v5_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v5_1_2 = QCx * v5_0_2 + WQx * v5_0_3 + (VT)1.0 * oo2ze * v2_0_3;
            const VT v6_1_0 = QCx * v6_0_0 + WQx * v6_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v6_1_1 = QCx * v6_0_1 + WQx * v6_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v6_1_2 = QCx * v6_0_2 + WQx * v6_0_3 + (VT)1.0 * oo2ze * v3_0_3;
            const VT v7_1_0 = QCx * v7_0_0 + WQx * v7_0_1;
            const VT v7_1_1 = QCx * v7_0_1 + WQx * v7_0_2;
            const VT v7_1_2 = QCx * v7_0_2 + WQx * v7_0_3;
            const VT v8_1_0 = QCx * v8_0_0 + WQx * v8_0_1;
            const VT v8_1_1 = QCx * v8_0_1 + WQx * v8_0_2;
            const VT v8_1_2 = QCx * v8_0_2 + WQx * v8_0_3;
            const VT v9_1_0 = QCx * v9_0_0 + WQx * v9_0_1;
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
            const VT v0_2_2 = QCy * v0_0_2 + WQy * v0_0_3;
            const VT v1_2_1 = QCy * v1_0_1 + WQy * v1_0_2;
            const VT v1_2_2 = QCy * v1_0_2 + WQy * v1_0_3;
            const VT v2_2_1 = QCy * v2_0_1 + WQy * v2_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v2_2_2 = QCy * v2_0_2 + WQy * v2_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v3_2_1 = QCy * v3_0_1 + WQy * v3_0_2;
            const VT v3_2_2 = QCy * v3_0_2 + WQy * v3_0_3;
            const VT v4_2_0 = QCy * v4_0_0 + WQy * v4_0_1;
            const VT v4_2_1 = QCy * v4_0_1 + WQy * v4_0_2;
            const VT v4_2_2 = QCy * v4_0_2 + WQy * v4_0_3;
            const VT v5_2_0 = QCy * v5_0_0 + WQy * v5_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v5_2_1 = QCy * v5_0_1 + WQy * v5_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v5_2_2 = QCy * v5_0_2 + WQy * v5_0_3 + (VT)1.0 * oo2ze * v1_0_3;
            const VT v6_2_0 = QCy * v6_0_0 + WQy * v6_0_1;
            const VT v6_2_1 = QCy * v6_0_1 + WQy * v6_0_2;
            const VT v6_2_2 = QCy * v6_0_2 + WQy * v6_0_3;
            const VT v7_2_0 = QCy * v7_0_0 + WQy * v7_0_1 + (VT)2.0 * oo2ze * v2_0_1;
            const VT v7_2_1 = QCy * v7_0_1 + WQy * v7_0_2 + (VT)2.0 * oo2ze * v2_0_2;
            const VT v7_2_2 = QCy * v7_0_2 + WQy * v7_0_3 + (VT)2.0 * oo2ze * v2_0_3;
            const VT v8_2_0 = QCy * v8_0_0 + WQy * v8_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v8_2_1 = QCy * v8_0_1 + WQy * v8_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v8_2_2 = QCy * v8_0_2 + WQy * v8_0_3 + (VT)1.0 * oo2ze * v3_0_3;
            const VT v9_2_0 = QCy * v9_0_0 + WQy * v9_0_1;
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
            const VT v0_3_2 = QCz * v0_0_2 + WQz * v0_0_3;
            const VT v1_3_1 = QCz * v1_0_1 + WQz * v1_0_2;
            const VT v1_3_2 = QCz * v1_0_2 + WQz * v1_0_3;
            const VT v2_3_1 = QCz * v2_0_1 + WQz * v2_0_2;
            const VT v2_3_2 = QCz * v2_0_2 + WQz * v2_0_3;
            const VT v3_3_1 = QCz * v3_0_1 + WQz * v3_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v3_3_2 = QCz * v3_0_2 + WQz * v3_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v4_3_0 = QCz * v4_0_0 + WQz * v4_0_1;
            const VT v4_3_1 = QCz * v4_0_1 + WQz * v4_0_2;
            const VT v4_3_2 = QCz * v4_0_2 + WQz * v4_0_3;
            const VT v5_3_0 = QCz * v5_0_0 + WQz * v5_0_1;
            const VT v5_3_1 = QCz * v5_0_1 + WQz * v5_0_2;
            const VT v5_3_2 = QCz * v5_0_2 + WQz * v5_0_3;
            const VT v6_3_0 = QCz * v6_0_0 + WQz * v6_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v6_3_1 = QCz * v6_0_1 + WQz * v6_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v6_3_2 = QCz * v6_0_2 + WQz * v6_0_3 + (VT)1.0 * oo2ze * v1_0_3;
            const VT v7_3_0 = QCz * v7_0_0 + WQz * v7_0_1;
            const VT v7_3_1 = QCz * v7_0_1 + WQz * v7_0_2;
            const VT v7_3_2 = QCz * v7_0_2 + WQz * v7_0_3;
            const VT v8_3_0 = QCz * v8_0_0 + WQz * v8_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v8_3_1 = QCz * v8_0_1 + WQz * v8_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v8_3_2 = QCz * v8_0_2 + WQz * v8_0_3 + (VT)1.0 * oo2ze * v2_0_3;
            const VT v9_3_0 = QCz * v9_0_0 + WQz * v9_0_1 + (VT)2.0 * oo2ze * v3_0_1;
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
            const VT v1_4_1 = QCx * v1_1_1 + WQx * v1_1_2 + (VT)1.0 * oo2ze * v0_1_2 + (VT)1.0 * oo2e * (v1_0_1 - rho_e * v1_0_2);
            const VT v2_4_1 = QCx * v2_1_1 + WQx * v2_1_2 + (VT)1.0 * oo2e * (v2_0_1 - rho_e * v2_0_2);
            const VT v3_4_1 = QCx * v3_1_1 + WQx * v3_1_2 + (VT)1.0 * oo2e * (v3_0_1 - rho_e * v3_0_2);
            const VT v4_4_0 = QCx * v4_1_0 + WQx * v4_1_1 + (VT)2.0 * oo2ze * v1_1_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v4_4_1 = QCx * v4_1_1 + WQx * v4_1_2 + (VT)2.0 * oo2ze * v1_1_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v5_4_0 = QCx * v5_1_0 + WQx * v5_1_1 + (VT)1.0 * oo2ze * v2_1_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v5_4_1 = QCx * v5_1_1 + WQx * v5_1_2 + (VT)1.0 * oo2ze * v2_1_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v6_4_0 = QCx * v6_1_0 + WQx * v6_1_1 + (VT)1.0 * oo2ze * v3_1_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v6_4_1 = QCx * v6_1_1 + WQx * v6_1_2 + (VT)1.0 * oo2ze * v3_1_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v7_4_0 = QCx * v7_1_0 + WQx * v7_1_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v7_4_1 = QCx * v7_1_1 + WQx * v7_1_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v8_4_0 = QCx * v8_1_0 + WQx * v8_1_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v8_4_1 = QCx * v8_1_1 + WQx * v8_1_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v9_4_0 = QCx * v9_1_0 + WQx * v9_1_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
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
            const VT v1_5_1 = QCx * v1_2_1 + WQx * v1_2_2 + (VT)1.0 * oo2ze * v0_2_2;
            const VT v2_5_1 = QCx * v2_2_1 + WQx * v2_2_2;
            const VT v3_5_1 = QCx * v3_2_1 + WQx * v3_2_2;
            const VT v4_5_0 = QCx * v4_2_0 + WQx * v4_2_1 + (VT)2.0 * oo2ze * v1_2_1;
            const VT v4_5_1 = QCx * v4_2_1 + WQx * v4_2_2 + (VT)2.0 * oo2ze * v1_2_2;
            const VT v5_5_0 = QCx * v5_2_0 + WQx * v5_2_1 + (VT)1.0 * oo2ze * v2_2_1;
            const VT v5_5_1 = QCx * v5_2_1 + WQx * v5_2_2 + (VT)1.0 * oo2ze * v2_2_2;
            const VT v6_5_0 = QCx * v6_2_0 + WQx * v6_2_1 + (VT)1.0 * oo2ze * v3_2_1;
            const VT v6_5_1 = QCx * v6_2_1 + WQx * v6_2_2 + (VT)1.0 * oo2ze * v3_2_2;
            const VT v7_5_0 = QCx * v7_2_0 + WQx * v7_2_1;
            const VT v7_5_1 = QCx * v7_2_1 + WQx * v7_2_2;
            const VT v8_5_0 = QCx * v8_2_0 + WQx * v8_2_1;
            const VT v8_5_1 = QCx * v8_2_1 + WQx * v8_2_2;
            const VT v9_5_0 = QCx * v9_2_0 + WQx * v9_2_1;
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
            const VT v1_6_1 = QCx * v1_3_1 + WQx * v1_3_2 + (VT)1.0 * oo2ze * v0_3_2;
            const VT v2_6_1 = QCx * v2_3_1 + WQx * v2_3_2;
            const VT v3_6_1 = QCx * v3_3_1 + WQx * v3_3_2;
            const VT v4_6_0 = QCx * v4_3_0 + WQx * v4_3_1 + (VT)2.0 * oo2ze * v1_3_1;
            const VT v4_6_1 = QCx * v4_3_1 + WQx * v4_3_2 + (VT)2.0 * oo2ze * v1_3_2;
            const VT v5_6_0 = QCx * v5_3_0 + WQx * v5_3_1 + (VT)1.0 * oo2ze * v2_3_1;
            const VT v5_6_1 = QCx * v5_3_1 + WQx * v5_3_2 + (VT)1.0 * oo2ze * v2_3_2;
            const VT v6_6_0 = QCx * v6_3_0 + WQx * v6_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v6_6_1 = QCx * v6_3_1 + WQx * v6_3_2 + (VT)1.0 * oo2ze * v3_3_2;
            const VT v7_6_0 = QCx * v7_3_0 + WQx * v7_3_1;
            const VT v7_6_1 = QCx * v7_3_1 + WQx * v7_3_2;
            const VT v8_6_0 = QCx * v8_3_0 + WQx * v8_3_1;
            const VT v8_6_1 = QCx * v8_3_1 + WQx * v8_3_2;
            const VT v9_6_0 = QCx * v9_3_0 + WQx * v9_3_1;
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
            const VT v1_7_1 = QCy * v1_2_1 + WQy * v1_2_2 + (VT)1.0 * oo2e * (v1_0_1 - rho_e * v1_0_2);
            const VT v2_7_1 = QCy * v2_2_1 + WQy * v2_2_2 + (VT)1.0 * oo2ze * v0_2_2 + (VT)1.0 * oo2e * (v2_0_1 - rho_e * v2_0_2);
            const VT v3_7_1 = QCy * v3_2_1 + WQy * v3_2_2 + (VT)1.0 * oo2e * (v3_0_1 - rho_e * v3_0_2);
            const VT v4_7_0 = QCy * v4_2_0 + WQy * v4_2_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v4_7_1 = QCy * v4_2_1 + WQy * v4_2_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v5_7_0 = QCy * v5_2_0 + WQy * v5_2_1 + (VT)1.0 * oo2ze * v1_2_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v5_7_1 = QCy * v5_2_1 + WQy * v5_2_2 + (VT)1.0 * oo2ze * v1_2_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v6_7_0 = QCy * v6_2_0 + WQy * v6_2_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v6_7_1 = QCy * v6_2_1 + WQy * v6_2_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v7_7_0 = QCy * v7_2_0 + WQy * v7_2_1 + (VT)2.0 * oo2ze * v2_2_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v7_7_1 = QCy * v7_2_1 + WQy * v7_2_2 + (VT)2.0 * oo2ze * v2_2_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v8_7_0 = QCy * v8_2_0 + WQy * v8_2_1 + (VT)1.0 * oo2ze * v3_2_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v8_7_1 = QCy * v8_2_1 + WQy * v8_2_2 + (VT)1.0 * oo2ze * v3_2_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v9_7_0 = QCy * v9_2_0 + WQy * v9_2_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
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
            const VT v1_8_1 = QCy * v1_3_1 + WQy * v1_3_2;
            const VT v2_8_1 = QCy * v2_3_1 + WQy * v2_3_2 + (VT)1.0 * oo2ze * v0_3_2;
            const VT v3_8_1 = QCy * v3_3_1 + WQy * v3_3_2;
            const VT v4_8_0 = QCy * v4_3_0 + WQy * v4_3_1;
            const VT v4_8_1 = QCy * v4_3_1 + WQy * v4_3_2;
            const VT v5_8_0 = QCy * v5_3_0 + WQy * v5_3_1 + (VT)1.0 * oo2ze * v1_3_1;
            const VT v5_8_1 = QCy * v5_3_1 + WQy * v5_3_2 + (VT)1.0 * oo2ze * v1_3_2;
            const VT v6_8_0 = QCy * v6_3_0 + WQy * v6_3_1;
            const VT v6_8_1 = QCy * v6_3_1 + WQy * v6_3_2;
            const VT v7_8_0 = QCy * v7_3_0 + WQy * v7_3_1 + (VT)2.0 * oo2ze * v2_3_1;
            const VT v7_8_1 = QCy * v7_3_1 + WQy * v7_3_2 + (VT)2.0 * oo2ze * v2_3_2;
            const VT v8_8_0 = QCy * v8_3_0 + WQy * v8_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v8_8_1 = QCy * v8_3_1 + WQy * v8_3_2 + (VT)1.0 * oo2ze * v3_3_2;
            const VT v9_8_0 = QCy * v9_3_0 + WQy * v9_3_1;
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
            const VT v1_9_1 = QCz * v1_3_1 + WQz * v1_3_2 + (VT)1.0 * oo2e * (v1_0_1 - rho_e * v1_0_2);
            const VT v2_9_1 = QCz * v2_3_1 + WQz * v2_3_2 + (VT)1.0 * oo2e * (v2_0_1 - rho_e * v2_0_2);
            const VT v3_9_1 = QCz * v3_3_1 + WQz * v3_3_2 + (VT)1.0 * oo2ze * v0_3_2 + (VT)1.0 * oo2e * (v3_0_1 - rho_e * v3_0_2);
            const VT v4_9_0 = QCz * v4_3_0 + WQz * v4_3_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v4_9_1 = QCz * v4_3_1 + WQz * v4_3_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v5_9_0 = QCz * v5_3_0 + WQz * v5_3_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v5_9_1 = QCz * v5_3_1 + WQz * v5_3_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v6_9_0 = QCz * v6_3_0 + WQz * v6_3_1 + (VT)1.0 * oo2ze * v1_3_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v6_9_1 = QCz * v6_3_1 + WQz * v6_3_2 + (VT)1.0 * oo2ze * v1_3_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v7_9_0 = QCz * v7_3_0 + WQz * v7_3_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v7_9_1 = QCz * v7_3_1 + WQz * v7_3_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v8_9_0 = QCz * v8_3_0 + WQz * v8_3_1 + (VT)1.0 * oo2ze * v2_3_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v8_9_1 = QCz * v8_3_1 + WQz * v8_3_2 + (VT)1.0 * oo2ze * v2_3_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v9_9_0 = QCz * v9_3_0 + WQz * v9_3_1 + (VT)2.0 * oo2ze * v3_3_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
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
            const VT v4_10_0 = QCx * v4_4_0 + WQx * v4_4_1 + (VT)2.0 * oo2ze * v1_4_1 + (VT)2.0 * oo2e * (v4_1_0 - rho_e * v4_1_1);
            const VT v5_10_0 = QCx * v5_4_0 + WQx * v5_4_1 + (VT)1.0 * oo2ze * v2_4_1 + (VT)2.0 * oo2e * (v5_1_0 - rho_e * v5_1_1);
            const VT v6_10_0 = QCx * v6_4_0 + WQx * v6_4_1 + (VT)1.0 * oo2ze * v3_4_1 + (VT)2.0 * oo2e * (v6_1_0 - rho_e * v6_1_1);
            const VT v7_10_0 = QCx * v7_4_0 + WQx * v7_4_1 + (VT)2.0 * oo2e * (v7_1_0 - rho_e * v7_1_1);
            const VT v8_10_0 = QCx * v8_4_0 + WQx * v8_4_1 + (VT)2.0 * oo2e * (v8_1_0 - rho_e * v8_1_1);
            const VT v9_10_0 = QCx * v9_4_0 + WQx * v9_4_1 + (VT)2.0 * oo2e * (v9_1_0 - rho_e * v9_1_1);
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
            const VT v4_11_0 = QCx * v4_5_0 + WQx * v4_5_1 + (VT)2.0 * oo2ze * v1_5_1 + (VT)1.0 * oo2e * (v4_2_0 - rho_e * v4_2_1);
            const VT v5_11_0 = QCx * v5_5_0 + WQx * v5_5_1 + (VT)1.0 * oo2ze * v2_5_1 + (VT)1.0 * oo2e * (v5_2_0 - rho_e * v5_2_1);
            const VT v6_11_0 = QCx * v6_5_0 + WQx * v6_5_1 + (VT)1.0 * oo2ze * v3_5_1 + (VT)1.0 * oo2e * (v6_2_0 - rho_e * v6_2_1);
            const VT v7_11_0 = QCx * v7_5_0 + WQx * v7_5_1 + (VT)1.0 * oo2e * (v7_2_0 - rho_e * v7_2_1);
            const VT v8_11_0 = QCx * v8_5_0 + WQx * v8_5_1 + (VT)1.0 * oo2e * (v8_2_0 - rho_e * v8_2_1);
            const VT v9_11_0 = QCx * v9_5_0 + WQx * v9_5_1 + (VT)1.0 * oo2e * (v9_2_0 - rho_e * v9_2_1);
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
            const VT v4_12_0 = QCx * v4_6_0 + WQx * v4_6_1 + (VT)2.0 * oo2ze * v1_6_1 + (VT)1.0 * oo2e * (v4_3_0 - rho_e * v4_3_1);
            const VT v5_12_0 = QCx * v5_6_0 + WQx * v5_6_1 + (VT)1.0 * oo2ze * v2_6_1 + (VT)1.0 * oo2e * (v5_3_0 - rho_e * v5_3_1);
            const VT v6_12_0 = QCx * v6_6_0 + WQx * v6_6_1 + (VT)1.0 * oo2ze * v3_6_1 + (VT)1.0 * oo2e * (v6_3_0 - rho_e * v6_3_1);
            const VT v7_12_0 = QCx * v7_6_0 + WQx * v7_6_1 + (VT)1.0 * oo2e * (v7_3_0 - rho_e * v7_3_1);
            const VT v8_12_0 = QCx * v8_6_0 + WQx * v8_6_1 + (VT)1.0 * oo2e * (v8_3_0 - rho_e * v8_3_1);
            const VT v9_12_0 = QCx * v9_6_0 + WQx * v9_6_1 + (VT)1.0 * oo2e * (v9_3_0 - rho_e * v9_3_1);
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
            const VT v4_13_0 = QCy * v4_5_0 + WQy * v4_5_1 + (VT)1.0 * oo2e * (v4_1_0 - rho_e * v4_1_1);
            const VT v5_13_0 = QCy * v5_5_0 + WQy * v5_5_1 + (VT)1.0 * oo2ze * v1_5_1 + (VT)1.0 * oo2e * (v5_1_0 - rho_e * v5_1_1);
            const VT v6_13_0 = QCy * v6_5_0 + WQy * v6_5_1 + (VT)1.0 * oo2e * (v6_1_0 - rho_e * v6_1_1);
            const VT v7_13_0 = QCy * v7_5_0 + WQy * v7_5_1 + (VT)2.0 * oo2ze * v2_5_1 + (VT)1.0 * oo2e * (v7_1_0 - rho_e * v7_1_1);
            const VT v8_13_0 = QCy * v8_5_0 + WQy * v8_5_1 + (VT)1.0 * oo2ze * v3_5_1 + (VT)1.0 * oo2e * (v8_1_0 - rho_e * v8_1_1);
            const VT v9_13_0 = QCy * v9_5_0 + WQy * v9_5_1 + (VT)1.0 * oo2e * (v9_1_0 - rho_e * v9_1_1);
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
            const VT v4_14_0 = QCz * v4_6_0 + WQz * v4_6_1 + (VT)1.0 * oo2e * (v4_1_0 - rho_e * v4_1_1);
            const VT v5_14_0 = QCz * v5_6_0 + WQz * v5_6_1 + (VT)1.0 * oo2e * (v5_1_0 - rho_e * v5_1_1);
            const VT v6_14_0 = QCz * v6_6_0 + WQz * v6_6_1 + (VT)1.0 * oo2ze * v1_6_1 + (VT)1.0 * oo2e * (v6_1_0 - rho_e * v6_1_1);
            const VT v7_14_0 = QCz * v7_6_0 + WQz * v7_6_1 + (VT)1.0 * oo2e * (v7_1_0 - rho_e * v7_1_1);
            const VT v8_14_0 = QCz * v8_6_0 + WQz * v8_6_1 + (VT)1.0 * oo2ze * v2_6_1 + (VT)1.0 * oo2e * (v8_1_0 - rho_e * v8_1_1);
            const VT v9_14_0 = QCz * v9_6_0 + WQz * v9_6_1 + (VT)2.0 * oo2ze * v3_6_1 + (VT)1.0 * oo2e * (v9_1_0 - rho_e * v9_1_1);
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
            const VT v4_15_0 = QCx * v4_8_0 + WQx * v4_8_1 + (VT)2.0 * oo2ze * v1_8_1;
            const VT v5_15_0 = QCx * v5_8_0 + WQx * v5_8_1 + (VT)1.0 * oo2ze * v2_8_1;
            const VT v6_15_0 = QCx * v6_8_0 + WQx * v6_8_1 + (VT)1.0 * oo2ze * v3_8_1;
            const VT v7_15_0 = QCx * v7_8_0 + WQx * v7_8_1;
            const VT v8_15_0 = QCx * v8_8_0 + WQx * v8_8_1;
            const VT v9_15_0 = QCx * v9_8_0 + WQx * v9_8_1;
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
            const VT v4_16_0 = QCy * v4_7_0 + WQy * v4_7_1 + (VT)2.0 * oo2e * (v4_2_0 - rho_e * v4_2_1);
            const VT v5_16_0 = QCy * v5_7_0 + WQy * v5_7_1 + (VT)1.0 * oo2ze * v1_7_1 + (VT)2.0 * oo2e * (v5_2_0 - rho_e * v5_2_1);
            const VT v6_16_0 = QCy * v6_7_0 + WQy * v6_7_1 + (VT)2.0 * oo2e * (v6_2_0 - rho_e * v6_2_1);
            const VT v7_16_0 = QCy * v7_7_0 + WQy * v7_7_1 + (VT)2.0 * oo2ze * v2_7_1 + (VT)2.0 * oo2e * (v7_2_0 - rho_e * v7_2_1);
            const VT v8_16_0 = QCy * v8_7_0 + WQy * v8_7_1 + (VT)1.0 * oo2ze * v3_7_1 + (VT)2.0 * oo2e * (v8_2_0 - rho_e * v8_2_1);
            const VT v9_16_0 = QCy * v9_7_0 + WQy * v9_7_1 + (VT)2.0 * oo2e * (v9_2_0 - rho_e * v9_2_1);
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
            const VT v4_17_0 = QCy * v4_8_0 + WQy * v4_8_1 + (VT)1.0 * oo2e * (v4_3_0 - rho_e * v4_3_1);
            const VT v5_17_0 = QCy * v5_8_0 + WQy * v5_8_1 + (VT)1.0 * oo2ze * v1_8_1 + (VT)1.0 * oo2e * (v5_3_0 - rho_e * v5_3_1);
            const VT v6_17_0 = QCy * v6_8_0 + WQy * v6_8_1 + (VT)1.0 * oo2e * (v6_3_0 - rho_e * v6_3_1);
            const VT v7_17_0 = QCy * v7_8_0 + WQy * v7_8_1 + (VT)2.0 * oo2ze * v2_8_1 + (VT)1.0 * oo2e * (v7_3_0 - rho_e * v7_3_1);
            const VT v8_17_0 = QCy * v8_8_0 + WQy * v8_8_1 + (VT)1.0 * oo2ze * v3_8_1 + (VT)1.0 * oo2e * (v8_3_0 - rho_e * v8_3_1);
            const VT v9_17_0 = QCy * v9_8_0 + WQy * v9_8_1 + (VT)1.0 * oo2e * (v9_3_0 - rho_e * v9_3_1);
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
            const VT v4_18_0 = QCz * v4_8_0 + WQz * v4_8_1 + (VT)1.0 * oo2e * (v4_2_0 - rho_e * v4_2_1);
            const VT v5_18_0 = QCz * v5_8_0 + WQz * v5_8_1 + (VT)1.0 * oo2e * (v5_2_0 - rho_e * v5_2_1);
            const VT v6_18_0 = QCz * v6_8_0 + WQz * v6_8_1 + (VT)1.0 * oo2ze * v1_8_1 + (VT)1.0 * oo2e * (v6_2_0 - rho_e * v6_2_1);
            const VT v7_18_0 = QCz * v7_8_0 + WQz * v7_8_1 + (VT)1.0 * oo2e * (v7_2_0 - rho_e * v7_2_1);
            const VT v8_18_0 = QCz * v8_8_0 + WQz * v8_8_1 + (VT)1.0 * oo2ze * v2_8_1 + (VT)1.0 * oo2e * (v8_2_0 - rho_e * v8_2_1);
            const VT v9_18_0 = QCz * v9_8_0 + WQz * v9_8_1 + (VT)2.0 * oo2ze * v3_8_1 + (VT)1.0 * oo2e * (v9_2_0 - rho_e * v9_2_1);
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
            const VT v4_19_0 = QCz * v4_9_0 + WQz * v4_9_1 + (VT)2.0 * oo2e * (v4_3_0 - rho_e * v4_3_1);
            const VT v5_19_0 = QCz * v5_9_0 + WQz * v5_9_1 + (VT)2.0 * oo2e * (v5_3_0 - rho_e * v5_3_1);
            const VT v6_19_0 = QCz * v6_9_0 + WQz * v6_9_1 + (VT)1.0 * oo2ze * v1_9_1 + (VT)2.0 * oo2e * (v6_3_0 - rho_e * v6_3_1);
            const VT v7_19_0 = QCz * v7_9_0 + WQz * v7_9_1 + (VT)2.0 * oo2e * (v7_3_0 - rho_e * v7_3_1);
            const VT v8_19_0 = QCz * v8_9_0 + WQz * v8_9_1 + (VT)1.0 * oo2ze * v2_9_1 + (VT)2.0 * oo2e * (v8_3_0 - rho_e * v8_3_1);
            const VT v9_19_0 = QCz * v9_9_0 + WQz * v9_9_1 + (VT)2.0 * oo2ze * v3_9_1 + (VT)2.0 * oo2e * (v9_3_0 - rho_e * v9_3_1);
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
            acc[0] += (double)v4_4_0;
            acc[1] += (double)v4_5_0;
            acc[2] += (double)v4_6_0;
            acc[3] += (double)v4_7_0;
            acc[4] += (double)v4_8_0;
            acc[5] += (double)v4_9_0;
            acc[6] += (double)v4_10_0;
            acc[7] += (double)v4_11_0;
            acc[8] += (double)v4_12_0;
            acc[9] += (double)v4_13_0;
            acc[10] += (double)v4_14_0;
            acc[11] += (double)v4_15_0;
            acc[12] += (double)v4_16_0;
            acc[13] += (double)v4_17_0;
            acc[14] += (double)v4_18_0;
            acc[15] += (double)v4_19_0;
            acc[16] += (double)v5_4_0;
            acc[17] += (double)v5_5_0;
            acc[18] += (double)v5_6_0;
            acc[19] += (double)v5_7_0;
            acc[20] += (double)v5_8_0;
            acc[21] += (double)v5_9_0;
            acc[22] += (double)v5_10_0;
            acc[23] += (double)v5_11_0;
            acc[24] += (double)v5_12_0;
            acc[25] += (double)v5_13_0;
            acc[26] += (double)v5_14_0;
            acc[27] += (double)v5_15_0;
            acc[28] += (double)v5_16_0;
            acc[29] += (double)v5_17_0;
            acc[30] += (double)v5_18_0;
            acc[31] += (double)v5_19_0;
            acc[32] += (double)v6_4_0;
            acc[33] += (double)v6_5_0;
            acc[34] += (double)v6_6_0;
            acc[35] += (double)v6_7_0;
            acc[36] += (double)v6_8_0;
            acc[37] += (double)v6_9_0;
            acc[38] += (double)v6_10_0;
            acc[39] += (double)v6_11_0;
            acc[40] += (double)v6_12_0;
            acc[41] += (double)v6_13_0;
            acc[42] += (double)v6_14_0;
            acc[43] += (double)v6_15_0;
            acc[44] += (double)v6_16_0;
            acc[45] += (double)v6_17_0;
            acc[46] += (double)v6_18_0;
            acc[47] += (double)v6_19_0;
            acc[48] += (double)v7_4_0;
            acc[49] += (double)v7_5_0;
            acc[50] += (double)v7_6_0;
            acc[51] += (double)v7_7_0;
            acc[52] += (double)v7_8_0;
            acc[53] += (double)v7_9_0;
            acc[54] += (double)v7_10_0;
            acc[55] += (double)v7_11_0;
            acc[56] += (double)v7_12_0;
            acc[57] += (double)v7_13_0;
            acc[58] += (double)v7_14_0;
            acc[59] += (double)v7_15_0;
            acc[60] += (double)v7_16_0;
            acc[61] += (double)v7_17_0;
            acc[62] += (double)v7_18_0;
            acc[63] += (double)v7_19_0;
            acc[64] += (double)v8_4_0;
            acc[65] += (double)v8_5_0;
            acc[66] += (double)v8_6_0;
            acc[67] += (double)v8_7_0;
            acc[68] += (double)v8_8_0;
            acc[69] += (double)v8_9_0;
            acc[70] += (double)v8_10_0;
            acc[71] += (double)v8_11_0;
            acc[72] += (double)v8_12_0;
            acc[73] += (double)v8_13_0;
            acc[74] += (double)v8_14_0;
            acc[75] += (double)v8_15_0;
            acc[76] += (double)v8_16_0;
            acc[77] += (double)v8_17_0;
            acc[78] += (double)v8_18_0;
            acc[79] += (double)v8_19_0;
            acc[80] += (double)v9_4_0;
            acc[81] += (double)v9_5_0;
            acc[82] += (double)v9_6_0;
            acc[83] += (double)v9_7_0;
            acc[84] += (double)v9_8_0;
            acc[85] += (double)v9_9_0;
            acc[86] += (double)v9_10_0;
            acc[87] += (double)v9_11_0;
            acc[88] += (double)v9_12_0;
            acc[89] += (double)v9_13_0;
            acc[90] += (double)v9_14_0;
            acc[91] += (double)v9_15_0;
            acc[92] += (double)v9_16_0;
            acc[93] += (double)v9_17_0;
            acc[94] += (double)v9_18_0;
            acc[95] += (double)v9_19_0;
            acc[96] += (double)v10_4_0;
            acc[97] += (double)v10_5_0;
            acc[98] += (double)v10_6_0;
            acc[99] += (double)v10_7_0;
            acc[100] += (double)v10_8_0;
            acc[101] += (double)v10_9_0;
            acc[102] += (double)v10_10_0;
            acc[103] += (double)v10_11_0;
            acc[104] += (double)v10_12_0;
            acc[105] += (double)v10_13_0;
            acc[106] += (double)v10_14_0;
            acc[107] += (double)v10_15_0;
            acc[108] += (double)v10_16_0;
            acc[109] += (double)v10_17_0;
            acc[110] += (double)v10_18_0;
            acc[111] += (double)v10_19_0;
            acc[112] += (double)v11_4_0;
            acc[113] += (double)v11_5_0;
            acc[114] += (double)v11_6_0;
            acc[115] += (double)v11_7_0;
            acc[116] += (double)v11_8_0;
            acc[117] += (double)v11_9_0;
            acc[118] += (double)v11_10_0;
            acc[119] += (double)v11_11_0;
            acc[120] += (double)v11_12_0;
            acc[121] += (double)v11_13_0;
            acc[122] += (double)v11_14_0;
            acc[123] += (double)v11_15_0;
            acc[124] += (double)v11_16_0;
            acc[125] += (double)v11_17_0;
            acc[126] += (double)v11_18_0;
            acc[127] += (double)v11_19_0;
            acc[128] += (double)v12_4_0;
            acc[129] += (double)v12_5_0;
            acc[130] += (double)v12_6_0;
            acc[131] += (double)v12_7_0;
            acc[132] += (double)v12_8_0;
            acc[133] += (double)v12_9_0;
            acc[134] += (double)v12_10_0;
            acc[135] += (double)v12_11_0;
            acc[136] += (double)v12_12_0;
            acc[137] += (double)v12_13_0;
            acc[138] += (double)v12_14_0;
            acc[139] += (double)v12_15_0;
            acc[140] += (double)v12_16_0;
            acc[141] += (double)v12_17_0;
            acc[142] += (double)v12_18_0;
            acc[143] += (double)v12_19_0;
            acc[144] += (double)v13_4_0;
            acc[145] += (double)v13_5_0;
            acc[146] += (double)v13_6_0;
            acc[147] += (double)v13_7_0;
            acc[148] += (double)v13_8_0;
            acc[149] += (double)v13_9_0;
            acc[150] += (double)v13_10_0;
            acc[151] += (double)v13_11_0;
            acc[152] += (double)v13_12_0;
            acc[153] += (double)v13_13_0;
            acc[154] += (double)v13_14_0;
            acc[155] += (double)v13_15_0;
            acc[156] += (double)v13_16_0;
            acc[157] += (double)v13_17_0;
            acc[158] += (double)v13_18_0;
            acc[159] += (double)v13_19_0;
            acc[160] += (double)v14_4_0;
            acc[161] += (double)v14_5_0;
            acc[162] += (double)v14_6_0;
            acc[163] += (double)v14_7_0;
            acc[164] += (double)v14_8_0;
            acc[165] += (double)v14_9_0;
            acc[166] += (double)v14_10_0;
            acc[167] += (double)v14_11_0;
            acc[168] += (double)v14_12_0;
            acc[169] += (double)v14_13_0;
            acc[170] += (double)v14_14_0;
            acc[171] += (double)v14_15_0;
            acc[172] += (double)v14_16_0;
            acc[173] += (double)v14_17_0;
            acc[174] += (double)v14_18_0;
            acc[175] += (double)v14_19_0;
            acc[176] += (double)v15_4_0;
            acc[177] += (double)v15_5_0;
            acc[178] += (double)v15_6_0;
            acc[179] += (double)v15_7_0;
            acc[180] += (double)v15_8_0;
            acc[181] += (double)v15_9_0;
            acc[182] += (double)v15_10_0;
            acc[183] += (double)v15_11_0;
            acc[184] += (double)v15_12_0;
            acc[185] += (double)v15_13_0;
            acc[186] += (double)v15_14_0;
            acc[187] += (double)v15_15_0;
            acc[188] += (double)v15_16_0;
            acc[189] += (double)v15_17_0;
            acc[190] += (double)v15_18_0;
            acc[191] += (double)v15_19_0;
            acc[192] += (double)v16_4_0;
            acc[193] += (double)v16_5_0;
            acc[194] += (double)v16_6_0;
            acc[195] += (double)v16_7_0;
            acc[196] += (double)v16_8_0;
            acc[197] += (double)v16_9_0;
            acc[198] += (double)v16_10_0;
            acc[199] += (double)v16_11_0;
            acc[200] += (double)v16_12_0;
            acc[201] += (double)v16_13_0;
            acc[202] += (double)v16_14_0;
            acc[203] += (double)v16_15_0;
            acc[204] += (double)v16_16_0;
            acc[205] += (double)v16_17_0;
            acc[206] += (double)v16_18_0;
            acc[207] += (double)v16_19_0;
            acc[208] += (double)v17_4_0;
            acc[209] += (double)v17_5_0;
            acc[210] += (double)v17_6_0;
            acc[211] += (double)v17_7_0;
            acc[212] += (double)v17_8_0;
            acc[213] += (double)v17_9_0;
            acc[214] += (double)v17_10_0;
            acc[215] += (double)v17_11_0;
            acc[216] += (double)v17_12_0;
            acc[217] += (double)v17_13_0;
            acc[218] += (double)v17_14_0;
            acc[219] += (double)v17_15_0;
            acc[220] += (double)v17_16_0;
            acc[221] += (double)v17_17_0;
            acc[222] += (double)v17_18_0;
            acc[223] += (double)v17_19_0;
            acc[224] += (double)v18_4_0;
            acc[225] += (double)v18_5_0;
            acc[226] += (double)v18_6_0;
            acc[227] += (double)v18_7_0;
            acc[228] += (double)v18_8_0;
            acc[229] += (double)v18_9_0;
            acc[230] += (double)v18_10_0;
            acc[231] += (double)v18_11_0;
            acc[232] += (double)v18_12_0;
            acc[233] += (double)v18_13_0;
            acc[234] += (double)v18_14_0;
            acc[235] += (double)v18_15_0;
            acc[236] += (double)v18_16_0;
            acc[237] += (double)v18_17_0;
            acc[238] += (double)v18_18_0;
            acc[239] += (double)v18_19_0;
            acc[240] += (double)v19_4_0;
            acc[241] += (double)v19_5_0;
            acc[242] += (double)v19_6_0;
            acc[243] += (double)v19_7_0;
            acc[244] += (double)v19_8_0;
            acc[245] += (double)v19_9_0;
            acc[246] += (double)v19_10_0;
            acc[247] += (double)v19_11_0;
            acc[248] += (double)v19_12_0;
            acc[249] += (double)v19_13_0;
            acc[250] += (double)v19_14_0;
            acc[251] += (double)v19_15_0;
            acc[252] += (double)v19_16_0;
            acc[253] += (double)v19_17_0;
            acc[254] += (double)v19_18_0;
            acc[255] += (double)v19_19_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[324] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_dpdp(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h4_1_10 = acc[102] + ABx * acc[6];
    const double h4_1_4 = acc[96] + ABx * acc[0];
    const double k4_1_4_1 = h4_1_10 + CDx * h4_1_4;
    const double h4_1_11 = acc[103] + ABx * acc[7];
    const double k4_1_4_2 = h4_1_11 + CDy * h4_1_4;
    const double h4_1_12 = acc[104] + ABx * acc[8];
    const double k4_1_4_3 = h4_1_12 + CDz * h4_1_4;
    const double h4_1_5 = acc[97] + ABx * acc[1];
    const double k4_1_5_1 = h4_1_11 + CDx * h4_1_5;
    const double h4_1_13 = acc[105] + ABx * acc[9];
    const double k4_1_5_2 = h4_1_13 + CDy * h4_1_5;
    const double h4_1_15 = acc[107] + ABx * acc[11];
    const double k4_1_5_3 = h4_1_15 + CDz * h4_1_5;
    const double h4_1_6 = acc[98] + ABx * acc[2];
    const double k4_1_6_1 = h4_1_12 + CDx * h4_1_6;
    const double k4_1_6_2 = h4_1_15 + CDy * h4_1_6;
    const double h4_1_14 = acc[106] + ABx * acc[10];
    const double k4_1_6_3 = h4_1_14 + CDz * h4_1_6;
    const double h4_1_7 = acc[99] + ABx * acc[3];
    const double k4_1_7_1 = h4_1_13 + CDx * h4_1_7;
    const double h4_1_16 = acc[108] + ABx * acc[12];
    const double k4_1_7_2 = h4_1_16 + CDy * h4_1_7;
    const double h4_1_17 = acc[109] + ABx * acc[13];
    const double k4_1_7_3 = h4_1_17 + CDz * h4_1_7;
    const double h4_1_8 = acc[100] + ABx * acc[4];
    const double k4_1_8_1 = h4_1_15 + CDx * h4_1_8;
    const double k4_1_8_2 = h4_1_17 + CDy * h4_1_8;
    const double h4_1_18 = acc[110] + ABx * acc[14];
    const double k4_1_8_3 = h4_1_18 + CDz * h4_1_8;
    const double h4_1_9 = acc[101] + ABx * acc[5];
    const double k4_1_9_1 = h4_1_14 + CDx * h4_1_9;
    const double k4_1_9_2 = h4_1_18 + CDy * h4_1_9;
    const double h4_1_19 = acc[111] + ABx * acc[15];
    const double k4_1_9_3 = h4_1_19 + CDz * h4_1_9;
    const double h4_2_10 = acc[118] + ABy * acc[6];
    const double h4_2_4 = acc[112] + ABy * acc[0];
    const double k4_2_4_1 = h4_2_10 + CDx * h4_2_4;
    const double h4_2_11 = acc[119] + ABy * acc[7];
    const double k4_2_4_2 = h4_2_11 + CDy * h4_2_4;
    const double h4_2_12 = acc[120] + ABy * acc[8];
    const double k4_2_4_3 = h4_2_12 + CDz * h4_2_4;
    const double h4_2_5 = acc[113] + ABy * acc[1];
    const double k4_2_5_1 = h4_2_11 + CDx * h4_2_5;
    const double h4_2_13 = acc[121] + ABy * acc[9];
    const double k4_2_5_2 = h4_2_13 + CDy * h4_2_5;
    const double h4_2_15 = acc[123] + ABy * acc[11];
    const double k4_2_5_3 = h4_2_15 + CDz * h4_2_5;
    const double h4_2_6 = acc[114] + ABy * acc[2];
    const double k4_2_6_1 = h4_2_12 + CDx * h4_2_6;
    const double k4_2_6_2 = h4_2_15 + CDy * h4_2_6;
    const double h4_2_14 = acc[122] + ABy * acc[10];
    const double k4_2_6_3 = h4_2_14 + CDz * h4_2_6;
    const double h4_2_7 = acc[115] + ABy * acc[3];
    const double k4_2_7_1 = h4_2_13 + CDx * h4_2_7;
    const double h4_2_16 = acc[124] + ABy * acc[12];
    const double k4_2_7_2 = h4_2_16 + CDy * h4_2_7;
    const double h4_2_17 = acc[125] + ABy * acc[13];
    const double k4_2_7_3 = h4_2_17 + CDz * h4_2_7;
    const double h4_2_8 = acc[116] + ABy * acc[4];
    const double k4_2_8_1 = h4_2_15 + CDx * h4_2_8;
    const double k4_2_8_2 = h4_2_17 + CDy * h4_2_8;
    const double h4_2_18 = acc[126] + ABy * acc[14];
    const double k4_2_8_3 = h4_2_18 + CDz * h4_2_8;
    const double h4_2_9 = acc[117] + ABy * acc[5];
    const double k4_2_9_1 = h4_2_14 + CDx * h4_2_9;
    const double k4_2_9_2 = h4_2_18 + CDy * h4_2_9;
    const double h4_2_19 = acc[127] + ABy * acc[15];
    const double k4_2_9_3 = h4_2_19 + CDz * h4_2_9;
    const double h4_3_10 = acc[134] + ABz * acc[6];
    const double h4_3_4 = acc[128] + ABz * acc[0];
    const double k4_3_4_1 = h4_3_10 + CDx * h4_3_4;
    const double h4_3_11 = acc[135] + ABz * acc[7];
    const double k4_3_4_2 = h4_3_11 + CDy * h4_3_4;
    const double h4_3_12 = acc[136] + ABz * acc[8];
    const double k4_3_4_3 = h4_3_12 + CDz * h4_3_4;
    const double h4_3_5 = acc[129] + ABz * acc[1];
    const double k4_3_5_1 = h4_3_11 + CDx * h4_3_5;
    const double h4_3_13 = acc[137] + ABz * acc[9];
    const double k4_3_5_2 = h4_3_13 + CDy * h4_3_5;
    const double h4_3_15 = acc[139] + ABz * acc[11];
    const double k4_3_5_3 = h4_3_15 + CDz * h4_3_5;
    const double h4_3_6 = acc[130] + ABz * acc[2];
    const double k4_3_6_1 = h4_3_12 + CDx * h4_3_6;
    const double k4_3_6_2 = h4_3_15 + CDy * h4_3_6;
    const double h4_3_14 = acc[138] + ABz * acc[10];
    const double k4_3_6_3 = h4_3_14 + CDz * h4_3_6;
    const double h4_3_7 = acc[131] + ABz * acc[3];
    const double k4_3_7_1 = h4_3_13 + CDx * h4_3_7;
    const double h4_3_16 = acc[140] + ABz * acc[12];
    const double k4_3_7_2 = h4_3_16 + CDy * h4_3_7;
    const double h4_3_17 = acc[141] + ABz * acc[13];
    const double k4_3_7_3 = h4_3_17 + CDz * h4_3_7;
    const double h4_3_8 = acc[132] + ABz * acc[4];
    const double k4_3_8_1 = h4_3_15 + CDx * h4_3_8;
    const double k4_3_8_2 = h4_3_17 + CDy * h4_3_8;
    const double h4_3_18 = acc[142] + ABz * acc[14];
    const double k4_3_8_3 = h4_3_18 + CDz * h4_3_8;
    const double h4_3_9 = acc[133] + ABz * acc[5];
    const double k4_3_9_1 = h4_3_14 + CDx * h4_3_9;
    const double k4_3_9_2 = h4_3_18 + CDy * h4_3_9;
    const double h4_3_19 = acc[143] + ABz * acc[15];
    const double k4_3_9_3 = h4_3_19 + CDz * h4_3_9;
    const double h5_1_10 = acc[118] + ABx * acc[22];
    const double h5_1_4 = acc[112] + ABx * acc[16];
    const double k5_1_4_1 = h5_1_10 + CDx * h5_1_4;
    const double h5_1_11 = acc[119] + ABx * acc[23];
    const double k5_1_4_2 = h5_1_11 + CDy * h5_1_4;
    const double h5_1_12 = acc[120] + ABx * acc[24];
    const double k5_1_4_3 = h5_1_12 + CDz * h5_1_4;
    const double h5_1_5 = acc[113] + ABx * acc[17];
    const double k5_1_5_1 = h5_1_11 + CDx * h5_1_5;
    const double h5_1_13 = acc[121] + ABx * acc[25];
    const double k5_1_5_2 = h5_1_13 + CDy * h5_1_5;
    const double h5_1_15 = acc[123] + ABx * acc[27];
    const double k5_1_5_3 = h5_1_15 + CDz * h5_1_5;
    const double h5_1_6 = acc[114] + ABx * acc[18];
    const double k5_1_6_1 = h5_1_12 + CDx * h5_1_6;
    const double k5_1_6_2 = h5_1_15 + CDy * h5_1_6;
    const double h5_1_14 = acc[122] + ABx * acc[26];
    const double k5_1_6_3 = h5_1_14 + CDz * h5_1_6;
    const double h5_1_7 = acc[115] + ABx * acc[19];
    const double k5_1_7_1 = h5_1_13 + CDx * h5_1_7;
    const double h5_1_16 = acc[124] + ABx * acc[28];
    const double k5_1_7_2 = h5_1_16 + CDy * h5_1_7;
    const double h5_1_17 = acc[125] + ABx * acc[29];
    const double k5_1_7_3 = h5_1_17 + CDz * h5_1_7;
    const double h5_1_8 = acc[116] + ABx * acc[20];
    const double k5_1_8_1 = h5_1_15 + CDx * h5_1_8;
    const double k5_1_8_2 = h5_1_17 + CDy * h5_1_8;
    const double h5_1_18 = acc[126] + ABx * acc[30];
    const double k5_1_8_3 = h5_1_18 + CDz * h5_1_8;
    const double h5_1_9 = acc[117] + ABx * acc[21];
    const double k5_1_9_1 = h5_1_14 + CDx * h5_1_9;
    const double k5_1_9_2 = h5_1_18 + CDy * h5_1_9;
    const double h5_1_19 = acc[127] + ABx * acc[31];
    const double k5_1_9_3 = h5_1_19 + CDz * h5_1_9;
    const double h5_2_10 = acc[150] + ABy * acc[22];
    const double h5_2_4 = acc[144] + ABy * acc[16];
    const double k5_2_4_1 = h5_2_10 + CDx * h5_2_4;
    const double h5_2_11 = acc[151] + ABy * acc[23];
    const double k5_2_4_2 = h5_2_11 + CDy * h5_2_4;
    const double h5_2_12 = acc[152] + ABy * acc[24];
    const double k5_2_4_3 = h5_2_12 + CDz * h5_2_4;
    const double h5_2_5 = acc[145] + ABy * acc[17];
    const double k5_2_5_1 = h5_2_11 + CDx * h5_2_5;
    const double h5_2_13 = acc[153] + ABy * acc[25];
    const double k5_2_5_2 = h5_2_13 + CDy * h5_2_5;
    const double h5_2_15 = acc[155] + ABy * acc[27];
    const double k5_2_5_3 = h5_2_15 + CDz * h5_2_5;
    const double h5_2_6 = acc[146] + ABy * acc[18];
    const double k5_2_6_1 = h5_2_12 + CDx * h5_2_6;
    const double k5_2_6_2 = h5_2_15 + CDy * h5_2_6;
    const double h5_2_14 = acc[154] + ABy * acc[26];
    const double k5_2_6_3 = h5_2_14 + CDz * h5_2_6;
    const double h5_2_7 = acc[147] + ABy * acc[19];
    const double k5_2_7_1 = h5_2_13 + CDx * h5_2_7;
    const double h5_2_16 = acc[156] + ABy * acc[28];
    const double k5_2_7_2 = h5_2_16 + CDy * h5_2_7;
    const double h5_2_17 = acc[157] + ABy * acc[29];
    const double k5_2_7_3 = h5_2_17 + CDz * h5_2_7;
    const double h5_2_8 = acc[148] + ABy * acc[20];
    const double k5_2_8_1 = h5_2_15 + CDx * h5_2_8;
    const double k5_2_8_2 = h5_2_17 + CDy * h5_2_8;
    const double h5_2_18 = acc[158] + ABy * acc[30];
    const double k5_2_8_3 = h5_2_18 + CDz * h5_2_8;
    const double h5_2_9 = acc[149] + ABy * acc[21];
    const double k5_2_9_1 = h5_2_14 + CDx * h5_2_9;
    const double k5_2_9_2 = h5_2_18 + CDy * h5_2_9;
    const double h5_2_19 = acc[159] + ABy * acc[31];
    const double k5_2_9_3 = h5_2_19 + CDz * h5_2_9;
    const double h5_3_10 = acc[182] + ABz * acc[22];
    const double h5_3_4 = acc[176] + ABz * acc[16];
    const double k5_3_4_1 = h5_3_10 + CDx * h5_3_4;
    const double h5_3_11 = acc[183] + ABz * acc[23];
    const double k5_3_4_2 = h5_3_11 + CDy * h5_3_4;
    const double h5_3_12 = acc[184] + ABz * acc[24];
    const double k5_3_4_3 = h5_3_12 + CDz * h5_3_4;
    const double h5_3_5 = acc[177] + ABz * acc[17];
    const double k5_3_5_1 = h5_3_11 + CDx * h5_3_5;
    const double h5_3_13 = acc[185] + ABz * acc[25];
    const double k5_3_5_2 = h5_3_13 + CDy * h5_3_5;
    const double h5_3_15 = acc[187] + ABz * acc[27];
    const double k5_3_5_3 = h5_3_15 + CDz * h5_3_5;
    const double h5_3_6 = acc[178] + ABz * acc[18];
    const double k5_3_6_1 = h5_3_12 + CDx * h5_3_6;
    const double k5_3_6_2 = h5_3_15 + CDy * h5_3_6;
    const double h5_3_14 = acc[186] + ABz * acc[26];
    const double k5_3_6_3 = h5_3_14 + CDz * h5_3_6;
    const double h5_3_7 = acc[179] + ABz * acc[19];
    const double k5_3_7_1 = h5_3_13 + CDx * h5_3_7;
    const double h5_3_16 = acc[188] + ABz * acc[28];
    const double k5_3_7_2 = h5_3_16 + CDy * h5_3_7;
    const double h5_3_17 = acc[189] + ABz * acc[29];
    const double k5_3_7_3 = h5_3_17 + CDz * h5_3_7;
    const double h5_3_8 = acc[180] + ABz * acc[20];
    const double k5_3_8_1 = h5_3_15 + CDx * h5_3_8;
    const double k5_3_8_2 = h5_3_17 + CDy * h5_3_8;
    const double h5_3_18 = acc[190] + ABz * acc[30];
    const double k5_3_8_3 = h5_3_18 + CDz * h5_3_8;
    const double h5_3_9 = acc[181] + ABz * acc[21];
    const double k5_3_9_1 = h5_3_14 + CDx * h5_3_9;
    const double k5_3_9_2 = h5_3_18 + CDy * h5_3_9;
    const double h5_3_19 = acc[191] + ABz * acc[31];
    const double k5_3_9_3 = h5_3_19 + CDz * h5_3_9;
    const double h6_1_10 = acc[134] + ABx * acc[38];
    const double h6_1_4 = acc[128] + ABx * acc[32];
    const double k6_1_4_1 = h6_1_10 + CDx * h6_1_4;
    const double h6_1_11 = acc[135] + ABx * acc[39];
    const double k6_1_4_2 = h6_1_11 + CDy * h6_1_4;
    const double h6_1_12 = acc[136] + ABx * acc[40];
    const double k6_1_4_3 = h6_1_12 + CDz * h6_1_4;
    const double h6_1_5 = acc[129] + ABx * acc[33];
    const double k6_1_5_1 = h6_1_11 + CDx * h6_1_5;
    const double h6_1_13 = acc[137] + ABx * acc[41];
    const double k6_1_5_2 = h6_1_13 + CDy * h6_1_5;
    const double h6_1_15 = acc[139] + ABx * acc[43];
    const double k6_1_5_3 = h6_1_15 + CDz * h6_1_5;
    const double h6_1_6 = acc[130] + ABx * acc[34];
    const double k6_1_6_1 = h6_1_12 + CDx * h6_1_6;
    const double k6_1_6_2 = h6_1_15 + CDy * h6_1_6;
    const double h6_1_14 = acc[138] + ABx * acc[42];
    const double k6_1_6_3 = h6_1_14 + CDz * h6_1_6;
    const double h6_1_7 = acc[131] + ABx * acc[35];
    const double k6_1_7_1 = h6_1_13 + CDx * h6_1_7;
    const double h6_1_16 = acc[140] + ABx * acc[44];
    const double k6_1_7_2 = h6_1_16 + CDy * h6_1_7;
    const double h6_1_17 = acc[141] + ABx * acc[45];
    const double k6_1_7_3 = h6_1_17 + CDz * h6_1_7;
    const double h6_1_8 = acc[132] + ABx * acc[36];
    const double k6_1_8_1 = h6_1_15 + CDx * h6_1_8;
    const double k6_1_8_2 = h6_1_17 + CDy * h6_1_8;
    const double h6_1_18 = acc[142] + ABx * acc[46];
    const double k6_1_8_3 = h6_1_18 + CDz * h6_1_8;
    const double h6_1_9 = acc[133] + ABx * acc[37];
    const double k6_1_9_1 = h6_1_14 + CDx * h6_1_9;
    const double k6_1_9_2 = h6_1_18 + CDy * h6_1_9;
    const double h6_1_19 = acc[143] + ABx * acc[47];
    const double k6_1_9_3 = h6_1_19 + CDz * h6_1_9;
    const double h6_2_10 = acc[182] + ABy * acc[38];
    const double h6_2_4 = acc[176] + ABy * acc[32];
    const double k6_2_4_1 = h6_2_10 + CDx * h6_2_4;
    const double h6_2_11 = acc[183] + ABy * acc[39];
    const double k6_2_4_2 = h6_2_11 + CDy * h6_2_4;
    const double h6_2_12 = acc[184] + ABy * acc[40];
    const double k6_2_4_3 = h6_2_12 + CDz * h6_2_4;
    const double h6_2_5 = acc[177] + ABy * acc[33];
    const double k6_2_5_1 = h6_2_11 + CDx * h6_2_5;
    const double h6_2_13 = acc[185] + ABy * acc[41];
    const double k6_2_5_2 = h6_2_13 + CDy * h6_2_5;
    const double h6_2_15 = acc[187] + ABy * acc[43];
    const double k6_2_5_3 = h6_2_15 + CDz * h6_2_5;
    const double h6_2_6 = acc[178] + ABy * acc[34];
    const double k6_2_6_1 = h6_2_12 + CDx * h6_2_6;
    const double k6_2_6_2 = h6_2_15 + CDy * h6_2_6;
    const double h6_2_14 = acc[186] + ABy * acc[42];
    const double k6_2_6_3 = h6_2_14 + CDz * h6_2_6;
    const double h6_2_7 = acc[179] + ABy * acc[35];
    const double k6_2_7_1 = h6_2_13 + CDx * h6_2_7;
    const double h6_2_16 = acc[188] + ABy * acc[44];
    const double k6_2_7_2 = h6_2_16 + CDy * h6_2_7;
    const double h6_2_17 = acc[189] + ABy * acc[45];
    const double k6_2_7_3 = h6_2_17 + CDz * h6_2_7;
    const double h6_2_8 = acc[180] + ABy * acc[36];
    const double k6_2_8_1 = h6_2_15 + CDx * h6_2_8;
    const double k6_2_8_2 = h6_2_17 + CDy * h6_2_8;
    const double h6_2_18 = acc[190] + ABy * acc[46];
    const double k6_2_8_3 = h6_2_18 + CDz * h6_2_8;
    const double h6_2_9 = acc[181] + ABy * acc[37];
    const double k6_2_9_1 = h6_2_14 + CDx * h6_2_9;
    const double k6_2_9_2 = h6_2_18 + CDy * h6_2_9;
    const double h6_2_19 = acc[191] + ABy * acc[47];
    const double k6_2_9_3 = h6_2_19 + CDz * h6_2_9;
    const double h6_3_10 = acc[166] + ABz * acc[38];
    const double h6_3_4 = acc[160] + ABz * acc[32];
    const double k6_3_4_1 = h6_3_10 + CDx * h6_3_4;
    const double h6_3_11 = acc[167] + ABz * acc[39];
    const double k6_3_4_2 = h6_3_11 + CDy * h6_3_4;
    const double h6_3_12 = acc[168] + ABz * acc[40];
    const double k6_3_4_3 = h6_3_12 + CDz * h6_3_4;
    const double h6_3_5 = acc[161] + ABz * acc[33];
    const double k6_3_5_1 = h6_3_11 + CDx * h6_3_5;
    const double h6_3_13 = acc[169] + ABz * acc[41];
    const double k6_3_5_2 = h6_3_13 + CDy * h6_3_5;
    const double h6_3_15 = acc[171] + ABz * acc[43];
    const double k6_3_5_3 = h6_3_15 + CDz * h6_3_5;
    const double h6_3_6 = acc[162] + ABz * acc[34];
    const double k6_3_6_1 = h6_3_12 + CDx * h6_3_6;
    const double k6_3_6_2 = h6_3_15 + CDy * h6_3_6;
    const double h6_3_14 = acc[170] + ABz * acc[42];
    const double k6_3_6_3 = h6_3_14 + CDz * h6_3_6;
    const double h6_3_7 = acc[163] + ABz * acc[35];
    const double k6_3_7_1 = h6_3_13 + CDx * h6_3_7;
    const double h6_3_16 = acc[172] + ABz * acc[44];
    const double k6_3_7_2 = h6_3_16 + CDy * h6_3_7;
    const double h6_3_17 = acc[173] + ABz * acc[45];
    const double k6_3_7_3 = h6_3_17 + CDz * h6_3_7;
    const double h6_3_8 = acc[164] + ABz * acc[36];
    const double k6_3_8_1 = h6_3_15 + CDx * h6_3_8;
    const double k6_3_8_2 = h6_3_17 + CDy * h6_3_8;
    const double h6_3_18 = acc[174] + ABz * acc[46];
    const double k6_3_8_3 = h6_3_18 + CDz * h6_3_8;
    const double h6_3_9 = acc[165] + ABz * acc[37];
    const double k6_3_9_1 = h6_3_14 + CDx * h6_3_9;
    const double k6_3_9_2 = h6_3_18 + CDy * h6_3_9;
    const double h6_3_19 = acc[175] + ABz * acc[47];
    const double k6_3_9_3 = h6_3_19 + CDz * h6_3_9;
    const double h7_1_10 = acc[150] + ABx * acc[54];
    const double h7_1_4 = acc[144] + ABx * acc[48];
    const double k7_1_4_1 = h7_1_10 + CDx * h7_1_4;
    const double h7_1_11 = acc[151] + ABx * acc[55];
    const double k7_1_4_2 = h7_1_11 + CDy * h7_1_4;
    const double h7_1_12 = acc[152] + ABx * acc[56];
    const double k7_1_4_3 = h7_1_12 + CDz * h7_1_4;
    const double h7_1_5 = acc[145] + ABx * acc[49];
    const double k7_1_5_1 = h7_1_11 + CDx * h7_1_5;
    const double h7_1_13 = acc[153] + ABx * acc[57];
    const double k7_1_5_2 = h7_1_13 + CDy * h7_1_5;
    const double h7_1_15 = acc[155] + ABx * acc[59];
    const double k7_1_5_3 = h7_1_15 + CDz * h7_1_5;
    const double h7_1_6 = acc[146] + ABx * acc[50];
    const double k7_1_6_1 = h7_1_12 + CDx * h7_1_6;
    const double k7_1_6_2 = h7_1_15 + CDy * h7_1_6;
    const double h7_1_14 = acc[154] + ABx * acc[58];
    const double k7_1_6_3 = h7_1_14 + CDz * h7_1_6;
    const double h7_1_7 = acc[147] + ABx * acc[51];
    const double k7_1_7_1 = h7_1_13 + CDx * h7_1_7;
    const double h7_1_16 = acc[156] + ABx * acc[60];
    const double k7_1_7_2 = h7_1_16 + CDy * h7_1_7;
    const double h7_1_17 = acc[157] + ABx * acc[61];
    const double k7_1_7_3 = h7_1_17 + CDz * h7_1_7;
    const double h7_1_8 = acc[148] + ABx * acc[52];
    const double k7_1_8_1 = h7_1_15 + CDx * h7_1_8;
    const double k7_1_8_2 = h7_1_17 + CDy * h7_1_8;
    const double h7_1_18 = acc[158] + ABx * acc[62];
    const double k7_1_8_3 = h7_1_18 + CDz * h7_1_8;
    const double h7_1_9 = acc[149] + ABx * acc[53];
    const double k7_1_9_1 = h7_1_14 + CDx * h7_1_9;
    const double k7_1_9_2 = h7_1_18 + CDy * h7_1_9;
    const double h7_1_19 = acc[159] + ABx * acc[63];
    const double k7_1_9_3 = h7_1_19 + CDz * h7_1_9;
    const double h7_2_10 = acc[198] + ABy * acc[54];
    const double h7_2_4 = acc[192] + ABy * acc[48];
    const double k7_2_4_1 = h7_2_10 + CDx * h7_2_4;
    const double h7_2_11 = acc[199] + ABy * acc[55];
    const double k7_2_4_2 = h7_2_11 + CDy * h7_2_4;
    const double h7_2_12 = acc[200] + ABy * acc[56];
    const double k7_2_4_3 = h7_2_12 + CDz * h7_2_4;
    const double h7_2_5 = acc[193] + ABy * acc[49];
    const double k7_2_5_1 = h7_2_11 + CDx * h7_2_5;
    const double h7_2_13 = acc[201] + ABy * acc[57];
    const double k7_2_5_2 = h7_2_13 + CDy * h7_2_5;
    const double h7_2_15 = acc[203] + ABy * acc[59];
    const double k7_2_5_3 = h7_2_15 + CDz * h7_2_5;
    const double h7_2_6 = acc[194] + ABy * acc[50];
    const double k7_2_6_1 = h7_2_12 + CDx * h7_2_6;
    const double k7_2_6_2 = h7_2_15 + CDy * h7_2_6;
    const double h7_2_14 = acc[202] + ABy * acc[58];
    const double k7_2_6_3 = h7_2_14 + CDz * h7_2_6;
    const double h7_2_7 = acc[195] + ABy * acc[51];
    const double k7_2_7_1 = h7_2_13 + CDx * h7_2_7;
    const double h7_2_16 = acc[204] + ABy * acc[60];
    const double k7_2_7_2 = h7_2_16 + CDy * h7_2_7;
    const double h7_2_17 = acc[205] + ABy * acc[61];
    const double k7_2_7_3 = h7_2_17 + CDz * h7_2_7;
    const double h7_2_8 = acc[196] + ABy * acc[52];
    const double k7_2_8_1 = h7_2_15 + CDx * h7_2_8;
    const double k7_2_8_2 = h7_2_17 + CDy * h7_2_8;
    const double h7_2_18 = acc[206] + ABy * acc[62];
    const double k7_2_8_3 = h7_2_18 + CDz * h7_2_8;
    const double h7_2_9 = acc[197] + ABy * acc[53];
    const double k7_2_9_1 = h7_2_14 + CDx * h7_2_9;
    const double k7_2_9_2 = h7_2_18 + CDy * h7_2_9;
    const double h7_2_19 = acc[207] + ABy * acc[63];
    const double k7_2_9_3 = h7_2_19 + CDz * h7_2_9;
    const double h7_3_10 = acc[214] + ABz * acc[54];
    const double h7_3_4 = acc[208] + ABz * acc[48];
    const double k7_3_4_1 = h7_3_10 + CDx * h7_3_4;
    const double h7_3_11 = acc[215] + ABz * acc[55];
    const double k7_3_4_2 = h7_3_11 + CDy * h7_3_4;
    const double h7_3_12 = acc[216] + ABz * acc[56];
    const double k7_3_4_3 = h7_3_12 + CDz * h7_3_4;
    const double h7_3_5 = acc[209] + ABz * acc[49];
    const double k7_3_5_1 = h7_3_11 + CDx * h7_3_5;
    const double h7_3_13 = acc[217] + ABz * acc[57];
    const double k7_3_5_2 = h7_3_13 + CDy * h7_3_5;
    const double h7_3_15 = acc[219] + ABz * acc[59];
    const double k7_3_5_3 = h7_3_15 + CDz * h7_3_5;
    const double h7_3_6 = acc[210] + ABz * acc[50];
    const double k7_3_6_1 = h7_3_12 + CDx * h7_3_6;
    const double k7_3_6_2 = h7_3_15 + CDy * h7_3_6;
    const double h7_3_14 = acc[218] + ABz * acc[58];
    const double k7_3_6_3 = h7_3_14 + CDz * h7_3_6;
    const double h7_3_7 = acc[211] + ABz * acc[51];
    const double k7_3_7_1 = h7_3_13 + CDx * h7_3_7;
    const double h7_3_16 = acc[220] + ABz * acc[60];
    const double k7_3_7_2 = h7_3_16 + CDy * h7_3_7;
    const double h7_3_17 = acc[221] + ABz * acc[61];
    const double k7_3_7_3 = h7_3_17 + CDz * h7_3_7;
    const double h7_3_8 = acc[212] + ABz * acc[52];
    const double k7_3_8_1 = h7_3_15 + CDx * h7_3_8;
    const double k7_3_8_2 = h7_3_17 + CDy * h7_3_8;
    const double h7_3_18 = acc[222] + ABz * acc[62];
    const double k7_3_8_3 = h7_3_18 + CDz * h7_3_8;
    const double h7_3_9 = acc[213] + ABz * acc[53];
    const double k7_3_9_1 = h7_3_14 + CDx * h7_3_9;
    const double k7_3_9_2 = h7_3_18 + CDy * h7_3_9;
    const double h7_3_19 = acc[223] + ABz * acc[63];
    const double k7_3_9_3 = h7_3_19 + CDz * h7_3_9;
    const double h8_1_10 = acc[182] + ABx * acc[70];
    const double h8_1_4 = acc[176] + ABx * acc[64];
    const double k8_1_4_1 = h8_1_10 + CDx * h8_1_4;
    const double h8_1_11 = acc[183] + ABx * acc[71];
    const double k8_1_4_2 = h8_1_11 + CDy * h8_1_4;
    const double h8_1_12 = acc[184] + ABx * acc[72];
    const double k8_1_4_3 = h8_1_12 + CDz * h8_1_4;
    const double h8_1_5 = acc[177] + ABx * acc[65];
    const double k8_1_5_1 = h8_1_11 + CDx * h8_1_5;
    const double h8_1_13 = acc[185] + ABx * acc[73];
    const double k8_1_5_2 = h8_1_13 + CDy * h8_1_5;
    const double h8_1_15 = acc[187] + ABx * acc[75];
    const double k8_1_5_3 = h8_1_15 + CDz * h8_1_5;
    const double h8_1_6 = acc[178] + ABx * acc[66];
    const double k8_1_6_1 = h8_1_12 + CDx * h8_1_6;
    const double k8_1_6_2 = h8_1_15 + CDy * h8_1_6;
    const double h8_1_14 = acc[186] + ABx * acc[74];
    const double k8_1_6_3 = h8_1_14 + CDz * h8_1_6;
    const double h8_1_7 = acc[179] + ABx * acc[67];
    const double k8_1_7_1 = h8_1_13 + CDx * h8_1_7;
    const double h8_1_16 = acc[188] + ABx * acc[76];
    const double k8_1_7_2 = h8_1_16 + CDy * h8_1_7;
    const double h8_1_17 = acc[189] + ABx * acc[77];
    const double k8_1_7_3 = h8_1_17 + CDz * h8_1_7;
    const double h8_1_8 = acc[180] + ABx * acc[68];
    const double k8_1_8_1 = h8_1_15 + CDx * h8_1_8;
    const double k8_1_8_2 = h8_1_17 + CDy * h8_1_8;
    const double h8_1_18 = acc[190] + ABx * acc[78];
    const double k8_1_8_3 = h8_1_18 + CDz * h8_1_8;
    const double h8_1_9 = acc[181] + ABx * acc[69];
    const double k8_1_9_1 = h8_1_14 + CDx * h8_1_9;
    const double k8_1_9_2 = h8_1_18 + CDy * h8_1_9;
    const double h8_1_19 = acc[191] + ABx * acc[79];
    const double k8_1_9_3 = h8_1_19 + CDz * h8_1_9;
    const double h8_2_10 = acc[214] + ABy * acc[70];
    const double h8_2_4 = acc[208] + ABy * acc[64];
    const double k8_2_4_1 = h8_2_10 + CDx * h8_2_4;
    const double h8_2_11 = acc[215] + ABy * acc[71];
    const double k8_2_4_2 = h8_2_11 + CDy * h8_2_4;
    const double h8_2_12 = acc[216] + ABy * acc[72];
    const double k8_2_4_3 = h8_2_12 + CDz * h8_2_4;
    const double h8_2_5 = acc[209] + ABy * acc[65];
    const double k8_2_5_1 = h8_2_11 + CDx * h8_2_5;
    const double h8_2_13 = acc[217] + ABy * acc[73];
    const double k8_2_5_2 = h8_2_13 + CDy * h8_2_5;
    const double h8_2_15 = acc[219] + ABy * acc[75];
    const double k8_2_5_3 = h8_2_15 + CDz * h8_2_5;
    const double h8_2_6 = acc[210] + ABy * acc[66];
    const double k8_2_6_1 = h8_2_12 + CDx * h8_2_6;
    const double k8_2_6_2 = h8_2_15 + CDy * h8_2_6;
    const double h8_2_14 = acc[218] + ABy * acc[74];
    const double k8_2_6_3 = h8_2_14 + CDz * h8_2_6;
    const double h8_2_7 = acc[211] + ABy * acc[67];
    const double k8_2_7_1 = h8_2_13 + CDx * h8_2_7;
    const double h8_2_16 = acc[220] + ABy * acc[76];
    const double k8_2_7_2 = h8_2_16 + CDy * h8_2_7;
    const double h8_2_17 = acc[221] + ABy * acc[77];
    const double k8_2_7_3 = h8_2_17 + CDz * h8_2_7;
    const double h8_2_8 = acc[212] + ABy * acc[68];
    const double k8_2_8_1 = h8_2_15 + CDx * h8_2_8;
    const double k8_2_8_2 = h8_2_17 + CDy * h8_2_8;
    const double h8_2_18 = acc[222] + ABy * acc[78];
    const double k8_2_8_3 = h8_2_18 + CDz * h8_2_8;
    const double h8_2_9 = acc[213] + ABy * acc[69];
    const double k8_2_9_1 = h8_2_14 + CDx * h8_2_9;
    const double k8_2_9_2 = h8_2_18 + CDy * h8_2_9;
    const double h8_2_19 = acc[223] + ABy * acc[79];
    const double k8_2_9_3 = h8_2_19 + CDz * h8_2_9;
    const double h8_3_10 = acc[230] + ABz * acc[70];
    const double h8_3_4 = acc[224] + ABz * acc[64];
    const double k8_3_4_1 = h8_3_10 + CDx * h8_3_4;
    const double h8_3_11 = acc[231] + ABz * acc[71];
    const double k8_3_4_2 = h8_3_11 + CDy * h8_3_4;
    const double h8_3_12 = acc[232] + ABz * acc[72];
    const double k8_3_4_3 = h8_3_12 + CDz * h8_3_4;
    const double h8_3_5 = acc[225] + ABz * acc[65];
    const double k8_3_5_1 = h8_3_11 + CDx * h8_3_5;
    const double h8_3_13 = acc[233] + ABz * acc[73];
    const double k8_3_5_2 = h8_3_13 + CDy * h8_3_5;
    const double h8_3_15 = acc[235] + ABz * acc[75];
    const double k8_3_5_3 = h8_3_15 + CDz * h8_3_5;
    const double h8_3_6 = acc[226] + ABz * acc[66];
    const double k8_3_6_1 = h8_3_12 + CDx * h8_3_6;
    const double k8_3_6_2 = h8_3_15 + CDy * h8_3_6;
    const double h8_3_14 = acc[234] + ABz * acc[74];
    const double k8_3_6_3 = h8_3_14 + CDz * h8_3_6;
    const double h8_3_7 = acc[227] + ABz * acc[67];
    const double k8_3_7_1 = h8_3_13 + CDx * h8_3_7;
    const double h8_3_16 = acc[236] + ABz * acc[76];
    const double k8_3_7_2 = h8_3_16 + CDy * h8_3_7;
    const double h8_3_17 = acc[237] + ABz * acc[77];
    const double k8_3_7_3 = h8_3_17 + CDz * h8_3_7;
    const double h8_3_8 = acc[228] + ABz * acc[68];
    const double k8_3_8_1 = h8_3_15 + CDx * h8_3_8;
    const double k8_3_8_2 = h8_3_17 + CDy * h8_3_8;
    const double h8_3_18 = acc[238] + ABz * acc[78];
    const double k8_3_8_3 = h8_3_18 + CDz * h8_3_8;
    const double h8_3_9 = acc[229] + ABz * acc[69];
    const double k8_3_9_1 = h8_3_14 + CDx * h8_3_9;
    const double k8_3_9_2 = h8_3_18 + CDy * h8_3_9;
    const double h8_3_19 = acc[239] + ABz * acc[79];
    const double k8_3_9_3 = h8_3_19 + CDz * h8_3_9;
    const double h9_1_10 = acc[166] + ABx * acc[86];
    const double h9_1_4 = acc[160] + ABx * acc[80];
    const double k9_1_4_1 = h9_1_10 + CDx * h9_1_4;
    const double h9_1_11 = acc[167] + ABx * acc[87];
    const double k9_1_4_2 = h9_1_11 + CDy * h9_1_4;
    const double h9_1_12 = acc[168] + ABx * acc[88];
    const double k9_1_4_3 = h9_1_12 + CDz * h9_1_4;
    const double h9_1_5 = acc[161] + ABx * acc[81];
    const double k9_1_5_1 = h9_1_11 + CDx * h9_1_5;
    const double h9_1_13 = acc[169] + ABx * acc[89];
    const double k9_1_5_2 = h9_1_13 + CDy * h9_1_5;
    const double h9_1_15 = acc[171] + ABx * acc[91];
    const double k9_1_5_3 = h9_1_15 + CDz * h9_1_5;
    const double h9_1_6 = acc[162] + ABx * acc[82];
    const double k9_1_6_1 = h9_1_12 + CDx * h9_1_6;
    const double k9_1_6_2 = h9_1_15 + CDy * h9_1_6;
    const double h9_1_14 = acc[170] + ABx * acc[90];
    const double k9_1_6_3 = h9_1_14 + CDz * h9_1_6;
    const double h9_1_7 = acc[163] + ABx * acc[83];
    const double k9_1_7_1 = h9_1_13 + CDx * h9_1_7;
    const double h9_1_16 = acc[172] + ABx * acc[92];
    const double k9_1_7_2 = h9_1_16 + CDy * h9_1_7;
    const double h9_1_17 = acc[173] + ABx * acc[93];
    const double k9_1_7_3 = h9_1_17 + CDz * h9_1_7;
    const double h9_1_8 = acc[164] + ABx * acc[84];
    const double k9_1_8_1 = h9_1_15 + CDx * h9_1_8;
    const double k9_1_8_2 = h9_1_17 + CDy * h9_1_8;
    const double h9_1_18 = acc[174] + ABx * acc[94];
    const double k9_1_8_3 = h9_1_18 + CDz * h9_1_8;
    const double h9_1_9 = acc[165] + ABx * acc[85];
    const double k9_1_9_1 = h9_1_14 + CDx * h9_1_9;
    const double k9_1_9_2 = h9_1_18 + CDy * h9_1_9;
    const double h9_1_19 = acc[175] + ABx * acc[95];
    const double k9_1_9_3 = h9_1_19 + CDz * h9_1_9;
    const double h9_2_10 = acc[230] + ABy * acc[86];
    const double h9_2_4 = acc[224] + ABy * acc[80];
    const double k9_2_4_1 = h9_2_10 + CDx * h9_2_4;
    const double h9_2_11 = acc[231] + ABy * acc[87];
    const double k9_2_4_2 = h9_2_11 + CDy * h9_2_4;
    const double h9_2_12 = acc[232] + ABy * acc[88];
    const double k9_2_4_3 = h9_2_12 + CDz * h9_2_4;
    const double h9_2_5 = acc[225] + ABy * acc[81];
    const double k9_2_5_1 = h9_2_11 + CDx * h9_2_5;
    const double h9_2_13 = acc[233] + ABy * acc[89];
    const double k9_2_5_2 = h9_2_13 + CDy * h9_2_5;
    const double h9_2_15 = acc[235] + ABy * acc[91];
    const double k9_2_5_3 = h9_2_15 + CDz * h9_2_5;
    const double h9_2_6 = acc[226] + ABy * acc[82];
    const double k9_2_6_1 = h9_2_12 + CDx * h9_2_6;
    const double k9_2_6_2 = h9_2_15 + CDy * h9_2_6;
    const double h9_2_14 = acc[234] + ABy * acc[90];
    const double k9_2_6_3 = h9_2_14 + CDz * h9_2_6;
    const double h9_2_7 = acc[227] + ABy * acc[83];
    const double k9_2_7_1 = h9_2_13 + CDx * h9_2_7;
    const double h9_2_16 = acc[236] + ABy * acc[92];
    const double k9_2_7_2 = h9_2_16 + CDy * h9_2_7;
    const double h9_2_17 = acc[237] + ABy * acc[93];
    const double k9_2_7_3 = h9_2_17 + CDz * h9_2_7;
    const double h9_2_8 = acc[228] + ABy * acc[84];
    const double k9_2_8_1 = h9_2_15 + CDx * h9_2_8;
    const double k9_2_8_2 = h9_2_17 + CDy * h9_2_8;
    const double h9_2_18 = acc[238] + ABy * acc[94];
    const double k9_2_8_3 = h9_2_18 + CDz * h9_2_8;
    const double h9_2_9 = acc[229] + ABy * acc[85];
    const double k9_2_9_1 = h9_2_14 + CDx * h9_2_9;
    const double k9_2_9_2 = h9_2_18 + CDy * h9_2_9;
    const double h9_2_19 = acc[239] + ABy * acc[95];
    const double k9_2_9_3 = h9_2_19 + CDz * h9_2_9;
    const double h9_3_10 = acc[246] + ABz * acc[86];
    const double h9_3_4 = acc[240] + ABz * acc[80];
    const double k9_3_4_1 = h9_3_10 + CDx * h9_3_4;
    const double h9_3_11 = acc[247] + ABz * acc[87];
    const double k9_3_4_2 = h9_3_11 + CDy * h9_3_4;
    const double h9_3_12 = acc[248] + ABz * acc[88];
    const double k9_3_4_3 = h9_3_12 + CDz * h9_3_4;
    const double h9_3_5 = acc[241] + ABz * acc[81];
    const double k9_3_5_1 = h9_3_11 + CDx * h9_3_5;
    const double h9_3_13 = acc[249] + ABz * acc[89];
    const double k9_3_5_2 = h9_3_13 + CDy * h9_3_5;
    const double h9_3_15 = acc[251] + ABz * acc[91];
    const double k9_3_5_3 = h9_3_15 + CDz * h9_3_5;
    const double h9_3_6 = acc[242] + ABz * acc[82];
    const double k9_3_6_1 = h9_3_12 + CDx * h9_3_6;
    const double k9_3_6_2 = h9_3_15 + CDy * h9_3_6;
    const double h9_3_14 = acc[250] + ABz * acc[90];
    const double k9_3_6_3 = h9_3_14 + CDz * h9_3_6;
    const double h9_3_7 = acc[243] + ABz * acc[83];
    const double k9_3_7_1 = h9_3_13 + CDx * h9_3_7;
    const double h9_3_16 = acc[252] + ABz * acc[92];
    const double k9_3_7_2 = h9_3_16 + CDy * h9_3_7;
    const double h9_3_17 = acc[253] + ABz * acc[93];
    const double k9_3_7_3 = h9_3_17 + CDz * h9_3_7;
    const double h9_3_8 = acc[244] + ABz * acc[84];
    const double k9_3_8_1 = h9_3_15 + CDx * h9_3_8;
    const double k9_3_8_2 = h9_3_17 + CDy * h9_3_8;
    const double h9_3_18 = acc[254] + ABz * acc[94];
    const double k9_3_8_3 = h9_3_18 + CDz * h9_3_8;
    const double h9_3_9 = acc[245] + ABz * acc[85];
    const double k9_3_9_1 = h9_3_14 + CDx * h9_3_9;
    const double k9_3_9_2 = h9_3_18 + CDy * h9_3_9;
    const double h9_3_19 = acc[255] + ABz * acc[95];
    const double k9_3_9_3 = h9_3_19 + CDz * h9_3_9;
    res[0] = k4_1_4_1 * 0.3333333333333334;
    res[1] = k4_1_4_2 * 0.3333333333333334;
    res[2] = k4_1_4_3 * 0.3333333333333334;
    res[3] = k4_1_5_1 * 0.5773502691896258;
    res[4] = k4_1_5_2 * 0.5773502691896258;
    res[5] = k4_1_5_3 * 0.5773502691896258;
    res[6] = k4_1_6_1 * 0.5773502691896258;
    res[7] = k4_1_6_2 * 0.5773502691896258;
    res[8] = k4_1_6_3 * 0.5773502691896258;
    res[9] = k4_1_7_1 * 0.3333333333333334;
    res[10] = k4_1_7_2 * 0.3333333333333334;
    res[11] = k4_1_7_3 * 0.3333333333333334;
    res[12] = k4_1_8_1 * 0.5773502691896258;
    res[13] = k4_1_8_2 * 0.5773502691896258;
    res[14] = k4_1_8_3 * 0.5773502691896258;
    res[15] = k4_1_9_1 * 0.3333333333333334;
    res[16] = k4_1_9_2 * 0.3333333333333334;
    res[17] = k4_1_9_3 * 0.3333333333333334;
    res[18] = k4_2_4_1 * 0.3333333333333334;
    res[19] = k4_2_4_2 * 0.3333333333333334;
    res[20] = k4_2_4_3 * 0.3333333333333334;
    res[21] = k4_2_5_1 * 0.5773502691896258;
    res[22] = k4_2_5_2 * 0.5773502691896258;
    res[23] = k4_2_5_3 * 0.5773502691896258;
    res[24] = k4_2_6_1 * 0.5773502691896258;
    res[25] = k4_2_6_2 * 0.5773502691896258;
    res[26] = k4_2_6_3 * 0.5773502691896258;
    res[27] = k4_2_7_1 * 0.3333333333333334;
    res[28] = k4_2_7_2 * 0.3333333333333334;
    res[29] = k4_2_7_3 * 0.3333333333333334;
    res[30] = k4_2_8_1 * 0.5773502691896258;
    res[31] = k4_2_8_2 * 0.5773502691896258;
    res[32] = k4_2_8_3 * 0.5773502691896258;
    res[33] = k4_2_9_1 * 0.3333333333333334;
    res[34] = k4_2_9_2 * 0.3333333333333334;
    res[35] = k4_2_9_3 * 0.3333333333333334;
    res[36] = k4_3_4_1 * 0.3333333333333334;
    res[37] = k4_3_4_2 * 0.3333333333333334;
    res[38] = k4_3_4_3 * 0.3333333333333334;
    res[39] = k4_3_5_1 * 0.5773502691896258;
    res[40] = k4_3_5_2 * 0.5773502691896258;
    res[41] = k4_3_5_3 * 0.5773502691896258;
    res[42] = k4_3_6_1 * 0.5773502691896258;
    res[43] = k4_3_6_2 * 0.5773502691896258;
    res[44] = k4_3_6_3 * 0.5773502691896258;
    res[45] = k4_3_7_1 * 0.3333333333333334;
    res[46] = k4_3_7_2 * 0.3333333333333334;
    res[47] = k4_3_7_3 * 0.3333333333333334;
    res[48] = k4_3_8_1 * 0.5773502691896258;
    res[49] = k4_3_8_2 * 0.5773502691896258;
    res[50] = k4_3_8_3 * 0.5773502691896258;
    res[51] = k4_3_9_1 * 0.3333333333333334;
    res[52] = k4_3_9_2 * 0.3333333333333334;
    res[53] = k4_3_9_3 * 0.3333333333333334;
    res[54] = k5_1_4_1 * 0.5773502691896258;
    res[55] = k5_1_4_2 * 0.5773502691896258;
    res[56] = k5_1_4_3 * 0.5773502691896258;
    res[57] = k5_1_5_1;
    res[58] = k5_1_5_2;
    res[59] = k5_1_5_3;
    res[60] = k5_1_6_1;
    res[61] = k5_1_6_2;
    res[62] = k5_1_6_3;
    res[63] = k5_1_7_1 * 0.5773502691896258;
    res[64] = k5_1_7_2 * 0.5773502691896258;
    res[65] = k5_1_7_3 * 0.5773502691896258;
    res[66] = k5_1_8_1;
    res[67] = k5_1_8_2;
    res[68] = k5_1_8_3;
    res[69] = k5_1_9_1 * 0.5773502691896258;
    res[70] = k5_1_9_2 * 0.5773502691896258;
    res[71] = k5_1_9_3 * 0.5773502691896258;
    res[72] = k5_2_4_1 * 0.5773502691896258;
    res[73] = k5_2_4_2 * 0.5773502691896258;
    res[74] = k5_2_4_3 * 0.5773502691896258;
    res[75] = k5_2_5_1;
    res[76] = k5_2_5_2;
    res[77] = k5_2_5_3;
    res[78] = k5_2_6_1;
    res[79] = k5_2_6_2;
    res[80] = k5_2_6_3;
    res[81] = k5_2_7_1 * 0.5773502691896258;
    res[82] = k5_2_7_2 * 0.5773502691896258;
    res[83] = k5_2_7_3 * 0.5773502691896258;
    res[84] = k5_2_8_1;
    res[85] = k5_2_8_2;
    res[86] = k5_2_8_3;
    res[87] = k5_2_9_1 * 0.5773502691896258;
    res[88] = k5_2_9_2 * 0.5773502691896258;
    res[89] = k5_2_9_3 * 0.5773502691896258;
    res[90] = k5_3_4_1 * 0.5773502691896258;
    res[91] = k5_3_4_2 * 0.5773502691896258;
    res[92] = k5_3_4_3 * 0.5773502691896258;
    res[93] = k5_3_5_1;
    res[94] = k5_3_5_2;
    res[95] = k5_3_5_3;
    res[96] = k5_3_6_1;
    res[97] = k5_3_6_2;
    res[98] = k5_3_6_3;
    res[99] = k5_3_7_1 * 0.5773502691896258;
    res[100] = k5_3_7_2 * 0.5773502691896258;
    res[101] = k5_3_7_3 * 0.5773502691896258;
    res[102] = k5_3_8_1;
    res[103] = k5_3_8_2;
    res[104] = k5_3_8_3;
    res[105] = k5_3_9_1 * 0.5773502691896258;
    res[106] = k5_3_9_2 * 0.5773502691896258;
    res[107] = k5_3_9_3 * 0.5773502691896258;
    res[108] = k6_1_4_1 * 0.5773502691896258;
    res[109] = k6_1_4_2 * 0.5773502691896258;
    res[110] = k6_1_4_3 * 0.5773502691896258;
    res[111] = k6_1_5_1;
    res[112] = k6_1_5_2;
    res[113] = k6_1_5_3;
    res[114] = k6_1_6_1;
    res[115] = k6_1_6_2;
    res[116] = k6_1_6_3;
    res[117] = k6_1_7_1 * 0.5773502691896258;
    res[118] = k6_1_7_2 * 0.5773502691896258;
    res[119] = k6_1_7_3 * 0.5773502691896258;
    res[120] = k6_1_8_1;
    res[121] = k6_1_8_2;
    res[122] = k6_1_8_3;
    res[123] = k6_1_9_1 * 0.5773502691896258;
    res[124] = k6_1_9_2 * 0.5773502691896258;
    res[125] = k6_1_9_3 * 0.5773502691896258;
    res[126] = k6_2_4_1 * 0.5773502691896258;
    res[127] = k6_2_4_2 * 0.5773502691896258;
    res[128] = k6_2_4_3 * 0.5773502691896258;
    res[129] = k6_2_5_1;
    res[130] = k6_2_5_2;
    res[131] = k6_2_5_3;
    res[132] = k6_2_6_1;
    res[133] = k6_2_6_2;
    res[134] = k6_2_6_3;
    res[135] = k6_2_7_1 * 0.5773502691896258;
    res[136] = k6_2_7_2 * 0.5773502691896258;
    res[137] = k6_2_7_3 * 0.5773502691896258;
    res[138] = k6_2_8_1;
    res[139] = k6_2_8_2;
    res[140] = k6_2_8_3;
    res[141] = k6_2_9_1 * 0.5773502691896258;
    res[142] = k6_2_9_2 * 0.5773502691896258;
    res[143] = k6_2_9_3 * 0.5773502691896258;
    res[144] = k6_3_4_1 * 0.5773502691896258;
    res[145] = k6_3_4_2 * 0.5773502691896258;
    res[146] = k6_3_4_3 * 0.5773502691896258;
    res[147] = k6_3_5_1;
    res[148] = k6_3_5_2;
    res[149] = k6_3_5_3;
    res[150] = k6_3_6_1;
    res[151] = k6_3_6_2;
    res[152] = k6_3_6_3;
    res[153] = k6_3_7_1 * 0.5773502691896258;
    res[154] = k6_3_7_2 * 0.5773502691896258;
    res[155] = k6_3_7_3 * 0.5773502691896258;
    res[156] = k6_3_8_1;
    res[157] = k6_3_8_2;
    res[158] = k6_3_8_3;
    res[159] = k6_3_9_1 * 0.5773502691896258;
    res[160] = k6_3_9_2 * 0.5773502691896258;
    res[161] = k6_3_9_3 * 0.5773502691896258;
    res[162] = k7_1_4_1 * 0.3333333333333334;
    res[163] = k7_1_4_2 * 0.3333333333333334;
    res[164] = k7_1_4_3 * 0.3333333333333334;
    res[165] = k7_1_5_1 * 0.5773502691896258;
    res[166] = k7_1_5_2 * 0.5773502691896258;
    res[167] = k7_1_5_3 * 0.5773502691896258;
    res[168] = k7_1_6_1 * 0.5773502691896258;
    res[169] = k7_1_6_2 * 0.5773502691896258;
    res[170] = k7_1_6_3 * 0.5773502691896258;
    res[171] = k7_1_7_1 * 0.3333333333333334;
    res[172] = k7_1_7_2 * 0.3333333333333334;
    res[173] = k7_1_7_3 * 0.3333333333333334;
    res[174] = k7_1_8_1 * 0.5773502691896258;
    res[175] = k7_1_8_2 * 0.5773502691896258;
    res[176] = k7_1_8_3 * 0.5773502691896258;
    res[177] = k7_1_9_1 * 0.3333333333333334;
    res[178] = k7_1_9_2 * 0.3333333333333334;
    res[179] = k7_1_9_3 * 0.3333333333333334;
    res[180] = k7_2_4_1 * 0.3333333333333334;
    res[181] = k7_2_4_2 * 0.3333333333333334;
    res[182] = k7_2_4_3 * 0.3333333333333334;
    res[183] = k7_2_5_1 * 0.5773502691896258;
    res[184] = k7_2_5_2 * 0.5773502691896258;
    res[185] = k7_2_5_3 * 0.5773502691896258;
    res[186] = k7_2_6_1 * 0.5773502691896258;
    res[187] = k7_2_6_2 * 0.5773502691896258;
    res[188] = k7_2_6_3 * 0.5773502691896258;
    res[189] = k7_2_7_1 * 0.3333333333333334;
    res[190] = k7_2_7_2 * 0.3333333333333334;
    res[191] = k7_2_7_3 * 0.3333333333333334;
    res[192] = k7_2_8_1 * 0.5773502691896258;
    res[193] = k7_2_8_2 * 0.5773502691896258;
    res[194] = k7_2_8_3 * 0.5773502691896258;
    res[195] = k7_2_9_1 * 0.3333333333333334;
    res[196] = k7_2_9_2 * 0.3333333333333334;
    res[197] = k7_2_9_3 * 0.3333333333333334;
    res[198] = k7_3_4_1 * 0.3333333333333334;
    res[199] = k7_3_4_2 * 0.3333333333333334;
    res[200] = k7_3_4_3 * 0.3333333333333334;
    res[201] = k7_3_5_1 * 0.5773502691896258;
    res[202] = k7_3_5_2 * 0.5773502691896258;
    res[203] = k7_3_5_3 * 0.5773502691896258;
    res[204] = k7_3_6_1 * 0.5773502691896258;
    res[205] = k7_3_6_2 * 0.5773502691896258;
    res[206] = k7_3_6_3 * 0.5773502691896258;
    res[207] = k7_3_7_1 * 0.3333333333333334;
    res[208] = k7_3_7_2 * 0.3333333333333334;
    res[209] = k7_3_7_3 * 0.3333333333333334;
    res[210] = k7_3_8_1 * 0.5773502691896258;
    res[211] = k7_3_8_2 * 0.5773502691896258;
    res[212] = k7_3_8_3 * 0.5773502691896258;
    res[213] = k7_3_9_1 * 0.3333333333333334;
    res[214] = k7_3_9_2 * 0.3333333333333334;
    res[215] = k7_3_9_3 * 0.3333333333333334;
    res[216] = k8_1_4_1 * 0.5773502691896258;
    res[217] = k8_1_4_2 * 0.5773502691896258;
    res[218] = k8_1_4_3 * 0.5773502691896258;
    res[219] = k8_1_5_1;
    res[220] = k8_1_5_2;
    res[221] = k8_1_5_3;
    res[222] = k8_1_6_1;
    res[223] = k8_1_6_2;
    res[224] = k8_1_6_3;
    res[225] = k8_1_7_1 * 0.5773502691896258;
    res[226] = k8_1_7_2 * 0.5773502691896258;
    res[227] = k8_1_7_3 * 0.5773502691896258;
    res[228] = k8_1_8_1;
    res[229] = k8_1_8_2;
    res[230] = k8_1_8_3;
    res[231] = k8_1_9_1 * 0.5773502691896258;
    res[232] = k8_1_9_2 * 0.5773502691896258;
    res[233] = k8_1_9_3 * 0.5773502691896258;
    res[234] = k8_2_4_1 * 0.5773502691896258;
    res[235] = k8_2_4_2 * 0.5773502691896258;
    res[236] = k8_2_4_3 * 0.5773502691896258;
    res[237] = k8_2_5_1;
    res[238] = k8_2_5_2;
    res[239] = k8_2_5_3;
    res[240] = k8_2_6_1;
    res[241] = k8_2_6_2;
    res[242] = k8_2_6_3;
    res[243] = k8_2_7_1 * 0.5773502691896258;
    res[244] = k8_2_7_2 * 0.5773502691896258;
    res[245] = k8_2_7_3 * 0.5773502691896258;
    res[246] = k8_2_8_1;
    res[247] = k8_2_8_2;
    res[248] = k8_2_8_3;
    res[249] = k8_2_9_1 * 0.5773502691896258;
    res[250] = k8_2_9_2 * 0.5773502691896258;
    res[251] = k8_2_9_3 * 0.5773502691896258;
    res[252] = k8_3_4_1 * 0.5773502691896258;
    res[253] = k8_3_4_2 * 0.5773502691896258;
    res[254] = k8_3_4_3 * 0.5773502691896258;
    res[255] = k8_3_5_1;
    res[256] = k8_3_5_2;
    res[257] = k8_3_5_3;
    res[258] = k8_3_6_1;
    res[259] = k8_3_6_2;
    res[260] = k8_3_6_3;
    res[261] = k8_3_7_1 * 0.5773502691896258;
    res[262] = k8_3_7_2 * 0.5773502691896258;
    res[263] = k8_3_7_3 * 0.5773502691896258;
    res[264] = k8_3_8_1;
    res[265] = k8_3_8_2;
    res[266] = k8_3_8_3;
    res[267] = k8_3_9_1 * 0.5773502691896258;
    res[268] = k8_3_9_2 * 0.5773502691896258;
    res[269] = k8_3_9_3 * 0.5773502691896258;
    res[270] = k9_1_4_1 * 0.3333333333333334;
    res[271] = k9_1_4_2 * 0.3333333333333334;
    res[272] = k9_1_4_3 * 0.3333333333333334;
    res[273] = k9_1_5_1 * 0.5773502691896258;
    res[274] = k9_1_5_2 * 0.5773502691896258;
    res[275] = k9_1_5_3 * 0.5773502691896258;
    res[276] = k9_1_6_1 * 0.5773502691896258;
    res[277] = k9_1_6_2 * 0.5773502691896258;
    res[278] = k9_1_6_3 * 0.5773502691896258;
    res[279] = k9_1_7_1 * 0.3333333333333334;
    res[280] = k9_1_7_2 * 0.3333333333333334;
    res[281] = k9_1_7_3 * 0.3333333333333334;
    res[282] = k9_1_8_1 * 0.5773502691896258;
    res[283] = k9_1_8_2 * 0.5773502691896258;
    res[284] = k9_1_8_3 * 0.5773502691896258;
    res[285] = k9_1_9_1 * 0.3333333333333334;
    res[286] = k9_1_9_2 * 0.3333333333333334;
    res[287] = k9_1_9_3 * 0.3333333333333334;
    res[288] = k9_2_4_1 * 0.3333333333333334;
    res[289] = k9_2_4_2 * 0.3333333333333334;
    res[290] = k9_2_4_3 * 0.3333333333333334;
    res[291] = k9_2_5_1 * 0.5773502691896258;
    res[292] = k9_2_5_2 * 0.5773502691896258;
    res[293] = k9_2_5_3 * 0.5773502691896258;
    res[294] = k9_2_6_1 * 0.5773502691896258;
    res[295] = k9_2_6_2 * 0.5773502691896258;
    res[296] = k9_2_6_3 * 0.5773502691896258;
    res[297] = k9_2_7_1 * 0.3333333333333334;
    res[298] = k9_2_7_2 * 0.3333333333333334;
    res[299] = k9_2_7_3 * 0.3333333333333334;
    res[300] = k9_2_8_1 * 0.5773502691896258;
    res[301] = k9_2_8_2 * 0.5773502691896258;
    res[302] = k9_2_8_3 * 0.5773502691896258;
    res[303] = k9_2_9_1 * 0.3333333333333334;
    res[304] = k9_2_9_2 * 0.3333333333333334;
    res[305] = k9_2_9_3 * 0.3333333333333334;
    res[306] = k9_3_4_1 * 0.3333333333333334;
    res[307] = k9_3_4_2 * 0.3333333333333334;
    res[308] = k9_3_4_3 * 0.3333333333333334;
    res[309] = k9_3_5_1 * 0.5773502691896258;
    res[310] = k9_3_5_2 * 0.5773502691896258;
    res[311] = k9_3_5_3 * 0.5773502691896258;
    res[312] = k9_3_6_1 * 0.5773502691896258;
    res[313] = k9_3_6_2 * 0.5773502691896258;
    res[314] = k9_3_6_3 * 0.5773502691896258;
    res[315] = k9_3_7_1 * 0.3333333333333334;
    res[316] = k9_3_7_2 * 0.3333333333333334;
    res[317] = k9_3_7_3 * 0.3333333333333334;
    res[318] = k9_3_8_1 * 0.5773502691896258;
    res[319] = k9_3_8_2 * 0.5773502691896258;
    res[320] = k9_3_8_3 * 0.5773502691896258;
    res[321] = k9_3_9_1 * 0.3333333333333334;
    res[322] = k9_3_9_2 * 0.3333333333333334;
    res[323] = k9_3_9_3 * 0.3333333333333334;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[324]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_dpdp(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[256];
    vrr_dpdp<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 256; ++x) acc_out[x] = acc[x];
    }
    hrr_dpdp(P, p, q, acc, res);
}

__device__ __forceinline__ void store_dpdp(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    const long long kl_0_1 = pair_index(ik_.z + 0, ik_.w + 1);
    const long long kl_0_2 = pair_index(ik_.z + 0, ik_.w + 2);
    const long long kl_1_0 = pair_index(ik_.z + 1, ik_.w + 0);
    const long long kl_1_1 = pair_index(ik_.z + 1, ik_.w + 1);
    const long long kl_1_2 = pair_index(ik_.z + 1, ik_.w + 2);
    const long long kl_2_0 = pair_index(ik_.z + 2, ik_.w + 0);
    const long long kl_2_1 = pair_index(ik_.z + 2, ik_.w + 1);
    const long long kl_2_2 = pair_index(ik_.z + 2, ik_.w + 2);
    const long long kl_3_0 = pair_index(ik_.z + 3, ik_.w + 0);
    const long long kl_3_1 = pair_index(ik_.z + 3, ik_.w + 1);
    const long long kl_3_2 = pair_index(ik_.z + 3, ik_.w + 2);
    const long long kl_4_0 = pair_index(ik_.z + 4, ik_.w + 0);
    const long long kl_4_1 = pair_index(ik_.z + 4, ik_.w + 1);
    const long long kl_4_2 = pair_index(ik_.z + 4, ik_.w + 2);
    const long long kl_5_0 = pair_index(ik_.z + 5, ik_.w + 0);
    const long long kl_5_1 = pair_index(ik_.z + 5, ik_.w + 1);
    const long long kl_5_2 = pair_index(ik_.z + 5, ik_.w + 2);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_0, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_0, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_0, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_0, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_0_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_0_0, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_0_0, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_0_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_0_0, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_0_0, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_0_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_0_0, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_0_0, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_0_1, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_0_1, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_0_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_0_1, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_0_1, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_0_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_0_1, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_0_1, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_0_1, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_0_1, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_0_1, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_0_1, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_0_1, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_0_1, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_0_1, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_0_1, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_0_1, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_0_2, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_0_2, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_0_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_0_2, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_0_2, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_0_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_0_2, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_0_2, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_0_2, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_0_2, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_0_2, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_0_2, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_0_2, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_0_2, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_0_2, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_0_2, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_0_2, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_1_0, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_1_0, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_1_0, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_1_0, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_1_0, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_1_0, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_1_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_1_0, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_1_0, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_1_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_1_0, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_1_0, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_1_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_1_0, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_1_0, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_1_1, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_1_1, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_1_1, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_1_1, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_1_1, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_1_1, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_1_1, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_1_1, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_1_1, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_1_1, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_1_1, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_1_1, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_1_1, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_1_1, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_1_1, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_1_2, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_1_2, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_1_2, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_1_2, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_1_2, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_1_2, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_1_2, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
    { const long long ij = ij_1_2, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[100]; }
    { const long long ij = ij_1_2, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[101]; }
    { const long long ij = ij_1_2, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[102]; }
    { const long long ij = ij_1_2, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[103]; }
    { const long long ij = ij_1_2, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[104]; }
    { const long long ij = ij_1_2, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[105]; }
    { const long long ij = ij_1_2, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[106]; }
    { const long long ij = ij_1_2, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[107]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[108]; }
    { const long long ij = ij_2_0, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[109]; }
    { const long long ij = ij_2_0, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[110]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[111]; }
    { const long long ij = ij_2_0, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[112]; }
    { const long long ij = ij_2_0, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[113]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[114]; }
    { const long long ij = ij_2_0, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[115]; }
    { const long long ij = ij_2_0, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[116]; }
    { const long long ij = ij_2_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[117]; }
    { const long long ij = ij_2_0, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[118]; }
    { const long long ij = ij_2_0, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[119]; }
    { const long long ij = ij_2_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[120]; }
    { const long long ij = ij_2_0, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[121]; }
    { const long long ij = ij_2_0, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[122]; }
    { const long long ij = ij_2_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[123]; }
    { const long long ij = ij_2_0, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[124]; }
    { const long long ij = ij_2_0, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[125]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[126]; }
    { const long long ij = ij_2_1, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[127]; }
    { const long long ij = ij_2_1, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[128]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[129]; }
    { const long long ij = ij_2_1, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[130]; }
    { const long long ij = ij_2_1, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[131]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[132]; }
    { const long long ij = ij_2_1, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[133]; }
    { const long long ij = ij_2_1, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[134]; }
    { const long long ij = ij_2_1, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[135]; }
    { const long long ij = ij_2_1, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[136]; }
    { const long long ij = ij_2_1, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[137]; }
    { const long long ij = ij_2_1, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[138]; }
    { const long long ij = ij_2_1, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[139]; }
    { const long long ij = ij_2_1, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[140]; }
    { const long long ij = ij_2_1, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[141]; }
    { const long long ij = ij_2_1, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[142]; }
    { const long long ij = ij_2_1, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[143]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[144]; }
    { const long long ij = ij_2_2, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[145]; }
    { const long long ij = ij_2_2, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[146]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[147]; }
    { const long long ij = ij_2_2, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[148]; }
    { const long long ij = ij_2_2, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[149]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[150]; }
    { const long long ij = ij_2_2, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[151]; }
    { const long long ij = ij_2_2, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[152]; }
    { const long long ij = ij_2_2, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[153]; }
    { const long long ij = ij_2_2, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[154]; }
    { const long long ij = ij_2_2, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[155]; }
    { const long long ij = ij_2_2, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[156]; }
    { const long long ij = ij_2_2, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[157]; }
    { const long long ij = ij_2_2, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[158]; }
    { const long long ij = ij_2_2, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[159]; }
    { const long long ij = ij_2_2, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[160]; }
    { const long long ij = ij_2_2, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[161]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[162]; }
    { const long long ij = ij_3_0, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[163]; }
    { const long long ij = ij_3_0, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[164]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[165]; }
    { const long long ij = ij_3_0, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[166]; }
    { const long long ij = ij_3_0, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[167]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[168]; }
    { const long long ij = ij_3_0, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[169]; }
    { const long long ij = ij_3_0, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[170]; }
    { const long long ij = ij_3_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[171]; }
    { const long long ij = ij_3_0, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[172]; }
    { const long long ij = ij_3_0, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[173]; }
    { const long long ij = ij_3_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[174]; }
    { const long long ij = ij_3_0, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[175]; }
    { const long long ij = ij_3_0, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[176]; }
    { const long long ij = ij_3_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[177]; }
    { const long long ij = ij_3_0, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[178]; }
    { const long long ij = ij_3_0, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[179]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[180]; }
    { const long long ij = ij_3_1, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[181]; }
    { const long long ij = ij_3_1, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[182]; }
    { const long long ij = ij_3_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[183]; }
    { const long long ij = ij_3_1, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[184]; }
    { const long long ij = ij_3_1, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[185]; }
    { const long long ij = ij_3_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[186]; }
    { const long long ij = ij_3_1, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[187]; }
    { const long long ij = ij_3_1, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[188]; }
    { const long long ij = ij_3_1, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[189]; }
    { const long long ij = ij_3_1, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[190]; }
    { const long long ij = ij_3_1, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[191]; }
    { const long long ij = ij_3_1, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[192]; }
    { const long long ij = ij_3_1, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[193]; }
    { const long long ij = ij_3_1, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[194]; }
    { const long long ij = ij_3_1, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[195]; }
    { const long long ij = ij_3_1, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[196]; }
    { const long long ij = ij_3_1, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[197]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[198]; }
    { const long long ij = ij_3_2, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[199]; }
    { const long long ij = ij_3_2, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[200]; }
    { const long long ij = ij_3_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[201]; }
    { const long long ij = ij_3_2, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[202]; }
    { const long long ij = ij_3_2, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[203]; }
    { const long long ij = ij_3_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[204]; }
    { const long long ij = ij_3_2, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[205]; }
    { const long long ij = ij_3_2, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[206]; }
    { const long long ij = ij_3_2, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[207]; }
    { const long long ij = ij_3_2, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[208]; }
    { const long long ij = ij_3_2, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[209]; }
    { const long long ij = ij_3_2, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[210]; }
    { const long long ij = ij_3_2, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[211]; }
    { const long long ij = ij_3_2, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[212]; }
    { const long long ij = ij_3_2, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[213]; }
    { const long long ij = ij_3_2, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[214]; }
    { const long long ij = ij_3_2, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[215]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[216]; }
    { const long long ij = ij_4_0, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[217]; }
    { const long long ij = ij_4_0, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[218]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[219]; }
    { const long long ij = ij_4_0, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[220]; }
    { const long long ij = ij_4_0, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[221]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[222]; }
    { const long long ij = ij_4_0, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[223]; }
    { const long long ij = ij_4_0, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[224]; }
    { const long long ij = ij_4_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[225]; }
    { const long long ij = ij_4_0, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[226]; }
    { const long long ij = ij_4_0, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[227]; }
    { const long long ij = ij_4_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[228]; }
    { const long long ij = ij_4_0, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[229]; }
    { const long long ij = ij_4_0, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[230]; }
    { const long long ij = ij_4_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[231]; }
    { const long long ij = ij_4_0, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[232]; }
    { const long long ij = ij_4_0, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[233]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[234]; }
    { const long long ij = ij_4_1, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[235]; }
    { const long long ij = ij_4_1, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[236]; }
    { const long long ij = ij_4_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[237]; }
    { const long long ij = ij_4_1, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[238]; }
    { const long long ij = ij_4_1, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[239]; }
    { const long long ij = ij_4_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[240]; }
    { const long long ij = ij_4_1, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[241]; }
    { const long long ij = ij_4_1, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[242]; }
    { const long long ij = ij_4_1, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[243]; }
    { const long long ij = ij_4_1, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[244]; }
    { const long long ij = ij_4_1, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[245]; }
    { const long long ij = ij_4_1, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[246]; }
    { const long long ij = ij_4_1, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[247]; }
    { const long long ij = ij_4_1, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[248]; }
    { const long long ij = ij_4_1, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[249]; }
    { const long long ij = ij_4_1, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[250]; }
    { const long long ij = ij_4_1, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[251]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[252]; }
    { const long long ij = ij_4_2, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[253]; }
    { const long long ij = ij_4_2, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[254]; }
    { const long long ij = ij_4_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[255]; }
    { const long long ij = ij_4_2, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[256]; }
    { const long long ij = ij_4_2, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[257]; }
    { const long long ij = ij_4_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[258]; }
    { const long long ij = ij_4_2, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[259]; }
    { const long long ij = ij_4_2, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[260]; }
    { const long long ij = ij_4_2, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[261]; }
    { const long long ij = ij_4_2, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[262]; }
    { const long long ij = ij_4_2, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[263]; }
    { const long long ij = ij_4_2, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[264]; }
    { const long long ij = ij_4_2, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[265]; }
    { const long long ij = ij_4_2, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[266]; }
    { const long long ij = ij_4_2, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[267]; }
    { const long long ij = ij_4_2, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[268]; }
    { const long long ij = ij_4_2, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[269]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[270]; }
    { const long long ij = ij_5_0, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[271]; }
    { const long long ij = ij_5_0, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[272]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[273]; }
    { const long long ij = ij_5_0, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[274]; }
    { const long long ij = ij_5_0, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[275]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[276]; }
    { const long long ij = ij_5_0, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[277]; }
    { const long long ij = ij_5_0, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[278]; }
    { const long long ij = ij_5_0, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[279]; }
    { const long long ij = ij_5_0, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[280]; }
    { const long long ij = ij_5_0, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[281]; }
    { const long long ij = ij_5_0, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[282]; }
    { const long long ij = ij_5_0, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[283]; }
    { const long long ij = ij_5_0, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[284]; }
    { const long long ij = ij_5_0, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[285]; }
    { const long long ij = ij_5_0, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[286]; }
    { const long long ij = ij_5_0, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[287]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[288]; }
    { const long long ij = ij_5_1, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[289]; }
    { const long long ij = ij_5_1, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[290]; }
    { const long long ij = ij_5_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[291]; }
    { const long long ij = ij_5_1, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[292]; }
    { const long long ij = ij_5_1, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[293]; }
    { const long long ij = ij_5_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[294]; }
    { const long long ij = ij_5_1, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[295]; }
    { const long long ij = ij_5_1, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[296]; }
    { const long long ij = ij_5_1, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[297]; }
    { const long long ij = ij_5_1, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[298]; }
    { const long long ij = ij_5_1, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[299]; }
    { const long long ij = ij_5_1, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[300]; }
    { const long long ij = ij_5_1, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[301]; }
    { const long long ij = ij_5_1, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[302]; }
    { const long long ij = ij_5_1, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[303]; }
    { const long long ij = ij_5_1, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[304]; }
    { const long long ij = ij_5_1, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[305]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[306]; }
    { const long long ij = ij_5_2, kl = kl_0_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[307]; }
    { const long long ij = ij_5_2, kl = kl_0_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[308]; }
    { const long long ij = ij_5_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[309]; }
    { const long long ij = ij_5_2, kl = kl_1_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[310]; }
    { const long long ij = ij_5_2, kl = kl_1_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[311]; }
    { const long long ij = ij_5_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[312]; }
    { const long long ij = ij_5_2, kl = kl_2_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[313]; }
    { const long long ij = ij_5_2, kl = kl_2_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[314]; }
    { const long long ij = ij_5_2, kl = kl_3_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[315]; }
    { const long long ij = ij_5_2, kl = kl_3_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[316]; }
    { const long long ij = ij_5_2, kl = kl_3_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[317]; }
    { const long long ij = ij_5_2, kl = kl_4_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[318]; }
    { const long long ij = ij_5_2, kl = kl_4_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[319]; }
    { const long long ij = ij_5_2, kl = kl_4_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[320]; }
    { const long long ij = ij_5_2, kl = kl_5_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[321]; }
    { const long long ij = ij_5_2, kl = kl_5_1;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[322]; }
    { const long long ij = ij_5_2, kl = kl_5_2;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[323]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_dpdp(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 324; ++x) {
        const int ia = x / 54, ibb = (x / 18) % 3, ic = (x / 3) % 6, id = x % 3;
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
__global__ void __launch_bounds__(128) eri_queue_dpdp(const EriQueue Q) {
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
        double acc[256];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 256; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_dpdp<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_dpdp<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 256; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: each leader stores its quartet's whole block at its slot
            if (lead) {
                double res[324];
                hrr_dpdp(Q.pairs, p, q, acc, res);
                double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                    (__ldg(&Q.chunk_slot[c]) + base + kq) * (long long)324;
#pragma unroll
                for (int x = 0; x < 324; ++x) dst[x] = res[x];
            }
        } else if (lead) {
            double res[324];
            hrr_dpdp(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_dpdp(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_dpdp(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_dpdp(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    constexpr size_t smem = 0;
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_dpdp<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_dpdp<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_dpdp<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_dpdp<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_dpdp(int mixed) {

    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dpdp<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dpdp<0, 0>, 128, 0);
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
__global__ void __launch_bounds__(128) schwarz_kernel_dpdp(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[324];
    if (full) {
        quartet_dpdp<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[19]));
    m = fmax(m, fabs(res[38]));
    m = fmax(m, fabs(res[57]));
    m = fmax(m, fabs(res[76]));
    m = fmax(m, fabs(res[95]));
    m = fmax(m, fabs(res[114]));
    m = fmax(m, fabs(res[133]));
    m = fmax(m, fabs(res[152]));
    m = fmax(m, fabs(res[171]));
    m = fmax(m, fabs(res[190]));
    m = fmax(m, fabs(res[209]));
    m = fmax(m, fabs(res[228]));
    m = fmax(m, fabs(res[247]));
    m = fmax(m, fabs(res[266]));
    m = fmax(m, fabs(res[285]));
    m = fmax(m, fabs(res[304]));
    m = fmax(m, fabs(res[323]));
        qout[p] = sqrt(m);
        return;
    }
    double acc[256];
    for (int k = 0; k < in.y; ++k) {
        quartet_dpdp<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[19]));
    m = fmax(m, fabs(res[38]));
    m = fmax(m, fabs(res[57]));
    m = fmax(m, fabs(res[76]));
    m = fmax(m, fabs(res[95]));
    m = fmax(m, fabs(res[114]));
    m = fmax(m, fabs(res[133]));
    m = fmax(m, fabs(res[152]));
    m = fmax(m, fabs(res[171]));
    m = fmax(m, fabs(res[190]));
    m = fmax(m, fabs(res[209]));
    m = fmax(m, fabs(res[228]));
    m = fmax(m, fabs(res[247]));
    m = fmax(m, fabs(res[266]));
    m = fmax(m, fabs(res[285]));
    m = fmax(m, fabs(res[304]));
    m = fmax(m, fabs(res[323]));
        w = fmax(w, fabs(acc[0]));
        w = fmax(w, fabs(acc[17]));
        w = fmax(w, fabs(acc[34]));
        w = fmax(w, fabs(acc[51]));
        w = fmax(w, fabs(acc[68]));
        w = fmax(w, fabs(acc[85]));
        w = fmax(w, fabs(acc[102]));
        w = fmax(w, fabs(acc[119]));
        w = fmax(w, fabs(acc[136]));
        w = fmax(w, fabs(acc[153]));
        w = fmax(w, fabs(acc[170]));
        w = fmax(w, fabs(acc[187]));
        w = fmax(w, fabs(acc[204]));
        w = fmax(w, fabs(acc[221]));
        w = fmax(w, fabs(acc[238]));
        w = fmax(w, fabs(acc[255]));
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }
}

void launch_schwarz_dpdp(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    schwarz_kernel_dpdp<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}

}  // namespace molints

// Generated by gen_eri.py -- class (fs|pp).  Do not edit.
// VRR entries: 213, contracted block: 90, HRR lines: 90, outputs: 90.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[90], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_fspp(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 90; ++x) acc[x] = 0.0;
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
            const VT v4_1_1 = QCx * v4_0_1 + WQx * v4_0_2 + (VT)2.0 * oo2ze * v1_0_2;
            const VT v5_1_1 = QCx * v5_0_1 + WQx * v5_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v6_1_1 = QCx * v6_0_1 + WQx * v6_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v7_1_1 = QCx * v7_0_1 + WQx * v7_0_2;
            const VT v8_1_1 = QCx * v8_0_1 + WQx * v8_0_2;
            const VT v9_1_1 = QCx * v9_0_1 + WQx * v9_0_2;
            const VT v10_1_0 = QCx * v10_0_0 + WQx * v10_0_1 + (VT)3.0 * oo2ze * v4_0_1;
            const VT v10_1_1 = QCx * v10_0_1 + WQx * v10_0_2 + (VT)3.0 * oo2ze * v4_0_2;
            const VT v11_1_0 = QCx * v11_0_0 + WQx * v11_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v11_1_1 = QCx * v11_0_1 + WQx * v11_0_2 + (VT)2.0 * oo2ze * v5_0_2;
            const VT v12_1_0 = QCx * v12_0_0 + WQx * v12_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v12_1_1 = QCx * v12_0_1 + WQx * v12_0_2 + (VT)2.0 * oo2ze * v6_0_2;
            const VT v13_1_0 = QCx * v13_0_0 + WQx * v13_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v13_1_1 = QCx * v13_0_1 + WQx * v13_0_2 + (VT)1.0 * oo2ze * v7_0_2;
            const VT v14_1_0 = QCx * v14_0_0 + WQx * v14_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v14_1_1 = QCx * v14_0_1 + WQx * v14_0_2 + (VT)1.0 * oo2ze * v9_0_2;
            const VT v15_1_0 = QCx * v15_0_0 + WQx * v15_0_1 + (VT)1.0 * oo2ze * v8_0_1;
            const VT v15_1_1 = QCx * v15_0_1 + WQx * v15_0_2 + (VT)1.0 * oo2ze * v8_0_2;
            const VT v16_1_0 = QCx * v16_0_0 + WQx * v16_0_1;
            const VT v16_1_1 = QCx * v16_0_1 + WQx * v16_0_2;
            const VT v17_1_0 = QCx * v17_0_0 + WQx * v17_0_1;
            const VT v17_1_1 = QCx * v17_0_1 + WQx * v17_0_2;
            const VT v18_1_0 = QCx * v18_0_0 + WQx * v18_0_1;
            const VT v18_1_1 = QCx * v18_0_1 + WQx * v18_0_2;
            const VT v19_1_0 = QCx * v19_0_0 + WQx * v19_0_1;
            const VT v19_1_1 = QCx * v19_0_1 + WQx * v19_0_2;
            const VT v4_2_1 = QCy * v4_0_1 + WQy * v4_0_2;
            const VT v5_2_1 = QCy * v5_0_1 + WQy * v5_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v6_2_1 = QCy * v6_0_1 + WQy * v6_0_2;
            const VT v7_2_1 = QCy * v7_0_1 + WQy * v7_0_2 + (VT)2.0 * oo2ze * v2_0_2;
            const VT v8_2_1 = QCy * v8_0_1 + WQy * v8_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v9_2_1 = QCy * v9_0_1 + WQy * v9_0_2;
            const VT v10_2_0 = QCy * v10_0_0 + WQy * v10_0_1;
            const VT v10_2_1 = QCy * v10_0_1 + WQy * v10_0_2;
            const VT v11_2_0 = QCy * v11_0_0 + WQy * v11_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v11_2_1 = QCy * v11_0_1 + WQy * v11_0_2 + (VT)1.0 * oo2ze * v4_0_2;
            const VT v12_2_0 = QCy * v12_0_0 + WQy * v12_0_1;
            const VT v12_2_1 = QCy * v12_0_1 + WQy * v12_0_2;
            const VT v13_2_0 = QCy * v13_0_0 + WQy * v13_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v13_2_1 = QCy * v13_0_1 + WQy * v13_0_2 + (VT)2.0 * oo2ze * v5_0_2;
            const VT v14_2_0 = QCy * v14_0_0 + WQy * v14_0_1;
            const VT v14_2_1 = QCy * v14_0_1 + WQy * v14_0_2;
            const VT v15_2_0 = QCy * v15_0_0 + WQy * v15_0_1 + (VT)1.0 * oo2ze * v6_0_1;
            const VT v15_2_1 = QCy * v15_0_1 + WQy * v15_0_2 + (VT)1.0 * oo2ze * v6_0_2;
            const VT v16_2_0 = QCy * v16_0_0 + WQy * v16_0_1 + (VT)3.0 * oo2ze * v7_0_1;
            const VT v16_2_1 = QCy * v16_0_1 + WQy * v16_0_2 + (VT)3.0 * oo2ze * v7_0_2;
            const VT v17_2_0 = QCy * v17_0_0 + WQy * v17_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v17_2_1 = QCy * v17_0_1 + WQy * v17_0_2 + (VT)2.0 * oo2ze * v8_0_2;
            const VT v18_2_0 = QCy * v18_0_0 + WQy * v18_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v18_2_1 = QCy * v18_0_1 + WQy * v18_0_2 + (VT)1.0 * oo2ze * v9_0_2;
            const VT v19_2_0 = QCy * v19_0_0 + WQy * v19_0_1;
            const VT v19_2_1 = QCy * v19_0_1 + WQy * v19_0_2;
            const VT v4_3_1 = QCz * v4_0_1 + WQz * v4_0_2;
            const VT v5_3_1 = QCz * v5_0_1 + WQz * v5_0_2;
            const VT v6_3_1 = QCz * v6_0_1 + WQz * v6_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v7_3_1 = QCz * v7_0_1 + WQz * v7_0_2;
            const VT v8_3_1 = QCz * v8_0_1 + WQz * v8_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v9_3_1 = QCz * v9_0_1 + WQz * v9_0_2 + (VT)2.0 * oo2ze * v3_0_2;
            const VT v10_3_0 = QCz * v10_0_0 + WQz * v10_0_1;
            const VT v10_3_1 = QCz * v10_0_1 + WQz * v10_0_2;
            const VT v11_3_0 = QCz * v11_0_0 + WQz * v11_0_1;
            const VT v11_3_1 = QCz * v11_0_1 + WQz * v11_0_2;
            const VT v12_3_0 = QCz * v12_0_0 + WQz * v12_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v12_3_1 = QCz * v12_0_1 + WQz * v12_0_2 + (VT)1.0 * oo2ze * v4_0_2;
            const VT v13_3_0 = QCz * v13_0_0 + WQz * v13_0_1;
            const VT v13_3_1 = QCz * v13_0_1 + WQz * v13_0_2;
            const VT v14_3_0 = QCz * v14_0_0 + WQz * v14_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v14_3_1 = QCz * v14_0_1 + WQz * v14_0_2 + (VT)2.0 * oo2ze * v6_0_2;
            const VT v15_3_0 = QCz * v15_0_0 + WQz * v15_0_1 + (VT)1.0 * oo2ze * v5_0_1;
            const VT v15_3_1 = QCz * v15_0_1 + WQz * v15_0_2 + (VT)1.0 * oo2ze * v5_0_2;
            const VT v16_3_0 = QCz * v16_0_0 + WQz * v16_0_1;
            const VT v16_3_1 = QCz * v16_0_1 + WQz * v16_0_2;
            const VT v17_3_0 = QCz * v17_0_0 + WQz * v17_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v17_3_1 = QCz * v17_0_1 + WQz * v17_0_2 + (VT)1.0 * oo2ze * v7_0_2;
            const VT v18_3_0 = QCz * v18_0_0 + WQz * v18_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v18_3_1 = QCz * v18_0_1 + WQz * v18_0_2 + (VT)2.0 * oo2ze * v8_0_2;
            const VT v19_3_0 = QCz * v19_0_0 + WQz * v19_0_1 + (VT)3.0 * oo2ze * v9_0_1;
            const VT v19_3_1 = QCz * v19_0_1 + WQz * v19_0_2 + (VT)3.0 * oo2ze * v9_0_2;
            const VT v10_4_0 = QCx * v10_1_0 + WQx * v10_1_1 + (VT)3.0 * oo2ze * v4_1_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v11_4_0 = QCx * v11_1_0 + WQx * v11_1_1 + (VT)2.0 * oo2ze * v5_1_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v12_4_0 = QCx * v12_1_0 + WQx * v12_1_1 + (VT)2.0 * oo2ze * v6_1_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v13_4_0 = QCx * v13_1_0 + WQx * v13_1_1 + (VT)1.0 * oo2ze * v7_1_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v14_4_0 = QCx * v14_1_0 + WQx * v14_1_1 + (VT)1.0 * oo2ze * v9_1_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v15_4_0 = QCx * v15_1_0 + WQx * v15_1_1 + (VT)1.0 * oo2ze * v8_1_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v16_4_0 = QCx * v16_1_0 + WQx * v16_1_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v17_4_0 = QCx * v17_1_0 + WQx * v17_1_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v18_4_0 = QCx * v18_1_0 + WQx * v18_1_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v19_4_0 = QCx * v19_1_0 + WQx * v19_1_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v10_5_0 = QCx * v10_2_0 + WQx * v10_2_1 + (VT)3.0 * oo2ze * v4_2_1;
            const VT v11_5_0 = QCx * v11_2_0 + WQx * v11_2_1 + (VT)2.0 * oo2ze * v5_2_1;
            const VT v12_5_0 = QCx * v12_2_0 + WQx * v12_2_1 + (VT)2.0 * oo2ze * v6_2_1;
            const VT v13_5_0 = QCx * v13_2_0 + WQx * v13_2_1 + (VT)1.0 * oo2ze * v7_2_1;
            const VT v14_5_0 = QCx * v14_2_0 + WQx * v14_2_1 + (VT)1.0 * oo2ze * v9_2_1;
            const VT v15_5_0 = QCx * v15_2_0 + WQx * v15_2_1 + (VT)1.0 * oo2ze * v8_2_1;
            const VT v16_5_0 = QCx * v16_2_0 + WQx * v16_2_1;
            const VT v17_5_0 = QCx * v17_2_0 + WQx * v17_2_1;
            const VT v18_5_0 = QCx * v18_2_0 + WQx * v18_2_1;
            const VT v19_5_0 = QCx * v19_2_0 + WQx * v19_2_1;
            const VT v10_6_0 = QCx * v10_3_0 + WQx * v10_3_1 + (VT)3.0 * oo2ze * v4_3_1;
            const VT v11_6_0 = QCx * v11_3_0 + WQx * v11_3_1 + (VT)2.0 * oo2ze * v5_3_1;
            const VT v12_6_0 = QCx * v12_3_0 + WQx * v12_3_1 + (VT)2.0 * oo2ze * v6_3_1;
            const VT v13_6_0 = QCx * v13_3_0 + WQx * v13_3_1 + (VT)1.0 * oo2ze * v7_3_1;
            const VT v14_6_0 = QCx * v14_3_0 + WQx * v14_3_1 + (VT)1.0 * oo2ze * v9_3_1;
            const VT v15_6_0 = QCx * v15_3_0 + WQx * v15_3_1 + (VT)1.0 * oo2ze * v8_3_1;
            const VT v16_6_0 = QCx * v16_3_0 + WQx * v16_3_1;
            const VT v17_6_0 = QCx * v17_3_0 + WQx * v17_3_1;
            const VT v18_6_0 = QCx * v18_3_0 + WQx * v18_3_1;
            const VT v19_6_0 = QCx * v19_3_0 + WQx * v19_3_1;
            const VT v10_7_0 = QCy * v10_2_0 + WQy * v10_2_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v11_7_0 = QCy * v11_2_0 + WQy * v11_2_1 + (VT)1.0 * oo2ze * v4_2_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v12_7_0 = QCy * v12_2_0 + WQy * v12_2_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v13_7_0 = QCy * v13_2_0 + WQy * v13_2_1 + (VT)2.0 * oo2ze * v5_2_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v14_7_0 = QCy * v14_2_0 + WQy * v14_2_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v15_7_0 = QCy * v15_2_0 + WQy * v15_2_1 + (VT)1.0 * oo2ze * v6_2_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v16_7_0 = QCy * v16_2_0 + WQy * v16_2_1 + (VT)3.0 * oo2ze * v7_2_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v17_7_0 = QCy * v17_2_0 + WQy * v17_2_1 + (VT)2.0 * oo2ze * v8_2_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v18_7_0 = QCy * v18_2_0 + WQy * v18_2_1 + (VT)1.0 * oo2ze * v9_2_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v19_7_0 = QCy * v19_2_0 + WQy * v19_2_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v10_8_0 = QCy * v10_3_0 + WQy * v10_3_1;
            const VT v11_8_0 = QCy * v11_3_0 + WQy * v11_3_1 + (VT)1.0 * oo2ze * v4_3_1;
            const VT v12_8_0 = QCy * v12_3_0 + WQy * v12_3_1;
            const VT v13_8_0 = QCy * v13_3_0 + WQy * v13_3_1 + (VT)2.0 * oo2ze * v5_3_1;
            const VT v14_8_0 = QCy * v14_3_0 + WQy * v14_3_1;
            const VT v15_8_0 = QCy * v15_3_0 + WQy * v15_3_1 + (VT)1.0 * oo2ze * v6_3_1;
            const VT v16_8_0 = QCy * v16_3_0 + WQy * v16_3_1 + (VT)3.0 * oo2ze * v7_3_1;
            const VT v17_8_0 = QCy * v17_3_0 + WQy * v17_3_1 + (VT)2.0 * oo2ze * v8_3_1;
            const VT v18_8_0 = QCy * v18_3_0 + WQy * v18_3_1 + (VT)1.0 * oo2ze * v9_3_1;
            const VT v19_8_0 = QCy * v19_3_0 + WQy * v19_3_1;
            const VT v10_9_0 = QCz * v10_3_0 + WQz * v10_3_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v11_9_0 = QCz * v11_3_0 + WQz * v11_3_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v12_9_0 = QCz * v12_3_0 + WQz * v12_3_1 + (VT)1.0 * oo2ze * v4_3_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v13_9_0 = QCz * v13_3_0 + WQz * v13_3_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v14_9_0 = QCz * v14_3_0 + WQz * v14_3_1 + (VT)2.0 * oo2ze * v6_3_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v15_9_0 = QCz * v15_3_0 + WQz * v15_3_1 + (VT)1.0 * oo2ze * v5_3_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v16_9_0 = QCz * v16_3_0 + WQz * v16_3_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v17_9_0 = QCz * v17_3_0 + WQz * v17_3_1 + (VT)1.0 * oo2ze * v7_3_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v18_9_0 = QCz * v18_3_0 + WQz * v18_3_1 + (VT)2.0 * oo2ze * v8_3_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v19_9_0 = QCz * v19_3_0 + WQz * v19_3_1 + (VT)3.0 * oo2ze * v9_3_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            acc[0] += (double)v10_1_0;
            acc[1] += (double)v10_2_0;
            acc[2] += (double)v10_3_0;
            acc[3] += (double)v10_4_0;
            acc[4] += (double)v10_5_0;
            acc[5] += (double)v10_6_0;
            acc[6] += (double)v10_7_0;
            acc[7] += (double)v10_8_0;
            acc[8] += (double)v10_9_0;
            acc[9] += (double)v11_1_0;
            acc[10] += (double)v11_2_0;
            acc[11] += (double)v11_3_0;
            acc[12] += (double)v11_4_0;
            acc[13] += (double)v11_5_0;
            acc[14] += (double)v11_6_0;
            acc[15] += (double)v11_7_0;
            acc[16] += (double)v11_8_0;
            acc[17] += (double)v11_9_0;
            acc[18] += (double)v12_1_0;
            acc[19] += (double)v12_2_0;
            acc[20] += (double)v12_3_0;
            acc[21] += (double)v12_4_0;
            acc[22] += (double)v12_5_0;
            acc[23] += (double)v12_6_0;
            acc[24] += (double)v12_7_0;
            acc[25] += (double)v12_8_0;
            acc[26] += (double)v12_9_0;
            acc[27] += (double)v13_1_0;
            acc[28] += (double)v13_2_0;
            acc[29] += (double)v13_3_0;
            acc[30] += (double)v13_4_0;
            acc[31] += (double)v13_5_0;
            acc[32] += (double)v13_6_0;
            acc[33] += (double)v13_7_0;
            acc[34] += (double)v13_8_0;
            acc[35] += (double)v13_9_0;
            acc[36] += (double)v14_1_0;
            acc[37] += (double)v14_2_0;
            acc[38] += (double)v14_3_0;
            acc[39] += (double)v14_4_0;
            acc[40] += (double)v14_5_0;
            acc[41] += (double)v14_6_0;
            acc[42] += (double)v14_7_0;
            acc[43] += (double)v14_8_0;
            acc[44] += (double)v14_9_0;
            acc[45] += (double)v15_1_0;
            acc[46] += (double)v15_2_0;
            acc[47] += (double)v15_3_0;
            acc[48] += (double)v15_4_0;
            acc[49] += (double)v15_5_0;
            acc[50] += (double)v15_6_0;
            acc[51] += (double)v15_7_0;
            acc[52] += (double)v15_8_0;
            acc[53] += (double)v15_9_0;
            acc[54] += (double)v16_1_0;
            acc[55] += (double)v16_2_0;
            acc[56] += (double)v16_3_0;
            acc[57] += (double)v16_4_0;
            acc[58] += (double)v16_5_0;
            acc[59] += (double)v16_6_0;
            acc[60] += (double)v16_7_0;
            acc[61] += (double)v16_8_0;
            acc[62] += (double)v16_9_0;
            acc[63] += (double)v17_1_0;
            acc[64] += (double)v17_2_0;
            acc[65] += (double)v17_3_0;
            acc[66] += (double)v17_4_0;
            acc[67] += (double)v17_5_0;
            acc[68] += (double)v17_6_0;
            acc[69] += (double)v17_7_0;
            acc[70] += (double)v17_8_0;
            acc[71] += (double)v17_9_0;
            acc[72] += (double)v18_1_0;
            acc[73] += (double)v18_2_0;
            acc[74] += (double)v18_3_0;
            acc[75] += (double)v18_4_0;
            acc[76] += (double)v18_5_0;
            acc[77] += (double)v18_6_0;
            acc[78] += (double)v18_7_0;
            acc[79] += (double)v18_8_0;
            acc[80] += (double)v18_9_0;
            acc[81] += (double)v19_1_0;
            acc[82] += (double)v19_2_0;
            acc[83] += (double)v19_3_0;
            acc[84] += (double)v19_4_0;
            acc[85] += (double)v19_5_0;
            acc[86] += (double)v19_6_0;
            acc[87] += (double)v19_7_0;
            acc[88] += (double)v19_8_0;
            acc[89] += (double)v19_9_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[90] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_fspp(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double k10_0_1_1 = acc[3] + CDx * acc[0];
    const double k10_0_1_2 = acc[4] + CDy * acc[0];
    const double k10_0_1_3 = acc[5] + CDz * acc[0];
    const double k10_0_2_1 = acc[4] + CDx * acc[1];
    const double k10_0_2_2 = acc[6] + CDy * acc[1];
    const double k10_0_2_3 = acc[7] + CDz * acc[1];
    const double k10_0_3_1 = acc[5] + CDx * acc[2];
    const double k10_0_3_2 = acc[7] + CDy * acc[2];
    const double k10_0_3_3 = acc[8] + CDz * acc[2];
    const double k11_0_1_1 = acc[12] + CDx * acc[9];
    const double k11_0_1_2 = acc[13] + CDy * acc[9];
    const double k11_0_1_3 = acc[14] + CDz * acc[9];
    const double k11_0_2_1 = acc[13] + CDx * acc[10];
    const double k11_0_2_2 = acc[15] + CDy * acc[10];
    const double k11_0_2_3 = acc[16] + CDz * acc[10];
    const double k11_0_3_1 = acc[14] + CDx * acc[11];
    const double k11_0_3_2 = acc[16] + CDy * acc[11];
    const double k11_0_3_3 = acc[17] + CDz * acc[11];
    const double k12_0_1_1 = acc[21] + CDx * acc[18];
    const double k12_0_1_2 = acc[22] + CDy * acc[18];
    const double k12_0_1_3 = acc[23] + CDz * acc[18];
    const double k12_0_2_1 = acc[22] + CDx * acc[19];
    const double k12_0_2_2 = acc[24] + CDy * acc[19];
    const double k12_0_2_3 = acc[25] + CDz * acc[19];
    const double k12_0_3_1 = acc[23] + CDx * acc[20];
    const double k12_0_3_2 = acc[25] + CDy * acc[20];
    const double k12_0_3_3 = acc[26] + CDz * acc[20];
    const double k13_0_1_1 = acc[30] + CDx * acc[27];
    const double k13_0_1_2 = acc[31] + CDy * acc[27];
    const double k13_0_1_3 = acc[32] + CDz * acc[27];
    const double k13_0_2_1 = acc[31] + CDx * acc[28];
    const double k13_0_2_2 = acc[33] + CDy * acc[28];
    const double k13_0_2_3 = acc[34] + CDz * acc[28];
    const double k13_0_3_1 = acc[32] + CDx * acc[29];
    const double k13_0_3_2 = acc[34] + CDy * acc[29];
    const double k13_0_3_3 = acc[35] + CDz * acc[29];
    const double k14_0_1_1 = acc[39] + CDx * acc[36];
    const double k14_0_1_2 = acc[40] + CDy * acc[36];
    const double k14_0_1_3 = acc[41] + CDz * acc[36];
    const double k14_0_2_1 = acc[40] + CDx * acc[37];
    const double k14_0_2_2 = acc[42] + CDy * acc[37];
    const double k14_0_2_3 = acc[43] + CDz * acc[37];
    const double k14_0_3_1 = acc[41] + CDx * acc[38];
    const double k14_0_3_2 = acc[43] + CDy * acc[38];
    const double k14_0_3_3 = acc[44] + CDz * acc[38];
    const double k15_0_1_1 = acc[48] + CDx * acc[45];
    const double k15_0_1_2 = acc[49] + CDy * acc[45];
    const double k15_0_1_3 = acc[50] + CDz * acc[45];
    const double k15_0_2_1 = acc[49] + CDx * acc[46];
    const double k15_0_2_2 = acc[51] + CDy * acc[46];
    const double k15_0_2_3 = acc[52] + CDz * acc[46];
    const double k15_0_3_1 = acc[50] + CDx * acc[47];
    const double k15_0_3_2 = acc[52] + CDy * acc[47];
    const double k15_0_3_3 = acc[53] + CDz * acc[47];
    const double k16_0_1_1 = acc[57] + CDx * acc[54];
    const double k16_0_1_2 = acc[58] + CDy * acc[54];
    const double k16_0_1_3 = acc[59] + CDz * acc[54];
    const double k16_0_2_1 = acc[58] + CDx * acc[55];
    const double k16_0_2_2 = acc[60] + CDy * acc[55];
    const double k16_0_2_3 = acc[61] + CDz * acc[55];
    const double k16_0_3_1 = acc[59] + CDx * acc[56];
    const double k16_0_3_2 = acc[61] + CDy * acc[56];
    const double k16_0_3_3 = acc[62] + CDz * acc[56];
    const double k17_0_1_1 = acc[66] + CDx * acc[63];
    const double k17_0_1_2 = acc[67] + CDy * acc[63];
    const double k17_0_1_3 = acc[68] + CDz * acc[63];
    const double k17_0_2_1 = acc[67] + CDx * acc[64];
    const double k17_0_2_2 = acc[69] + CDy * acc[64];
    const double k17_0_2_3 = acc[70] + CDz * acc[64];
    const double k17_0_3_1 = acc[68] + CDx * acc[65];
    const double k17_0_3_2 = acc[70] + CDy * acc[65];
    const double k17_0_3_3 = acc[71] + CDz * acc[65];
    const double k18_0_1_1 = acc[75] + CDx * acc[72];
    const double k18_0_1_2 = acc[76] + CDy * acc[72];
    const double k18_0_1_3 = acc[77] + CDz * acc[72];
    const double k18_0_2_1 = acc[76] + CDx * acc[73];
    const double k18_0_2_2 = acc[78] + CDy * acc[73];
    const double k18_0_2_3 = acc[79] + CDz * acc[73];
    const double k18_0_3_1 = acc[77] + CDx * acc[74];
    const double k18_0_3_2 = acc[79] + CDy * acc[74];
    const double k18_0_3_3 = acc[80] + CDz * acc[74];
    const double k19_0_1_1 = acc[84] + CDx * acc[81];
    const double k19_0_1_2 = acc[85] + CDy * acc[81];
    const double k19_0_1_3 = acc[86] + CDz * acc[81];
    const double k19_0_2_1 = acc[85] + CDx * acc[82];
    const double k19_0_2_2 = acc[87] + CDy * acc[82];
    const double k19_0_2_3 = acc[88] + CDz * acc[82];
    const double k19_0_3_1 = acc[86] + CDx * acc[83];
    const double k19_0_3_2 = acc[88] + CDy * acc[83];
    const double k19_0_3_3 = acc[89] + CDz * acc[83];
    res[0] = k10_0_1_1 * 0.2581988897471611;
    res[1] = k10_0_1_2 * 0.2581988897471611;
    res[2] = k10_0_1_3 * 0.2581988897471611;
    res[3] = k10_0_2_1 * 0.2581988897471611;
    res[4] = k10_0_2_2 * 0.2581988897471611;
    res[5] = k10_0_2_3 * 0.2581988897471611;
    res[6] = k10_0_3_1 * 0.2581988897471611;
    res[7] = k10_0_3_2 * 0.2581988897471611;
    res[8] = k10_0_3_3 * 0.2581988897471611;
    res[9] = k11_0_1_1 * 0.5773502691896258;
    res[10] = k11_0_1_2 * 0.5773502691896258;
    res[11] = k11_0_1_3 * 0.5773502691896258;
    res[12] = k11_0_2_1 * 0.5773502691896258;
    res[13] = k11_0_2_2 * 0.5773502691896258;
    res[14] = k11_0_2_3 * 0.5773502691896258;
    res[15] = k11_0_3_1 * 0.5773502691896258;
    res[16] = k11_0_3_2 * 0.5773502691896258;
    res[17] = k11_0_3_3 * 0.5773502691896258;
    res[18] = k12_0_1_1 * 0.5773502691896258;
    res[19] = k12_0_1_2 * 0.5773502691896258;
    res[20] = k12_0_1_3 * 0.5773502691896258;
    res[21] = k12_0_2_1 * 0.5773502691896258;
    res[22] = k12_0_2_2 * 0.5773502691896258;
    res[23] = k12_0_2_3 * 0.5773502691896258;
    res[24] = k12_0_3_1 * 0.5773502691896258;
    res[25] = k12_0_3_2 * 0.5773502691896258;
    res[26] = k12_0_3_3 * 0.5773502691896258;
    res[27] = k13_0_1_1 * 0.5773502691896258;
    res[28] = k13_0_1_2 * 0.5773502691896258;
    res[29] = k13_0_1_3 * 0.5773502691896258;
    res[30] = k13_0_2_1 * 0.5773502691896258;
    res[31] = k13_0_2_2 * 0.5773502691896258;
    res[32] = k13_0_2_3 * 0.5773502691896258;
    res[33] = k13_0_3_1 * 0.5773502691896258;
    res[34] = k13_0_3_2 * 0.5773502691896258;
    res[35] = k13_0_3_3 * 0.5773502691896258;
    res[36] = k14_0_1_1 * 0.5773502691896258;
    res[37] = k14_0_1_2 * 0.5773502691896258;
    res[38] = k14_0_1_3 * 0.5773502691896258;
    res[39] = k14_0_2_1 * 0.5773502691896258;
    res[40] = k14_0_2_2 * 0.5773502691896258;
    res[41] = k14_0_2_3 * 0.5773502691896258;
    res[42] = k14_0_3_1 * 0.5773502691896258;
    res[43] = k14_0_3_2 * 0.5773502691896258;
    res[44] = k14_0_3_3 * 0.5773502691896258;
    res[45] = k15_0_1_1;
    res[46] = k15_0_1_2;
    res[47] = k15_0_1_3;
    res[48] = k15_0_2_1;
    res[49] = k15_0_2_2;
    res[50] = k15_0_2_3;
    res[51] = k15_0_3_1;
    res[52] = k15_0_3_2;
    res[53] = k15_0_3_3;
    res[54] = k16_0_1_1 * 0.2581988897471611;
    res[55] = k16_0_1_2 * 0.2581988897471611;
    res[56] = k16_0_1_3 * 0.2581988897471611;
    res[57] = k16_0_2_1 * 0.2581988897471611;
    res[58] = k16_0_2_2 * 0.2581988897471611;
    res[59] = k16_0_2_3 * 0.2581988897471611;
    res[60] = k16_0_3_1 * 0.2581988897471611;
    res[61] = k16_0_3_2 * 0.2581988897471611;
    res[62] = k16_0_3_3 * 0.2581988897471611;
    res[63] = k17_0_1_1 * 0.5773502691896258;
    res[64] = k17_0_1_2 * 0.5773502691896258;
    res[65] = k17_0_1_3 * 0.5773502691896258;
    res[66] = k17_0_2_1 * 0.5773502691896258;
    res[67] = k17_0_2_2 * 0.5773502691896258;
    res[68] = k17_0_2_3 * 0.5773502691896258;
    res[69] = k17_0_3_1 * 0.5773502691896258;
    res[70] = k17_0_3_2 * 0.5773502691896258;
    res[71] = k17_0_3_3 * 0.5773502691896258;
    res[72] = k18_0_1_1 * 0.5773502691896258;
    res[73] = k18_0_1_2 * 0.5773502691896258;
    res[74] = k18_0_1_3 * 0.5773502691896258;
    res[75] = k18_0_2_1 * 0.5773502691896258;
    res[76] = k18_0_2_2 * 0.5773502691896258;
    res[77] = k18_0_2_3 * 0.5773502691896258;
    res[78] = k18_0_3_1 * 0.5773502691896258;
    res[79] = k18_0_3_2 * 0.5773502691896258;
    res[80] = k18_0_3_3 * 0.5773502691896258;
    res[81] = k19_0_1_1 * 0.2581988897471611;
    res[82] = k19_0_1_2 * 0.2581988897471611;
    res[83] = k19_0_1_3 * 0.2581988897471611;
    res[84] = k19_0_2_1 * 0.2581988897471611;
    res[85] = k19_0_2_2 * 0.2581988897471611;
    res[86] = k19_0_2_3 * 0.2581988897471611;
    res[87] = k19_0_3_1 * 0.2581988897471611;
    res[88] = k19_0_3_2 * 0.2581988897471611;
    res[89] = k19_0_3_3 * 0.2581988897471611;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[90]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_fspp(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[90];
    vrr_fspp<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 90; ++x) acc_out[x] = acc[x];
    }
    hrr_fspp(P, p, q, acc, res);
}

__device__ __forceinline__ void store_fspp(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
    const long long kl_0_1 = pair_index(ik_.z + 0, ik_.w + 1);
    const long long kl_0_2 = pair_index(ik_.z + 0, ik_.w + 2);
    const long long kl_1_0 = pair_index(ik_.z + 1, ik_.w + 0);
    const long long kl_1_1 = pair_index(ik_.z + 1, ik_.w + 1);
    const long long kl_1_2 = pair_index(ik_.z + 1, ik_.w + 2);
    const long long kl_2_0 = pair_index(ik_.z + 2, ik_.w + 0);
    const long long kl_2_1 = pair_index(ik_.z + 2, ik_.w + 1);
    const long long kl_2_2 = pair_index(ik_.z + 2, ik_.w + 2);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_1_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_1_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_1_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_1_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_1_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_1_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_2_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_2_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_2_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_2_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_2_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_2_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_3_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_3_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_3_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_3_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_3_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_3_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_4_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_4_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_4_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_4_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_4_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_4_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_5_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_5_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_5_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_5_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_5_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_5_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_6_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_6_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_6_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_6_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_6_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_6_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_6_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_6_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_7_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_7_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_7_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_7_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_7_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_7_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_7_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_7_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_8_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_8_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_8_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_8_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_8_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_8_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_8_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_8_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_9_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_9_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_9_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_9_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_9_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_9_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_9_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_9_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_fspp(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 90; ++x) {
        const int ia = x / 9, ibb = (x / 9) % 1, ic = (x / 3) % 3, id = x % 3;
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
__global__ void __launch_bounds__(128) eri_queue_fspp(const EriQueue Q) {
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
        double acc[90];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 90; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_fspp<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_fspp<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 90; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 90 doubles (launch_eri_fspp)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 90);
            if (lead) hrr_fspp(Q.pairs, p, q, acc, sb + kq * 90);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)90;
            for (int t = lane; t < nlive * 90; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[90];
            hrr_fspp(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_fspp(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_fspp(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (92160 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_fspp() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_fspp<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 92160);
        cudaFuncSetAttribute(eri_queue_fspp<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 92160);
        done[dev] = true;
    }
}

void launch_eri_fspp(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 92160 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 92160 : 0;
    if (smem) eri_prepare_fspp();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_fspp<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_fspp<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_fspp<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_fspp<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_fspp(int mixed) {
    eri_prepare_fspp();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fspp<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fspp<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

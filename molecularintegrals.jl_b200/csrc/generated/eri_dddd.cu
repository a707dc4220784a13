// Generated by gen_eri.py -- class (dd|dd).  Do not edit.
// VRR entries: 2330, contracted block: 961, HRR lines: 5293, outputs: 1296.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[961], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_dddd(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 961; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[9];
            boys_fm<8>(T, B, F);
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
            const VT v0_0_7 = (VT)(pref * F[7]);
            const VT v0_0_8 = (VT)(pref * F[8]);
            const VT v1_0_0 = PAx * v0_0_0 + WPx * v0_0_1;
            const VT v1_0_1 = PAx * v0_0_1 + WPx * v0_0_2;
            const VT v1_0_2 = PAx * v0_0_2 + WPx * v0_0_3;
            const VT v1_0_3 = PAx * v0_0_3 + WPx * v0_0_4;
            const VT v1_0_4 = PAx * v0_0_4 + WPx * v0_0_5;
            const VT v1_0_5 = PAx * v0_0_5 + WPx * v0_0_6;
            const VT v1_0_6 = PAx * v0_0_6 + WPx * v0_0_7;
            const VT v1_0_7 = PAx * v0_0_7 + WPx * v0_0_8;
            const VT v2_0_0 = PAy * v0_0_0 + WPy * v0_0_1;
            const VT v2_0_1 = PAy * v0_0_1 + WPy * v0_0_2;
            const VT v2_0_2 = PAy * v0_0_2 + WPy * v0_0_3;
            const VT v2_0_3 = PAy * v0_0_3 + WPy * v0_0_4;
            const VT v2_0_4 = PAy * v0_0_4 + WPy * v0_0_5;
            const VT v2_0_5 = PAy * v0_0_5 + WPy * v0_0_6;
            const VT v2_0_6 = PAy * v0_0_6 + WPy * v0_0_7;
            const VT v2_0_7 = PAy * v0_0_7 + WPy * v0_0_8;
            const VT v3_0_0 = PAz * v0_0_0 + WPz * v0_0_1;
            const VT v3_0_1 = PAz * v0_0_1 + WPz * v0_0_2;
            const VT v3_0_2 = PAz * v0_0_2 + WPz * v0_0_3;
            const VT v3_0_3 = PAz * v0_0_3 + WPz * v0_0_4;
            const VT v3_0_4 = PAz * v0_0_4 + WPz * v0_0_5;
            const VT v3_0_5 = PAz * v0_0_5 + WPz * v0_0_6;
            const VT v3_0_6 = PAz * v0_0_6 + WPz * v0_0_7;
            const VT v3_0_7 = PAz * v0_0_7 + WPz * v0_0_8;
            const VT v4_0_0 = PAx * v1_0_0 + WPx * v1_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v4_0_1 = PAx * v1_0_1 + WPx * v1_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v4_0_2 = PAx * v1_0_2 + WPx * v1_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v4_0_3 = PAx * v1_0_3 + WPx * v1_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v4_0_4 = PAx * v1_0_4 + WPx * v1_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v4_0_5 = PAx * v1_0_5 + WPx * v1_0_6 + (VT)1.0 * oo2z * (v0_0_5 - rho_z * v0_0_6);
            const VT v4_0_6 = PAx * v1_0_6 + WPx * v1_0_7 + (VT)1.0 * oo2z * (v0_0_6 - rho_z * v0_0_7);
            const VT v5_0_0 = PAx * v2_0_0 + WPx * v2_0_1;
            const VT v5_0_1 = PAx * v2_0_1 + WPx * v2_0_2;
            const VT v5_0_2 = PAx * v2_0_2 + WPx * v2_0_3;
            const VT v5_0_3 = PAx * v2_0_3 + WPx * v2_0_4;
            const VT v5_0_4 = PAx * v2_0_4 + WPx * v2_0_5;
            const VT v5_0_5 = PAx * v2_0_5 + WPx * v2_0_6;
            const VT v5_0_6 = PAx * v2_0_6 + WPx * v2_0_7;
            const VT v6_0_0 = PAx * v3_0_0 + WPx * v3_0_1;
            const VT v6_0_1 = PAx * v3_0_1 + WPx * v3_0_2;
            const VT v6_0_2 = PAx * v3_0_2 + WPx * v3_0_3;
            const VT v6_0_3 = PAx * v3_0_3 + WPx * v3_0_4;
            const VT v6_0_4 = PAx * v3_0_4 + WPx * v3_0_5;
            const VT v6_0_5 = PAx * v3_0_5 + WPx * v3_0_6;
            const VT v6_0_6 = PAx * v3_0_6 + WPx * v3_0_7;
            const VT v7_0_0 = PAy * v2_0_0 + WPy * v2_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v7_0_1 = PAy * v2_0_1 + WPy * v2_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v7_0_2 = PAy * v2_0_2 + WPy * v2_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v7_0_3 = PAy * v2_0_3 + WPy * v2_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v7_0_4 = PAy * v2_0_4 + WPy * v2_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v7_0_5 = PAy * v2_0_5 + WPy * v2_0_6 + (VT)1.0 * oo2z * (v0_0_5 - rho_z * v0_0_6);
            const VT v7_0_6 = PAy * v2_0_6 + WPy * v2_0_7 + (VT)1.0 * oo2z * (v0_0_6 - rho_z * v0_0_7);
            const VT v8_0_0 = PAy * v3_0_0 + WPy * v3_0_1;
            const VT v8_0_1 = PAy * v3_0_1 + WPy * v3_0_2;
            const VT v8_0_2 = PAy * v3_0_2 + WPy * v3_0_3;
            const VT v8_0_3 = PAy * v3_0_3 + WPy * v3_0_4;
            const VT v8_0_4 = PAy * v3_0_4 + WPy * v3_0_5;
            const VT v8_0_5 = PAy * v3_0_5 + WPy * v3_0_6;
            const VT v8_0_6 = PAy * v3_0_6 + WPy * v3_0_7;
            const VT v9_0_0 = PAz * v3_0_0 + WPz * v3_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v9_0_1 = PAz * v3_0_1 + WPz * v3_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v9_0_2 = PAz * v3_0_2 + WPz * v3_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v9_0_3 = PAz * v3_0_3 + WPz * v3_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v9_0_4 = PAz * v3_0_4 + WPz * v3_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v9_0_5 = PAz * v3_0_5 + WPz * v3_0_6 + (VT)1.0 * oo2z * (v0_0_5 - rho_z * v0_0_6);
            const VT v9_0_6 = PAz * v3_0_6 + WPz * v3_0_7 + (VT)1.0 * oo2z * (v0_0_6 - rho_z * v0_0_7);
            const VT v10_0_0 = PAx * v4_0_0 + WPx * v4_0_1 + (VT)2.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v10_0_1 = PAx * v4_0_1 + WPx * v4_0_2 + (VT)2.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v10_0_2 = PAx * v4_0_2 + WPx * v4_0_3 + (VT)2.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v10_0_3 = PAx * v4_0_3 + WPx * v4_0_4 + (VT)2.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v10_0_4 = PAx * v4_0_4 + WPx * v4_0_5 + (VT)2.0 * oo2z * (v1_0_4 - rho_z * v1_0_5);
            const VT v10_0_5 = PAx * v4_0_5 + WPx * v4_0_6 + (VT)2.0 * oo2z * (v1_0_5 - rho_z * v1_0_6);
            const VT v11_0_0 = PAx * v5_0_0 + WPx * v5_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v11_0_1 = PAx * v5_0_1 + WPx * v5_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v11_0_2 = PAx * v5_0_2 + WPx * v5_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v11_0_3 = PAx * v5_0_3 + WPx * v5_0_4 + (VT)1.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v11_0_4 = PAx * v5_0_4 + WPx * v5_0_5 + (VT)1.0 * oo2z * (v2_0_4 - rho_z * v2_0_5);
            const VT v11_0_5 = PAx * v5_0_5 + WPx * v5_0_6 + (VT)1.0 * oo2z * (v2_0_5 - rho_z * v2_0_6);
            const VT v12_0_0 = PAx * v6_0_0 + WPx * v6_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v12_0_1 = PAx * v6_0_1 + WPx * v6_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v12_0_2 = PAx * v6_0_2 + WPx * v6_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v12_0_3 = PAx * v6_0_3 + WPx * v6_0_4 + (VT)1.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v12_0_4 = PAx * v6_0_4 + WPx * v6_0_5 + (VT)1.0 * oo2z * (v3_0_4 - rho_z * v3_0_5);
            const VT v12_0_5 = PAx * v6_0_5 + WPx * v6_0_6 + (VT)1.0 * oo2z * (v3_0_5 - rho_z * v3_0_6);
            const VT v13_0_0 = PAy * v5_0_0 + WPy * v5_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v13_0_1 = PAy * v5_0_1 + WPy * v5_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v13_0_2 = PAy * v5_0_2 + WPy * v5_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v13_0_3 = PAy * v5_0_3 + WPy * v5_0_4 + (VT)1.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v13_0_4 = PAy * v5_0_4 + WPy * v5_0_5 + (VT)1.0 * oo2z * (v1_0_4 - rho_z * v1_0_5);
            const VT v13_0_5 = PAy * v5_0_5 + WPy * v5_0_6 + (VT)1.0 * oo2z * (v1_0_5 - rho_z * v1_0_6);
            const VT v14_0_0 = PAz * v6_0_0 + WPz * v6_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v14_0_1 = PAz * v6_0_1 + WPz * v6_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v14_0_2 = PAz * v6_0_2 + WPz * v6_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v14_0_3 = PAz * v6_0_3 + WPz * v6_0_4 + (VT)1.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v14_0_4 = PAz * v6_0_4 + WPz * v6_0_5 + (VT)1.0 * oo2z * (v1_0_4 - rho_z * v1_0_5);
            const VT v14_0_5 = PAz * v6_0_5 + WPz * v6_0_6 + (VT)1.0 * oo2z * (v1_0_5 - rho_z * v1_0_6);
            const VT v15_0_0 = PAx * v8_0_0 + WPx * v8_0_1;
            const VT v15_0_1 = PAx * v8_0_1 + WPx * v8_0_2;
            const VT v15_0_2 = PAx * v8_0_2 + WPx * v8_0_3;
            const VT v15_0_3 = PAx * v8_0_3 + WPx * v8_0_4;
            const VT v15_0_4 = PAx * v8_0_4 + WPx * v8_0_5;
            const VT v15_0_5 = PAx * v8_0_5 + WPx * v8_0_6;
            const VT v16_0_0 = PAy * v7_0_0 + WPy * v7_0_1 + (VT)2.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v16_0_1 = PAy * v7_0_1 + WPy * v7_0_2 + (VT)2.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v16_0_2 = PAy * v7_0_2 + WPy * v7_0_3 + (VT)2.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v16_0_3 = PAy * v7_0_3 + WPy * v7_0_4 + (VT)2.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v16_0_4 = PAy * v7_0_4 + WPy * v7_0_5 + (VT)2.0 * oo2z * (v2_0_4 - rho_z * v2_0_5);
            const VT v16_0_5 = PAy * v7_0_5 + WPy * v7_0_6 + (VT)2.0 * oo2z * (v2_0_5 - rho_z * v2_0_6);
            const VT v17_0_0 = PAy * v8_0_0 + WPy * v8_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v17_0_1 = PAy * v8_0_1 + WPy * v8_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v17_0_2 = PAy * v8_0_2 + WPy * v8_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v17_0_3 = PAy * v8_0_3 + WPy * v8_0_4 + (VT)1.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v17_0_4 = PAy * v8_0_4 + WPy * v8_0_5 + (VT)1.0 * oo2z * (v3_0_4 - rho_z * v3_0_5);
            const VT v17_0_5 = PAy * v8_0_5 + WPy * v8_0_6 + (VT)1.0 * oo2z * (v3_0_5 - rho_z * v3_0_6);
            const VT v18_0_0 = PAz * v8_0_0 + WPz * v8_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v18_0_1 = PAz * v8_0_1 + WPz * v8_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v18_0_2 = PAz * v8_0_2 + WPz * v8_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v18_0_3 = PAz * v8_0_3 + WPz * v8_0_4 + (VT)1.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v18_0_4 = PAz * v8_0_4 + WPz * v8_0_5 + (VT)1.0 * oo2z * (v2_0_4 - rho_z * v2_0_5);
            const VT v18_0_5 = PAz * v8_0_5 + WPz * v8_0_6 + (VT)1.0 * oo2z * (v2_0_5 - rho_z * v2_0_6);
            const VT v19_0_0 = PAz * v9_0_0 + WPz * v9_0_1 + (VT)2.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v19_0_1 = PAz * v9_0_1 + WPz * v9_0_2 + (VT)2.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v19_0_2 = PAz * v9_0_2 + WPz * v9_0_3 + (VT)2.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v19_0_3 = PAz * v9_0_3 + WPz * v9_0_4 + (VT)2.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v19_0_4 = PAz * v9_0_4 + WPz * v9_0_5 + (VT)2.0 * oo2z * (v3_0_4 - rho_z * v3_0_5);
            const VT v19_0_5 = PAz * v9_0_5 + WPz * v9_0_6 + (VT)2.0 * oo2z * (v3_0_5 - rho_z * v3_0_6);
            const VT v20_0_0 = PAx * v10_0_0 + WPx * v10_0_1 + (VT)3.0 * oo2z * (v4_0_0 - rho_z * v4_0_1);
            const VT v20_0_1 = PAx * v10_0_1 + WPx * v10_0_2 + (VT)3.0 * oo2z * (v4_0_1 - rho_z * v4_0_2);
            const VT v20_0_2 = PAx * v10_0_2 + WPx * v10_0_3 + (VT)3.0 * oo2z * (v4_0_2 - rho_z * v4_0_3);
            const VT v20_0_3 = PAx * v10_0_3 + WPx * v10_0_4 + (VT)3.0 * oo2z * (v4_0_3 - rho_z * v4_0_4);
            const VT v20_0_4 = PAx * v10_0_4 + WPx * v10_0_5 + (VT)3.0 * oo2z * (v4_0_4 - rho_z * v4_0_5);
            const VT v21_0_0 = PAx * v11_0_0 + WPx * v11_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v21_0_1 = PAx * v11_0_1 + WPx * v11_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v21_0_2 = PAx * v11_0_2 + WPx * v11_0_3 + (VT)2.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v21_0_3 = PAx * v11_0_3 + WPx * v11_0_4 + (VT)2.0 * oo2z * (v5_0_3 - rho_z * v5_0_4);
            const VT v21_0_4 = PAx * v11_0_4 + WPx * v11_0_5 + (VT)2.0 * oo2z * (v5_0_4 - rho_z * v5_0_5);
            const VT v22_0_0 = PAx * v12_0_0 + WPx * v12_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v22_0_1 = PAx * v12_0_1 + WPx * v12_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v22_0_2 = PAx * v12_0_2 + WPx * v12_0_3 + (VT)2.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v22_0_3 = PAx * v12_0_3 + WPx * v12_0_4 + (VT)2.0 * oo2z * (v6_0_3 - rho_z * v6_0_4);
            const VT v22_0_4 = PAx * v12_0_4 + WPx * v12_0_5 + (VT)2.0 * oo2z * (v6_0_4 - rho_z * v6_0_5);
            const VT v23_0_0 = PAx * v13_0_0 + WPx * v13_0_1 + (VT)1.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v23_0_1 = PAx * v13_0_1 + WPx * v13_0_2 + (VT)1.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v23_0_2 = PAx * v13_0_2 + WPx * v13_0_3 + (VT)1.0 * oo2z * (v7_0_2 - rho_z * v7_0_3);
            const VT v23_0_3 = PAx * v13_0_3 + WPx * v13_0_4 + (VT)1.0 * oo2z * (v7_0_3 - rho_z * v7_0_4);
            const VT v23_0_4 = PAx * v13_0_4 + WPx * v13_0_5 + (VT)1.0 * oo2z * (v7_0_4 - rho_z * v7_0_5);
            const VT v24_0_0 = PAx * v15_0_0 + WPx * v15_0_1 + (VT)1.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v24_0_1 = PAx * v15_0_1 + WPx * v15_0_2 + (VT)1.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v24_0_2 = PAx * v15_0_2 + WPx * v15_0_3 + (VT)1.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v24_0_3 = PAx * v15_0_3 + WPx * v15_0_4 + (VT)1.0 * oo2z * (v8_0_3 - rho_z * v8_0_4);
            const VT v24_0_4 = PAx * v15_0_4 + WPx * v15_0_5 + (VT)1.0 * oo2z * (v8_0_4 - rho_z * v8_0_5);
            const VT v25_0_0 = PAx * v14_0_0 + WPx * v14_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v25_0_1 = PAx * v14_0_1 + WPx * v14_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v25_0_2 = PAx * v14_0_2 + WPx * v14_0_3 + (VT)1.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v25_0_3 = PAx * v14_0_3 + WPx * v14_0_4 + (VT)1.0 * oo2z * (v9_0_3 - rho_z * v9_0_4);
            const VT v25_0_4 = PAx * v14_0_4 + WPx * v14_0_5 + (VT)1.0 * oo2z * (v9_0_4 - rho_z * v9_0_5);
            const VT v26_0_0 = PAy * v13_0_0 + WPy * v13_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v26_0_1 = PAy * v13_0_1 + WPy * v13_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v26_0_2 = PAy * v13_0_2 + WPy * v13_0_3 + (VT)2.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v26_0_3 = PAy * v13_0_3 + WPy * v13_0_4 + (VT)2.0 * oo2z * (v5_0_3 - rho_z * v5_0_4);
            const VT v26_0_4 = PAy * v13_0_4 + WPy * v13_0_5 + (VT)2.0 * oo2z * (v5_0_4 - rho_z * v5_0_5);
            const VT v27_0_0 = PAy * v15_0_0 + WPy * v15_0_1 + (VT)1.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v27_0_1 = PAy * v15_0_1 + WPy * v15_0_2 + (VT)1.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v27_0_2 = PAy * v15_0_2 + WPy * v15_0_3 + (VT)1.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v27_0_3 = PAy * v15_0_3 + WPy * v15_0_4 + (VT)1.0 * oo2z * (v6_0_3 - rho_z * v6_0_4);
            const VT v27_0_4 = PAy * v15_0_4 + WPy * v15_0_5 + (VT)1.0 * oo2z * (v6_0_4 - rho_z * v6_0_5);
            const VT v28_0_0 = PAz * v15_0_0 + WPz * v15_0_1 + (VT)1.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v28_0_1 = PAz * v15_0_1 + WPz * v15_0_2 + (VT)1.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v28_0_2 = PAz * v15_0_2 + WPz * v15_0_3 + (VT)1.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v28_0_3 = PAz * v15_0_3 + WPz * v15_0_4 + (VT)1.0 * oo2z * (v5_0_3 - rho_z * v5_0_4);
            const VT v28_0_4 = PAz * v15_0_4 + WPz * v15_0_5 + (VT)1.0 * oo2z * (v5_0_4 - rho_z * v5_0_5);
            const VT v29_0_0 = PAz * v14_0_0 + WPz * v14_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v29_0_1 = PAz * v14_0_1 + WPz * v14_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v29_0_2 = PAz * v14_0_2 + WPz * v14_0_3 + (VT)2.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v29_0_3 = PAz * v14_0_3 + WPz * v14_0_4 + (VT)2.0 * oo2z * (v6_0_3 - rho_z * v6_0_4);
            const VT v29_0_4 = PAz * v14_0_4 + WPz * v14_0_5 + (VT)2.0 * oo2z * (v6_0_4 - rho_z * v6_0_5);
            const VT v30_0_0 = PAy * v16_0_0 + WPy * v16_0_1 + (VT)3.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v30_0_1 = PAy * v16_0_1 + WPy * v16_0_2 + (VT)3.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v30_0_2 = PAy * v16_0_2 + WPy * v16_0_3 + (VT)3.0 * oo2z * (v7_0_2 - rho_z * v7_0_3);
            const VT v30_0_3 = PAy * v16_0_3 + WPy * v16_0_4 + (VT)3.0 * oo2z * (v7_0_3 - rho_z * v7_0_4);
            const VT v30_0_4 = PAy * v16_0_4 + WPy * v16_0_5 + (VT)3.0 * oo2z * (v7_0_4 - rho_z * v7_0_5);
            const VT v31_0_0 = PAy * v17_0_0 + WPy * v17_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v31_0_1 = PAy * v17_0_1 + WPy * v17_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v31_0_2 = PAy * v17_0_2 + WPy * v17_0_3 + (VT)2.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v31_0_3 = PAy * v17_0_3 + WPy * v17_0_4 + (VT)2.0 * oo2z * (v8_0_3 - rho_z * v8_0_4);
            const VT v31_0_4 = PAy * v17_0_4 + WPy * v17_0_5 + (VT)2.0 * oo2z * (v8_0_4 - rho_z * v8_0_5);
            const VT v32_0_0 = PAy * v18_0_0 + WPy * v18_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v32_0_1 = PAy * v18_0_1 + WPy * v18_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v32_0_2 = PAy * v18_0_2 + WPy * v18_0_3 + (VT)1.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v32_0_3 = PAy * v18_0_3 + WPy * v18_0_4 + (VT)1.0 * oo2z * (v9_0_3 - rho_z * v9_0_4);
            const VT v32_0_4 = PAy * v18_0_4 + WPy * v18_0_5 + (VT)1.0 * oo2z * (v9_0_4 - rho_z * v9_0_5);
            const VT v33_0_0 = PAz * v18_0_0 + WPz * v18_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v33_0_1 = PAz * v18_0_1 + WPz * v18_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v33_0_2 = PAz * v18_0_2 + WPz * v18_0_3 + (VT)2.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v33_0_3 = PAz * v18_0_3 + WPz * v18_0_4 + (VT)2.0 * oo2z * (v8_0_3 - rho_z * v8_0_4);
            const VT v33_0_4 = PAz * v18_0_4 + WPz * v18_0_5 + (VT)2.0 * oo2z * (v8_0_4 - rho_z * v8_0_5);
            const VT v34_0_0 = PAz * v19_0_0 + WPz * v19_0_1 + (VT)3.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v34_0_1 = PAz * v19_0_1 + WPz * v19_0_2 + (VT)3.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v34_0_2 = PAz * v19_0_2 + WPz * v19_0_3 + (VT)3.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v34_0_3 = PAz * v19_0_3 + WPz * v19_0_4 + (VT)3.0 * oo2z * (v9_0_3 - rho_z * v9_0_4);
            const VT v34_0_4 = PAz * v19_0_4 + WPz * v19_0_5 + (VT)3.0 * oo2z * (v9_0_4 - rho_z * v9_0_5);
            const VT v0_1_2 = QCx * v0_0_2 + WQx * v0_0_3;
            const VT v0_1_3 = QCx * v0_0_3 + WQx * v0_0_4;
            const VT v1_1_1 = QCx * v1_0_1 + WQx * v1_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v1_1_2 = QCx * v1_0_2 + WQx * v1_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v1_1_3 = QCx * v1_0_3 + WQx * v1_0_4 + (VT)1.0 * oo2ze * v0_0_4;
            const VT v2_1_1 = QCx * v2_0_1 + WQx * v2_0_2;
            const VT v2_1_2 = QCx * v2_0_2 + WQx * v2_0_3;
            const VT v2_1_3 = QCx * v2_0_3 + WQx * v2_0_4;
            const VT v3_1_1 = QCx * v3_0_1 + WQx * v3_0_2;
            const VT v3_1_2 = QCx * v3_0_2 + WQx * v3_0_3;
            const VT v3_1_3 = QCx * v3_0_3 + WQx * v3_0_4;
            const VT v4_1_0 = QCx * v4_0_0 + WQx * v4_0_1 + (VT)2.0 * oo2ze * v1_0_1;
            const VT v4_1_1 = QCx * v4_0_1 + WQx * v4_0_2 + (VT)2.0 * oo2ze * v1_0_2;
            const VT v4_1_2 = QCx * v4_0_2 + WQx * v4_0_3 + (VT)2.0 * oo2ze * v1_0_3;
            const VT v4_1_3 = QCx * v4_0_3 + WQx * v4_0_4 + (VT)2.0 * oo2ze * v1_0_4;
            const VT v5_1_0 = QCx * v5_0_0 + WQx * v5_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v5_1_1 = QCx * v5_0_1 + WQx * v5_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v5_1_2 = QCx * v5_0_2 + WQx * v5_0_3 + (VT)1.0 * oo2ze * v2_0_3;
            const VT v5_1_3 = QCx * v5_0_3 + WQx * v5_0_4 + (VT)1.0 * oo2ze * v2_0_4;
            const VT v6_1_0 = QCx * v6_0_0 + WQx * v6_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v6_1_1 = QCx * v6_0_1 + WQx * v6_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v6_1_2 = QCx * v6_0_2 + WQx * v6_0_3 + (VT)1.0 * oo2ze * v3_0_3;
            const VT v6_1_3 = QCx * v6_0_3 + WQx * v6_0_4 + (VT)1.0 * oo2ze * v3_0_4;
            const VT v7_1_0 = QCx * v7_0_0 + WQx * v7_0_1;
            const VT v7_1_1 = QCx * v7_0_1 + WQx * v7_0_2;
            const VT v7_1_2 = QCx * v7_0_2 + WQx * v7_0_3;
            const VT v7_1_3 = QCx * v7_0_3 + WQx * v7_0_4;
            const VT v8_1_0 = QCx * v8_0_0 + WQx * v8_0_1;
            const VT v8_1_1 = QCx * v8_0_1 + WQx * v8_0_2;
            const VT v8_1_2 = QCx * v8_0_2 + WQx * v8_0_3;
            const VT v8_1_3 = QCx * v8_0_3 + WQx * v8_0_4;
            const VT v9_1_0 = QCx * v9_0_0 + WQx * v9_0_1;
            const VT v9_1_1 = QCx * v9_0_1 + WQx * v9_0_2;
            const VT v9_1_2 = QCx * v9_0_2 + WQx * v9_0_3;
            const VT v9_1_3 = QCx * v9_0_3 + WQx * v9_0_4;
            const VT v10_1_0 = QCx * v10_0_0 + WQx * v10_0_1 + (VT)3.0 * oo2ze * v4_0_1;
            const VT v10_1_1 = QCx * v10_0_1 + WQx * v10_0_2 + (VT)3.0 * oo2ze * v4_0_2;
            const VT v10_1_2 = QCx * v10_0_2 + WQx * v10_0_3 + (VT)3.0 * oo2ze * v4_0_3;
            const VT v10_1_3 = QCx * v10_0_3 + WQx * v10_0_4 + (VT)3.0 * oo2ze * v4_0_4;
            const VT v11_1_0 = QCx * v11_0_0 + WQx * v11_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v11_1_1 = QCx * v11_0_1 + WQx * v11_0_2 + (VT)2.0 * oo2ze * v5_0_2;
            const VT v11_1_2 = QCx * v11_0_2 + WQx * v11_0_3 + (VT)2.0 * oo2ze * v5_0_3;
            const VT v11_1_3 = QCx * v11_0_3 + WQx * v11_0_4 + (VT)2.0 * oo2ze * v5_0_4;
            const VT v12_1_0 = QCx * v12_0_0 + WQx * v12_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v12_1_1 = QCx * v12_0_1 + WQx * v12_0_2 + (VT)2.0 * oo2ze * v6_0_2;
            const VT v12_1_2 = QCx * v12_0_2 + WQx * v12_0_3 + (VT)2.0 * oo2ze * v6_0_3;
            const VT v12_1_3 = QCx * v12_0_3 + WQx * v12_0_4 + (VT)2.0 * oo2ze * v6_0_4;
            const VT v13_1_0 = QCx * v13_0_0 + WQx * v13_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v13_1_1 = QCx * v13_0_1 + WQx * v13_0_2 + (VT)1.0 * oo2ze * v7_0_2;
            const VT v13_1_2 = QCx * v13_0_2 + WQx * v13_0_3 + (VT)1.0 * oo2ze * v7_0_3;
            const VT v13_1_3 = QCx * v13_0_3 + WQx * v13_0_4 + (VT)1.0 * oo2ze * v7_0_4;
            const VT v14_1_0 = QCx * v14_0_0 + WQx * v14_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v14_1_1 = QCx * v14_0_1 + WQx * v14_0_2 + (VT)1.0 * oo2ze * v9_0_2;
            const VT v14_1_2 = QCx * v14_0_2 + WQx * v14_0_3 + (VT)1.0 * oo2ze * v9_0_3;
            const VT v14_1_3 = QCx * v14_0_3 + WQx * v14_0_4 + (VT)1.0 * oo2ze * v9_0_4;
            const VT v15_1_0 = QCx * v15_0_0 + WQx * v15_0_1 + (VT)1.0 * oo2ze * v8_0_1;
            const VT v15_1_1 = QCx * v15_0_1 + WQx * v15_0_2 + (VT)1.0 * oo2ze * v8_0_2;
            const VT v15_1_2 = QCx * v15_0_2 + WQx * v15_0_3 + (VT)1.0 * oo2ze * v8_0_3;
            const VT v15_1_3 = QCx * v15_0_3 + WQx * v15_0_4 + (VT)1.0 * oo2ze * v8_0_4;
            const VT v16_1_0 = QCx * v16_0_0 + WQx * v16_0_1;
            const VT v16_1_1 = QCx * v16_0_1 + WQx * v16_0_2;
            const VT v16_1_2 = QCx * v16_0_2 + WQx * v16_0_3;
            const VT v16_1_3 = QCx * v16_0_3 + WQx * v16_0_4;
            const VT v17_1_0 = QCx * v17_0_0 + WQx * v17_0_1;
            const VT v17_1_1 = QCx * v17_0_1 + WQx * v17_0_2;
            const VT v17_1_2 = QCx * v17_0_2 + WQx * v17_0_3;
            const VT v17_1_3 = QCx * v17_0_3 + WQx * v17_0_4;
            const VT v18_1_0 = QCx * v18_0_0 + WQx * v18_0_1;
            const VT v18_1_1 = QCx * v18_0_1 + WQx * v18_0_2;
            const VT v18_1_2 = QCx * v18_0_2 + WQx * v18_0_3;
            const VT v18_1_3 = QCx * v18_0_3 + WQx * v18_0_4;
            const VT v19_1_0 = QCx * v19_0_0 + WQx * v19_0_1;
            const VT v19_1_1 = QCx * v19_0_1 + WQx * v19_0_2;
            const VT v19_1_2 = QCx * v19_0_2 + WQx * v19_0_3;
            const VT v19_1_3 = QCx * v19_0_3 + WQx * v19_0_4;
            const VT v20_1_0 = QCx * v20_0_0 + WQx * v20_0_1 + (VT)4.0 * oo2ze * v10_0_1;
            const VT v20_1_1 = QCx * v20_0_1 + WQx * v20_0_2 + (VT)4.0 * oo2ze * v10_0_2;
            const VT v20_1_2 = QCx * v20_0_2 + WQx * v20_0_3 + (VT)4.0 * oo2ze * v10_0_3;
            const VT v20_1_3 = QCx * v20_0_3 + WQx * v20_0_4 + (VT)4.0 * oo2ze * v10_0_4;
            const VT v21_1_0 = QCx * v21_0_0 + WQx * v21_0_1 + (VT)3.0 * oo2ze * v11_0_1;
            const VT v21_1_1 = QCx * v21_0_1 + WQx * v21_0_2 + (VT)3.0 * oo2ze * v11_0_2;
            const VT v21_1_2 = QCx * v21_0_2 + WQx * v21_0_3 + (VT)3.0 * oo2ze * v11_0_3;
            const VT v21_1_3 = QCx * v21_0_3 + WQx * v21_0_4 + (VT)3.0 * oo2ze * v11_0_4;
            const VT v22_1_0 = QCx * v22_0_0 + WQx * v22_0_1 + (VT)3.0 * oo2ze * v12_0_1;
            const VT v22_1_1 = QCx * v22_0_1 + WQx * v22_0_2 + (VT)3.0 * oo2ze * v12_0_2;
            const VT v22_1_2 = QCx * v22_0_2 + WQx * v22_0_3 + (VT)3.0 * oo2ze * v12_0_3;
            const VT v22_1_3 = QCx * v22_0_3 + WQx * v22_0_4 + (VT)3.0 * oo2ze * v12_0_4;
            const VT v23_1_0 = QCx * v23_0_0 + WQx * v23_0_1 + (VT)2.0 * oo2ze * v13_0_1;
            const VT v23_1_1 = QCx * v23_0_1 + WQx * v23_0_2 + (VT)2.0 * oo2ze * v13_0_2;
            const VT v23_1_2 = QCx * v23_0_2 + WQx * v23_0_3 + (VT)2.0 * oo2ze * v13_0_3;
            const VT v23_1_3 = QCx * v23_0_3 + WQx * v23_0_4 + (VT)2.0 * oo2ze * v13_0_4;
            const VT v24_1_0 = QCx * v24_0_0 + WQx * v24_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v24_1_1 = QCx * v24_0_1 + WQx * v24_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v24_1_2 = QCx * v24_0_2 + WQx * v24_0_3 + (VT)2.0 * oo2ze * v15_0_3;
            const VT v24_1_3 = QCx * v24_0_3 + WQx * v24_0_4 + (VT)2.0 * oo2ze * v15_0_4;
            const VT v25_1_0 = QCx * v25_0_0 + WQx * v25_0_1 + (VT)2.0 * oo2ze * v14_0_1;
            const VT v25_1_1 = QCx * v25_0_1 + WQx * v25_0_2 + (VT)2.0 * oo2ze * v14_0_2;
            const VT v25_1_2 = QCx * v25_0_2 + WQx * v25_0_3 + (VT)2.0 * oo2ze * v14_0_3;
            const VT v25_1_3 = QCx * v25_0_3 + WQx * v25_0_4 + (VT)2.0 * oo2ze * v14_0_4;
            const VT v26_1_0 = QCx * v26_0_0 + WQx * v26_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v26_1_1 = QCx * v26_0_1 + WQx * v26_0_2 + (VT)1.0 * oo2ze * v16_0_2;
            const VT v26_1_2 = QCx * v26_0_2 + WQx * v26_0_3 + (VT)1.0 * oo2ze * v16_0_3;
            const VT v26_1_3 = QCx * v26_0_3 + WQx * v26_0_4 + (VT)1.0 * oo2ze * v16_0_4;
            const VT v27_1_0 = QCx * v27_0_0 + WQx * v27_0_1 + (VT)1.0 * oo2ze * v17_0_1;
            const VT v27_1_1 = QCx * v27_0_1 + WQx * v27_0_2 + (VT)1.0 * oo2ze * v17_0_2;
            const VT v27_1_2 = QCx * v27_0_2 + WQx * v27_0_3 + (VT)1.0 * oo2ze * v17_0_3;
            const VT v27_1_3 = QCx * v27_0_3 + WQx * v27_0_4 + (VT)1.0 * oo2ze * v17_0_4;
            const VT v28_1_0 = QCx * v28_0_0 + WQx * v28_0_1 + (VT)1.0 * oo2ze * v18_0_1;
            const VT v28_1_1 = QCx * v28_0_1 + WQx * v28_0_2 + (VT)1.0 * oo2ze * v18_0_2;
            const VT v28_1_2 = QCx * v28_0_2 + WQx * v28_0_3 + (VT)1.0 * oo2ze * v18_0_3;
            const VT v28_1_3 = QCx * v28_0_3 + WQx * v28_0_4 + (VT)1.0 * oo2ze * v18_0_4;
            const VT v29_1_0 = QCx * v29_0_0 + WQx * v29_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v29_1_1 = QCx * v29_0_1 + WQx * v29_0_2 + (VT)1.0 * oo2ze * v19_0_2;
            const VT v29_1_2 = QCx * v29_0_2 + WQx * v29_0_3 + (VT)1.0 * oo2ze * v19_0_3;
            const VT v29_1_3 = QCx * v29_0_3 + WQx * v29_0_4 + (VT)1.0 * oo2ze * v19_0_4;
            const VT v30_1_0 = QCx * v30_0_0 + WQx * v30_0_1;
            const VT v30_1_1 = QCx * v30_0_1 + WQx * v30_0_2;
            const VT v30_1_2 = QCx * v30_0_2 + WQx * v30_0_3;
            const VT v30_1_3 = QCx * v30_0_3 + WQx * v30_0_4;
            const VT v31_1_0 = QCx * v31_0_0 + WQx * v31_0_1;
            const VT v31_1_1 = QCx * v31_0_1 + WQx * v31_0_2;
            const VT v31_1_2 = QCx * v31_0_2 + WQx * v31_0_3;
            const VT v31_1_3 = QCx * v31_0_3 + WQx * v31_0_4;
            const VT v32_1_0 = QCx * v32_0_0 + WQx * v32_0_1;
            const VT v32_1_1 = QCx * v32_0_1 + WQx * v32_0_2;
            const VT v32_1_2 = QCx * v32_0_2 + WQx * v32_0_3;
            const VT v32_1_3 = QCx * v32_0_3 + WQx * v32_0_4;
            const VT v33_1_0 = QCx * v33_0_0 + WQx * v33_0_1;
            const VT v33_1_1 = QCx * v33_0_1 + WQx * v33_0_2;
            const VT v33_1_2 = QCx * v33_0_2 + WQx * v33_0_3;
            const VT v33_1_3 = QCx * v33_0_3 + WQx * v33_0_4;
            const VT v34_1_0 = QCx * v34_0_0 + WQx * v34_0_1;
            const VT v34_1_1 = QCx * v34_0_1 + WQx * v34_0_2;
            const VT v34_1_2 = QCx * v34_0_2 + WQx * v34_0_3;
            const VT v34_1_3 = QCx * v34_0_3 + WQx * v34_0_4;
            const VT v0_2_2 = QCy * v0_0_2 + WQy * v0_0_3;
            const VT v0_2_3 = QCy * v0_0_3 + WQy * v0_0_4;
            const VT v1_2_1 = QCy * v1_0_1 + WQy * v1_0_2;
            const VT v1_2_2 = QCy * v1_0_2 + WQy * v1_0_3;
            const VT v1_2_3 = QCy * v1_0_3 + WQy * v1_0_4;
            const VT v2_2_1 = QCy * v2_0_1 + WQy * v2_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v2_2_2 = QCy * v2_0_2 + WQy * v2_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v2_2_3 = QCy * v2_0_3 + WQy * v2_0_4 + (VT)1.0 * oo2ze * v0_0_4;
            const VT v3_2_1 = QCy * v3_0_1 + WQy * v3_0_2;
            const VT v3_2_2 = QCy * v3_0_2 + WQy * v3_0_3;
            const VT v3_2_3 = QCy * v3_0_3 + WQy * v3_0_4;
            const VT v4_2_0 = QCy * v4_0_0 + WQy * v4_0_1;
            const VT v4_2_1 = QCy * v4_0_1 + WQy * v4_0_2;
            const VT v4_2_2 = QCy * v4_0_2 + WQy * v4_0_3;
            const VT v4_2_3 = QCy * v4_0_3 + WQy * v4_0_4;
            const VT v5_2_0 = QCy * v5_0_0 + WQy * v5_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v5_2_1 = QCy * v5_0_1 + WQy * v5_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v5_2_2 = QCy * v5_0_2 + WQy * v5_0_3 + (VT)1.0 * oo2ze * v1_0_3;
            const VT v5_2_3 = QCy * v5_0_3 + WQy * v5_0_4 + (VT)1.0 * oo2ze * v1_0_4;
            const VT v6_2_0 = QCy * v6_0_0 + WQy * v6_0_1;
            const VT v6_2_1 = QCy * v6_0_1 + WQy * v6_0_2;
            const VT v6_2_2 = QCy * v6_0_2 + WQy * v6_0_3;
            const VT v6_2_3 = QCy * v6_0_3 + WQy * v6_0_4;
            const VT v7_2_0 = QCy * v7_0_0 + WQy * v7_0_1 + (VT)2.0 * oo2ze * v2_0_1;
            const VT v7_2_1 = QCy * v7_0_1 + WQy * v7_0_2 + (VT)2.0 * oo2ze * v2_0_2;
            const VT v7_2_2 = QCy * v7_0_2 + WQy * v7_0_3 + (VT)2.0 * oo2ze * v2_0_3;
            const VT v7_2_3 = QCy * v7_0_3 + WQy * v7_0_4 + (VT)2.0 * oo2ze * v2_0_4;
            const VT v8_2_0 = QCy * v8_0_0 + WQy * v8_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v8_2_1 = QCy * v8_0_1 + WQy * v8_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v8_2_2 = QCy * v8_0_2 + WQy * v8_0_3 + (VT)1.0 * oo2ze * v3_0_3;
            const VT v8_2_3 = QCy * v8_0_3 + WQy * v8_0_4 + (VT)1.0 * oo2ze * v3_0_4;
            const VT v9_2_0 = QCy * v9_0_0 + WQy * v9_0_1;
            const VT v9_2_1 = QCy * v9_0_1 + WQy * v9_0_2;
            const VT v9_2_2 = QCy * v9_0_2 + WQy * v9_0_3;
            const VT v9_2_3 = QCy * v9_0_3 + WQy * v9_0_4;
            const VT v10_2_0 = QCy * v10_0_0 + WQy * v10_0_1;
            const VT v10_2_1 = QCy * v10_0_1 + WQy * v10_0_2;
            const VT v10_2_2 = QCy * v10_0_2 + WQy * v10_0_3;
            const VT v10_2_3 = QCy * v10_0_3 + WQy * v10_0_4;
            const VT v11_2_0 = QCy * v11_0_0 + WQy * v11_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v11_2_1 = QCy * v11_0_1 + WQy * v11_0_2 + (VT)1.0 * oo2ze * v4_0_2;
            const VT v11_2_2 = QCy * v11_0_2 + WQy * v11_0_3 + (VT)1.0 * oo2ze * v4_0_3;
            const VT v11_2_3 = QCy * v11_0_3 + WQy * v11_0_4 + (VT)1.0 * oo2ze * v4_0_4;
            const VT v12_2_0 = QCy * v12_0_0 + WQy * v12_0_1;
            const VT v12_2_1 = QCy * v12_0_1 + WQy * v12_0_2;
            const VT v12_2_2 = QCy * v12_0_2 + WQy * v12_0_3;
            const VT v12_2_3 = QCy * v12_0_3 + WQy * v12_0_4;
            const VT v13_2_0 = QCy * v13_0_0 + WQy * v13_0_1 + (VT)2.0 * oo2ze * v5_0_1;
            const VT v13_2_1 = QCy * v13_0_1 + WQy * v13_0_2 + (VT)2.0 * oo2ze * v5_0_2;
            const VT v13_2_2 = QCy * v13_0_2 + WQy * v13_0_3 + (VT)2.0 * oo2ze * v5_0_3;
            const VT v13_2_3 = QCy * v13_0_3 + WQy * v13_0_4 + (VT)2.0 * oo2ze * v5_0_4;
            const VT v14_2_0 = QCy * v14_0_0 + WQy * v14_0_1;
            const VT v14_2_1 = QCy * v14_0_1 + WQy * v14_0_2;
            const VT v14_2_2 = QCy * v14_0_2 + WQy * v14_0_3;
            const VT v14_2_3 = QCy * v14_0_3 + WQy * v14_0_4;
            const VT v15_2_0 = QCy * v15_0_0 + WQy * v15_0_1 + (VT)1.0 * oo2ze * v6_0_1;
            const VT v15_2_1 = QCy * v15_0_1 + WQy * v15_0_2 + (VT)1.0 * oo2ze * v6_0_2;
            const VT v15_2_2 = QCy * v15_0_2 + WQy * v15_0_3 + (VT)1.0 * oo2ze * v6_0_3;
            const VT v15_2_3 = QCy * v15_0_3 + WQy * v15_0_4 + (VT)1.0 * oo2ze * v6_0_4;
            const VT v16_2_0 = QCy * v16_0_0 + WQy * v16_0_1 + (VT)3.0 * oo2ze * v7_0_1;
            const VT v16_2_1 = QCy * v16_0_1 + WQy * v16_0_2 + (VT)3.0 * oo2ze * v7_0_2;
            const VT v16_2_2 = QCy * v16_0_2 + WQy * v16_0_3 + (VT)3.0 * oo2ze * v7_0_3;
            const VT v16_2_3 = QCy * v16_0_3 + WQy * v16_0_4 + (VT)3.0 * oo2ze * v7_0_4;
            const VT v17_2_0 = QCy * v17_0_0 + WQy * v17_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v17_2_1 = QCy * v17_0_1 + WQy * v17_0_2 + (VT)2.0 * oo2ze * v8_0_2;
            const VT v17_2_2 = QCy * v17_0_2 + WQy * v17_0_3 + (VT)2.0 * oo2ze * v8_0_3;
            const VT v17_2_3 = QCy * v17_0_3 + WQy * v17_0_4 + (VT)2.0 * oo2ze * v8_0_4;
            const VT v18_2_0 = QCy * v18_0_0 + WQy * v18_0_1 + (VT)1.0 * oo2ze * v9_0_1;
            const VT v18_2_1 = QCy * v18_0_1 + WQy * v18_0_2 + (VT)1.0 * oo2ze * v9_0_2;
            const VT v18_2_2 = QCy * v18_0_2 + WQy * v18_0_3 + (VT)1.0 * oo2ze * v9_0_3;
            const VT v18_2_3 = QCy * v18_0_3 + WQy * v18_0_4 + (VT)1.0 * oo2ze * v9_0_4;
            const VT v19_2_0 = QCy * v19_0_0 + WQy * v19_0_1;
            const VT v19_2_1 = QCy * v19_0_1 + WQy * v19_0_2;
            const VT v19_2_2 = QCy * v19_0_2 + WQy * v19_0_3;
            const VT v19_2_3 = QCy * v19_0_3 + WQy * v19_0_4;
            const VT v20_2_0 = QCy * v20_0_0 + WQy * v20_0_1;
            const VT v20_2_1 = QCy * v20_0_1 + WQy * v20_0_2;
            const VT v20_2_2 = QCy * v20_0_2 + WQy * v20_0_3;
            const VT v20_2_3 = QCy * v20_0_3 + WQy * v20_0_4;
            const VT v21_2_0 = QCy * v21_0_0 + WQy * v21_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v21_2_1 = QCy * v21_0_1 + WQy * v21_0_2 + (VT)1.0 * oo2ze * v10_0_2;
            const VT v21_2_2 = QCy * v21_0_2 + WQy * v21_0_3 + (VT)1.0 * oo2ze * v10_0_3;
            const VT v21_2_3 = QCy * v21_0_3 + WQy * v21_0_4 + (VT)1.0 * oo2ze * v10_0_4;
            const VT v22_2_0 = QCy * v22_0_0 + WQy * v22_0_1;
            const VT v22_2_1 = QCy * v22_0_1 + WQy * v22_0_2;
            const VT v22_2_2 = QCy * v22_0_2 + WQy * v22_0_3;
            const VT v22_2_3 = QCy * v22_0_3 + WQy * v22_0_4;
            const VT v23_2_0 = QCy * v23_0_0 + WQy * v23_0_1 + (VT)2.0 * oo2ze * v11_0_1;
            const VT v23_2_1 = QCy * v23_0_1 + WQy * v23_0_2 + (VT)2.0 * oo2ze * v11_0_2;
            const VT v23_2_2 = QCy * v23_0_2 + WQy * v23_0_3 + (VT)2.0 * oo2ze * v11_0_3;
            const VT v23_2_3 = QCy * v23_0_3 + WQy * v23_0_4 + (VT)2.0 * oo2ze * v11_0_4;
            const VT v24_2_0 = QCy * v24_0_0 + WQy * v24_0_1 + (VT)1.0 * oo2ze * v12_0_1;
            const VT v24_2_1 = QCy * v24_0_1 + WQy * v24_0_2 + (VT)1.0 * oo2ze * v12_0_2;
            const VT v24_2_2 = QCy * v24_0_2 + WQy * v24_0_3 + (VT)1.0 * oo2ze * v12_0_3;
            const VT v24_2_3 = QCy * v24_0_3 + WQy * v24_0_4 + (VT)1.0 * oo2ze * v12_0_4;
            const VT v25_2_0 = QCy * v25_0_0 + WQy * v25_0_1;
            const VT v25_2_1 = QCy * v25_0_1 + WQy * v25_0_2;
            const VT v25_2_2 = QCy * v25_0_2 + WQy * v25_0_3;
            const VT v25_2_3 = QCy * v25_0_3 + WQy * v25_0_4;
            const VT v26_2_0 = QCy * v26_0_0 + WQy * v26_0_1 + (VT)3.0 * oo2ze * v13_0_1;
            const VT v26_2_1 = QCy * v26_0_1 + WQy * v26_0_2 + (VT)3.0 * oo2ze * v13_0_2;
            const VT v26_2_2 = QCy * v26_0_2 + WQy * v26_0_3 + (VT)3.0 * oo2ze * v13_0_3;
            const VT v26_2_3 = QCy * v26_0_3 + WQy * v26_0_4 + (VT)3.0 * oo2ze * v13_0_4;
            const VT v27_2_0 = QCy * v27_0_0 + WQy * v27_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v27_2_1 = QCy * v27_0_1 + WQy * v27_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v27_2_2 = QCy * v27_0_2 + WQy * v27_0_3 + (VT)2.0 * oo2ze * v15_0_3;
            const VT v27_2_3 = QCy * v27_0_3 + WQy * v27_0_4 + (VT)2.0 * oo2ze * v15_0_4;
            const VT v28_2_0 = QCy * v28_0_0 + WQy * v28_0_1 + (VT)1.0 * oo2ze * v14_0_1;
            const VT v28_2_1 = QCy * v28_0_1 + WQy * v28_0_2 + (VT)1.0 * oo2ze * v14_0_2;
            const VT v28_2_2 = QCy * v28_0_2 + WQy * v28_0_3 + (VT)1.0 * oo2ze * v14_0_3;
            const VT v28_2_3 = QCy * v28_0_3 + WQy * v28_0_4 + (VT)1.0 * oo2ze * v14_0_4;
            const VT v29_2_0 = QCy * v29_0_0 + WQy * v29_0_1;
            const VT v29_2_1 = QCy * v29_0_1 + WQy * v29_0_2;
            const VT v29_2_2 = QCy * v29_0_2 + WQy * v29_0_3;
            const VT v29_2_3 = QCy * v29_0_3 + WQy * v29_0_4;
            const VT v30_2_0 = QCy * v30_0_0 + WQy * v30_0_1 + (VT)4.0 * oo2ze * v16_0_1;
            const VT v30_2_1 = QCy * v30_0_1 + WQy * v30_0_2 + (VT)4.0 * oo2ze * v16_0_2;
            const VT v30_2_2 = QCy * v30_0_2 + WQy * v30_0_3 + (VT)4.0 * oo2ze * v16_0_3;
            const VT v30_2_3 = QCy * v30_0_3 + WQy * v30_0_4 + (VT)4.0 * oo2ze * v16_0_4;
            const VT v31_2_0 = QCy * v31_0_0 + WQy * v31_0_1 + (VT)3.0 * oo2ze * v17_0_1;
            const VT v31_2_1 = QCy * v31_0_1 + WQy * v31_0_2 + (VT)3.0 * oo2ze * v17_0_2;
            const VT v31_2_2 = QCy * v31_0_2 + WQy * v31_0_3 + (VT)3.0 * oo2ze * v17_0_3;
            const VT v31_2_3 = QCy * v31_0_3 + WQy * v31_0_4 + (VT)3.0 * oo2ze * v17_0_4;
            const VT v32_2_0 = QCy * v32_0_0 + WQy * v32_0_1 + (VT)2.0 * oo2ze * v18_0_1;
            const VT v32_2_1 = QCy * v32_0_1 + WQy * v32_0_2 + (VT)2.0 * oo2ze * v18_0_2;
            const VT v32_2_2 = QCy * v32_0_2 + WQy * v32_0_3 + (VT)2.0 * oo2ze * v18_0_3;
            const VT v32_2_3 = QCy * v32_0_3 + WQy * v32_0_4 + (VT)2.0 * oo2ze * v18_0_4;
            const VT v33_2_0 = QCy * v33_0_0 + WQy * v33_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v33_2_1 = QCy * v33_0_1 + WQy * v33_0_2 + (VT)1.0 * oo2ze * v19_0_2;
            const VT v33_2_2 = QCy * v33_0_2 + WQy * v33_0_3 + (VT)1.0 * oo2ze * v19_0_3;
            const VT v33_2_3 = QCy * v33_0_3 + WQy * v33_0_4 + (VT)1.0 * oo2ze * v19_0_4;
            const VT v34_2_0 = QCy * v34_0_0 + WQy * v34_0_1;
            const VT v34_2_1 = QCy * v34_0_1 + WQy * v34_0_2;
            const VT v34_2_2 = QCy * v34_0_2 + WQy * v34_0_3;
            const VT v34_2_3 = QCy * v34_0_3 + WQy * v34_0_4;
            const VT v0_3_2 = QCz * v0_0_2 + WQz * v0_0_3;
            const VT v0_3_3 = QCz * v0_0_3 + WQz * v0_0_4;
            const VT v1_3_1 = QCz * v1_0_1 + WQz * v1_0_2;
            const VT v1_3_2 = QCz * v1_0_2 + WQz * v1_0_3;
            const VT v1_3_3 = QCz * v1_0_3 + WQz * v1_0_4;
            const VT v2_3_1 = QCz * v2_0_1 + WQz * v2_0_2;
            const VT v2_3_2 = QCz * v2_0_2 + WQz * v2_0_3;
            const VT v2_3_3 = QCz * v2_0_3 + WQz * v2_0_4;
            const VT v3_3_1 = QCz * v3_0_1 + WQz * v3_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v3_3_2 = QCz * v3_0_2 + WQz * v3_0_3 + (VT)1.0 * oo2ze * v0_0_3;
            const VT v3_3_3 = QCz * v3_0_3 + WQz * v3_0_4 + (VT)1.0 * oo2ze * v0_0_4;
            const VT v4_3_0 = QCz * v4_0_0 + WQz * v4_0_1;
            const VT v4_3_1 = QCz * v4_0_1 + WQz * v4_0_2;
            const VT v4_3_2 = QCz * v4_0_2 + WQz * v4_0_3;
            const VT v4_3_3 = QCz * v4_0_3 + WQz * v4_0_4;
            const VT v5_3_0 = QCz * v5_0_0 + WQz * v5_0_1;
            const VT v5_3_1 = QCz * v5_0_1 + WQz * v5_0_2;
            const VT v5_3_2 = QCz * v5_0_2 + WQz * v5_0_3;
            const VT v5_3_3 = QCz * v5_0_3 + WQz * v5_0_4;
            const VT v6_3_0 = QCz * v6_0_0 + WQz * v6_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v6_3_1 = QCz * v6_0_1 + WQz * v6_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v6_3_2 = QCz * v6_0_2 + WQz * v6_0_3 + (VT)1.0 * oo2ze * v1_0_3;
            const VT v6_3_3 = QCz * v6_0_3 + WQz * v6_0_4 + (VT)1.0 * oo2ze * v1_0_4;
            const VT v7_3_0 = QCz * v7_0_0 + WQz * v7_0_1;
            const VT v7_3_1 = QCz * v7_0_1 + WQz * v7_0_2;
            const VT v7_3_2 = QCz * v7_0_2 + WQz * v7_0_3;
            const VT v7_3_3 = QCz * v7_0_3 + WQz * v7_0_4;
            const VT v8_3_0 = QCz * v8_0_0 + WQz * v8_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v8_3_1 = QCz * v8_0_1 + WQz * v8_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v8_3_2 = QCz * v8_0_2 + WQz * v8_0_3 + (VT)1.0 * oo2ze * v2_0_3;
            const VT v8_3_3 = QCz * v8_0_3 + WQz * v8_0_4 + (VT)1.0 * oo2ze * v2_0_4;
            const VT v9_3_0 = QCz * v9_0_0 + WQz * v9_0_1 + (VT)2.0 * oo2ze * v3_0_1;
            const VT v9_3_1 = QCz * v9_0_1 + WQz * v9_0_2 + (VT)2.0 * oo2ze * v3_0_2;
            const VT v9_3_2 = QCz * v9_0_2 + WQz * v9_0_3 + (VT)2.0 * oo2ze * v3_0_3;
            const VT v9_3_3 = QCz * v9_0_3 + WQz * v9_0_4 + (VT)2.0 * oo2ze * v3_0_4;
            const VT v10_3_0 = QCz * v10_0_0 + WQz * v10_0_1;
            const VT v10_3_1 = QCz * v10_0_1 + WQz * v10_0_2;
            const VT v10_3_2 = QCz * v10_0_2 + WQz * v10_0_3;
            const VT v10_3_3 = QCz * v10_0_3 + WQz * v10_0_4;
            const VT v11_3_0 = QCz * v11_0_0 + WQz * v11_0_1;
            const VT v11_3_1 = QCz * v11_0_1 + WQz * v11_0_2;
            const VT v11_3_2 = QCz * v11_0_2 + WQz * v11_0_3;
            const VT v11_3_3 = QCz * v11_0_3 + WQz * v11_0_4;
            const VT v12_3_0 = QCz * v12_0_0 + WQz * v12_0_1 + (VT)1.0 * oo2ze * v4_0_1;
            const VT v12_3_1 = QCz * v12_0_1 + WQz * v12_0_2 + (VT)1.0 * oo2ze * v4_0_2;
            const VT v12_3_2 = QCz * v12_0_2 + WQz * v12_0_3 + (VT)1.0 * oo2ze * v4_0_3;
            const VT v12_3_3 = QCz * v12_0_3 + WQz * v12_0_4 + (VT)1.0 * oo2ze * v4_0_4;
            const VT v13_3_0 = QCz * v13_0_0 + WQz * v13_0_1;
            const VT v13_3_1 = QCz * v13_0_1 + WQz * v13_0_2;
            const VT v13_3_2 = QCz * v13_0_2 + WQz * v13_0_3;
            const VT v13_3_3 = QCz * v13_0_3 + WQz * v13_0_4;
            const VT v14_3_0 = QCz * v14_0_0 + WQz * v14_0_1 + (VT)2.0 * oo2ze * v6_0_1;
            const VT v14_3_1 = QCz * v14_0_1 + WQz * v14_0_2 + (VT)2.0 * oo2ze * v6_0_2;
            const VT v14_3_2 = QCz * v14_0_2 + WQz * v14_0_3 + (VT)2.0 * oo2ze * v6_0_3;
            const VT v14_3_3 = QCz * v14_0_3 + WQz * v14_0_4 + (VT)2.0 * oo2ze * v6_0_4;
            const VT v15_3_0 = QCz * v15_0_0 + WQz * v15_0_1 + (VT)1.0 * oo2ze * v5_0_1;
            const VT v15_3_1 = QCz * v15_0_1 + WQz * v15_0_2 + (VT)1.0 * oo2ze * v5_0_2;
            const VT v15_3_2 = QCz * v15_0_2 + WQz * v15_0_3 + (VT)1.0 * oo2ze * v5_0_3;
            const VT v15_3_3 = QCz * v15_0_3 + WQz * v15_0_4 + (VT)1.0 * oo2ze * v5_0_4;
            const VT v16_3_0 = QCz * v16_0_0 + WQz * v16_0_1;
            const VT v16_3_1 = QCz * v16_0_1 + WQz * v16_0_2;
            const VT v16_3_2 = QCz * v16_0_2 + WQz * v16_0_3;
            const VT v16_3_3 = QCz * v16_0_3 + WQz * v16_0_4;
            const VT v17_3_0 = QCz * v17_0_0 + WQz * v17_0_1 + (VT)1.0 * oo2ze * v7_0_1;
            const VT v17_3_1 = QCz * v17_0_1 + WQz * v17_0_2 + (VT)1.0 * oo2ze * v7_0_2;
            const VT v17_3_2 = QCz * v17_0_2 + WQz * v17_0_3 + (VT)1.0 * oo2ze * v7_0_3;
            const VT v17_3_3 = QCz * v17_0_3 + WQz * v17_0_4 + (VT)1.0 * oo2ze * v7_0_4;
            const VT v18_3_0 = QCz * v18_0_0 + WQz * v18_0_1 + (VT)2.0 * oo2ze * v8_0_1;
            const VT v18_3_1 = QCz * v18_0_1 + WQz * v18_0_2 + (VT)2.0 * oo2ze * v8_0_2;
            const VT v18_3_2 = QCz * v18_0_2 + WQz * v18_0_3 + (VT)2.0 * oo2ze * v8_0_3;
            const VT v18_3_3 = QCz * v18_0_3 + WQz * v18_0_4 + (VT)2.0 * oo2ze * v8_0_4;
            const VT v19_3_0 = QCz * v19_0_0 + WQz * v19_0_1 + (VT)3.0 * oo2ze * v9_0_1;
            const VT v19_3_1 = QCz * v19_0_1 + WQz * v19_0_2 + (VT)3.0 * oo2ze * v9_0_2;
            const VT v19_3_2 = QCz * v19_0_2 + WQz * v19_0_3 + (VT)3.0 * oo2ze * v9_0_3;
            const VT v19_3_3 = QCz * v19_0_3 + WQz * v19_0_4 + (VT)3.0 * oo2ze * v9_0_4;
            const VT v20_3_0 = QCz * v20_0_0 + WQz * v20_0_1;
            const VT v20_3_1 = QCz * v20_0_1 + WQz * v20_0_2;
            const VT v20_3_2 = QCz * v20_0_2 + WQz * v20_0_3;
            const VT v20_3_3 = QCz * v20_0_3 + WQz * v20_0_4;
            const VT v21_3_0 = QCz * v21_0_0 + WQz * v21_0_1;
            const VT v21_3_1 = QCz * v21_0_1 + WQz * v21_0_2;
            const VT v21_3_2 = QCz * v21_0_2 + WQz * v21_0_3;
            const VT v21_3_3 = QCz * v21_0_3 + WQz * v21_0_4;
            const VT v22_3_0 = QCz * v22_0_0 + WQz * v22_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v22_3_1 = QCz * v22_0_1 + WQz * v22_0_2 + (VT)1.0 * oo2ze * v10_0_2;
            const VT v22_3_2 = QCz * v22_0_2 + WQz * v22_0_3 + (VT)1.0 * oo2ze * v10_0_3;
            const VT v22_3_3 = QCz * v22_0_3 + WQz * v22_0_4 + (VT)1.0 * oo2ze * v10_0_4;
            const VT v23_3_0 = QCz * v23_0_0 + WQz * v23_0_1;
            const VT v23_3_1 = QCz * v23_0_1 + WQz * v23_0_2;
            const VT v23_3_2 = QCz * v23_0_2 + WQz * v23_0_3;
            const VT v23_3_3 = QCz * v23_0_3 + WQz * v23_0_4;
            const VT v24_3_0 = QCz * v24_0_0 + WQz * v24_0_1 + (VT)1.0 * oo2ze * v11_0_1;
            const VT v24_3_1 = QCz * v24_0_1 + WQz * v24_0_2 + (VT)1.0 * oo2ze * v11_0_2;
            const VT v24_3_2 = QCz * v24_0_2 + WQz * v24_0_3 + (VT)1.0 * oo2ze * v11_0_3;
            const VT v24_3_3 = QCz * v24_0_3 + WQz * v24_0_4 + (VT)1.0 * oo2ze * v11_0_4;
            const VT v25_3_0 = QCz * v25_0_0 + WQz * v25_0_1 + (VT)2.0 * oo2ze * v12_0_1;
            const VT v25_3_1 = QCz * v25_0_1 + WQz * v25_0_2 + (VT)2.0 * oo2ze * v12_0_2;
            const VT v25_3_2 = QCz * v25_0_2 + WQz * v25_0_3 + (VT)2.0 * oo2ze * v12_0_3;
            const VT v25_3_3 = QCz * v25_0_3 + WQz * v25_0_4 + (VT)2.0 * oo2ze * v12_0_4;
            const VT v26_3_0 = QCz * v26_0_0 + WQz * v26_0_1;
            const VT v26_3_1 = QCz * v26_0_1 + WQz * v26_0_2;
            const VT v26_3_2 = QCz * v26_0_2 + WQz * v26_0_3;
            const VT v26_3_3 = QCz * v26_0_3 + WQz * v26_0_4;
            const VT v27_3_0 = QCz * v27_0_0 + WQz * v27_0_1 + (VT)1.0 * oo2ze * v13_0_1;
            const VT v27_3_1 = QCz * v27_0_1 + WQz * v27_0_2 + (VT)1.0 * oo2ze * v13_0_2;
            const VT v27_3_2 = QCz * v27_0_2 + WQz * v27_0_3 + (VT)1.0 * oo2ze * v13_0_3;
            const VT v27_3_3 = QCz * v27_0_3 + WQz * v27_0_4 + (VT)1.0 * oo2ze * v13_0_4;
            const VT v28_3_0 = QCz * v28_0_0 + WQz * v28_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v28_3_1 = QCz * v28_0_1 + WQz * v28_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v28_3_2 = QCz * v28_0_2 + WQz * v28_0_3 + (VT)2.0 * oo2ze * v15_0_3;
            const VT v28_3_3 = QCz * v28_0_3 + WQz * v28_0_4 + (VT)2.0 * oo2ze * v15_0_4;
            const VT v29_3_0 = QCz * v29_0_0 + WQz * v29_0_1 + (VT)3.0 * oo2ze * v14_0_1;
            const VT v29_3_1 = QCz * v29_0_1 + WQz * v29_0_2 + (VT)3.0 * oo2ze * v14_0_2;
            const VT v29_3_2 = QCz * v29_0_2 + WQz * v29_0_3 + (VT)3.0 * oo2ze * v14_0_3;
            const VT v29_3_3 = QCz * v29_0_3 + WQz * v29_0_4 + (VT)3.0 * oo2ze * v14_0_4;
            const VT v30_3_0 = QCz * v30_0_0 + WQz * v30_0_1;
            const VT v30_3_1 = QCz * v30_0_1 + WQz * v30_0_2;
            const VT v30_3_2 = QCz * v30_0_2 + WQz * v30_0_3;
            const VT v30_3_3 = QCz * v30_0_3 + WQz * v30_0_4;
            const VT v31_3_0 = QCz * v31_0_0 + WQz * v31_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v31_3_1 = QCz * v31_0_1 + WQz * v31_0_2 + (VT)1.0 * oo2ze * v16_0_2;
            const VT v31_3_2 = QCz * v31_0_2 + WQz * v31_0_3 + (VT)1.0 * oo2ze * v16_0_3;
            const VT v31_3_3 = QCz * v31_0_3 + WQz * v31_0_4 + (VT)1.0 * oo2ze * v16_0_4;
            const VT v32_3_0 = QCz * v32_0_0 + WQz * v32_0_1 + (VT)2.0 * oo2ze * v17_0_1;
            const VT v32_3_1 = QCz * v32_0_1 + WQz * v32_0_2 + (VT)2.0 * oo2ze * v17_0_2;
            const VT v32_3_2 = QCz * v32_0_2 + WQz * v32_0_3 + (VT)2.0 * oo2ze * v17_0_3;
            const VT v32_3_3 = QCz * v32_0_3 + WQz * v32_0_4 + (VT)2.0 * oo2ze * v17_0_4;
            const VT v33_3_0 = QCz * v33_0_0 + WQz * v33_0_1 + (VT)3.0 * oo2ze * v18_0_1;
            const VT v33_3_1 = QCz * v33_0_1 + WQz * v33_0_2 + (VT)3.0 * oo2ze * v18_0_2;
            const VT v33_3_2 = QCz * v33_0_2 + WQz * v33_0_3 + (VT)3.0 * oo2ze * v18_0_3;
            const VT v33_3_3 = QCz * v33_0_3 + WQz * v33_0_4 + (VT)3.0 * oo2ze * v18_0_4;
            const VT v34_3_0 = QCz * v34_0_0 + WQz * v34_0_1 + (VT)4.0 * oo2ze * v19_0_1;
            const VT v34_3_1 = QCz * v34_0_1 + WQz * v34_0_2 + (VT)4.0 * oo2ze * v19_0_2;
            const VT v34_3_2 = QCz * v34_0_2 + WQz * v34_0_3 + (VT)4.0 * oo2ze * v19_0_3;
            const VT v34_3_3 = QCz * v34_0_3 + WQz * v34_0_4 + (VT)4.0 * oo2ze * v19_0_4;
            const VT v0_4_2 = QCx * v0_1_2 + WQx * v0_1_3 + (VT)1.0 * oo2e * (v0_0_2 - rho_e * v0_0_3);
            const VT v1_4_1 = QCx * v1_1_1 + WQx * v1_1_2 + (VT)1.0 * oo2ze * v0_1_2 + (VT)1.0 * oo2e * (v1_0_1 - rho_e * v1_0_2);
            const VT v1_4_2 = QCx * v1_1_2 + WQx * v1_1_3 + (VT)1.0 * oo2ze * v0_1_3 + (VT)1.0 * oo2e * (v1_0_2 - rho_e * v1_0_3);
            const VT v2_4_1 = QCx * v2_1_1 + WQx * v2_1_2 + (VT)1.0 * oo2e * (v2_0_1 - rho_e * v2_0_2);
            const VT v2_4_2 = QCx * v2_1_2 + WQx * v2_1_3 + (VT)1.0 * oo2e * (v2_0_2 - rho_e * v2_0_3);
            const VT v3_4_1 = QCx * v3_1_1 + WQx * v3_1_2 + (VT)1.0 * oo2e * (v3_0_1 - rho_e * v3_0_2);
            const VT v3_4_2 = QCx * v3_1_2 + WQx * v3_1_3 + (VT)1.0 * oo2e * (v3_0_2 - rho_e * v3_0_3);
            const VT v4_4_0 = QCx * v4_1_0 + WQx * v4_1_1 + (VT)2.0 * oo2ze * v1_1_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v4_4_1 = QCx * v4_1_1 + WQx * v4_1_2 + (VT)2.0 * oo2ze * v1_1_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v4_4_2 = QCx * v4_1_2 + WQx * v4_1_3 + (VT)2.0 * oo2ze * v1_1_3 + (VT)1.0 * oo2e * (v4_0_2 - rho_e * v4_0_3);
            const VT v5_4_0 = QCx * v5_1_0 + WQx * v5_1_1 + (VT)1.0 * oo2ze * v2_1_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v5_4_1 = QCx * v5_1_1 + WQx * v5_1_2 + (VT)1.0 * oo2ze * v2_1_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v5_4_2 = QCx * v5_1_2 + WQx * v5_1_3 + (VT)1.0 * oo2ze * v2_1_3 + (VT)1.0 * oo2e * (v5_0_2 - rho_e * v5_0_3);
            const VT v6_4_0 = QCx * v6_1_0 + WQx * v6_1_1 + (VT)1.0 * oo2ze * v3_1_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v6_4_1 = QCx * v6_1_1 + WQx * v6_1_2 + (VT)1.0 * oo2ze * v3_1_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v6_4_2 = QCx * v6_1_2 + WQx * v6_1_3 + (VT)1.0 * oo2ze * v3_1_3 + (VT)1.0 * oo2e * (v6_0_2 - rho_e * v6_0_3);
            const VT v7_4_0 = QCx * v7_1_0 + WQx * v7_1_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v7_4_1 = QCx * v7_1_1 + WQx * v7_1_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v7_4_2 = QCx * v7_1_2 + WQx * v7_1_3 + (VT)1.0 * oo2e * (v7_0_2 - rho_e * v7_0_3);
            const VT v8_4_0 = QCx * v8_1_0 + WQx * v8_1_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v8_4_1 = QCx * v8_1_1 + WQx * v8_1_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v8_4_2 = QCx * v8_1_2 + WQx * v8_1_3 + (VT)1.0 * oo2e * (v8_0_2 - rho_e * v8_0_3);
            const VT v9_4_0 = QCx * v9_1_0 + WQx * v9_1_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v9_4_1 = QCx * v9_1_1 + WQx * v9_1_2 + (VT)1.0 * oo2e * (v9_0_1 - rho_e * v9_0_2);
            const VT v9_4_2 = QCx * v9_1_2 + WQx * v9_1_3 + (VT)1.0 * oo2e * (v9_0_2 - rho_e * v9_0_3);
            const VT v10_4_0 = QCx * v10_1_0 + WQx * v10_1_1 + (VT)3.0 * oo2ze * v4_1_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v10_4_1 = QCx * v10_1_1 + WQx * v10_1_2 + (VT)3.0 * oo2ze * v4_1_2 + (VT)1.0 * oo2e * (v10_0_1 - rho_e * v10_0_2);
            const VT v10_4_2 = QCx * v10_1_2 + WQx * v10_1_3 + (VT)3.0 * oo2ze * v4_1_3 + (VT)1.0 * oo2e * (v10_0_2 - rho_e * v10_0_3);
            const VT v11_4_0 = QCx * v11_1_0 + WQx * v11_1_1 + (VT)2.0 * oo2ze * v5_1_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v11_4_1 = QCx * v11_1_1 + WQx * v11_1_2 + (VT)2.0 * oo2ze * v5_1_2 + (VT)1.0 * oo2e * (v11_0_1 - rho_e * v11_0_2);
            const VT v11_4_2 = QCx * v11_1_2 + WQx * v11_1_3 + (VT)2.0 * oo2ze * v5_1_3 + (VT)1.0 * oo2e * (v11_0_2 - rho_e * v11_0_3);
            const VT v12_4_0 = QCx * v12_1_0 + WQx * v12_1_1 + (VT)2.0 * oo2ze * v6_1_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v12_4_1 = QCx * v12_1_1 + WQx * v12_1_2 + (VT)2.0 * oo2ze * v6_1_2 + (VT)1.0 * oo2e * (v12_0_1 - rho_e * v12_0_2);
            const VT v12_4_2 = QCx * v12_1_2 + WQx * v12_1_3 + (VT)2.0 * oo2ze * v6_1_3 + (VT)1.0 * oo2e * (v12_0_2 - rho_e * v12_0_3);
            const VT v13_4_0 = QCx * v13_1_0 + WQx * v13_1_1 + (VT)1.0 * oo2ze * v7_1_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v13_4_1 = QCx * v13_1_1 + WQx * v13_1_2 + (VT)1.0 * oo2ze * v7_1_2 + (VT)1.0 * oo2e * (v13_0_1 - rho_e * v13_0_2);
            const VT v13_4_2 = QCx * v13_1_2 + WQx * v13_1_3 + (VT)1.0 * oo2ze * v7_1_3 + (VT)1.0 * oo2e * (v13_0_2 - rho_e * v13_0_3);
            const VT v14_4_0 = QCx * v14_1_0 + WQx * v14_1_1 + (VT)1.0 * oo2ze * v9_1_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v14_4_1 = QCx * v14_1_1 + WQx * v14_1_2 + (VT)1.0 * oo2ze * v9_1_2 + (VT)1.0 * oo2e * (v14_0_1 - rho_e * v14_0_2);
            const VT v14_4_2 = QCx * v14_1_2 + WQx * v14_1_3 + (VT)1.0 * oo2ze * v9_1_3 + (VT)1.0 * oo2e * (v14_0_2 - rho_e * v14_0_3);
            const VT v15_4_0 = QCx * v15_1_0 + WQx * v15_1_1 + (VT)1.0 * oo2ze * v8_1_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v15_4_1 = QCx * v15_1_1 + WQx * v15_1_2 + (VT)1.0 * oo2ze * v8_1_2 + (VT)1.0 * oo2e * (v15_0_1 - rho_e * v15_0_2);
            const VT v15_4_2 = QCx * v15_1_2 + WQx * v15_1_3 + (VT)1.0 * oo2ze * v8_1_3 + (VT)1.0 * oo2e * (v15_0_2 - rho_e * v15_0_3);
            const VT v16_4_0 = QCx * v16_1_0 + WQx * v16_1_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v16_4_1 = QCx * v16_1_1 + WQx * v16_1_2 + (VT)1.0 * oo2e * (v16_0_1 - rho_e * v16_0_2);
            const VT v16_4_2 = QCx * v16_1_2 + WQx * v16_1_3 + (VT)1.0 * oo2e * (v16_0_2 - rho_e * v16_0_3);
            const VT v17_4_0 = QCx * v17_1_0 + WQx * v17_1_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v17_4_1 = QCx * v17_1_1 + WQx * v17_1_2 + (VT)1.0 * oo2e * (v17_0_1 - rho_e * v17_0_2);
            const VT v17_4_2 = QCx * v17_1_2 + WQx * v17_1_3 + (VT)1.0 * oo2e * (v17_0_2 - rho_e * v17_0_3);
            const VT v18_4_0 = QCx * v18_1_0 + WQx * v18_1_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v18_4_1 = QCx * v18_1_1 + WQx * v18_1_2 + (VT)1.0 * oo2e * (v18_0_1 - rho_e * v18_0_2);
            const VT v18_4_2 = QCx * v18_1_2 + WQx * v18_1_3 + (VT)1.0 * oo2e * (v18_0_2 - rho_e * v18_0_3);
            const VT v19_4_0 = QCx * v19_1_0 + WQx * v19_1_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v19_4_1 = QCx * v19_1_1 + WQx * v19_1_2 + (VT)1.0 * oo2e * (v19_0_1 - rho_e * v19_0_2);
            const VT v19_4_2 = QCx * v19_1_2 + WQx * v19_1_3 + (VT)1.0 * oo2e * (v19_0_2 - rho_e * v19_0_3);
            const VT v20_4_0 = QCx * v20_1_0 + WQx * v20_1_1 + (VT)4.0 * oo2ze * v10_1_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v20_4_1 = QCx * v20_1_1 + WQx * v20_1_2 + (VT)4.0 * oo2ze * v10_1_2 + (VT)1.0 * oo2e * (v20_0_1 - rho_e * v20_0_2);
            const VT v20_4_2 = QCx * v20_1_2 + WQx * v20_1_3 + (VT)4.0 * oo2ze * v10_1_3 + (VT)1.0 * oo2e * (v20_0_2 - rho_e * v20_0_3);
            const VT v21_4_0 = QCx * v21_1_0 + WQx * v21_1_1 + (VT)3.0 * oo2ze * v11_1_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v21_4_1 = QCx * v21_1_1 + WQx * v21_1_2 + (VT)3.0 * oo2ze * v11_1_2 + (VT)1.0 * oo2e * (v21_0_1 - rho_e * v21_0_2);
            const VT v21_4_2 = QCx * v21_1_2 + WQx * v21_1_3 + (VT)3.0 * oo2ze * v11_1_3 + (VT)1.0 * oo2e * (v21_0_2 - rho_e * v21_0_3);
            const VT v22_4_0 = QCx * v22_1_0 + WQx * v22_1_1 + (VT)3.0 * oo2ze * v12_1_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v22_4_1 = QCx * v22_1_1 + WQx * v22_1_2 + (VT)3.0 * oo2ze * v12_1_2 + (VT)1.0 * oo2e * (v22_0_1 - rho_e * v22_0_2);
            const VT v22_4_2 = QCx * v22_1_2 + WQx * v22_1_3 + (VT)3.0 * oo2ze * v12_1_3 + (VT)1.0 * oo2e * (v22_0_2 - rho_e * v22_0_3);
            const VT v23_4_0 = QCx * v23_1_0 + WQx * v23_1_1 + (VT)2.0 * oo2ze * v13_1_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v23_4_1 = QCx * v23_1_1 + WQx * v23_1_2 + (VT)2.0 * oo2ze * v13_1_2 + (VT)1.0 * oo2e * (v23_0_1 - rho_e * v23_0_2);
            const VT v23_4_2 = QCx * v23_1_2 + WQx * v23_1_3 + (VT)2.0 * oo2ze * v13_1_3 + (VT)1.0 * oo2e * (v23_0_2 - rho_e * v23_0_3);
            const VT v24_4_0 = QCx * v24_1_0 + WQx * v24_1_1 + (VT)2.0 * oo2ze * v15_1_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v24_4_1 = QCx * v24_1_1 + WQx * v24_1_2 + (VT)2.0 * oo2ze * v15_1_2 + (VT)1.0 * oo2e * (v24_0_1 - rho_e * v24_0_2);
            const VT v24_4_2 = QCx * v24_1_2 + WQx * v24_1_3 + (VT)2.0 * oo2ze * v15_1_3 + (VT)1.0 * oo2e * (v24_0_2 - rho_e * v24_0_3);
            const VT v25_4_0 = QCx * v25_1_0 + WQx * v25_1_1 + (VT)2.0 * oo2ze * v14_1_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v25_4_1 = QCx * v25_1_1 + WQx * v25_1_2 + (VT)2.0 * oo2ze * v14_1_2 + (VT)1.0 * oo2e * (v25_0_1 - rho_e * v25_0_2);
            const VT v25_4_2 = QCx * v25_1_2 + WQx * v25_1_3 + (VT)2.0 * oo2ze * v14_1_3 + (VT)1.0 * oo2e * (v25_0_2 - rho_e * v25_0_3);
            const VT v26_4_0 = QCx * v26_1_0 + WQx * v26_1_1 + (VT)1.0 * oo2ze * v16_1_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v26_4_1 = QCx * v26_1_1 + WQx * v26_1_2 + (VT)1.0 * oo2ze * v16_1_2 + (VT)1.0 * oo2e * (v26_0_1 - rho_e * v26_0_2);
            const VT v26_4_2 = QCx * v26_1_2 + WQx * v26_1_3 + (VT)1.0 * oo2ze * v16_1_3 + (VT)1.0 * oo2e * (v26_0_2 - rho_e * v26_0_3);
            const VT v27_4_0 = QCx * v27_1_0 + WQx * v27_1_1 + (VT)1.0 * oo2ze * v17_1_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v27_4_1 = QCx * v27_1_1 + WQx * v27_1_2 + (VT)1.0 * oo2ze * v17_1_2 + (VT)1.0 * oo2e * (v27_0_1 - rho_e * v27_0_2);
            const VT v27_4_2 = QCx * v27_1_2 + WQx * v27_1_3 + (VT)1.0 * oo2ze * v17_1_3 + (VT)1.0 * oo2e * (v27_0_2 - rho_e * v27_0_3);
            const VT v28_4_0 = QCx * v28_1_0 + WQx * v28_1_1 + (VT)1.0 * oo2ze * v18_1_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v28_4_1 = QCx * v28_1_1 + WQx * v28_1_2 + (VT)1.0 * oo2ze * v18_1_2 + (VT)1.0 * oo2e * (v28_0_1 - rho_e * v28_0_2);
            const VT v28_4_2 = QCx * v28_1_2 + WQx * v28_1_3 + (VT)1.0 * oo2ze * v18_1_3 + (VT)1.0 * oo2e * (v28_0_2 - rho_e * v28_0_3);
            const VT v29_4_0 = QCx * v29_1_0 + WQx * v29_1_1 + (VT)1.0 * oo2ze * v19_1_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v29_4_1 = QCx * v29_1_1 + WQx * v29_1_2 + (VT)1.0 * oo2ze * v19_1_2 + (VT)1.0 * oo2e * (v29_0_1 - rho_e * v29_0_2);
            const VT v29_4_2 = QCx * v29_1_2 + WQx * v29_1_3 + (VT)1.0 * oo2ze * v19_1_3 + (VT)1.0 * oo2e * (v29_0_2 - rho_e * v29_0_3);
            const VT v30_4_0 = QCx * v30_1_0 + WQx * v30_1_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v30_4_1 = QCx * v30_1_1 + WQx * v30_1_2 + (VT)1.0 * oo2e * (v30_0_1 - rho_e * v30_0_2);
            const VT v30_4_2 = QCx * v30_1_2 + WQx * v30_1_3 + (VT)1.0 * oo2e * (v30_0_2 - rho_e * v30_0_3);
            const VT v31_4_0 = QCx * v31_1_0 + WQx * v31_1_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v31_4_1 = QCx * v31_1_1 + WQx * v31_1_2 + (VT)1.0 * oo2e * (v31_0_1 - rho_e * v31_0_2);
            const VT v31_4_2 = QCx * v31_1_2 + WQx * v31_1_3 + (VT)1.0 * oo2e * (v31_0_2 - rho_e * v31_0_3);
            const VT v32_4_0 = QCx * v32_1_0 + WQx * v32_1_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v32_4_1 = QCx * v32_1_1 + WQx * v32_1_2 + (VT)1.0 * oo2e * (v32_0_1 - rho_e * v32_0_2);
            const VT v32_4_2 = QCx * v32_1_2 + WQx * v32_1_3 + (VT)1.0 * oo2e * (v32_0_2 - rho_e * v32_0_3);
            const VT v33_4_0 = QCx * v33_1_0 + WQx * v33_1_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v33_4_1 = QCx * v33_1_1 + WQx * v33_1_2 + (VT)1.0 * oo2e * (v33_0_1 - rho_e * v33_0_2);
            const VT v33_4_2 = QCx * v33_1_2 + WQx * v33_1_3 + (VT)1.0 * oo2e * (v33_0_2 - rho_e * v33_0_3);
            const VT v34_4_0 = QCx * v34_1_0 + WQx * v34_1_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
            const VT v34_4_1 = QCx * v34_1_1 + WQx * v34_1_2 + (VT)1.0 * oo2e * (v34_0_1 - rho_e * v34_0_2);
            const VT v34_4_2 = QCx * v34_1_2 + WQx * v34_1_3 + (VT)1.0 * oo2e * (v34_0_2 - rho_e * v34_0_3);
            const VT v0_5_2 = QCx * v0_2_2 + WQx * v0_2_3;
            const VT v1_5_1 = QCx * v1_2_1 + WQx * v1_2_2 + (VT)1.0 * oo2ze * v0_2_2;
            const VT v1_5_2 = QCx * v1_2_2 + WQx * v1_2_3 + (VT)1.0 * oo2ze * v0_2_3;
            const VT v2_5_1 = QCx * v2_2_1 + WQx * v2_2_2;
            const VT v2_5_2 = QCx * v2_2_2 + WQx * v2_2_3;
            const VT v3_5_1 = QCx * v3_2_1 + WQx * v3_2_2;
            const VT v3_5_2 = QCx * v3_2_2 + WQx * v3_2_3;
            const VT v4_5_0 = QCx * v4_2_0 + WQx * v4_2_1 + (VT)2.0 * oo2ze * v1_2_1;
            const VT v4_5_1 = QCx * v4_2_1 + WQx * v4_2_2 + (VT)2.0 * oo2ze * v1_2_2;
            const VT v4_5_2 = QCx * v4_2_2 + WQx * v4_2_3 + (VT)2.0 * oo2ze * v1_2_3;
            const VT v5_5_0 = QCx * v5_2_0 + WQx * v5_2_1 + (VT)1.0 * oo2ze * v2_2_1;
            const VT v5_5_1 = QCx * v5_2_1 + WQx * v5_2_2 + (VT)1.0 * oo2ze * v2_2_2;
            const VT v5_5_2 = QCx * v5_2_2 + WQx * v5_2_3 + (VT)1.0 * oo2ze * v2_2_3;
            const VT v6_5_0 = QCx * v6_2_0 + WQx * v6_2_1 + (VT)1.0 * oo2ze * v3_2_1;
            const VT v6_5_1 = QCx * v6_2_1 + WQx * v6_2_2 + (VT)1.0 * oo2ze * v3_2_2;
            const VT v6_5_2 = QCx * v6_2_2 + WQx * v6_2_3 + (VT)1.0 * oo2ze * v3_2_3;
            const VT v7_5_0 = QCx * v7_2_0 + WQx * v7_2_1;
            const VT v7_5_1 = QCx * v7_2_1 + WQx * v7_2_2;
            const VT v7_5_2 = QCx * v7_2_2 + WQx * v7_2_3;
            const VT v8_5_0 = QCx * v8_2_0 + WQx * v8_2_1;
            const VT v8_5_1 = QCx * v8_2_1 + WQx * v8_2_2;
            const VT v8_5_2 = QCx * v8_2_2 + WQx * v8_2_3;
            const VT v9_5_0 = QCx * v9_2_0 + WQx * v9_2_1;
            const VT v9_5_1 = QCx * v9_2_1 + WQx * v9_2_2;
            const VT v9_5_2 = QCx * v9_2_2 + WQx * v9_2_3;
            const VT v10_5_0 = QCx * v10_2_0 + WQx * v10_2_1 + (VT)3.0 * oo2ze * v4_2_1;
            const VT v10_5_1 = QCx * v10_2_1 + WQx * v10_2_2 + (VT)3.0 * oo2ze * v4_2_2;
            const VT v10_5_2 = QCx * v10_2_2 + WQx * v10_2_3 + (VT)3.0 * oo2ze * v4_2_3;
            const VT v11_5_0 = QCx * v11_2_0 + WQx * v11_2_1 + (VT)2.0 * oo2ze * v5_2_1;
            const VT v11_5_1 = QCx * v11_2_1 + WQx * v11_2_2 + (VT)2.0 * oo2ze * v5_2_2;
            const VT v11_5_2 = QCx * v11_2_2 + WQx * v11_2_3 + (VT)2.0 * oo2ze * v5_2_3;
            const VT v12_5_0 = QCx * v12_2_0 + WQx * v12_2_1 + (VT)2.0 * oo2ze * v6_2_1;
            const VT v12_5_1 = QCx * v12_2_1 + WQx * v12_2_2 + (VT)2.0 * oo2ze * v6_2_2;
            const VT v12_5_2 = QCx * v12_2_2 + WQx * v12_2_3 + (VT)2.0 * oo2ze * v6_2_3;
            const VT v13_5_0 = QCx * v13_2_0 + WQx * v13_2_1 + (VT)1.0 * oo2ze * v7_2_1;
            const VT v13_5_1 = QCx * v13_2_1 + WQx * v13_2_2 + (VT)1.0 * oo2ze * v7_2_2;
            const VT v13_5_2 = QCx * v13_2_2 + WQx * v13_2_3 + (VT)1.0 * oo2ze * v7_2_3;
            const VT v14_5_0 = QCx * v14_2_0 + WQx * v14_2_1 + (VT)1.0 * oo2ze * v9_2_1;
            const VT v14_5_1 = QCx * v14_2_1 + WQx * v14_2_2 + (VT)1.0 * oo2ze * v9_2_2;
            const VT v14_5_2 = QCx * v14_2_2 + WQx * v14_2_3 + (VT)1.0 * oo2ze * v9_2_3;
            const VT v15_5_0 = QCx * v15_2_0 + WQx * v15_2_1 + (VT)1.0 * oo2ze * v8_2_1;
            const VT v15_5_1 = QCx * v15_2_1 + WQx * v15_2_2 + (VT)1.0 * oo2ze * v8_2_2;
            const VT v15_5_2 = QCx * v15_2_2 + WQx * v15_2_3 + (VT)1.0 * oo2ze * v8_2_3;
            const VT v16_5_0 = QCx * v16_2_0 + WQx * v16_2_1;
            const VT v16_5_1 = QCx * v16_2_1 + WQx * v16_2_2;
            const VT v16_5_2 = QCx * v16_2_2 + WQx * v16_2_3;
            const VT v17_5_0 = QCx * v17_2_0 + WQx * v17_2_1;
            const VT v17_5_1 = QCx * v17_2_1 + WQx * v17_2_2;
            const VT v17_5_2 = QCx * v17_2_2 + WQx * v17_2_3;
            const VT v18_5_0 = QCx * v18_2_0 + WQx * v18_2_1;
            const VT v18_5_1 = QCx * v18_2_1 + WQx * v18_2_2;
            const VT v18_5_2 = QCx * v18_2_2 + WQx * v18_2_3;
            const VT v19_5_0 = QCx * v19_2_0 + WQx * v19_2_1;
            const VT v19_5_1 = QCx * v19_2_1 + WQx * v19_2_2;
            const VT v19_5_2 = QCx * v19_2_2 + WQx * v19_2_3;
            const VT v20_5_0 = QCx * v20_2_0 + WQx * v20_2_1 + (VT)4.0 * oo2ze * v10_2_1;
            const VT v20_5_1 = QCx * v20_2_1 + WQx * v20_2_2 + (VT)4.0 * oo2ze * v10_2_2;
            const VT v20_5_2 = QCx * v20_2_2 + WQx * v20_2_3 + (VT)4.0 * oo2ze * v10_2_3;
            const VT v21_5_0 = QCx * v21_2_0 + WQx * v21_2_1 + (VT)3.0 * oo2ze * v11_2_1;
            const VT v21_5_1 = QCx * v21_2_1 + WQx * v21_2_2 + (VT)3.0 * oo2ze * v11_2_2;
            const VT v21_5_2 = QCx * v21_2_2 + WQx * v21_2_3 + (VT)3.0 * oo2ze * v11_2_3;
            const VT v22_5_0 = QCx * v22_2_0 + WQx * v22_2_1 + (VT)3.0 * oo2ze * v12_2_1;
            const VT v22_5_1 = QCx * v22_2_1 + WQx * v22_2_2 + (VT)3.0 * oo2ze * v12_2_2;
            const VT v22_5_2 = QCx * v22_2_2 + WQx * v22_2_3 + (VT)3.0 * oo2ze * v12_2_3;
            const VT v23_5_0 = QCx * v23_2_0 + WQx * v23_2_1 + (VT)2.0 * oo2ze * v13_2_1;
            const VT v23_5_1 = QCx * v23_2_1 + WQx * v23_2_2 + (VT)2.0 * oo2ze * v13_2_2;
            const VT v23_5_2 = QCx * v23_2_2 + WQx * v23_2_3 + (VT)2.0 * oo2ze * v13_2_3;
            const VT v24_5_0 = QCx * v24_2_0 + WQx * v24_2_1 + (VT)2.0 * oo2ze * v15_2_1;
            const VT v24_5_1 = QCx * v24_2_1 + WQx * v24_2_2 + (VT)2.0 * oo2ze * v15_2_2;
            const VT v24_5_2 = QCx * v24_2_2 + WQx * v24_2_3 + (VT)2.0 * oo2ze * v15_2_3;
            const VT v25_5_0 = QCx * v25_2_0 + WQx * v25_2_1 + (VT)2.0 * oo2ze * v14_2_1;
            const VT v25_5_1 = QCx * v25_2_1 + WQx * v25_2_2 + (VT)2.0 * oo2ze * v14_2_2;
            const VT v25_5_2 = QCx * v25_2_2 + WQx * v25_2_3 + (VT)2.0 * oo2ze * v14_2_3;
            const VT v26_5_0 = QCx * v26_2_0 + WQx * v26_2_1 + (VT)1.0 * oo2ze * v16_2_1;
            const VT v26_5_1 = QCx * v26_2_1 + WQx * v26_2_2 + (VT)1.0 * oo2ze * v16_2_2;
            const VT v26_5_2 = QCx * v26_2_2 + WQx * v26_2_3 + (VT)1.0 * oo2ze * v16_2_3;
            const VT v27_5_0 = QCx * v27_2_0 + WQx * v27_2_1 + (VT)1.0 * oo2ze * v17_2_1;
            const VT v27_5_1 = QCx * v27_2_1 + WQx * v27_2_2 + (VT)1.0 * oo2ze * v17_2_2;
            const VT v27_5_2 = QCx * v27_2_2 + WQx * v27_2_3 + (VT)1.0 * oo2ze * v17_2_3;
            const VT v28_5_0 = QCx * v28_2_0 + WQx * v28_2_1 + (VT)1.0 * oo2ze * v18_2_1;
            const VT v28_5_1 = QCx * v28_2_1 + WQx * v28_2_2 + (VT)1.0 * oo2ze * v18_2_2;
            const VT v28_5_2 = QCx * v28_2_2 + WQx * v28_2_3 + (VT)1.0 * oo2ze * v18_2_3;
            const VT v29_5_0 = QCx * v29_2_0 + WQx * v29_2_1 + (VT)1.0 * oo2ze * v19_2_1;
            const VT v29_5_1 = QCx * v29_2_1 + WQx * v29_2_2 + (VT)1.0 * oo2ze * v19_2_2;
            const VT v29_5_2 = QCx * v29_2_2 + WQx * v29_2_3 + (VT)1.0 * oo2ze * v19_2_3;
            const VT v30_5_0 = QCx * v30_2_0 + WQx * v30_2_1;
            const VT v30_5_1 = QCx * v30_2_1 + WQx * v30_2_2;
            const VT v30_5_2 = QCx * v30_2_2 + WQx * v30_2_3;
            const VT v31_5_0 = QCx * v31_2_0 + WQx * v31_2_1;
            const VT v31_5_1 = QCx * v31_2_1 + WQx * v31_2_2;
            const VT v31_5_2 = QCx * v31_2_2 + WQx * v31_2_3;
            const VT v32_5_0 = QCx * v32_2_0 + WQx * v32_2_1;
            const VT v32_5_1 = QCx * v32_2_1 + WQx * v32_2_2;
            const VT v32_5_2 = QCx * v32_2_2 + WQx * v32_2_3;
            const VT v33_5_0 = QCx * v33_2_0 + WQx * v33_2_1;
            const VT v33_5_1 = QCx * v33_2_1 + WQx * v33_2_2;
            const VT v33_5_2 = QCx * v33_2_2 + WQx * v33_2_3;
            const VT v34_5_0 = QCx * v34_2_0 + WQx * v34_2_1;
            const VT v34_5_1 = QCx * v34_2_1 + WQx * v34_2_2;
            const VT v34_5_2 = QCx * v34_2_2 + WQx * v34_2_3;
            const VT v0_6_2 = QCx * v0_3_2 + WQx * v0_3_3;
            const VT v1_6_1 = QCx * v1_3_1 + WQx * v1_3_2 + (VT)1.0 * oo2ze * v0_3_2;
            const VT v1_6_2 = QCx * v1_3_2 + WQx * v1_3_3 + (VT)1.0 * oo2ze * v0_3_3;
            const VT v2_6_1 = QCx * v2_3_1 + WQx * v2_3_2;
            const VT v2_6_2 = QCx * v2_3_2 + WQx * v2_3_3;
            const VT v3_6_1 = QCx * v3_3_1 + WQx * v3_3_2;
            const VT v3_6_2 = QCx * v3_3_2 + WQx * v3_3_3;
            const VT v4_6_0 = QCx * v4_3_0 + WQx * v4_3_1 + (VT)2.0 * oo2ze * v1_3_1;
            const VT v4_6_1 = QCx * v4_3_1 + WQx * v4_3_2 + (VT)2.0 * oo2ze * v1_3_2;
            const VT v4_6_2 = QCx * v4_3_2 + WQx * v4_3_3 + (VT)2.0 * oo2ze * v1_3_3;
            const VT v5_6_0 = QCx * v5_3_0 + WQx * v5_3_1 + (VT)1.0 * oo2ze * v2_3_1;
            const VT v5_6_1 = QCx * v5_3_1 + WQx * v5_3_2 + (VT)1.0 * oo2ze * v2_3_2;
            const VT v5_6_2 = QCx * v5_3_2 + WQx * v5_3_3 + (VT)1.0 * oo2ze * v2_3_3;
            const VT v6_6_0 = QCx * v6_3_0 + WQx * v6_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v6_6_1 = QCx * v6_3_1 + WQx * v6_3_2 + (VT)1.0 * oo2ze * v3_3_2;
            const VT v6_6_2 = QCx * v6_3_2 + WQx * v6_3_3 + (VT)1.0 * oo2ze * v3_3_3;
            const VT v7_6_0 = QCx * v7_3_0 + WQx * v7_3_1;
            const VT v7_6_1 = QCx * v7_3_1 + WQx * v7_3_2;
            const VT v7_6_2 = QCx * v7_3_2 + WQx * v7_3_3;
            const VT v8_6_0 = QCx * v8_3_0 + WQx * v8_3_1;
            const VT v8_6_1 = QCx * v8_3_1 + WQx * v8_3_2;
            const VT v8_6_2 = QCx * v8_3_2 + WQx * v8_3_3;
            const VT v9_6_0 = QCx * v9_3_0 + WQx * v9_3_1;
            const VT v9_6_1 = QCx * v9_3_1 + WQx * v9_3_2;
            const VT v9_6_2 = QCx * v9_3_2 + WQx * v9_3_3;
            const VT v10_6_0 = QCx * v10_3_0 + WQx * v10_3_1 + (VT)3.0 * oo2ze * v4_3_1;
            const VT v10_6_1 = QCx * v10_3_1 + WQx * v10_3_2 + (VT)3.0 * oo2ze * v4_3_2;
            const VT v10_6_2 = QCx * v10_3_2 + WQx * v10_3_3 + (VT)3.0 * oo2ze * v4_3_3;
            const VT v11_6_0 = QCx * v11_3_0 + WQx * v11_3_1 + (VT)2.0 * oo2ze * v5_3_1;
            const VT v11_6_1 = QCx * v11_3_1 + WQx * v11_3_2 + (VT)2.0 * oo2ze * v5_3_2;
            const VT v11_6_2 = QCx * v11_3_2 + WQx * v11_3_3 + (VT)2.0 * oo2ze * v5_3_3;
            const VT v12_6_0 = QCx * v12_3_0 + WQx * v12_3_1 + (VT)2.0 * oo2ze * v6_3_1;
            const VT v12_6_1 = QCx * v12_3_1 + WQx * v12_3_2 + (VT)2.0 * oo2ze * v6_3_2;
            const VT v12_6_2 = QCx * v12_3_2 + WQx * v12_3_3 + (VT)2.0 * oo2ze * v6_3_3;
            const VT v13_6_0 = QCx * v13_3_0 + WQx * v13_3_1 + (VT)1.0 * oo2ze * v7_3_1;
            const VT v13_6_1 = QCx * v13_3_1 + WQx * v13_3_2 + (VT)1.0 * oo2ze * v7_3_2;
            const VT v13_6_2 = QCx * v13_3_2 + WQx * v13_3_3 + (VT)1.0 * oo2ze * v7_3_3;
            const VT v14_6_0 = QCx * v14_3_0 + WQx * v14_3_1 + (VT)1.0 * oo2ze * v9_3_1;
            const VT v14_6_1 = QCx * v14_3_1 + WQx * v14_3_2 + (VT)1.0 * oo2ze * v9_3_2;
            const VT v14_6_2 = QCx * v14_3_2 + WQx * v14_3_3 + (VT)1.0 * oo2ze * v9_3_3;
            const VT v15_6_0 = QCx * v15_3_0 + WQx * v15_3_1 + (VT)1.0 * oo2ze * v8_3_1;
            const VT v15_6_1 = QCx * v15_3_1 + WQx * v15_3_2 + (VT)1.0 * oo2ze * v8_3_2;
            const VT v15_6_2 = QCx * v15_3_2 + WQx * v15_3_3 + (VT)1.0 * oo2ze * v8_3_3;
            const VT v16_6_0 = QCx * v16_3_0 + WQx * v16_3_1;
            const VT v16_6_1 = QCx * v16_3_1 + WQx * v16_3_2;
            const VT v16_6_2 = QCx * v16_3_2 + WQx * v16_3_3;
            const VT v17_6_0 = QCx * v17_3_0 + WQx * v17_3_1;
            const VT v17_6_1 = QCx * v17_3_1 + WQx * v17_3_2;
            const VT v17_6_2 = QCx * v17_3_2 + WQx * v17_3_3;
            const VT v18_6_0 = QCx * v18_3_0 + WQx * v18_3_1;
            const VT v18_6_1 = QCx * v18_3_1 + WQx * v18_3_2;
            const VT v18_6_2 = QCx * v18_3_2 + WQx * v18_3_3;
            const VT v19_6_0 = QCx * v19_3_0 + WQx * v19_3_1;
            const VT v19_6_1 = QCx * v19_3_1 + WQx * v19_3_2;
            const VT v19_6_2 = QCx * v19_3_2 + WQx * v19_3_3;
            const VT v20_6_0 = QCx * v20_3_0 + WQx * v20_3_1 + (VT)4.0 * oo2ze * v10_3_1;
            const VT v20_6_1 = QCx * v20_3_1 + WQx * v20_3_2 + (VT)4.0 * oo2ze * v10_3_2;
            const VT v20_6_2 = QCx * v20_3_2 + WQx * v20_3_3 + (VT)4.0 * oo2ze * v10_3_3;
            const VT v21_6_0 = QCx * v21_3_0 + WQx * v21_3_1 + (VT)3.0 * oo2ze * v11_3_1;
            const VT v21_6_1 = QCx * v21_3_1 + WQx * v21_3_2 + (VT)3.0 * oo2ze * v11_3_2;
            const VT v21_6_2 = QCx * v21_3_2 + WQx * v21_3_3 + (VT)3.0 * oo2ze * v11_3_3;
            const VT v22_6_0 = QCx * v22_3_0 + WQx * v22_3_1 + (VT)3.0 * oo2ze * v12_3_1;
            const VT v22_6_1 = QCx * v22_3_1 + WQx * v22_3_2 + (VT)3.0 * oo2ze * v12_3_2;
            const VT v22_6_2 = QCx * v22_3_2 + WQx * v22_3_3 + (VT)3.0 * oo2ze * v12_3_3;
            const VT v23_6_0 = QCx * v23_3_0 + WQx * v23_3_1 + (VT)2.0 * oo2ze * v13_3_1;
            const VT v23_6_1 = QCx * v23_3_1 + WQx * v23_3_2 + (VT)2.0 * oo2ze * v13_3_2;
            const VT v23_6_2 = QCx * v23_3_2 + WQx * v23_3_3 + (VT)2.0 * oo2ze * v13_3_3;
            const VT v24_6_0 = QCx * v24_3_0 + WQx * v24_3_1 + (VT)2.0 * oo2ze * v15_3_1;
            const VT v24_6_1 = QCx * v24_3_1 + WQx * v24_3_2 + (VT)2.0 * oo2ze * v15_3_2;
            const VT v24_6_2 = QCx * v24_3_2 + WQx * v24_3_3 + (VT)2.0 * oo2ze * v15_3_3;
            const VT v25_6_0 = QCx * v25_3_0 + WQx * v25_3_1 + (VT)2.0 * oo2ze * v14_3_1;
            const VT v25_6_1 = QCx * v25_3_1 + WQx * v25_3_2 + (VT)2.0 * oo2ze * v14_3_2;
            const VT v25_6_2 = QCx * v25_3_2 + WQx * v25_3_3 + (VT)2.0 * oo2ze * v14_3_3;
            const VT v26_6_0 = QCx * v26_3_0 + WQx * v26_3_1 + (VT)1.0 * oo2ze * v16_3_1;
            const VT v26_6_1 = QCx * v26_3_1 + WQx * v26_3_2 + (VT)1.0 * oo2ze * v16_3_2;
            const VT v26_6_2 = QCx * v26_3_2 + WQx * v26_3_3 + (VT)1.0 * oo2ze * v16_3_3;
            const VT v27_6_0 = QCx * v27_3_0 + WQx * v27_3_1 + (VT)1.0 * oo2ze * v17_3_1;
            const VT v27_6_1 = QCx * v27_3_1 + WQx * v27_3_2 + (VT)1.0 * oo2ze * v17_3_2;
            const VT v27_6_2 = QCx * v27_3_2 + WQx * v27_3_3 + (VT)1.0 * oo2ze * v17_3_3;
            const VT v28_6_0 = QCx * v28_3_0 + WQx * v28_3_1 + (VT)1.0 * oo2ze * v18_3_1;
            const VT v28_6_1 = QCx * v28_3_1 + WQx * v28_3_2 + (VT)1.0 * oo2ze * v18_3_2;
            const VT v28_6_2 = QCx * v28_3_2 + WQx * v28_3_3 + (VT)1.0 * oo2ze * v18_3_3;
            const VT v29_6_0 = QCx * v29_3_0 + WQx * v29_3_1 + (VT)1.0 * oo2ze * v19_3_1;
            const VT v29_6_1 = QCx * v29_3_1 + WQx * v29_3_2 + (VT)1.0 * oo2ze * v19_3_2;
            const VT v29_6_2 = QCx * v29_3_2 + WQx * v29_3_3 + (VT)1.0 * oo2ze * v19_3_3;
            const VT v30_6_0 = QCx * v30_3_0 + WQx * v30_3_1;
            const VT v30_6_1 = QCx * v30_3_1 + WQx * v30_3_2;
            const VT v30_6_2 = QCx * v30_3_2 + WQx * v30_3_3;
            const VT v31_6_0 = QCx * v31_3_0 + WQx * v31_3_1;
            const VT v31_6_1 = QCx * v31_3_1 + WQx * v31_3_2;
            const VT v31_6_2 = QCx * v31_3_2 + WQx * v31_3_3;
            const VT v32_6_0 = QCx * v32_3_0 + WQx * v32_3_1;
            const VT v32_6_1 = QCx * v32_3_1 + WQx * v32_3_2;
            const VT v32_6_2 = QCx * v32_3_2 + WQx * v32_3_3;
            const VT v33_6_0 = QCx * v33_3_0 + WQx * v33_3_1;
            const VT v33_6_1 = QCx * v33_3_1 + WQx * v33_3_2;
            const VT v33_6_2 = QCx * v33_3_2 + WQx * v33_3_3;
            const VT v34_6_0 = QCx * v34_3_0 + WQx * v34_3_1;
            const VT v34_6_1 = QCx * v34_3_1 + WQx * v34_3_2;
            const VT v34_6_2 = QCx * v34_3_2 + WQx * v34_3_3;
            const VT v0_7_2 = QCy * v0_2_2 + WQy * v0_2_3 + (VT)1.0 * oo2e * (v0_0_2 - rho_e * v0_0_3);
            const VT v1_7_1 = QCy * v1_2_1 + WQy * v1_2_2 + (VT)1.0 * oo2e * (v1_0_1 - rho_e * v1_0_2);
            const VT v1_7_2 = QCy * v1_2_2 + WQy * v1_2_3 + (VT)1.0 * oo2e * (v1_0_2 - rho_e * v1_0_3);
            const VT v2_7_1 = QCy * v2_2_1 + WQy * v2_2_2 + (VT)1.0 * oo2ze * v0_2_2 + (VT)1.0 * oo2e * (v2_0_1 - rho_e * v2_0_2);
            const VT v2_7_2 = QCy * v2_2_2 + WQy * v2_2_3 + (VT)1.0 * oo2ze * v0_2_3 + (VT)1.0 * oo2e * (v2_0_2 - rho_e * v2_0_3);
            const VT v3_7_1 = QCy * v3_2_1 + WQy * v3_2_2 + (VT)1.0 * oo2e * (v3_0_1 - rho_e * v3_0_2);
            const VT v3_7_2 = QCy * v3_2_2 + WQy * v3_2_3 + (VT)1.0 * oo2e * (v3_0_2 - rho_e * v3_0_3);
            const VT v4_7_0 = QCy * v4_2_0 + WQy * v4_2_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v4_7_1 = QCy * v4_2_1 + WQy * v4_2_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v4_7_2 = QCy * v4_2_2 + WQy * v4_2_3 + (VT)1.0 * oo2e * (v4_0_2 - rho_e * v4_0_3);
            const VT v5_7_0 = QCy * v5_2_0 + WQy * v5_2_1 + (VT)1.0 * oo2ze * v1_2_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v5_7_1 = QCy * v5_2_1 + WQy * v5_2_2 + (VT)1.0 * oo2ze * v1_2_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v5_7_2 = QCy * v5_2_2 + WQy * v5_2_3 + (VT)1.0 * oo2ze * v1_2_3 + (VT)1.0 * oo2e * (v5_0_2 - rho_e * v5_0_3);
            const VT v6_7_0 = QCy * v6_2_0 + WQy * v6_2_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v6_7_1 = QCy * v6_2_1 + WQy * v6_2_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v6_7_2 = QCy * v6_2_2 + WQy * v6_2_3 + (VT)1.0 * oo2e * (v6_0_2 - rho_e * v6_0_3);
            const VT v7_7_0 = QCy * v7_2_0 + WQy * v7_2_1 + (VT)2.0 * oo2ze * v2_2_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v7_7_1 = QCy * v7_2_1 + WQy * v7_2_2 + (VT)2.0 * oo2ze * v2_2_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v7_7_2 = QCy * v7_2_2 + WQy * v7_2_3 + (VT)2.0 * oo2ze * v2_2_3 + (VT)1.0 * oo2e * (v7_0_2 - rho_e * v7_0_3);
            const VT v8_7_0 = QCy * v8_2_0 + WQy * v8_2_1 + (VT)1.0 * oo2ze * v3_2_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v8_7_1 = QCy * v8_2_1 + WQy * v8_2_2 + (VT)1.0 * oo2ze * v3_2_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v8_7_2 = QCy * v8_2_2 + WQy * v8_2_3 + (VT)1.0 * oo2ze * v3_2_3 + (VT)1.0 * oo2e * (v8_0_2 - rho_e * v8_0_3);
            const VT v9_7_0 = QCy * v9_2_0 + WQy * v9_2_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v9_7_1 = QCy * v9_2_1 + WQy * v9_2_2 + (VT)1.0 * oo2e * (v9_0_1 - rho_e * v9_0_2);
            const VT v9_7_2 = QCy * v9_2_2 + WQy * v9_2_3 + (VT)1.0 * oo2e * (v9_0_2 - rho_e * v9_0_3);
            const VT v10_7_0 = QCy * v10_2_0 + WQy * v10_2_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v10_7_1 = QCy * v10_2_1 + WQy * v10_2_2 + (VT)1.0 * oo2e * (v10_0_1 - rho_e * v10_0_2);
            const VT v10_7_2 = QCy * v10_2_2 + WQy * v10_2_3 + (VT)1.0 * oo2e * (v10_0_2 - rho_e * v10_0_3);
            const VT v11_7_0 = QCy * v11_2_0 + WQy * v11_2_1 + (VT)1.0 * oo2ze * v4_2_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v11_7_1 = QCy * v11_2_1 + WQy * v11_2_2 + (VT)1.0 * oo2ze * v4_2_2 + (VT)1.0 * oo2e * (v11_0_1 - rho_e * v11_0_2);
            const VT v11_7_2 = QCy * v11_2_2 + WQy * v11_2_3 + (VT)1.0 * oo2ze * v4_2_3 + (VT)1.0 * oo2e * (v11_0_2 - rho_e * v11_0_3);
            const VT v12_7_0 = QCy * v12_2_0 + WQy * v12_2_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v12_7_1 = QCy * v12_2_1 + WQy * v12_2_2 + (VT)1.0 * oo2e * (v12_0_1 - rho_e * v12_0_2);
            const VT v12_7_2 = QCy * v12_2_2 + WQy * v12_2_3 + (VT)1.0 * oo2e * (v12_0_2 - rho_e * v12_0_3);
            const VT v13_7_0 = QCy * v13_2_0 + WQy * v13_2_1 + (VT)2.0 * oo2ze * v5_2_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v13_7_1 = QCy * v13_2_1 + WQy * v13_2_2 + (VT)2.0 * oo2ze * v5_2_2 + (VT)1.0 * oo2e * (v13_0_1 - rho_e * v13_0_2);
            const VT v13_7_2 = QCy * v13_2_2 + WQy * v13_2_3 + (VT)2.0 * oo2ze * v5_2_3 + (VT)1.0 * oo2e * (v13_0_2 - rho_e * v13_0_3);
            const VT v14_7_0 = QCy * v14_2_0 + WQy * v14_2_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v14_7_1 = QCy * v14_2_1 + WQy * v14_2_2 + (VT)1.0 * oo2e * (v14_0_1 - rho_e * v14_0_2);
            const VT v14_7_2 = QCy * v14_2_2 + WQy * v14_2_3 + (VT)1.0 * oo2e * (v14_0_2 - rho_e * v14_0_3);
            const VT v15_7_0 = QCy * v15_2_0 + WQy * v15_2_1 + (VT)1.0 * oo2ze * v6_2_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v15_7_1 = QCy * v15_2_1 + WQy * v15_2_2 + (VT)1.0 * oo2ze * v6_2_2 + (VT)1.0 * oo2e * (v15_0_1 - rho_e * v15_0_2);
            const VT v15_7_2 = QCy * v15_2_2 + WQy * v15_2_3 + (VT)1.0 * oo2ze * v6_2_3 + (VT)1.0 * oo2e * (v15_0_2 - rho_e * v15_0_3);
            const VT v16_7_0 = QCy * v16_2_0 + WQy * v16_2_1 + (VT)3.0 * oo2ze * v7_2_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v16_7_1 = QCy * v16_2_1 + WQy * v16_2_2 + (VT)3.0 * oo2ze * v7_2_2 + (VT)1.0 * oo2e * (v16_0_1 - rho_e * v16_0_2);
            const VT v16_7_2 = QCy * v16_2_2 + WQy * v16_2_3 + (VT)3.0 * oo2ze * v7_2_3 + (VT)1.0 * oo2e * (v16_0_2 - rho_e * v16_0_3);
            const VT v17_7_0 = QCy * v17_2_0 + WQy * v17_2_1 + (VT)2.0 * oo2ze * v8_2_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v17_7_1 = QCy * v17_2_1 + WQy * v17_2_2 + (VT)2.0 * oo2ze * v8_2_2 + (VT)1.0 * oo2e * (v17_0_1 - rho_e * v17_0_2);
            const VT v17_7_2 = QCy * v17_2_2 + WQy * v17_2_3 + (VT)2.0 * oo2ze * v8_2_3 + (VT)1.0 * oo2e * (v17_0_2 - rho_e * v17_0_3);
            const VT v18_7_0 = QCy * v18_2_0 + WQy * v18_2_1 + (VT)1.0 * oo2ze * v9_2_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v18_7_1 = QCy * v18_2_1 + WQy * v18_2_2 + (VT)1.0 * oo2ze * v9_2_2 + (VT)1.0 * oo2e * (v18_0_1 - rho_e * v18_0_2);
            const VT v18_7_2 = QCy * v18_2_2 + WQy * v18_2_3 + (VT)1.0 * oo2ze * v9_2_3 + (VT)1.0 * oo2e * (v18_0_2 - rho_e * v18_0_3);
            const VT v19_7_0 = QCy * v19_2_0 + WQy * v19_2_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v19_7_1 = QCy * v19_2_1 + WQy * v19_2_2 + (VT)1.0 * oo2e * (v19_0_1 - rho_e * v19_0_2);
            const VT v19_7_2 = QCy * v19_2_2 + WQy * v19_2_3 + (VT)1.0 * oo2e * (v19_0_2 - rho_e * v19_0_3);
            const VT v20_7_0 = QCy * v20_2_0 + WQy * v20_2_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v20_7_1 = QCy * v20_2_1 + WQy * v20_2_2 + (VT)1.0 * oo2e * (v20_0_1 - rho_e * v20_0_2);
            const VT v20_7_2 = QCy * v20_2_2 + WQy * v20_2_3 + (VT)1.0 * oo2e * (v20_0_2 - rho_e * v20_0_3);
            const VT v21_7_0 = QCy * v21_2_0 + WQy * v21_2_1 + (VT)1.0 * oo2ze * v10_2_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v21_7_1 = QCy * v21_2_1 + WQy * v21_2_2 + (VT)1.0 * oo2ze * v10_2_2 + (VT)1.0 * oo2e * (v21_0_1 - rho_e * v21_0_2);
            const VT v21_7_2 = QCy * v21_2_2 + WQy * v21_2_3 + (VT)1.0 * oo2ze * v10_2_3 + (VT)1.0 * oo2e * (v21_0_2 - rho_e * v21_0_3);
            const VT v22_7_0 = QCy * v22_2_0 + WQy * v22_2_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v22_7_1 = QCy * v22_2_1 + WQy * v22_2_2 + (VT)1.0 * oo2e * (v22_0_1 - rho_e * v22_0_2);
            const VT v22_7_2 = QCy * v22_2_2 + WQy * v22_2_3 + (VT)1.0 * oo2e * (v22_0_2 - rho_e * v22_0_3);
            const VT v23_7_0 = QCy * v23_2_0 + WQy * v23_2_1 + (VT)2.0 * oo2ze * v11_2_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v23_7_1 = QCy * v23_2_1 + WQy * v23_2_2 + (VT)2.0 * oo2ze * v11_2_2 + (VT)1.0 * oo2e * (v23_0_1 - rho_e * v23_0_2);
            const VT v23_7_2 = QCy * v23_2_2 + WQy * v23_2_3 + (VT)2.0 * oo2ze * v11_2_3 + (VT)1.0 * oo2e * (v23_0_2 - rho_e * v23_0_3);
            const VT v24_7_0 = QCy * v24_2_0 + WQy * v24_2_1 + (VT)1.0 * oo2ze * v12_2_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v24_7_1 = QCy * v24_2_1 + WQy * v24_2_2 + (VT)1.0 * oo2ze * v12_2_2 + (VT)1.0 * oo2e * (v24_0_1 - rho_e * v24_0_2);
            const VT v24_7_2 = QCy * v24_2_2 + WQy * v24_2_3 + (VT)1.0 * oo2ze * v12_2_3 + (VT)1.0 * oo2e * (v24_0_2 - rho_e * v24_0_3);
            const VT v25_7_0 = QCy * v25_2_0 + WQy * v25_2_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v25_7_1 = QCy * v25_2_1 + WQy * v25_2_2 + (VT)1.0 * oo2e * (v25_0_1 - rho_e * v25_0_2);
            const VT v25_7_2 = QCy * v25_2_2 + WQy * v25_2_3 + (VT)1.0 * oo2e * (v25_0_2 - rho_e * v25_0_3);
            const VT v26_7_0 = QCy * v26_2_0 + WQy * v26_2_1 + (VT)3.0 * oo2ze * v13_2_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v26_7_1 = QCy * v26_2_1 + WQy * v26_2_2 + (VT)3.0 * oo2ze * v13_2_2 + (VT)1.0 * oo2e * (v26_0_1 - rho_e * v26_0_2);
            const VT v26_7_2 = QCy * v26_2_2 + WQy * v26_2_3 + (VT)3.0 * oo2ze * v13_2_3 + (VT)1.0 * oo2e * (v26_0_2 - rho_e * v26_0_3);
            const VT v27_7_0 = QCy * v27_2_0 + WQy * v27_2_1 + (VT)2.0 * oo2ze * v15_2_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v27_7_1 = QCy * v27_2_1 + WQy * v27_2_2 + (VT)2.0 * oo2ze * v15_2_2 + (VT)1.0 * oo2e * (v27_0_1 - rho_e * v27_0_2);
            const VT v27_7_2 = QCy * v27_2_2 + WQy * v27_2_3 + (VT)2.0 * oo2ze * v15_2_3 + (VT)1.0 * oo2e * (v27_0_2 - rho_e * v27_0_3);
            const VT v28_7_0 = QCy * v28_2_0 + WQy * v28_2_1 + (VT)1.0 * oo2ze * v14_2_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v28_7_1 = QCy * v28_2_1 + WQy * v28_2_2 + (VT)1.0 * oo2ze * v14_2_2 + (VT)1.0 * oo2e * (v28_0_1 - rho_e * v28_0_2);
            const VT v28_7_2 = QCy * v28_2_2 + WQy * v28_2_3 + (VT)1.0 * oo2ze * v14_2_3 + (VT)1.0 * oo2e * (v28_0_2 - rho_e * v28_0_3);
            const VT v29_7_0 = QCy * v29_2_0 + WQy * v29_2_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v29_7_1 = QCy * v29_2_1 + WQy * v29_2_2 + (VT)1.0 * oo2e * (v29_0_1 - rho_e * v29_0_2);
            const VT v29_7_2 = QCy * v29_2_2 + WQy * v29_2_3 + (VT)1.0 * oo2e * (v29_0_2 - rho_e * v29_0_3);
            const VT v30_7_0 = QCy * v30_2_0 + WQy * v30_2_1 + (VT)4.0 * oo2ze * v16_2_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v30_7_1 = QCy * v30_2_1 + WQy * v30_2_2 + (VT)4.0 * oo2ze * v16_2_2 + (VT)1.0 * oo2e * (v30_0_1 - rho_e * v30_0_2);
            const VT v30_7_2 = QCy * v30_2_2 + WQy * v30_2_3 + (VT)4.0 * oo2ze * v16_2_3 + (VT)1.0 * oo2e * (v30_0_2 - rho_e * v30_0_3);
            const VT v31_7_0 = QCy * v31_2_0 + WQy * v31_2_1 + (VT)3.0 * oo2ze * v17_2_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v31_7_1 = QCy * v31_2_1 + WQy * v31_2_2 + (VT)3.0 * oo2ze * v17_2_2 + (VT)1.0 * oo2e * (v31_0_1 - rho_e * v31_0_2);
            const VT v31_7_2 = QCy * v31_2_2 + WQy * v31_2_3 + (VT)3.0 * oo2ze * v17_2_3 + (VT)1.0 * oo2e * (v31_0_2 - rho_e * v31_0_3);
            const VT v32_7_0 = QCy * v32_2_0 + WQy * v32_2_1 + (VT)2.0 * oo2ze * v18_2_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v32_7_1 = QCy * v32_2_1 + WQy * v32_2_2 + (VT)2.0 * oo2ze * v18_2_2 + (VT)1.0 * oo2e * (v32_0_1 - rho_e * v32_0_2);
            const VT v32_7_2 = QCy * v32_2_2 + WQy * v32_2_3 + (VT)2.0 * oo2ze * v18_2_3 + (VT)1.0 * oo2e * (v32_0_2 - rho_e * v32_0_3);
            const VT v33_7_0 = QCy * v33_2_0 + WQy * v33_2_1 + (VT)1.0 * oo2ze * v19_2_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v33_7_1 = QCy * v33_2_1 + WQy * v33_2_2 + (VT)1.0 * oo2ze * v19_2_2 + (VT)1.0 * oo2e * (v33_0_1 - rho_e * v33_0_2);
            const VT v33_7_2 = QCy * v33_2_2 + WQy * v33_2_3 + (VT)1.0 * oo2ze * v19_2_3 + (VT)1.0 * oo2e * (v33_0_2 - rho_e * v33_0_3);
            const VT v34_7_0 = QCy * v34_2_0 + WQy * v34_2_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
            const VT v34_7_1 = QCy * v34_2_1 + WQy * v34_2_2 + (VT)1.0 * oo2e * (v34_0_1 - rho_e * v34_0_2);
            const VT v34_7_2 = QCy * v34_2_2 + WQy * v34_2_3 + (VT)1.0 * oo2e * (v34_0_2 - rho_e * v34_0_3);
            const VT v0_8_2 = QCy * v0_3_2 + WQy * v0_3_3;
            const VT v1_8_1 = QCy * v1_3_1 + WQy * v1_3_2;
            const VT v1_8_2 = QCy * v1_3_2 + WQy * v1_3_3;
            const VT v2_8_1 = QCy * v2_3_1 + WQy * v2_3_2 + (VT)1.0 * oo2ze * v0_3_2;
            const VT v2_8_2 = QCy * v2_3_2 + WQy * v2_3_3 + (VT)1.0 * oo2ze * v0_3_3;
            const VT v3_8_1 = QCy * v3_3_1 + WQy * v3_3_2;
            const VT v3_8_2 = QCy * v3_3_2 + WQy * v3_3_3;
            const VT v4_8_0 = QCy * v4_3_0 + WQy * v4_3_1;
            const VT v4_8_1 = QCy * v4_3_1 + WQy * v4_3_2;
            const VT v4_8_2 = QCy * v4_3_2 + WQy * v4_3_3;
            const VT v5_8_0 = QCy * v5_3_0 + WQy * v5_3_1 + (VT)1.0 * oo2ze * v1_3_1;
            const VT v5_8_1 = QCy * v5_3_1 + WQy * v5_3_2 + (VT)1.0 * oo2ze * v1_3_2;
            const VT v5_8_2 = QCy * v5_3_2 + WQy * v5_3_3 + (VT)1.0 * oo2ze * v1_3_3;
            const VT v6_8_0 = QCy * v6_3_0 + WQy * v6_3_1;
            const VT v6_8_1 = QCy * v6_3_1 + WQy * v6_3_2;
            const VT v6_8_2 = QCy * v6_3_2 + WQy * v6_3_3;
            const VT v7_8_0 = QCy * v7_3_0 + WQy * v7_3_1 + (VT)2.0 * oo2ze * v2_3_1;
            const VT v7_8_1 = QCy * v7_3_1 + WQy * v7_3_2 + (VT)2.0 * oo2ze * v2_3_2;
            const VT v7_8_2 = QCy * v7_3_2 + WQy * v7_3_3 + (VT)2.0 * oo2ze * v2_3_3;
            const VT v8_8_0 = QCy * v8_3_0 + WQy * v8_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v8_8_1 = QCy * v8_3_1 + WQy * v8_3_2 + (VT)1.0 * oo2ze * v3_3_2;
            const VT v8_8_2 = QCy * v8_3_2 + WQy * v8_3_3 + (VT)1.0 * oo2ze * v3_3_3;
            const VT v9_8_0 = QCy * v9_3_0 + WQy * v9_3_1;
            const VT v9_8_1 = QCy * v9_3_1 + WQy * v9_3_2;
            const VT v9_8_2 = QCy * v9_3_2 + WQy * v9_3_3;
            const VT v10_8_0 = QCy * v10_3_0 + WQy * v10_3_1;
            const VT v10_8_1 = QCy * v10_3_1 + WQy * v10_3_2;
            const VT v10_8_2 = QCy * v10_3_2 + WQy * v10_3_3;
            const VT v11_8_0 = QCy * v11_3_0 + WQy * v11_3_1 + (VT)1.0 * oo2ze * v4_3_1;
            const VT v11_8_1 = QCy * v11_3_1 + WQy * v11_3_2 + (VT)1.0 * oo2ze * v4_3_2;
            const VT v11_8_2 = QCy * v11_3_2 + WQy * v11_3_3 + (VT)1.0 * oo2ze * v4_3_3;
            const VT v12_8_0 = QCy * v12_3_0 + WQy * v12_3_1;
            const VT v12_8_1 = QCy * v12_3_1 + WQy * v12_3_2;
            const VT v12_8_2 = QCy * v12_3_2 + WQy * v12_3_3;
            const VT v13_8_0 = QCy * v13_3_0 + WQy * v13_3_1 + (VT)2.0 * oo2ze * v5_3_1;
            const VT v13_8_1 = QCy * v13_3_1 + WQy * v13_3_2 + (VT)2.0 * oo2ze * v5_3_2;
            const VT v13_8_2 = QCy * v13_3_2 + WQy * v13_3_3 + (VT)2.0 * oo2ze * v5_3_3;
            const VT v14_8_0 = QCy * v14_3_0 + WQy * v14_3_1;
            const VT v14_8_1 = QCy * v14_3_1 + WQy * v14_3_2;
            const VT v14_8_2 = QCy * v14_3_2 + WQy * v14_3_3;
            const VT v15_8_0 = QCy * v15_3_0 + WQy * v15_3_1 + (VT)1.0 * oo2ze * v6_3_1;
            const VT v15_8_1 = QCy * v15_3_1 + WQy * v15_3_2 + (VT)1.0 * oo2ze * v6_3_2;
            const VT v15_8_2 = QCy * v15_3_2 + WQy * v15_3_3 + (VT)1.0 * oo2ze * v6_3_3;
            const VT v16_8_0 = QCy * v16_3_0 + WQy * v16_3_1 + (VT)3.0 * oo2ze * v7_3_1;
            const VT v16_8_1 = QCy * v16_3_1 + WQy * v16_3_2 + (VT)3.0 * oo2ze * v7_3_2;
            const VT v16_8_2 = QCy * v16_3_2 + WQy * v16_3_3 + (VT)3.0 * oo2ze * v7_3_3;
            const VT v17_8_0 = QCy * v17_3_0 + WQy * v17_3_1 + (VT)2.0 * oo2ze * v8_3_1;
            const VT v17_8_1 = QCy * v17_3_1 + WQy * v17_3_2 + (VT)2.0 * oo2ze * v8_3_2;
            const VT v17_8_2 = QCy * v17_3_2 + WQy * v17_3_3 + (VT)2.0 * oo2ze * v8_3_3;
            const VT v18_8_0 = QCy * v18_3_0 + WQy * v18_3_1 + (VT)1.0 * oo2ze * v9_3_1;
            const VT v18_8_1 = QCy * v18_3_1 + WQy * v18_3_2 + (VT)1.0 * oo2ze * v9_3_2;
            const VT v18_8_2 = QCy * v18_3_2 + WQy * v18_3_3 + (VT)1.0 * oo2ze * v9_3_3;
            const VT v19_8_0 = QCy * v19_3_0 + WQy * v19_3_1;
            const VT v19_8_1 = QCy * v19_3_1 + WQy * v19_3_2;
            const VT v19_8_2 = QCy * v19_3_2 + WQy * v19_3_3;
            const VT v20_8_0 = QCy * v20_3_0 + WQy * v20_3_1;
            const VT v20_8_1 = QCy * v20_3_1 + WQy * v20_3_2;
            const VT v20_8_2 = QCy * v20_3_2 + WQy * v20_3_3;
            const VT v21_8_0 = QCy * v21_3_0 + WQy * v21_3_1 + (VT)1.0 * oo2ze * v10_3_1;
            const VT v21_8_1 = QCy * v21_3_1 + WQy * v21_3_2 + (VT)1.0 * oo2ze * v10_3_2;
            const VT v21_8_2 = QCy * v21_3_2 + WQy * v21_3_3 + (VT)1.0 * oo2ze * v10_3_3;
            const VT v22_8_0 = QCy * v22_3_0 + WQy * v22_3_1;
            const VT v22_8_1 = QCy * v22_3_1 + WQy * v22_3_2;
            const VT v22_8_2 = QCy * v22_3_2 + WQy * v22_3_3;
            const VT v23_8_0 = QCy * v23_3_0 + WQy * v23_3_1 + (VT)2.0 * oo2ze * v11_3_1;
            const VT v23_8_1 = QCy * v23_3_1 + WQy * v23_3_2 + (VT)2.0 * oo2ze * v11_3_2;
            const VT v23_8_2 = QCy * v23_3_2 + WQy * v23_3_3 + (VT)2.0 * oo2ze * v11_3_3;
            const VT v24_8_0 = QCy * v24_3_0 + WQy * v24_3_1 + (VT)1.0 * oo2ze * v12_3_1;
            const VT v24_8_1 = QCy * v24_3_1 + WQy * v24_3_2 + (VT)1.0 * oo2ze * v12_3_2;
            const VT v24_8_2 = QCy * v24_3_2 + WQy * v24_3_3 + (VT)1.0 * oo2ze * v12_3_3;
            const VT v25_8_0 = QCy * v25_3_0 + WQy * v25_3_1;
            const VT v25_8_1 = QCy * v25_3_1 + WQy * v25_3_2;
            const VT v25_8_2 = QCy * v25_3_2 + WQy * v25_3_3;
            const VT v26_8_0 = QCy * v26_3_0 + WQy * v26_3_1 + (VT)3.0 * oo2ze * v13_3_1;
            const VT v26_8_1 = QCy * v26_3_1 + WQy * v26_3_2 + (VT)3.0 * oo2ze * v13_3_2;
            const VT v26_8_2 = QCy * v26_3_2 + WQy * v26_3_3 + (VT)3.0 * oo2ze * v13_3_3;
            const VT v27_8_0 = QCy * v27_3_0 + WQy * v27_3_1 + (VT)2.0 * oo2ze * v15_3_1;
            const VT v27_8_1 = QCy * v27_3_1 + WQy * v27_3_2 + (VT)2.0 * oo2ze * v15_3_2;
            const VT v27_8_2 = QCy * v27_3_2 + WQy * v27_3_3 + (VT)2.0 * oo2ze * v15_3_3;
            const VT v28_8_0 = QCy * v28_3_0 + WQy * v28_3_1 + (VT)1.0 * oo2ze * v14_3_1;
            const VT v28_8_1 = QCy * v28_3_1 + WQy * v28_3_2 + (VT)1.0 * oo2ze * v14_3_2;
            const VT v28_8_2 = QCy * v28_3_2 + WQy * v28_3_3 + (VT)1.0 * oo2ze * v14_3_3;
            const VT v29_8_0 = QCy * v29_3_0 + WQy * v29_3_1;
            const VT v29_8_1 = QCy * v29_3_1 + WQy * v29_3_2;
            const VT v29_8_2 = QCy * v29_3_2 + WQy * v29_3_3;
            const VT v30_8_0 = QCy * v30_3_0 + WQy * v30_3_1 + (VT)4.0 * oo2ze * v16_3_1;
            const VT v30_8_1 = QCy * v30_3_1 + WQy * v30_3_2 + (VT)4.0 * oo2ze * v16_3_2;
            const VT v30_8_2 = QCy * v30_3_2 + WQy * v30_3_3 + (VT)4.0 * oo2ze * v16_3_3;
            const VT v31_8_0 = QCy * v31_3_0 + WQy * v31_3_1 + (VT)3.0 * oo2ze * v17_3_1;
            const VT v31_8_1 = QCy * v31_3_1 + WQy * v31_3_2 + (VT)3.0 * oo2ze * v17_3_2;
            const VT v31_8_2 = QCy * v31_3_2 + WQy * v31_3_3 + (VT)3.0 * oo2ze * v17_3_3;
            const VT v32_8_0 = QCy * v32_3_0 + WQy * v32_3_1 + (VT)2.0 * oo2ze * v18_3_1;
            const VT v32_8_1 = QCy * v32_3_1 + WQy * v32_3_2 + (VT)2.0 * oo2ze * v18_3_2;
            const VT v32_8_2 = QCy * v32_3_2 + WQy * v32_3_3 + (VT)2.0 * oo2ze * v18_3_3;
            const VT v33_8_0 = QCy * v33_3_0 + WQy * v33_3_1 + (VT)1.0 * oo2ze * v19_3_1;
            const VT v33_8_1 = QCy * v33_3_1 + WQy * v33_3_2 + (VT)1.0 * oo2ze * v19_3_2;
            const VT v33_8_2 = QCy * v33_3_2 + WQy * v33_3_3 + (VT)1.0 * oo2ze * v19_3_3;
            const VT v34_8_0 = QCy * v34_3_0 + WQy * v34_3_1;
            const VT v34_8_1 = QCy * v34_3_1 + WQy * v34_3_2;
            const VT v34_8_2 = QCy * v34_3_2 + WQy * v34_3_3;
            const VT v0_9_2 = QCz * v0_3_2 + WQz * v0_3_3 + (VT)1.0 * oo2e * (v0_0_2 - rho_e * v0_0_3);
            const VT v1_9_1 = QCz * v1_3_1 + WQz * v1_3_2 + (VT)1.0 * oo2e * (v1_0_1 - rho_e * v1_0_2);
            const VT v1_9_2 = QCz * v1_3_2 + WQz * v1_3_3 + (VT)1.0 * oo2e * (v1_0_2 - rho_e * v1_0_3);
            const VT v2_9_1 = QCz * v2_3_1 + WQz * v2_3_2 + (VT)1.0 * oo2e * (v2_0_1 - rho_e * v2_0_2);
            const VT v2_9_2 = QCz * v2_3_2 + WQz * v2_3_3 + (VT)1.0 * oo2e * (v2_0_2 - rho_e * v2_0_3);
            const VT v3_9_1 = QCz * v3_3_1 + WQz * v3_3_2 + (VT)1.0 * oo2ze * v0_3_2 + (VT)1.0 * oo2e * (v3_0_1 - rho_e * v3_0_2);
            const VT v3_9_2 = QCz * v3_3_2 + WQz * v3_3_3 + (VT)1.0 * oo2ze * v0_3_3 + (VT)1.0 * oo2e * (v3_0_2 - rho_e * v3_0_3);
            const VT v4_9_0 = QCz * v4_3_0 + WQz * v4_3_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v4_9_1 = QCz * v4_3_1 + WQz * v4_3_2 + (VT)1.0 * oo2e * (v4_0_1 - rho_e * v4_0_2);
            const VT v4_9_2 = QCz * v4_3_2 + WQz * v4_3_3 + (VT)1.0 * oo2e * (v4_0_2 - rho_e * v4_0_3);
            const VT v5_9_0 = QCz * v5_3_0 + WQz * v5_3_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v5_9_1 = QCz * v5_3_1 + WQz * v5_3_2 + (VT)1.0 * oo2e * (v5_0_1 - rho_e * v5_0_2);
            const VT v5_9_2 = QCz * v5_3_2 + WQz * v5_3_3 + (VT)1.0 * oo2e * (v5_0_2 - rho_e * v5_0_3);
            const VT v6_9_0 = QCz * v6_3_0 + WQz * v6_3_1 + (VT)1.0 * oo2ze * v1_3_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v6_9_1 = QCz * v6_3_1 + WQz * v6_3_2 + (VT)1.0 * oo2ze * v1_3_2 + (VT)1.0 * oo2e * (v6_0_1 - rho_e * v6_0_2);
            const VT v6_9_2 = QCz * v6_3_2 + WQz * v6_3_3 + (VT)1.0 * oo2ze * v1_3_3 + (VT)1.0 * oo2e * (v6_0_2 - rho_e * v6_0_3);
            const VT v7_9_0 = QCz * v7_3_0 + WQz * v7_3_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v7_9_1 = QCz * v7_3_1 + WQz * v7_3_2 + (VT)1.0 * oo2e * (v7_0_1 - rho_e * v7_0_2);
            const VT v7_9_2 = QCz * v7_3_2 + WQz * v7_3_3 + (VT)1.0 * oo2e * (v7_0_2 - rho_e * v7_0_3);
            const VT v8_9_0 = QCz * v8_3_0 + WQz * v8_3_1 + (VT)1.0 * oo2ze * v2_3_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v8_9_1 = QCz * v8_3_1 + WQz * v8_3_2 + (VT)1.0 * oo2ze * v2_3_2 + (VT)1.0 * oo2e * (v8_0_1 - rho_e * v8_0_2);
            const VT v8_9_2 = QCz * v8_3_2 + WQz * v8_3_3 + (VT)1.0 * oo2ze * v2_3_3 + (VT)1.0 * oo2e * (v8_0_2 - rho_e * v8_0_3);
            const VT v9_9_0 = QCz * v9_3_0 + WQz * v9_3_1 + (VT)2.0 * oo2ze * v3_3_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v9_9_1 = QCz * v9_3_1 + WQz * v9_3_2 + (VT)2.0 * oo2ze * v3_3_2 + (VT)1.0 * oo2e * (v9_0_1 - rho_e * v9_0_2);
            const VT v9_9_2 = QCz * v9_3_2 + WQz * v9_3_3 + (VT)2.0 * oo2ze * v3_3_3 + (VT)1.0 * oo2e * (v9_0_2 - rho_e * v9_0_3);
            const VT v10_9_0 = QCz * v10_3_0 + WQz * v10_3_1 + (VT)1.0 * oo2e * (v10_0_0 - rho_e * v10_0_1);
            const VT v10_9_1 = QCz * v10_3_1 + WQz * v10_3_2 + (VT)1.0 * oo2e * (v10_0_1 - rho_e * v10_0_2);
            const VT v10_9_2 = QCz * v10_3_2 + WQz * v10_3_3 + (VT)1.0 * oo2e * (v10_0_2 - rho_e * v10_0_3);
            const VT v11_9_0 = QCz * v11_3_0 + WQz * v11_3_1 + (VT)1.0 * oo2e * (v11_0_0 - rho_e * v11_0_1);
            const VT v11_9_1 = QCz * v11_3_1 + WQz * v11_3_2 + (VT)1.0 * oo2e * (v11_0_1 - rho_e * v11_0_2);
            const VT v11_9_2 = QCz * v11_3_2 + WQz * v11_3_3 + (VT)1.0 * oo2e * (v11_0_2 - rho_e * v11_0_3);
            const VT v12_9_0 = QCz * v12_3_0 + WQz * v12_3_1 + (VT)1.0 * oo2ze * v4_3_1 + (VT)1.0 * oo2e * (v12_0_0 - rho_e * v12_0_1);
            const VT v12_9_1 = QCz * v12_3_1 + WQz * v12_3_2 + (VT)1.0 * oo2ze * v4_3_2 + (VT)1.0 * oo2e * (v12_0_1 - rho_e * v12_0_2);
            const VT v12_9_2 = QCz * v12_3_2 + WQz * v12_3_3 + (VT)1.0 * oo2ze * v4_3_3 + (VT)1.0 * oo2e * (v12_0_2 - rho_e * v12_0_3);
            const VT v13_9_0 = QCz * v13_3_0 + WQz * v13_3_1 + (VT)1.0 * oo2e * (v13_0_0 - rho_e * v13_0_1);
            const VT v13_9_1 = QCz * v13_3_1 + WQz * v13_3_2 + (VT)1.0 * oo2e * (v13_0_1 - rho_e * v13_0_2);
            const VT v13_9_2 = QCz * v13_3_2 + WQz * v13_3_3 + (VT)1.0 * oo2e * (v13_0_2 - rho_e * v13_0_3);
            const VT v14_9_0 = QCz * v14_3_0 + WQz * v14_3_1 + (VT)2.0 * oo2ze * v6_3_1 + (VT)1.0 * oo2e * (v14_0_0 - rho_e * v14_0_1);
            const VT v14_9_1 = QCz * v14_3_1 + WQz * v14_3_2 + (VT)2.0 * oo2ze * v6_3_2 + (VT)1.0 * oo2e * (v14_0_1 - rho_e * v14_0_2);
            const VT v14_9_2 = QCz * v14_3_2 + WQz * v14_3_3 + (VT)2.0 * oo2ze * v6_3_3 + (VT)1.0 * oo2e * (v14_0_2 - rho_e * v14_0_3);
            const VT v15_9_0 = QCz * v15_3_0 + WQz * v15_3_1 + (VT)1.0 * oo2ze * v5_3_1 + (VT)1.0 * oo2e * (v15_0_0 - rho_e * v15_0_1);
            const VT v15_9_1 = QCz * v15_3_1 + WQz * v15_3_2 + (VT)1.0 * oo2ze * v5_3_2 + (VT)1.0 * oo2e * (v15_0_1 - rho_e * v15_0_2);
            const VT v15_9_2 = QCz * v15_3_2 + WQz * v15_3_3 + (VT)1.0 * oo2ze * v5_3_3 + (VT)1.0 * oo2e * (v15_0_2 - rho_e * v15_0_3);
            const VT v16_9_0 = QCz * v16_3_0 + WQz * v16_3_1 + (VT)1.0 * oo2e * (v16_0_0 - rho_e * v16_0_1);
            const VT v16_9_1 = QCz * v16_3_1 + WQz * v16_3_2 + (VT)1.0 * oo2e * (v16_0_1 - rho_e * v16_0_2);
            const VT v16_9_2 = QCz * v16_3_2 + WQz * v16_3_3 + (VT)1.0 * oo2e * (v16_0_2 - rho_e * v16_0_3);
            const VT v17_9_0 = QCz * v17_3_0 + WQz * v17_3_1 + (VT)1.0 * oo2ze * v7_3_1 + (VT)1.0 * oo2e * (v17_0_0 - rho_e * v17_0_1);
            const VT v17_9_1 = QCz * v17_3_1 + WQz * v17_3_2 + (VT)1.0 * oo2ze * v7_3_2 + (VT)1.0 * oo2e * (v17_0_1 - rho_e * v17_0_2);
            const VT v17_9_2 = QCz * v17_3_2 + WQz * v17_3_3 + (VT)1.0 * oo2ze * v7_3_3 + (VT)1.0 * oo2e * (v17_0_2 - rho_e * v17_0_3);
            const VT v18_9_0 = QCz * v18_3_0 + WQz * v18_3_1 + (VT)2.0 * oo2ze * v8_3_1 + (VT)1.0 * oo2e * (v18_0_0 - rho_e * v18_0_1);
            const VT v18_9_1 = QCz * v18_3_1 + WQz * v18_3_2 + (VT)2.0 * oo2ze * v8_3_2 + (VT)1.0 * oo2e * (v18_0_1 - rho_e * v18_0_2);
            const VT v18_9_2 = QCz * v18_3_2 + WQz * v18_3_3 + (VT)2.0 * oo2ze * v8_3_3 + (VT)1.0 * oo2e * (v18_0_2 - rho_e * v18_0_3);
            const VT v19_9_0 = QCz * v19_3_0 + WQz * v19_3_1 + (VT)3.0 * oo2ze * v9_3_1 + (VT)1.0 * oo2e * (v19_0_0 - rho_e * v19_0_1);
            const VT v19_9_1 = QCz * v19_3_1 + WQz * v19_3_2 + (VT)3.0 * oo2ze * v9_3_2 + (VT)1.0 * oo2e * (v19_0_1 - rho_e * v19_0_2);
            const VT v19_9_2 = QCz * v19_3_2 + WQz * v19_3_3 + (VT)3.0 * oo2ze * v9_3_3 + (VT)1.0 * oo2e * (v19_0_2 - rho_e * v19_0_3);
            const VT v20_9_0 = QCz * v20_3_0 + WQz * v20_3_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v20_9_1 = QCz * v20_3_1 + WQz * v20_3_2 + (VT)1.0 * oo2e * (v20_0_1 - rho_e * v20_0_2);
            const VT v20_9_2 = QCz * v20_3_2 + WQz * v20_3_3 + (VT)1.0 * oo2e * (v20_0_2 - rho_e * v20_0_3);
            const VT v21_9_0 = QCz * v21_3_0 + WQz * v21_3_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v21_9_1 = QCz * v21_3_1 + WQz * v21_3_2 + (VT)1.0 * oo2e * (v21_0_1 - rho_e * v21_0_2);
            const VT v21_9_2 = QCz * v21_3_2 + WQz * v21_3_3 + (VT)1.0 * oo2e * (v21_0_2 - rho_e * v21_0_3);
            const VT v22_9_0 = QCz * v22_3_0 + WQz * v22_3_1 + (VT)1.0 * oo2ze * v10_3_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v22_9_1 = QCz * v22_3_1 + WQz * v22_3_2 + (VT)1.0 * oo2ze * v10_3_2 + (VT)1.0 * oo2e * (v22_0_1 - rho_e * v22_0_2);
            const VT v22_9_2 = QCz * v22_3_2 + WQz * v22_3_3 + (VT)1.0 * oo2ze * v10_3_3 + (VT)1.0 * oo2e * (v22_0_2 - rho_e * v22_0_3);
            const VT v23_9_0 = QCz * v23_3_0 + WQz * v23_3_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v23_9_1 = QCz * v23_3_1 + WQz * v23_3_2 + (VT)1.0 * oo2e * (v23_0_1 - rho_e * v23_0_2);
            const VT v23_9_2 = QCz * v23_3_2 + WQz * v23_3_3 + (VT)1.0 * oo2e * (v23_0_2 - rho_e * v23_0_3);
            const VT v24_9_0 = QCz * v24_3_0 + WQz * v24_3_1 + (VT)1.0 * oo2ze * v11_3_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v24_9_1 = QCz * v24_3_1 + WQz * v24_3_2 + (VT)1.0 * oo2ze * v11_3_2 + (VT)1.0 * oo2e * (v24_0_1 - rho_e * v24_0_2);
            const VT v24_9_2 = QCz * v24_3_2 + WQz * v24_3_3 + (VT)1.0 * oo2ze * v11_3_3 + (VT)1.0 * oo2e * (v24_0_2 - rho_e * v24_0_3);
            const VT v25_9_0 = QCz * v25_3_0 + WQz * v25_3_1 + (VT)2.0 * oo2ze * v12_3_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v25_9_1 = QCz * v25_3_1 + WQz * v25_3_2 + (VT)2.0 * oo2ze * v12_3_2 + (VT)1.0 * oo2e * (v25_0_1 - rho_e * v25_0_2);
            const VT v25_9_2 = QCz * v25_3_2 + WQz * v25_3_3 + (VT)2.0 * oo2ze * v12_3_3 + (VT)1.0 * oo2e * (v25_0_2 - rho_e * v25_0_3);
            const VT v26_9_0 = QCz * v26_3_0 + WQz * v26_3_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v26_9_1 = QCz * v26_3_1 + WQz * v26_3_2 + (VT)1.0 * oo2e * (v26_0_1 - rho_e * v26_0_2);
            const VT v26_9_2 = QCz * v26_3_2 + WQz * v26_3_3 + (VT)1.0 * oo2e * (v26_0_2 - rho_e * v26_0_3);
            const VT v27_9_0 = QCz * v27_3_0 + WQz * v27_3_1 + (VT)1.0 * oo2ze * v13_3_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v27_9_1 = QCz * v27_3_1 + WQz * v27_3_2 + (VT)1.0 * oo2ze * v13_3_2 + (VT)1.0 * oo2e * (v27_0_1 - rho_e * v27_0_2);
            const VT v27_9_2 = QCz * v27_3_2 + WQz * v27_3_3 + (VT)1.0 * oo2ze * v13_3_3 + (VT)1.0 * oo2e * (v27_0_2 - rho_e * v27_0_3);
            const VT v28_9_0 = QCz * v28_3_0 + WQz * v28_3_1 + (VT)2.0 * oo2ze * v15_3_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v28_9_1 = QCz * v28_3_1 + WQz * v28_3_2 + (VT)2.0 * oo2ze * v15_3_2 + (VT)1.0 * oo2e * (v28_0_1 - rho_e * v28_0_2);
            const VT v28_9_2 = QCz * v28_3_2 + WQz * v28_3_3 + (VT)2.0 * oo2ze * v15_3_3 + (VT)1.0 * oo2e * (v28_0_2 - rho_e * v28_0_3);
            const VT v29_9_0 = QCz * v29_3_0 + WQz * v29_3_1 + (VT)3.0 * oo2ze * v14_3_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v29_9_1 = QCz * v29_3_1 + WQz * v29_3_2 + (VT)3.0 * oo2ze * v14_3_2 + (VT)1.0 * oo2e * (v29_0_1 - rho_e * v29_0_2);
            const VT v29_9_2 = QCz * v29_3_2 + WQz * v29_3_3 + (VT)3.0 * oo2ze * v14_3_3 + (VT)1.0 * oo2e * (v29_0_2 - rho_e * v29_0_3);
            const VT v30_9_0 = QCz * v30_3_0 + WQz * v30_3_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v30_9_1 = QCz * v30_3_1 + WQz * v30_3_2 + (VT)1.0 * oo2e * (v30_0_1 - rho_e * v30_0_2);
            const VT v30_9_2 = QCz * v30_3_2 + WQz * v30_3_3 + (VT)1.0 * oo2e * (v30_0_2 - rho_e * v30_0_3);
            const VT v31_9_0 = QCz * v31_3_0 + WQz * v31_3_1 + (VT)1.0 * oo2ze * v16_3_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v31_9_1 = QCz * v31_3_1 + WQz * v31_3_2 + (VT)1.0 * oo2ze * v16_3_2 + (VT)1.0 * oo2e * (v31_0_1 - rho_e * v31_0_2);
            const VT v31_9_2 = QCz * v31_3_2 + WQz * v31_3_3 + (VT)1.0 * oo2ze * v16_3_3 + (VT)1.0 * oo2e * (v31_0_2 - rho_e * v31_0_3);
            const VT v32_9_0 = QCz * v32_3_0 + WQz * v32_3_1 + (VT)2.0 * oo2ze * v17_3_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v32_9_1 = QCz * v32_3_1 + WQz * v32_3_2 + (VT)2.0 * oo2ze * v17_3_2 + (VT)1.0 * oo2e * (v32_0_1 - rho_e * v32_0_2);
            const VT v32_9_2 = QCz * v32_3_2 + WQz * v32_3_3 + (VT)2.0 * oo2ze * v17_3_3 + (VT)1.0 * oo2e * (v32_0_2 - rho_e * v32_0_3);
            const VT v33_9_0 = QCz * v33_3_0 + WQz * v33_3_1 + (VT)3.0 * oo2ze * v18_3_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v33_9_1 = QCz * v33_3_1 + WQz * v33_3_2 + (VT)3.0 * oo2ze * v18_3_2 + (VT)1.0 * oo2e * (v33_0_1 - rho_e * v33_0_2);
            const VT v33_9_2 = QCz * v33_3_2 + WQz * v33_3_3 + (VT)3.0 * oo2ze * v18_3_3 + (VT)1.0 * oo2e * (v33_0_2 - rho_e * v33_0_3);
            const VT v34_9_0 = QCz * v34_3_0 + WQz * v34_3_1 + (VT)4.0 * oo2ze * v19_3_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
            const VT v34_9_1 = QCz * v34_3_1 + WQz * v34_3_2 + (VT)4.0 * oo2ze * v19_3_2 + (VT)1.0 * oo2e * (v34_0_1 - rho_e * v34_0_2);
            const VT v34_9_2 = QCz * v34_3_2 + WQz * v34_3_3 + (VT)4.0 * oo2ze * v19_3_3 + (VT)1.0 * oo2e * (v34_0_2 - rho_e * v34_0_3);
            const VT v1_10_1 = QCx * v1_4_1 + WQx * v1_4_2 + (VT)1.0 * oo2ze * v0_4_2 + (VT)2.0 * oo2e * (v1_1_1 - rho_e * v1_1_2);
            const VT v2_10_1 = QCx * v2_4_1 + WQx * v2_4_2 + (VT)2.0 * oo2e * (v2_1_1 - rho_e * v2_1_2);
            const VT v3_10_1 = QCx * v3_4_1 + WQx * v3_4_2 + (VT)2.0 * oo2e * (v3_1_1 - rho_e * v3_1_2);
            const VT v4_10_0 = QCx * v4_4_0 + WQx * v4_4_1 + (VT)2.0 * oo2ze * v1_4_1 + (VT)2.0 * oo2e * (v4_1_0 - rho_e * v4_1_1);
            const VT v4_10_1 = QCx * v4_4_1 + WQx * v4_4_2 + (VT)2.0 * oo2ze * v1_4_2 + (VT)2.0 * oo2e * (v4_1_1 - rho_e * v4_1_2);
            const VT v5_10_0 = QCx * v5_4_0 + WQx * v5_4_1 + (VT)1.0 * oo2ze * v2_4_1 + (VT)2.0 * oo2e * (v5_1_0 - rho_e * v5_1_1);
            const VT v5_10_1 = QCx * v5_4_1 + WQx * v5_4_2 + (VT)1.0 * oo2ze * v2_4_2 + (VT)2.0 * oo2e * (v5_1_1 - rho_e * v5_1_2);
            const VT v6_10_0 = QCx * v6_4_0 + WQx * v6_4_1 + (VT)1.0 * oo2ze * v3_4_1 + (VT)2.0 * oo2e * (v6_1_0 - rho_e * v6_1_1);
            const VT v6_10_1 = QCx * v6_4_1 + WQx * v6_4_2 + (VT)1.0 * oo2ze * v3_4_2 + (VT)2.0 * oo2e * (v6_1_1 - rho_e * v6_1_2);
            const VT v7_10_0 = QCx * v7_4_0 + WQx * v7_4_1 + (VT)2.0 * oo2e * (v7_1_0 - rho_e * v7_1_1);
            const VT v7_10_1 = QCx * v7_4_1 + WQx * v7_4_2 + (VT)2.0 * oo2e * (v7_1_1 - rho_e * v7_1_2);
            const VT v8_10_0 = QCx * v8_4_0 + WQx * v8_4_1 + (VT)2.0 * oo2e * (v8_1_0 - rho_e * v8_1_1);
            const VT v8_10_1 = QCx * v8_4_1 + WQx * v8_4_2 + (VT)2.0 * oo2e * (v8_1_1 - rho_e * v8_1_2);
            const VT v9_10_0 = QCx * v9_4_0 + WQx * v9_4_1 + (VT)2.0 * oo2e * (v9_1_0 - rho_e * v9_1_1);
            const VT v9_10_1 = QCx * v9_4_1 + WQx * v9_4_2 + (VT)2.0 * oo2e * (v9_1_1 - rho_e * v9_1_2);
            const VT v10_10_0 = QCx * v10_4_0 + WQx * v10_4_1 + (VT)3.0 * oo2ze * v4_4_1 + (VT)2.0 * oo2e * (v10_1_0 - rho_e * v10_1_1);
            const VT v10_10_1 = QCx * v10_4_1 + WQx * v10_4_2 + (VT)3.0 * oo2ze * v4_4_2 + (VT)2.0 * oo2e * (v10_1_1 - rho_e * v10_1_2);
            const VT v11_10_0 = QCx * v11_4_0 + WQx * v11_4_1 + (VT)2.0 * oo2ze * v5_4_1 + (VT)2.0 * oo2e * (v11_1_0 - rho_e * v11_1_1);
            const VT v11_10_1 = QCx * v11_4_1 + WQx * v11_4_2 + (VT)2.0 * oo2ze * v5_4_2 + (VT)2.0 * oo2e * (v11_1_1 - rho_e * v11_1_2);
            const VT v12_10_0 = QCx * v12_4_0 + WQx * v12_4_1 + (VT)2.0 * oo2ze * v6_4_1 + (VT)2.0 * oo2e * (v12_1_0 - rho_e * v12_1_1);
            const VT v12_10_1 = QCx * v12_4_1 + WQx * v12_4_2 + (VT)2.0 * oo2ze * v6_4_2 + (VT)2.0 * oo2e * (v12_1_1 - rho_e * v12_1_2);
            const VT v13_10_0 = QCx * v13_4_0 + WQx * v13_4_1 + (VT)1.0 * oo2ze * v7_4_1 + (VT)2.0 * oo2e * (v13_1_0 - rho_e * v13_1_1);
            const VT v13_10_1 = QCx * v13_4_1 + WQx * v13_4_2 + (VT)1.0 * oo2ze * v7_4_2 + (VT)2.0 * oo2e * (v13_1_1 - rho_e * v13_1_2);
            const VT v14_10_0 = QCx * v14_4_0 + WQx * v14_4_1 + (VT)1.0 * oo2ze * v9_4_1 + (VT)2.0 * oo2e * (v14_1_0 - rho_e * v14_1_1);
            const VT v14_10_1 = QCx * v14_4_1 + WQx * v14_4_2 + (VT)1.0 * oo2ze * v9_4_2 + (VT)2.0 * oo2e * (v14_1_1 - rho_e * v14_1_2);
            const VT v15_10_0 = QCx * v15_4_0 + WQx * v15_4_1 + (VT)1.0 * oo2ze * v8_4_1 + (VT)2.0 * oo2e * (v15_1_0 - rho_e * v15_1_1);
            const VT v15_10_1 = QCx * v15_4_1 + WQx * v15_4_2 + (VT)1.0 * oo2ze * v8_4_2 + (VT)2.0 * oo2e * (v15_1_1 - rho_e * v15_1_2);
            const VT v16_10_0 = QCx * v16_4_0 + WQx * v16_4_1 + (VT)2.0 * oo2e * (v16_1_0 - rho_e * v16_1_1);
            const VT v16_10_1 = QCx * v16_4_1 + WQx * v16_4_2 + (VT)2.0 * oo2e * (v16_1_1 - rho_e * v16_1_2);
            const VT v17_10_0 = QCx * v17_4_0 + WQx * v17_4_1 + (VT)2.0 * oo2e * (v17_1_0 - rho_e * v17_1_1);
            const VT v17_10_1 = QCx * v17_4_1 + WQx * v17_4_2 + (VT)2.0 * oo2e * (v17_1_1 - rho_e * v17_1_2);
            const VT v18_10_0 = QCx * v18_4_0 + WQx * v18_4_1 + (VT)2.0 * oo2e * (v18_1_0 - rho_e * v18_1_1);
            const VT v18_10_1 = QCx * v18_4_1 + WQx * v18_4_2 + (VT)2.0 * oo2e * (v18_1_1 - rho_e * v18_1_2);
            const VT v19_10_0 = QCx * v19_4_0 + WQx * v19_4_1 + (VT)2.0 * oo2e * (v19_1_0 - rho_e * v19_1_1);
            const VT v19_10_1 = QCx * v19_4_1 + WQx * v19_4_2 + (VT)2.0 * oo2e * (v19_1_1 - rho_e * v19_1_2);
            const VT v20_10_0 = QCx * v20_4_0 + WQx * v20_4_1 + (VT)4.0 * oo2ze * v10_4_1 + (VT)2.0 * oo2e * (v20_1_0 - rho_e * v20_1_1);
            const VT v20_10_1 = QCx * v20_4_1 + WQx * v20_4_2 + (VT)4.0 * oo2ze * v10_4_2 + (VT)2.0 * oo2e * (v20_1_1 - rho_e * v20_1_2);
            const VT v21_10_0 = QCx * v21_4_0 + WQx * v21_4_1 + (VT)3.0 * oo2ze * v11_4_1 + (VT)2.0 * oo2e * (v21_1_0 - rho_e * v21_1_1);
            const VT v21_10_1 = QCx * v21_4_1 + WQx * v21_4_2 + (VT)3.0 * oo2ze * v11_4_2 + (VT)2.0 * oo2e * (v21_1_1 - rho_e * v21_1_2);
            const VT v22_10_0 = QCx * v22_4_0 + WQx * v22_4_1 + (VT)3.0 * oo2ze * v12_4_1 + (VT)2.0 * oo2e * (v22_1_0 - rho_e * v22_1_1);
            const VT v22_10_1 = QCx * v22_4_1 + WQx * v22_4_2 + (VT)3.0 * oo2ze * v12_4_2 + (VT)2.0 * oo2e * (v22_1_1 - rho_e * v22_1_2);
            const VT v23_10_0 = QCx * v23_4_0 + WQx * v23_4_1 + (VT)2.0 * oo2ze * v13_4_1 + (VT)2.0 * oo2e * (v23_1_0 - rho_e * v23_1_1);
            const VT v23_10_1 = QCx * v23_4_1 + WQx * v23_4_2 + (VT)2.0 * oo2ze * v13_4_2 + (VT)2.0 * oo2e * (v23_1_1 - rho_e * v23_1_2);
            const VT v24_10_0 = QCx * v24_4_0 + WQx * v24_4_1 + (VT)2.0 * oo2ze * v15_4_1 + (VT)2.0 * oo2e * (v24_1_0 - rho_e * v24_1_1);
            const VT v24_10_1 = QCx * v24_4_1 + WQx * v24_4_2 + (VT)2.0 * oo2ze * v15_4_2 + (VT)2.0 * oo2e * (v24_1_1 - rho_e * v24_1_2);
            const VT v25_10_0 = QCx * v25_4_0 + WQx * v25_4_1 + (VT)2.0 * oo2ze * v14_4_1 + (VT)2.0 * oo2e * (v25_1_0 - rho_e * v25_1_1);
            const VT v25_10_1 = QCx * v25_4_1 + WQx * v25_4_2 + (VT)2.0 * oo2ze * v14_4_2 + (VT)2.0 * oo2e * (v25_1_1 - rho_e * v25_1_2);
            const VT v26_10_0 = QCx * v26_4_0 + WQx * v26_4_1 + (VT)1.0 * oo2ze * v16_4_1 + (VT)2.0 * oo2e * (v26_1_0 - rho_e * v26_1_1);
            const VT v26_10_1 = QCx * v26_4_1 + WQx * v26_4_2 + (VT)1.0 * oo2ze * v16_4_2 + (VT)2.0 * oo2e * (v26_1_1 - rho_e * v26_1_2);
            const VT v27_10_0 = QCx * v27_4_0 + WQx * v27_4_1 + (VT)1.0 * oo2ze * v17_4_1 + (VT)2.0 * oo2e * (v27_1_0 - rho_e * v27_1_1);
            const VT v27_10_1 = QCx * v27_4_1 + WQx * v27_4_2 + (VT)1.0 * oo2ze * v17_4_2 + (VT)2.0 * oo2e * (v27_1_1 - rho_e * v27_1_2);
            const VT v28_10_0 = QCx * v28_4_0 + WQx * v28_4_1 + (VT)1.0 * oo2ze * v18_4_1 + (VT)2.0 * oo2e * (v28_1_0 - rho_e * v28_1_1);
            const VT v28_10_1 = QCx * v28_4_1 + WQx * v28_4_2 + (VT)1.0 * oo2ze * v18_4_2 + (VT)2.0 * oo2e * (v28_1_1 - rho_e * v28_1_2);
            const VT v29_10_0 = QCx * v29_4_0 + WQx * v29_4_1 + (VT)1.0 * oo2ze * v19_4_1 + (VT)2.0 * oo2e * (v29_1_0 - rho_e * v29_1_1);
            const VT v29_10_1 = QCx * v29_4_1 + WQx * v29_4_2 + (VT)1.0 * oo2ze * v19_4_2 + (VT)2.0 * oo2e * (v29_1_1 - rho_e * v29_1_2);
            const VT v30_10_0 = QCx * v30_4_0 + WQx * v30_4_1 + (VT)2.0 * oo2e * (v30_1_0 - rho_e * v30_1_1);
            const VT v30_10_1 = QCx * v30_4_1 + WQx * v30_4_2 + (VT)2.0 * oo2e * (v30_1_1 - rho_e * v30_1_2);
            const VT v31_10_0 = QCx * v31_4_0 + WQx * v31_4_1 + (VT)2.0 * oo2e * (v31_1_0 - rho_e * v31_1_1);
            const VT v31_10_1 = QCx * v31_4_1 + WQx * v31_4_2 + (VT)2.0 * oo2e * (v31_1_1 - rho_e * v31_1_2);
            const VT v32_10_0 = QCx * v32_4_0 + WQx * v32_4_1 + (VT)2.0 * oo2e * (v32_1_0 - rho_e * v32_1_1);
            const VT v32_10_1 = QCx * v32_4_1 + WQx * v32_4_2 + (VT)2.0 * oo2e * (v32_1_1 - rho_e * v32_1_2);
            const VT v33_10_0 = QCx * v33_4_0 + WQx * v33_4_1 + (VT)2.0 * oo2e * (v33_1_0 - rho_e * v33_1_1);
            const VT v33_10_1 = QCx * v33_4_1 + WQx * v33_4_2 + (VT)2.0 * oo2e * (v33_1_1 - rho_e * v33_1_2);
            const VT v34_10_0 = QCx * v34_4_0 + WQx * v34_4_1 + (VT)2.0 * oo2e * (v34_1_0 - rho_e * v34_1_1);
            const VT v34_10_1 = QCx * v34_4_1 + WQx * v34_4_2 + (VT)2.0 * oo2e * (v34_1_1 - rho_e * v34_1_2);
            const VT v1_11_1 = QCx * v1_5_1 + WQx * v1_5_2 + (VT)1.0 * oo2ze * v0_5_2 + (VT)1.0 * oo2e * (v1_2_1 - rho_e * v1_2_2);
            const VT v2_11_1 = QCx * v2_5_1 + WQx * v2_5_2 + (VT)1.0 * oo2e * (v2_2_1 - rho_e * v2_2_2);
            const VT v3_11_1 = QCx * v3_5_1 + WQx * v3_5_2 + (VT)1.0 * oo2e * (v3_2_1 - rho_e * v3_2_2);
            const VT v4_11_0 = QCx * v4_5_0 + WQx * v4_5_1 + (VT)2.0 * oo2ze * v1_5_1 + (VT)1.0 * oo2e * (v4_2_0 - rho_e * v4_2_1);
            const VT v4_11_1 = QCx * v4_5_1 + WQx * v4_5_2 + (VT)2.0 * oo2ze * v1_5_2 + (VT)1.0 * oo2e * (v4_2_1 - rho_e * v4_2_2);
            const VT v5_11_0 = QCx * v5_5_0 + WQx * v5_5_1 + (VT)1.0 * oo2ze * v2_5_1 + (VT)1.0 * oo2e * (v5_2_0 - rho_e * v5_2_1);
            const VT v5_11_1 = QCx * v5_5_1 + WQx * v5_5_2 + (VT)1.0 * oo2ze * v2_5_2 + (VT)1.0 * oo2e * (v5_2_1 - rho_e * v5_2_2);
            const VT v6_11_0 = QCx * v6_5_0 + WQx * v6_5_1 + (VT)1.0 * oo2ze * v3_5_1 + (VT)1.0 * oo2e * (v6_2_0 - rho_e * v6_2_1);
            const VT v6_11_1 = QCx * v6_5_1 + WQx * v6_5_2 + (VT)1.0 * oo2ze * v3_5_2 + (VT)1.0 * oo2e * (v6_2_1 - rho_e * v6_2_2);
            const VT v7_11_0 = QCx * v7_5_0 + WQx * v7_5_1 + (VT)1.0 * oo2e * (v7_2_0 - rho_e * v7_2_1);
            const VT v7_11_1 = QCx * v7_5_1 + WQx * v7_5_2 + (VT)1.0 * oo2e * (v7_2_1 - rho_e * v7_2_2);
            const VT v8_11_0 = QCx * v8_5_0 + WQx * v8_5_1 + (VT)1.0 * oo2e * (v8_2_0 - rho_e * v8_2_1);
            const VT v8_11_1 = QCx * v8_5_1 + WQx * v8_5_2 + (VT)1.0 * oo2e * (v8_2_1 - rho_e * v8_2_2);
            const VT v9_11_0 = QCx * v9_5_0 + WQx * v9_5_1 + (VT)1.0 * oo2e * (v9_2_0 - rho_e * v9_2_1);
            const VT v9_11_1 = QCx * v9_5_1 + WQx * v9_5_2 + (VT)1.0 * oo2e * (v9_2_1 - rho_e * v9_2_2);
            const VT v10_11_0 = QCx * v10_5_0 + WQx * v10_5_1 + (VT)3.0 * oo2ze * v4_5_1 + (VT)1.0 * oo2e * (v10_2_0 - rho_e * v10_2_1);
            const VT v10_11_1 = QCx * v10_5_1 + WQx * v10_5_2 + (VT)3.0 * oo2ze * v4_5_2 + (VT)1.0 * oo2e * (v10_2_1 - rho_e * v10_2_2);
            const VT v11_11_0 = QCx * v11_5_0 + WQx * v11_5_1 + (VT)2.0 * oo2ze * v5_5_1 + (VT)1.0 * oo2e * (v11_2_0 - rho_e * v11_2_1);
            const VT v11_11_1 = QCx * v11_5_1 + WQx * v11_5_2 + (VT)2.0 * oo2ze * v5_5_2 + (VT)1.0 * oo2e * (v11_2_1 - rho_e * v11_2_2);
            const VT v12_11_0 = QCx * v12_5_0 + WQx * v12_5_1 + (VT)2.0 * oo2ze * v6_5_1 + (VT)1.0 * oo2e * (v12_2_0 - rho_e * v12_2_1);
            const VT v12_11_1 = QCx * v12_5_1 + WQx * v12_5_2 + (VT)2.0 * oo2ze * v6_5_2 + (VT)1.0 * oo2e * (v12_2_1 - rho_e * v12_2_2);
            const VT v13_11_0 = QCx * v13_5_0 + WQx * v13_5_1 + (VT)1.0 * oo2ze * v7_5_1 + (VT)1.0 * oo2e * (v13_2_0 - rho_e * v13_2_1);
            const VT v13_11_1 = QCx * v13_5_1 + WQx * v13_5_2 + (VT)1.0 * oo2ze * v7_5_2 + (VT)1.0 * oo2e * (v13_2_1 - rho_e * v13_2_2);
            const VT v14_11_0 = QCx * v14_5_0 + WQx * v14_5_1 + (VT)1.0 * oo2ze * v9_5_1 + (VT)1.0 * oo2e * (v14_2_0 - rho_e * v14_2_1);
            const VT v14_11_1 = QCx * v14_5_1 + WQx * v14_5_2 + (VT)1.0 * oo2ze * v9_5_2 + (VT)1.0 * oo2e * (v14_2_1 - rho_e * v14_2_2);
            const VT v15_11_0 = QCx * v15_5_0 + WQx * v15_5_1 + (VT)1.0 * oo2ze * v8_5_1 + (VT)1.0 * oo2e * (v15_2_0 - rho_e * v15_2_1);
            const VT v15_11_1 = QCx * v15_5_1 + WQx * v15_5_2 + (VT)1.0 * oo2ze * v8_5_2 + (VT)1.0 * oo2e * (v15_2_1 - rho_e * v15_2_2);
            const VT v16_11_0 = QCx * v16_5_0 + WQx * v16_5_1 + (VT)1.0 * oo2e * (v16_2_0 - rho_e * v16_2_1);
            const VT v16_11_1 = QCx * v16_5_1 + WQx * v16_5_2 + (VT)1.0 * oo2e * (v16_2_1 - rho_e * v16_2_2);
            const VT v17_11_0 = QCx * v17_5_0 + WQx * v17_5_1 + (VT)1.0 * oo2e * (v17_2_0 - rho_e * v17_2_1);
            const VT v17_11_1 = QCx * v17_5_1 + WQx * v17_5_2 + (VT)1.0 * oo2e * (v17_2_1 - rho_e * v17_2_2);
            const VT v18_11_0 = QCx * v18_5_0 + WQx * v18_5_1 + (VT)1.0 * oo2e * (v18_2_0 - rho_e * v18_2_1);
            const VT v18_11_1 = QCx * v18_5_1 + WQx * v18_5_2 + (VT)1.0 * oo2e * (v18_2_1 - rho_e * v18_2_2);
            const VT v19_11_0 = QCx * v19_5_0 + WQx * v19_5_1 + (VT)1.0 * oo2e * (v19_2_0 - rho_e * v19_2_1);
            const VT v19_11_1 = QCx * v19_5_1 + WQx * v19_5_2 + (VT)1.0 * oo2e * (v19_2_1 - rho_e * v19_2_2);
            const VT v20_11_0 = QCx * v20_5_0 + WQx * v20_5_1 + (VT)4.0 * oo2ze * v10_5_1 + (VT)1.0 * oo2e * (v20_2_0 - rho_e * v20_2_1);
            const VT v20_11_1 = QCx * v20_5_1 + WQx * v20_5_2 + (VT)4.0 * oo2ze * v10_5_2 + (VT)1.0 * oo2e * (v20_2_1 - rho_e * v20_2_2);
            const VT v21_11_0 = QCx * v21_5_0 + WQx * v21_5_1 + (VT)3.0 * oo2ze * v11_5_1 + (VT)1.0 * oo2e * (v21_2_0 - rho_e * v21_2_1);
            const VT v21_11_1 = QCx * v21_5_1 + WQx * v21_5_2 + (VT)3.0 * oo2ze * v11_5_2 + (VT)1.0 * oo2e * (v21_2_1 - rho_e * v21_2_2);
            const VT v22_11_0 = QCx * v22_5_0 + WQx * v22_5_1 + (VT)3.0 * oo2ze * v12_5_1 + (VT)1.0 * oo2e * (v22_2_0 - rho_e * v22_2_1);
            const VT v22_11_1 = QCx * v22_5_1 + WQx * v22_5_2 + (VT)3.0 * oo2ze * v12_5_2 + (VT)1.0 * oo2e * (v22_2_1 - rho_e * v22_2_2);
            const VT v23_11_0 = QCx * v23_5_0 + WQx * v23_5_1 + (VT)2.0 * oo2ze * v13_5_1 + (VT)1.0 * oo2e * (v23_2_0 - rho_e * v23_2_1);
            const VT v23_11_1 = QCx * v23_5_1 + WQx * v23_5_2 + (VT)2.0 * oo2ze * v13_5_2 + (VT)1.0 * oo2e * (v23_2_1 - rho_e * v23_2_2);
            const VT v24_11_0 = QCx * v24_5_0 + WQx * v24_5_1 + (VT)2.0 * oo2ze * v15_5_1 + (VT)1.0 * oo2e * (v24_2_0 - rho_e * v24_2_1);
            const VT v24_11_1 = QCx * v24_5_1 + WQx * v24_5_2 + (VT)2.0 * oo2ze * v15_5_2 + (VT)1.0 * oo2e * (v24_2_1 - rho_e * v24_2_2);
            const VT v25_11_0 = QCx * v25_5_0 + WQx * v25_5_1 + (VT)2.0 * oo2ze * v14_5_1 + (VT)1.0 * oo2e * (v25_2_0 - rho_e * v25_2_1);
            const VT v25_11_1 = QCx * v25_5_1 + WQx * v25_5_2 + (VT)2.0 * oo2ze * v14_5_2 + (VT)1.0 * oo2e * (v25_2_1 - rho_e * v25_2_2);
            const VT v26_11_0 = QCx * v26_5_0 + WQx * v26_5_1 + (VT)1.0 * oo2ze * v16_5_1 + (VT)1.0 * oo2e * (v26_2_0 - rho_e * v26_2_1);
            const VT v26_11_1 = QCx * v26_5_1 + WQx * v26_5_2 + (VT)1.0 * oo2ze * v16_5_2 + (VT)1.0 * oo2e * (v26_2_1 - rho_e * v26_2_2);
            const VT v27_11_0 = QCx * v27_5_0 + WQx * v27_5_1 + (VT)1.0 * oo2ze * v17_5_1 + (VT)1.0 * oo2e * (v27_2_0 - rho_e * v27_2_1);
            const VT v27_11_1 = QCx * v27_5_1 + WQx * v27_5_2 + (VT)1.0 * oo2ze * v17_5_2 + (VT)1.0 * oo2e * (v27_2_1 - rho_e * v27_2_2);
            const VT v28_11_0 = QCx * v28_5_0 + WQx * v28_5_1 + (VT)1.0 * oo2ze * v18_5_1 + (VT)1.0 * oo2e * (v28_2_0 - rho_e * v28_2_1);
            const VT v28_11_1 = QCx * v28_5_1 + WQx * v28_5_2 + (VT)1.0 * oo2ze * v18_5_2 + (VT)1.0 * oo2e * (v28_2_1 - rho_e * v28_2_2);
            const VT v29_11_0 = QCx * v29_5_0 + WQx * v29_5_1 + (VT)1.0 * oo2ze * v19_5_1 + (VT)1.0 * oo2e * (v29_2_0 - rho_e * v29_2_1);
            const VT v29_11_1 = QCx * v29_5_1 + WQx * v29_5_2 + (VT)1.0 * oo2ze * v19_5_2 + (VT)1.0 * oo2e * (v29_2_1 - rho_e * v29_2_2);
            const VT v30_11_0 = QCx * v30_5_0 + WQx * v30_5_1 + (VT)1.0 * oo2e * (v30_2_0 - rho_e * v30_2_1);
            const VT v30_11_1 = QCx * v30_5_1 + WQx * v30_5_2 + (VT)1.0 * oo2e * (v30_2_1 - rho_e * v30_2_2);
            const VT v31_11_0 = QCx * v31_5_0 + WQx * v31_5_1 + (VT)1.0 * oo2e * (v31_2_0 - rho_e * v31_2_1);
            const VT v31_11_1 = QCx * v31_5_1 + WQx * v31_5_2 + (VT)1.0 * oo2e * (v31_2_1 - rho_e * v31_2_2);
            const VT v32_11_0 = QCx * v32_5_0 + WQx * v32_5_1 + (VT)1.0 * oo2e * (v32_2_0 - rho_e * v32_2_1);
            const VT v32_11_1 = QCx * v32_5_1 + WQx * v32_5_2 + (VT)1.0 * oo2e * (v32_2_1 - rho_e * v32_2_2);
            const VT v33_11_0 = QCx * v33_5_0 + WQx * v33_5_1 + (VT)1.0 * oo2e * (v33_2_0 - rho_e * v33_2_1);
            const VT v33_11_1 = QCx * v33_5_1 + WQx * v33_5_2 + (VT)1.0 * oo2e * (v33_2_1 - rho_e * v33_2_2);
            const VT v34_11_0 = QCx * v34_5_0 + WQx * v34_5_1 + (VT)1.0 * oo2e * (v34_2_0 - rho_e * v34_2_1);
            const VT v34_11_1 = QCx * v34_5_1 + WQx * v34_5_2 + (VT)1.0 * oo2e * (v34_2_1 - rho_e * v34_2_2);
            const VT v1_12_1 = QCx * v1_6_1 + WQx * v1_6_2 + (VT)1.0 * oo2ze * v0_6_2 + (VT)1.0 * oo2e * (v1_3_1 - rho_e * v1_3_2);
            const VT v2_12_1 = QCx * v2_6_1 + WQx * v2_6_2 + (VT)1.0 * oo2e * (v2_3_1 - rho_e * v2_3_2);
            const VT v3_12_1 = QCx * v3_6_1 + WQx * v3_6_2 + (VT)1.0 * oo2e * (v3_3_1 - rho_e * v3_3_2);
            const VT v4_12_0 = QCx * v4_6_0 + WQx * v4_6_1 + (VT)2.0 * oo2ze * v1_6_1 + (VT)1.0 * oo2e * (v4_3_0 - rho_e * v4_3_1);
            const VT v4_12_1 = QCx * v4_6_1 + WQx * v4_6_2 + (VT)2.0 * oo2ze * v1_6_2 + (VT)1.0 * oo2e * (v4_3_1 - rho_e * v4_3_2);
            const VT v5_12_0 = QCx * v5_6_0 + WQx * v5_6_1 + (VT)1.0 * oo2ze * v2_6_1 + (VT)1.0 * oo2e * (v5_3_0 - rho_e * v5_3_1);
            const VT v5_12_1 = QCx * v5_6_1 + WQx * v5_6_2 + (VT)1.0 * oo2ze * v2_6_2 + (VT)1.0 * oo2e * (v5_3_1 - rho_e * v5_3_2);
            const VT v6_12_0 = QCx * v6_6_0 + WQx * v6_6_1 + (VT)1.0 * oo2ze * v3_6_1 + (VT)1.0 * oo2e * (v6_3_0 - rho_e * v6_3_1);
            const VT v6_12_1 = QCx * v6_6_1 + WQx * v6_6_2 + (VT)1.0 * oo2ze * v3_6_2 + (VT)1.0 * oo2e * (v6_3_1 - rho_e * v6_3_2);
            const VT v7_12_0 = QCx * v7_6_0 + WQx * v7_6_1 + (VT)1.0 * oo2e * (v7_3_0 - rho_e * v7_3_1);
            const VT v7_12_1 = QCx * v7_6_1 + WQx * v7_6_2 + (VT)1.0 * oo2e * (v7_3_1 - rho_e * v7_3_2);
            const VT v8_12_0 = QCx * v8_6_0 + WQx * v8_6_1 + (VT)1.0 * oo2e * (v8_3_0 - rho_e * v8_3_1);
            const VT v8_12_1 = QCx * v8_6_1 + WQx * v8_6_2 + (VT)1.0 * oo2e * (v8_3_1 - rho_e * v8_3_2);
            const VT v9_12_0 = QCx * v9_6_0 + WQx * v9_6_1 + (VT)1.0 * oo2e * (v9_3_0 - rho_e * v9_3_1);
            const VT v9_12_1 = QCx * v9_6_1 + WQx * v9_6_2 + (VT)1.0 * oo2e * (v9_3_1 - rho_e * v9_3_2);
            const VT v10_12_0 = QCx * v10_6_0 + WQx * v10_6_1 + (VT)3.0 * oo2ze * v4_6_1 + (VT)1.0 * oo2e * (v10_3_0 - rho_e * v10_3_1);
            const VT v10_12_1 = QCx * v10_6_1 + WQx * v10_6_2 + (VT)3.0 * oo2ze * v4_6_2 + (VT)1.0 * oo2e * (v10_3_1 - rho_e * v10_3_2);
            const VT v11_12_0 = QCx * v11_6_0 + WQx * v11_6_1 + (VT)2.0 * oo2ze * v5_6_1 + (VT)1.0 * oo2e * (v11_3_0 - rho_e * v11_3_1);
            const VT v11_12_1 = QCx * v11_6_1 + WQx * v11_6_2 + (VT)2.0 * oo2ze * v5_6_2 + (VT)1.0 * oo2e * (v11_3_1 - rho_e * v11_3_2);
            const VT v12_12_0 = QCx * v12_6_0 + WQx * v12_6_1 + (VT)2.0 * oo2ze * v6_6_1 + (VT)1.0 * oo2e * (v12_3_0 - rho_e * v12_3_1);
            const VT v12_12_1 = QCx * v12_6_1 + WQx * v12_6_2 + (VT)2.0 * oo2ze * v6_6_2 + (VT)1.0 * oo2e * (v12_3_1 - rho_e * v12_3_2);
            const VT v13_12_0 = QCx * v13_6_0 + WQx * v13_6_1 + (VT)1.0 * oo2ze * v7_6_1 + (VT)1.0 * oo2e * (v13_3_0 - rho_e * v13_3_1);
            const VT v13_12_1 = QCx * v13_6_1 + WQx * v13_6_2 + (VT)1.0 * oo2ze * v7_6_2 + (VT)1.0 * oo2e * (v13_3_1 - rho_e * v13_3_2);
            const VT v14_12_0 = QCx * v14_6_0 + WQx * v14_6_1 + (VT)1.0 * oo2ze * v9_6_1 + (VT)1.0 * oo2e * (v14_3_0 - rho_e * v14_3_1);
            const VT v14_12_1 = QCx * v14_6_1 + WQx * v14_6_2 + (VT)1.0 * oo2ze * v9_6_2 + (VT)1.0 * oo2e * (v14_3_1 - rho_e * v14_3_2);
            const VT v15_12_0 = QCx * v15_6_0 + WQx * v15_6_1 + (VT)1.0 * oo2ze * v8_6_1 + (VT)1.0 * oo2e * (v15_3_0 - rho_e * v15_3_1);
            const VT v15_12_1 = QCx * v15_6_1 + WQx * v15_6_2 + (VT)1.0 * oo2ze * v8_6_2 + (VT)1.0 * oo2e * (v15_3_1 - rho_e * v15_3_2);
            const VT v16_12_0 = QCx * v16_6_0 + WQx * v16_6_1 + (VT)1.0 * oo2e * (v16_3_0 - rho_e * v16_3_1);
            const VT v16_12_1 = QCx * v16_6_1 + WQx * v16_6_2 + (VT)1.0 * oo2e * (v16_3_1 - rho_e * v16_3_2);
            const VT v17_12_0 = QCx * v17_6_0 + WQx * v17_6_1 + (VT)1.0 * oo2e * (v17_3_0 - rho_e * v17_3_1);
            const VT v17_12_1 = QCx * v17_6_1 + WQx * v17_6_2 + (VT)1.0 * oo2e * (v17_3_1 - rho_e * v17_3_2);
            const VT v18_12_0 = QCx * v18_6_0 + WQx * v18_6_1 + (VT)1.0 * oo2e * (v18_3_0 - rho_e * v18_3_1);
            const VT v18_12_1 = QCx * v18_6_1 + WQx * v18_6_2 + (VT)1.0 * oo2e * (v18_3_1 - rho_e * v18_3_2);
            const VT v19_12_0 = QCx * v19_6_0 + WQx * v19_6_1 + (VT)1.0 * oo2e * (v19_3_0 - rho_e * v19_3_1);
            const VT v19_12_1 = QCx * v19_6_1 + WQx * v19_6_2 + (VT)1.0 * oo2e * (v19_3_1 - rho_e * v19_3_2);
            const VT v20_12_0 = QCx * v20_6_0 + WQx * v20_6_1 + (VT)4.0 * oo2ze * v10_6_1 + (VT)1.0 * oo2e * (v20_3_0 - rho_e * v20_3_1);
            const VT v20_12_1 = QCx * v20_6_1 + WQx * v20_6_2 + (VT)4.0 * oo2ze * v10_6_2 + (VT)1.0 * oo2e * (v20_3_1 - rho_e * v20_3_2);
            const VT v21_12_0 = QCx * v21_6_0 + WQx * v21_6_1 + (VT)3.0 * oo2ze * v11_6_1 + (VT)1.0 * oo2e * (v21_3_0 - rho_e * v21_3_1);
            const VT v21_12_1 = QCx * v21_6_1 + WQx * v21_6_2 + (VT)3.0 * oo2ze * v11_6_2 + (VT)1.0 * oo2e * (v21_3_1 - rho_e * v21_3_2);
            const VT v22_12_0 = QCx * v22_6_0 + WQx * v22_6_1 + (VT)3.0 * oo2ze * v12_6_1 + (VT)1.0 * oo2e * (v22_3_0 - rho_e * v22_3_1);
            const VT v22_12_1 = QCx * v22_6_1 + WQx * v22_6_2 + (VT)3.0 * oo2ze * v12_6_2 + (VT)1.0 * oo2e * (v22_3_1 - rho_e * v22_3_2);
            const VT v23_12_0 = QCx * v23_6_0 + WQx * v23_6_1 + (VT)2.0 * oo2ze * v13_6_1 + (VT)1.0 * oo2e * (v23_3_0 - rho_e * v23_3_1);
            const VT v23_12_1 = QCx * v23_6_1 + WQx * v23_6_2 + (VT)2.0 * oo2ze * v13_6_2 + (VT)1.0 * oo2e * (v23_3_1 - rho_e * v23_3_2);
            const VT v24_12_0 = QCx * v24_6_0 + WQx * v24_6_1 + (VT)2.0 * oo2ze * v15_6_1 + (VT)1.0 * oo2e * (v24_3_0 - rho_e * v24_3_1);
            const VT v24_12_1 = QCx * v24_6_1 + WQx * v24_6_2 + (VT)2.0 * oo2ze * v15_6_2 + (VT)1.0 * oo2e * (v24_3_1 - rho_e * v24_3_2);
            const VT v25_12_0 = QCx * v25_6_0 + WQx * v25_6_1 + (VT)2.0 * oo2ze * v14_6_1 + (VT)1.0 * oo2e * (v25_3_0 - rho_e * v25_3_1);
            const VT v25_12_1 = QCx * v25_6_1 + WQx * v25_6_2 + (VT)2.0 * oo2ze * v14_6_2 + (VT)1.0 * oo2e * (v25_3_1 - rho_e * v25_3_2);
            const VT v26_12_0 = QCx * v26_6_0 + WQx * v26_6_1 + (VT)1.0 * oo2ze * v16_6_1 + (VT)1.0 * oo2e * (v26_3_0 - rho_e * v26_3_1);
            const VT v26_12_1 = QCx * v26_6_1 + WQx * v26_6_2 + (VT)1.0 * oo2ze * v16_6_2 + (VT)1.0 * oo2e * (v26_3_1 - rho_e * v26_3_2);
            const VT v27_12_0 = QCx * v27_6_0 + WQx * v27_6_1 + (VT)1.0 * oo2ze * v17_6_1 + (VT)1.0 * oo2e * (v27_3_0 - rho_e * v27_3_1);
            const VT v27_12_1 = QCx * v27_6_1 + WQx * v27_6_2 + (VT)1.0 * oo2ze * v17_6_2 + (VT)1.0 * oo2e * (v27_3_1 - rho_e * v27_3_2);
            const VT v28_12_0 = QCx * v28_6_0 + WQx * v28_6_1 + (VT)1.0 * oo2ze * v18_6_1 + (VT)1.0 * oo2e * (v28_3_0 - rho_e * v28_3_1);
            const VT v28_12_1 = QCx * v28_6_1 + WQx * v28_6_2 + (VT)1.0 * oo2ze * v18_6_2 + (VT)1.0 * oo2e * (v28_3_1 - rho_e * v28_3_2);
            const VT v29_12_0 = QCx * v29_6_0 + WQx * v29_6_1 + (VT)1.0 * oo2ze * v19_6_1 + (VT)1.0 * oo2e * (v29_3_0 - rho_e * v29_3_1);
            const VT v29_12_1 = QCx * v29_6_1 + WQx * v29_6_2 + (VT)1.0 * oo2ze * v19_6_2 + (VT)1.0 * oo2e * (v29_3_1 - rho_e * v29_3_2);
            const VT v30_12_0 = QCx * v30_6_0 + WQx * v30_6_1 + (VT)1.0 * oo2e * (v30_3_0 - rho_e * v30_3_1);
            const VT v30_12_1 = QCx * v30_6_1 + WQx * v30_6_2 + (VT)1.0 * oo2e * (v30_3_1 - rho_e * v30_3_2);
            const VT v31_12_0 = QCx * v31_6_0 + WQx * v31_6_1 + (VT)1.0 * oo2e * (v31_3_0 - rho_e * v31_3_1);
            const VT v31_12_1 = QCx * v31_6_1 + WQx * v31_6_2 + (VT)1.0 * oo2e * (v31_3_1 - rho_e * v31_3_2);
            const VT v32_12_0 = QCx * v32_6_0 + WQx * v32_6_1 + (VT)1.0 * oo2e * (v32_3_0 - rho_e * v32_3_1);
            const VT v32_12_1 = QCx * v32_6_1 + WQx * v32_6_2 + (VT)1.0 * oo2e * (v32_3_1 - rho_e * v32_3_2);
            const VT v33_12_0 = QCx * v33_6_0 + WQx * v33_6_1 + (VT)1.0 * oo2e * (v33_3_0 - rho_e * v33_3_1);
            const VT v33_12_1 = QCx * v33_6_1 + WQx * v33_6_2 + (VT)1.0 * oo2e * (v33_3_1 - rho_e * v33_3_2);
            const VT v34_12_0 = QCx * v34_6_0 + WQx * v34_6_1 + (VT)1.0 * oo2e * (v34_3_0 - rho_e * v34_3_1);
            const VT v34_12_1 = QCx * v34_6_1 + WQx * v34_6_2 + (VT)1.0 * oo2e * (v34_3_1 - rho_e * v34_3_2);
            const VT v1_13_1 = QCy * v1_5_1 + WQy * v1_5_2 + (VT)1.0 * oo2e * (v1_1_1 - rho_e * v1_1_2);
            const VT v2_13_1 = QCy * v2_5_1 + WQy * v2_5_2 + (VT)1.0 * oo2ze * v0_5_2 + (VT)1.0 * oo2e * (v2_1_1 - rho_e * v2_1_2);
            const VT v3_13_1 = QCy * v3_5_1 + WQy * v3_5_2 + (VT)1.0 * oo2e * (v3_1_1 - rho_e * v3_1_2);
            const VT v4_13_0 = QCy * v4_5_0 + WQy * v4_5_1 + (VT)1.0 * oo2e * (v4_1_0 - rho_e * v4_1_1);
            const VT v4_13_1 = QCy * v4_5_1 + WQy * v4_5_2 + (VT)1.0 * oo2e * (v4_1_1 - rho_e * v4_1_2);
            const VT v5_13_0 = QCy * v5_5_0 + WQy * v5_5_1 + (VT)1.0 * oo2ze * v1_5_1 + (VT)1.0 * oo2e * (v5_1_0 - rho_e * v5_1_1);
            const VT v5_13_1 = QCy * v5_5_1 + WQy * v5_5_2 + (VT)1.0 * oo2ze * v1_5_2 + (VT)1.0 * oo2e * (v5_1_1 - rho_e * v5_1_2);
            const VT v6_13_0 = QCy * v6_5_0 + WQy * v6_5_1 + (VT)1.0 * oo2e * (v6_1_0 - rho_e * v6_1_1);
            const VT v6_13_1 = QCy * v6_5_1 + WQy * v6_5_2 + (VT)1.0 * oo2e * (v6_1_1 - rho_e * v6_1_2);
            const VT v7_13_0 = QCy * v7_5_0 + WQy * v7_5_1 + (VT)2.0 * oo2ze * v2_5_1 + (VT)1.0 * oo2e * (v7_1_0 - rho_e * v7_1_1);
            const VT v7_13_1 = QCy * v7_5_1 + WQy * v7_5_2 + (VT)2.0 * oo2ze * v2_5_2 + (VT)1.0 * oo2e * (v7_1_1 - rho_e * v7_1_2);
            const VT v8_13_0 = QCy * v8_5_0 + WQy * v8_5_1 + (VT)1.0 * oo2ze * v3_5_1 + (VT)1.0 * oo2e * (v8_1_0 - rho_e * v8_1_1);
            const VT v8_13_1 = QCy * v8_5_1 + WQy * v8_5_2 + (VT)1.0 * oo2ze * v3_5_2 + (VT)1.0 * oo2e * (v8_1_1 - rho_e * v8_1_2);
            const VT v9_13_0 = QCy * v9_5_0 + WQy * v9_5_1 + (VT)1.0 * oo2e * (v9_1_0 - rho_e * v9_1_1);
            const VT v9_13_1 = QCy * v9_5_1 + WQy * v9_5_2 + (VT)1.0 * oo2e * (v9_1_1 - rho_e * v9_1_2);
            const VT v10_13_0 = QCy * v10_5_0 + WQy * v10_5_1 + (VT)1.0 * oo2e * (v10_1_0 - rho_e * v10_1_1);
            const VT v10_13_1 = QCy * v10_5_1 + WQy * v10_5_2 + (VT)1.0 * oo2e * (v10_1_1 - rho_e * v10_1_2);
            const VT v11_13_0 = QCy * v11_5_0 + WQy * v11_5_1 + (VT)1.0 * oo2ze * v4_5_1 + (VT)1.0 * oo2e * (v11_1_0 - rho_e * v11_1_1);
            const VT v11_13_1 = QCy * v11_5_1 + WQy * v11_5_2 + (VT)1.0 * oo2ze * v4_5_2 + (VT)1.0 * oo2e * (v11_1_1 - rho_e * v11_1_2);
            const VT v12_13_0 = QCy * v12_5_0 + WQy * v12_5_1 + (VT)1.0 * oo2e * (v12_1_0 - rho_e * v12_1_1);
            const VT v12_13_1 = QCy * v12_5_1 + WQy * v12_5_2 + (VT)1.0 * oo2e * (v12_1_1 - rho_e * v12_1_2);
            const VT v13_13_0 = QCy * v13_5_0 + WQy * v13_5_1 + (VT)2.0 * oo2ze * v5_5_1 + (VT)1.0 * oo2e * (v13_1_0 - rho_e * v13_1_1);
            const VT v13_13_1 = QCy * v13_5_1 + WQy * v13_5_2 + (VT)2.0 * oo2ze * v5_5_2 + (VT)1.0 * oo2e * (v13_1_1 - rho_e * v13_1_2);
            const VT v14_13_0 = QCy * v14_5_0 + WQy * v14_5_1 + (VT)1.0 * oo2e * (v14_1_0 - rho_e * v14_1_1);
            const VT v14_13_1 = QCy * v14_5_1 + WQy * v14_5_2 + (VT)1.0 * oo2e * (v14_1_1 - rho_e * v14_1_2);
            const VT v15_13_0 = QCy * v15_5_0 + WQy * v15_5_1 + (VT)1.0 * oo2ze * v6_5_1 + (VT)1.0 * oo2e * (v15_1_0 - rho_e * v15_1_1);
            const VT v15_13_1 = QCy * v15_5_1 + WQy * v15_5_2 + (VT)1.0 * oo2ze * v6_5_2 + (VT)1.0 * oo2e * (v15_1_1 - rho_e * v15_1_2);
            const VT v16_13_0 = QCy * v16_5_0 + WQy * v16_5_1 + (VT)3.0 * oo2ze * v7_5_1 + (VT)1.0 * oo2e * (v16_1_0 - rho_e * v16_1_1);
            const VT v16_13_1 = QCy * v16_5_1 + WQy * v16_5_2 + (VT)3.0 * oo2ze * v7_5_2 + (VT)1.0 * oo2e * (v16_1_1 - rho_e * v16_1_2);
            const VT v17_13_0 = QCy * v17_5_0 + WQy * v17_5_1 + (VT)2.0 * oo2ze * v8_5_1 + (VT)1.0 * oo2e * (v17_1_0 - rho_e * v17_1_1);
            const VT v17_13_1 = QCy * v17_5_1 + WQy * v17_5_2 + (VT)2.0 * oo2ze * v8_5_2 + (VT)1.0 * oo2e * (v17_1_1 - rho_e * v17_1_2);
            const VT v18_13_0 = QCy * v18_5_0 + WQy * v18_5_1 + (VT)1.0 * oo2ze * v9_5_1 + (VT)1.0 * oo2e * (v18_1_0 - rho_e * v18_1_1);
            const VT v18_13_1 = QCy * v18_5_1 + WQy * v18_5_2 + (VT)1.0 * oo2ze * v9_5_2 + (VT)1.0 * oo2e * (v18_1_1 - rho_e * v18_1_2);
            const VT v19_13_0 = QCy * v19_5_0 + WQy * v19_5_1 + (VT)1.0 * oo2e * (v19_1_0 - rho_e * v19_1_1);
            const VT v19_13_1 = QCy * v19_5_1 + WQy * v19_5_2 + (VT)1.0 * oo2e * (v19_1_1 - rho_e * v19_1_2);
            const VT v20_13_0 = QCy * v20_5_0 + WQy * v20_5_1 + (VT)1.0 * oo2e * (v20_1_0 - rho_e * v20_1_1);
            const VT v20_13_1 = QCy * v20_5_1 + WQy * v20_5_2 + (VT)1.0 * oo2e * (v20_1_1 - rho_e * v20_1_2);
            const VT v21_13_0 = QCy * v21_5_0 + WQy * v21_5_1 + (VT)1.0 * oo2ze * v10_5_1 + (VT)1.0 * oo2e * (v21_1_0 - rho_e * v21_1_1);
            const VT v21_13_1 = QCy * v21_5_1 + WQy * v21_5_2 + (VT)1.0 * oo2ze * v10_5_2 + (VT)1.0 * oo2e * (v21_1_1 - rho_e * v21_1_2);
            const VT v22_13_0 = QCy * v22_5_0 + WQy * v22_5_1 + (VT)1.0 * oo2e * (v22_1_0 - rho_e * v22_1_1);
            const VT v22_13_1 = QCy * v22_5_1 + WQy * v22_5_2 + (VT)1.0 * oo2e * (v22_1_1 - rho_e * v22_1_2);
            const VT v23_13_0 = QCy * v23_5_0 + WQy * v23_5_1 + (VT)2.0 * oo2ze * v11_5_1 + (VT)1.0 * oo2e * (v23_1_0 - rho_e * v23_1_1);
            const VT v23_13_1 = QCy * v23_5_1 + WQy * v23_5_2 + (VT)2.0 * oo2ze * v11_5_2 + (VT)1.0 * oo2e * (v23_1_1 - rho_e * v23_1_2);
            const VT v24_13_0 = QCy * v24_5_0 + WQy * v24_5_1 + (VT)1.0 * oo2ze * v12_5_1 + (VT)1.0 * oo2e * (v24_1_0 - rho_e * v24_1_1);
            const VT v24_13_1 = QCy * v24_5_1 + WQy * v24_5_2 + (VT)1.0 * oo2ze * v12_5_2 + (VT)1.0 * oo2e * (v24_1_1 - rho_e * v24_1_2);
            const VT v25_13_0 = QCy * v25_5_0 + WQy * v25_5_1 + (VT)1.0 * oo2e * (v25_1_0 - rho_e * v25_1_1);
            const VT v25_13_1 = QCy * v25_5_1 + WQy * v25_5_2 + (VT)1.0 * oo2e * (v25_1_1 - rho_e * v25_1_2);
            const VT v26_13_0 = QCy * v26_5_0 + WQy * v26_5_1 + (VT)3.0 * oo2ze * v13_5_1 + (VT)1.0 * oo2e * (v26_1_0 - rho_e * v26_1_1);
            const VT v26_13_1 = QCy * v26_5_1 + WQy * v26_5_2 + (VT)3.0 * oo2ze * v13_5_2 + (VT)1.0 * oo2e * (v26_1_1 - rho_e * v26_1_2);
            const VT v27_13_0 = QCy * v27_5_0 + WQy * v27_5_1 + (VT)2.0 * oo2ze * v15_5_1 + (VT)1.0 * oo2e * (v27_1_0 - rho_e * v27_1_1);
            const VT v27_13_1 = QCy * v27_5_1 + WQy * v27_5_2 + (VT)2.0 * oo2ze * v15_5_2 + (VT)1.0 * oo2e * (v27_1_1 - rho_e * v27_1_2);
            const VT v28_13_0 = QCy * v28_5_0 + WQy * v28_5_1 + (VT)1.0 * oo2ze * v14_5_1 + (VT)1.0 * oo2e * (v28_1_0 - rho_e * v28_1_1);
            const VT v28_13_1 = QCy * v28_5_1 + WQy * v28_5_2 + (VT)1.0 * oo2ze * v14_5_2 + (VT)1.0 * oo2e * (v28_1_1 - rho_e * v28_1_2);
            const VT v29_13_0 = QCy * v29_5_0 + WQy * v29_5_1 + (VT)1.0 * oo2e * (v29_1_0 - rho_e * v29_1_1);
            const VT v29_13_1 = QCy * v29_5_1 + WQy * v29_5_2 + (VT)1.0 * oo2e * (v29_1_1 - rho_e * v29_1_2);
            const VT v30_13_0 = QCy * v30_5_0 + WQy * v30_5_1 + (VT)4.0 * oo2ze * v16_5_1 + (VT)1.0 * oo2e * (v30_1_0 - rho_e * v30_1_1);
            const VT v30_13_1 = QCy * v30_5_1 + WQy * v30_5_2 + (VT)4.0 * oo2ze * v16_5_2 + (VT)1.0 * oo2e * (v30_1_1 - rho_e * v30_1_2);
            const VT v31_13_0 = QCy * v31_5_0 + WQy * v31_5_1 + (VT)3.0 * oo2ze * v17_5_1 + (VT)1.0 * oo2e * (v31_1_0 - rho_e * v31_1_1);
            const VT v31_13_1 = QCy * v31_5_1 + WQy * v31_5_2 + (VT)3.0 * oo2ze * v17_5_2 + (VT)1.0 * oo2e * (v31_1_1 - rho_e * v31_1_2);
            const VT v32_13_0 = QCy * v32_5_0 + WQy * v32_5_1 + (VT)2.0 * oo2ze * v18_5_1 + (VT)1.0 * oo2e * (v32_1_0 - rho_e * v32_1_1);
            const VT v32_13_1 = QCy * v32_5_1 + WQy * v32_5_2 + (VT)2.0 * oo2ze * v18_5_2 + (VT)1.0 * oo2e * (v32_1_1 - rho_e * v32_1_2);
            const VT v33_13_0 = QCy * v33_5_0 + WQy * v33_5_1 + (VT)1.0 * oo2ze * v19_5_1 + (VT)1.0 * oo2e * (v33_1_0 - rho_e * v33_1_1);
            const VT v33_13_1 = QCy * v33_5_1 + WQy * v33_5_2 + (VT)1.0 * oo2ze * v19_5_2 + (VT)1.0 * oo2e * (v33_1_1 - rho_e * v33_1_2);
            const VT v34_13_0 = QCy * v34_5_0 + WQy * v34_5_1 + (VT)1.0 * oo2e * (v34_1_0 - rho_e * v34_1_1);
            const VT v34_13_1 = QCy * v34_5_1 + WQy * v34_5_2 + (VT)1.0 * oo2e * (v34_1_1 - rho_e * v34_1_2);
            const VT v1_14_1 = QCz * v1_6_1 + WQz * v1_6_2 + (VT)1.0 * oo2e * (v1_1_1 - rho_e * v1_1_2);
            const VT v2_14_1 = QCz * v2_6_1 + WQz * v2_6_2 + (VT)1.0 * oo2e * (v2_1_1 - rho_e * v2_1_2);
            const VT v3_14_1 = QCz * v3_6_1 + WQz * v3_6_2 + (VT)1.0 * oo2ze * v0_6_2 + (VT)1.0 * oo2e * (v3_1_1 - rho_e * v3_1_2);
            const VT v4_14_0 = QCz * v4_6_0 + WQz * v4_6_1 + (VT)1.0 * oo2e * (v4_1_0 - rho_e * v4_1_1);
            const VT v4_14_1 = QCz * v4_6_1 + WQz * v4_6_2 + (VT)1.0 * oo2e * (v4_1_1 - rho_e * v4_1_2);
            const VT v5_14_0 = QCz * v5_6_0 + WQz * v5_6_1 + (VT)1.0 * oo2e * (v5_1_0 - rho_e * v5_1_1);
            const VT v5_14_1 = QCz * v5_6_1 + WQz * v5_6_2 + (VT)1.0 * oo2e * (v5_1_1 - rho_e * v5_1_2);
            const VT v6_14_0 = QCz * v6_6_0 + WQz * v6_6_1 + (VT)1.0 * oo2ze * v1_6_1 + (VT)1.0 * oo2e * (v6_1_0 - rho_e * v6_1_1);
            const VT v6_14_1 = QCz * v6_6_1 + WQz * v6_6_2 + (VT)1.0 * oo2ze * v1_6_2 + (VT)1.0 * oo2e * (v6_1_1 - rho_e * v6_1_2);
            const VT v7_14_0 = QCz * v7_6_0 + WQz * v7_6_1 + (VT)1.0 * oo2e * (v7_1_0 - rho_e * v7_1_1);
            const VT v7_14_1 = QCz * v7_6_1 + WQz * v7_6_2 + (VT)1.0 * oo2e * (v7_1_1 - rho_e * v7_1_2);
            const VT v8_14_0 = QCz * v8_6_0 + WQz * v8_6_1 + (VT)1.0 * oo2ze * v2_6_1 + (VT)1.0 * oo2e * (v8_1_0 - rho_e * v8_1_1);
            const VT v8_14_1 = QCz * v8_6_1 + WQz * v8_6_2 + (VT)1.0 * oo2ze * v2_6_2 + (VT)1.0 * oo2e * (v8_1_1 - rho_e * v8_1_2);
            const VT v9_14_0 = QCz * v9_6_0 + WQz * v9_6_1 + (VT)2.0 * oo2ze * v3_6_1 + (VT)1.0 * oo2e * (v9_1_0 - rho_e * v9_1_1);
            const VT v9_14_1 = QCz * v9_6_1 + WQz * v9_6_2 + (VT)2.0 * oo2ze * v3_6_2 + (VT)1.0 * oo2e * (v9_1_1 - rho_e * v9_1_2);
            const VT v10_14_0 = QCz * v10_6_0 + WQz * v10_6_1 + (VT)1.0 * oo2e * (v10_1_0 - rho_e * v10_1_1);
            const VT v10_14_1 = QCz * v10_6_1 + WQz * v10_6_2 + (VT)1.0 * oo2e * (v10_1_1 - rho_e * v10_1_2);
            const VT v11_14_0 = QCz * v11_6_0 + WQz * v11_6_1 + (VT)1.0 * oo2e * (v11_1_0 - rho_e * v11_1_1);
            const VT v11_14_1 = QCz * v11_6_1 + WQz * v11_6_2 + (VT)1.0 * oo2e * (v11_1_1 - rho_e * v11_1_2);
            const VT v12_14_0 = QCz * v12_6_0 + WQz * v12_6_1 + (VT)1.0 * oo2ze * v4_6_1 + (VT)1.0 * oo2e * (v12_1_0 - rho_e * v12_1_1);
            const VT v12_14_1 = QCz * v12_6_1 + WQz * v12_6_2 + (VT)1.0 * oo2ze * v4_6_2 + (VT)1.0 * oo2e * (v12_1_1 - rho_e * v12_1_2);
            const VT v13_14_0 = QCz * v13_6_0 + WQz * v13_6_1 + (VT)1.0 * oo2e * (v13_1_0 - rho_e * v13_1_1);
            const VT v13_14_1 = QCz * v13_6_1 + WQz * v13_6_2 + (VT)1.0 * oo2e * (v13_1_1 - rho_e * v13_1_2);
            const VT v14_14_0 = QCz * v14_6_0 + WQz * v14_6_1 + (VT)2.0 * oo2ze * v6_6_1 + (VT)1.0 * oo2e * (v14_1_0 - rho_e * v14_1_1);
            const VT v14_14_1 = QCz * v14_6_1 + WQz * v14_6_2 + (VT)2.0 * oo2ze * v6_6_2 + (VT)1.0 * oo2e * (v14_1_1 - rho_e * v14_1_2);
            const VT v15_14_0 = QCz * v15_6_0 + WQz * v15_6_1 + (VT)1.0 * oo2ze * v5_6_1 + (VT)1.0 * oo2e * (v15_1_0 - rho_e * v15_1_1);
            const VT v15_14_1 = QCz * v15_6_1 + WQz * v15_6_2 + (VT)1.0 * oo2ze * v5_6_2 + (VT)1.0 * oo2e * (v15_1_1 - rho_e * v15_1_2);
            const VT v16_14_0 = QCz * v16_6_0 + WQz * v16_6_1 + (VT)1.0 * oo2e * (v16_1_0 - rho_e * v16_1_1);
            const VT v16_14_1 = QCz * v16_6_1 + WQz * v16_6_2 + (VT)1.0 * oo2e * (v16_1_1 - rho_e * v16_1_2);
            const VT v17_14_0 = QCz * v17_6_0 + WQz * v17_6_1 + (VT)1.0 * oo2ze * v7_6_1 + (VT)1.0 * oo2e * (v17_1_0 - rho_e * v17_1_1);
            const VT v17_14_1 = QCz * v17_6_1 + WQz * v17_6_2 + (VT)1.0 * oo2ze * v7_6_2 + (VT)1.0 * oo2e * (v17_1_1 - rho_e * v17_1_2);
            const VT v18_14_0 = QCz * v18_6_0 + WQz * v18_6_1 + (VT)2.0 * oo2ze * v8_6_1 + (VT)1.0 * oo2e * (v18_1_0 - rho_e * v18_1_1);
            const VT v18_14_1 = QCz * v18_6_1 + WQz * v18_6_2 + (VT)2.0 * oo2ze * v8_6_2 + (VT)1.0 * oo2e * (v18_1_1 - rho_e * v18_1_2);
            const VT v19_14_0 = QCz * v19_6_0 + WQz * v19_6_1 + (VT)3.0 * oo2ze * v9_6_1 + (VT)1.0 * oo2e * (v19_1_0 - rho_e * v19_1_1);
            const VT v19_14_1 = QCz * v19_6_1 + WQz * v19_6_2 + (VT)3.0 * oo2ze * v9_6_2 + (VT)1.0 * oo2e * (v19_1_1 - rho_e * v19_1_2);
            const VT v20_14_0 = QCz * v20_6_0 + WQz * v20_6_1 + (VT)1.0 * oo2e * (v20_1_0 - rho_e * v20_1_1);
            const VT v20_14_1 = QCz * v20_6_1 + WQz * v20_6_2 + (VT)1.0 * oo2e * (v20_1_1 - rho_e * v20_1_2);
            const VT v21_14_0 = QCz * v21_6_0 + WQz * v21_6_1 + (VT)1.0 * oo2e * (v21_1_0 - rho_e * v21_1_1);
            const VT v21_14_1 = QCz * v21_6_1 + WQz * v21_6_2 + (VT)1.0 * oo2e * (v21_1_1 - rho_e * v21_1_2);
            const VT v22_14_0 = QCz * v22_6_0 + WQz * v22_6_1 + (VT)1.0 * oo2ze * v10_6_1 + (VT)1.0 * oo2e * (v22_1_0 - rho_e * v22_1_1);
            const VT v22_14_1 = QCz * v22_6_1 + WQz * v22_6_2 + (VT)1.0 * oo2ze * v10_6_2 + (VT)1.0 * oo2e * (v22_1_1 - rho_e * v22_1_2);
            const VT v23_14_0 = QCz * v23_6_0 + WQz * v23_6_1 + (VT)1.0 * oo2e * (v23_1_0 - rho_e * v23_1_1);
            const VT v23_14_1 = QCz * v23_6_1 + WQz * v23_6_2 + (VT)1.0 * oo2e * (v23_1_1 - rho_e * v23_1_2);
            const VT v24_14_0 = QCz * v24_6_0 + WQz * v24_6_1 + (VT)1.0 * oo2ze * v11_6_1 + (VT)1.0 * oo2e * (v24_1_0 - rho_e * v24_1_1);
            const VT v24_14_1 = QCz * v24_6_1 + WQz * v24_6_2 + (VT)1.0 * oo2ze * v11_6_2 + (VT)1.0 * oo2e * (v24_1_1 - rho_e * v24_1_2);
            const VT v25_14_0 = QCz * v25_6_0 + WQz * v25_6_1 + (VT)2.0 * oo2ze * v12_6_1 + (VT)1.0 * oo2e * (v25_1_0 - rho_e * v25_1_1);
            const VT v25_14_1 = QCz * v25_6_1 + WQz * v25_6_2 + (VT)2.0 * oo2ze * v12_6_2 + (VT)1.0 * oo2e * (v25_1_1 - rho_e * v25_1_2);
            const VT v26_14_0 = QCz * v26_6_0 + WQz * v26_6_1 + (VT)1.0 * oo2e * (v26_1_0 - rho_e * v26_1_1);
            const VT v26_14_1 = QCz * v26_6_1 + WQz * v26_6_2 + (VT)1.0 * oo2e * (v26_1_1 - rho_e * v26_1_2);
            const VT v27_14_0 = QCz * v27_6_0 + WQz * v27_6_1 + (VT)1.0 * oo2ze * v13_6_1 + (VT)1.0 * oo2e * (v27_1_0 - rho_e * v27_1_1);
            const VT v27_14_1 = QCz * v27_6_1 + WQz * v27_6_2 + (VT)1.0 * oo2ze * v13_6_2 + (VT)1.0 * oo2e * (v27_1_1 - rho_e * v27_1_2);
            const VT v28_14_0 = QCz * v28_6_0 + WQz * v28_6_1 + (VT)2.0 * oo2ze * v15_6_1 + (VT)1.0 * oo2e * (v28_1_0 - rho_e * v28_1_1);
            const VT v28_14_1 = QCz * v28_6_1 + WQz * v28_6_2 + (VT)2.0 * oo2ze * v15_6_2 + (VT)1.0 * oo2e * (v28_1_1 - rho_e * v28_1_2);
            const VT v29_14_0 = QCz * v29_6_0 + WQz * v29_6_1 + (VT)3.0 * oo2ze * v14_6_1 + (VT)1.0 * oo2e * (v29_1_0 - rho_e * v29_1_1);
            const VT v29_14_1 = QCz * v29_6_1 + WQz * v29_6_2 + (VT)3.0 * oo2ze * v14_6_2 + (VT)1.0 * oo2e * (v29_1_1 - rho_e * v29_1_2);
            const VT v30_14_0 = QCz * v30_6_0 + WQz * v30_6_1 + (VT)1.0 * oo2e * (v30_1_0 - rho_e * v30_1_1);
            const VT v30_14_1 = QCz * v30_6_1 + WQz * v30_6_2 + (VT)1.0 * oo2e * (v30_1_1 - rho_e * v30_1_2);
            const VT v31_14_0 = QCz * v31_6_0 + WQz * v31_6_1 + (VT)1.0 * oo2ze * v16_6_1 + (VT)1.0 * oo2e * (v31_1_0 - rho_e * v31_1_1);
            const VT v31_14_1 = QCz * v31_6_1 + WQz * v31_6_2 + (VT)1.0 * oo2ze * v16_6_2 + (VT)1.0 * oo2e * (v31_1_1 - rho_e * v31_1_2);
            const VT v32_14_0 = QCz * v32_6_0 + WQz * v32_6_1 + (VT)2.0 * oo2ze * v17_6_1 + (VT)1.0 * oo2e * (v32_1_0 - rho_e * v32_1_1);
            const VT v32_14_1 = QCz * v32_6_1 + WQz * v32_6_2 + (VT)2.0 * oo2ze * v17_6_2 + (VT)1.0 * oo2e * (v32_1_1 - rho_e * v32_1_2);
            const VT v33_14_0 = QCz * v33_6_0 + WQz * v33_6_1 + (VT)3.0 * oo2ze * v18_6_1 + (VT)1.0 * oo2e * (v33_1_0 - rho_e * v33_1_1);
            const VT v33_14_1 = QCz * v33_6_1 + WQz * v33_6_2 + (VT)3.0 * oo2ze * v18_6_2 + (VT)1.0 * oo2e * (v33_1_1 - rho_e * v33_1_2);
            const VT v34_14_0 = QCz * v34_6_0 + WQz * v34_6_1 + (VT)4.0 * oo2ze * v19_6_1 + (VT)1.0 * oo2e * (v34_1_0 - rho_e * v34_1_1);
            const VT v34_14_1 = QCz * v34_6_1 + WQz * v34_6_2 + (VT)4.0 * oo2ze * v19_6_2 + (VT)1.0 * oo2e * (v34_1_1 - rho_e * v34_1_2);
            const VT v1_15_1 = QCx * v1_8_1 + WQx * v1_8_2 + (VT)1.0 * oo2ze * v0_8_2;
            const VT v2_15_1 = QCx * v2_8_1 + WQx * v2_8_2;
            const VT v3_15_1 = QCx * v3_8_1 + WQx * v3_8_2;
            const VT v4_15_0 = QCx * v4_8_0 + WQx * v4_8_1 + (VT)2.0 * oo2ze * v1_8_1;
            const VT v4_15_1 = QCx * v4_8_1 + WQx * v4_8_2 + (VT)2.0 * oo2ze * v1_8_2;
            const VT v5_15_0 = QCx * v5_8_0 + WQx * v5_8_1 + (VT)1.0 * oo2ze * v2_8_1;
            const VT v5_15_1 = QCx * v5_8_1 + WQx * v5_8_2 + (VT)1.0 * oo2ze * v2_8_2;
            const VT v6_15_0 = QCx * v6_8_0 + WQx * v6_8_1 + (VT)1.0 * oo2ze * v3_8_1;
            const VT v6_15_1 = QCx * v6_8_1 + WQx * v6_8_2 + (VT)1.0 * oo2ze * v3_8_2;
            const VT v7_15_0 = QCx * v7_8_0 + WQx * v7_8_1;
            const VT v7_15_1 = QCx * v7_8_1 + WQx * v7_8_2;
            const VT v8_15_0 = QCx * v8_8_0 + WQx * v8_8_1;
            const VT v8_15_1 = QCx * v8_8_1 + WQx * v8_8_2;
            const VT v9_15_0 = QCx * v9_8_0 + WQx * v9_8_1;
            const VT v9_15_1 = QCx * v9_8_1 + WQx * v9_8_2;
            const VT v10_15_0 = QCx * v10_8_0 + WQx * v10_8_1 + (VT)3.0 * oo2ze * v4_8_1;
            const VT v10_15_1 = QCx * v10_8_1 + WQx * v10_8_2 + (VT)3.0 * oo2ze * v4_8_2;
            const VT v11_15_0 = QCx * v11_8_0 + WQx * v11_8_1 + (VT)2.0 * oo2ze * v5_8_1;
            const VT v11_15_1 = QCx * v11_8_1 + WQx * v11_8_2 + (VT)2.0 * oo2ze * v5_8_2;
            const VT v12_15_0 = QCx * v12_8_0 + WQx * v12_8_1 + (VT)2.0 * oo2ze * v6_8_1;
            const VT v12_15_1 = QCx * v12_8_1 + WQx * v12_8_2 + (VT)2.0 * oo2ze * v6_8_2;
            const VT v13_15_0 = QCx * v13_8_0 + WQx * v13_8_1 + (VT)1.0 * oo2ze * v7_8_1;
            const VT v13_15_1 = QCx * v13_8_1 + WQx * v13_8_2 + (VT)1.0 * oo2ze * v7_8_2;
            const VT v14_15_0 = QCx * v14_8_0 + WQx * v14_8_1 + (VT)1.0 * oo2ze * v9_8_1;
            const VT v14_15_1 = QCx * v14_8_1 + WQx * v14_8_2 + (VT)1.0 * oo2ze * v9_8_2;
            const VT v15_15_0 = QCx * v15_8_0 + WQx * v15_8_1 + (VT)1.0 * oo2ze * v8_8_1;
            const VT v15_15_1 = QCx * v15_8_1 + WQx * v15_8_2 + (VT)1.0 * oo2ze * v8_8_2;
            const VT v16_15_0 = QCx * v16_8_0 + WQx * v16_8_1;
            const VT v16_15_1 = QCx * v16_8_1 + WQx * v16_8_2;
            const VT v17_15_0 = QCx * v17_8_0 + WQx * v17_8_1;
            const VT v17_15_1 = QCx * v17_8_1 + WQx * v17_8_2;
            const VT v18_15_0 = QCx * v18_8_0 + WQx * v18_8_1;
            const VT v18_15_1 = QCx * v18_8_1 + WQx * v18_8_2;
            const VT v19_15_0 = QCx * v19_8_0 + WQx * v19_8_1;
            const VT v19_15_1 = QCx * v19_8_1 + WQx * v19_8_2;
            const VT v20_15_0 = QCx * v20_8_0 + WQx * v20_8_1 + (VT)4.0 * oo2ze * v10_8_1;
            const VT v20_15_1 = QCx * v20_8_1 + WQx * v20_8_2 + (VT)4.0 * oo2ze * v10_8_2;
            const VT v21_15_0 = QCx * v21_8_0 + WQx * v21_8_1 + (VT)3.0 * oo2ze * v11_8_1;
            const VT v21_15_1 = QCx * v21_8_1 + WQx * v21_8_2 + (VT)3.0 * oo2ze * v11_8_2;
            const VT v22_15_0 = QCx * v22_8_0 + WQx * v22_8_1 + (VT)3.0 * oo2ze * v12_8_1;
            const VT v22_15_1 = QCx * v22_8_1 + WQx * v22_8_2 + (VT)3.0 * oo2ze * v12_8_2;
            const VT v23_15_0 = QCx * v23_8_0 + WQx * v23_8_1 + (VT)2.0 * oo2ze * v13_8_1;
            const VT v23_15_1 = QCx * v23_8_1 + WQx * v23_8_2 + (VT)2.0 * oo2ze * v13_8_2;
            const VT v24_15_0 = QCx * v24_8_0 + WQx * v24_8_1 + (VT)2.0 * oo2ze * v15_8_1;
            const VT v24_15_1 = QCx * v24_8_1 + WQx * v24_8_2 + (VT)2.0 * oo2ze * v15_8_2;
            const VT v25_15_0 = QCx * v25_8_0 + WQx * v25_8_1 + (VT)2.0 * oo2ze * v14_8_1;
            const VT v25_15_1 = QCx * v25_8_1 + WQx * v25_8_2 + (VT)2.0 * oo2ze * v14_8_2;
            const VT v26_15_0 = QCx * v26_8_0 + WQx * v26_8_1 + (VT)1.0 * oo2ze * v16_8_1;
            const VT v26_15_1 = QCx * v26_8_1 + WQx * v26_8_2 + (VT)1.0 * oo2ze * v16_8_2;
            const VT v27_15_0 = QCx * v27_8_0 + WQx * v27_8_1 + (VT)1.0 * oo2ze * v17_8_1;
            const VT v27_15_1 = QCx * v27_8_1 + WQx * v27_8_2 + (VT)1.0 * oo2ze * v17_8_2;
            const VT v28_15_0 = QCx * v28_8_0 + WQx * v28_8_1 + (VT)1.0 * oo2ze * v18_8_1;
            const VT v28_15_1 = QCx * v28_8_1 + WQx * v28_8_2 + (VT)1.0 * oo2ze * v18_8_2;
            const VT v29_15_0 = QCx * v29_8_0 + WQx * v29_8_1 + (VT)1.0 * oo2ze * v19_8_1;
            const VT v29_15_1 = QCx * v29_8_1 + WQx * v29_8_2 + (VT)1.0 * oo2ze * v19_8_2;
            const VT v30_15_0 = QCx * v30_8_0 + WQx * v30_8_1;
            const VT v30_15_1 = QCx * v30_8_1 + WQx * v30_8_2;
            const VT v31_15_0 = QCx * v31_8_0 + WQx * v31_8_1;
            const VT v31_15_1 = QCx * v31_8_1 + WQx * v31_8_2;
            const VT v32_15_0 = QCx * v32_8_0 + WQx * v32_8_1;
            const VT v32_15_1 = QCx * v32_8_1 + WQx * v32_8_2;
            const VT v33_15_0 = QCx * v33_8_0 + WQx * v33_8_1;
            const VT v33_15_1 = QCx * v33_8_1 + WQx * v33_8_2;
            const VT v34_15_0 = QCx * v34_8_0 + WQx * v34_8_1;
            const VT v34_15_1 = QCx * v34_8_1 + WQx * v34_8_2;
            const VT v1_16_1 = QCy * v1_7_1 + WQy * v1_7_2 + (VT)2.0 * oo2e * (v1_2_1 - rho_e * v1_2_2);
            const VT v2_16_1 = QCy * v2_7_1 + WQy * v2_7_2 + (VT)1.0 * oo2ze * v0_7_2 + (VT)2.0 * oo2e * (v2_2_1 - rho_e * v2_2_2);
            const VT v3_16_1 = QCy * v3_7_1 + WQy * v3_7_2 + (VT)2.0 * oo2e * (v3_2_1 - rho_e * v3_2_2);
            const VT v4_16_0 = QCy * v4_7_0 + WQy * v4_7_1 + (VT)2.0 * oo2e * (v4_2_0 - rho_e * v4_2_1);
            const VT v4_16_1 = QCy * v4_7_1 + WQy * v4_7_2 + (VT)2.0 * oo2e * (v4_2_1 - rho_e * v4_2_2);
            const VT v5_16_0 = QCy * v5_7_0 + WQy * v5_7_1 + (VT)1.0 * oo2ze * v1_7_1 + (VT)2.0 * oo2e * (v5_2_0 - rho_e * v5_2_1);
            const VT v5_16_1 = QCy * v5_7_1 + WQy * v5_7_2 + (VT)1.0 * oo2ze * v1_7_2 + (VT)2.0 * oo2e * (v5_2_1 - rho_e * v5_2_2);
            const VT v6_16_0 = QCy * v6_7_0 + WQy * v6_7_1 + (VT)2.0 * oo2e * (v6_2_0 - rho_e * v6_2_1);
            const VT v6_16_1 = QCy * v6_7_1 + WQy * v6_7_2 + (VT)2.0 * oo2e * (v6_2_1 - rho_e * v6_2_2);
            const VT v7_16_0 = QCy * v7_7_0 + WQy * v7_7_1 + (VT)2.0 * oo2ze * v2_7_1 + (VT)2.0 * oo2e * (v7_2_0 - rho_e * v7_2_1);
            const VT v7_16_1 = QCy * v7_7_1 + WQy * v7_7_2 + (VT)2.0 * oo2ze * v2_7_2 + (VT)2.0 * oo2e * (v7_2_1 - rho_e * v7_2_2);
            const VT v8_16_0 = QCy * v8_7_0 + WQy * v8_7_1 + (VT)1.0 * oo2ze * v3_7_1 + (VT)2.0 * oo2e * (v8_2_0 - rho_e * v8_2_1);
            const VT v8_16_1 = QCy * v8_7_1 + WQy * v8_7_2 + (VT)1.0 * oo2ze * v3_7_2 + (VT)2.0 * oo2e * (v8_2_1 - rho_e * v8_2_2);
            const VT v9_16_0 = QCy * v9_7_0 + WQy * v9_7_1 + (VT)2.0 * oo2e * (v9_2_0 - rho_e * v9_2_1);
            const VT v9_16_1 = QCy * v9_7_1 + WQy * v9_7_2 + (VT)2.0 * oo2e * (v9_2_1 - rho_e * v9_2_2);
            const VT v10_16_0 = QCy * v10_7_0 + WQy * v10_7_1 + (VT)2.0 * oo2e * (v10_2_0 - rho_e * v10_2_1);
            const VT v10_16_1 = QCy * v10_7_1 + WQy * v10_7_2 + (VT)2.0 * oo2e * (v10_2_1 - rho_e * v10_2_2);
            const VT v11_16_0 = QCy * v11_7_0 + WQy * v11_7_1 + (VT)1.0 * oo2ze * v4_7_1 + (VT)2.0 * oo2e * (v11_2_0 - rho_e * v11_2_1);
            const VT v11_16_1 = QCy * v11_7_1 + WQy * v11_7_2 + (VT)1.0 * oo2ze * v4_7_2 + (VT)2.0 * oo2e * (v11_2_1 - rho_e * v11_2_2);
            const VT v12_16_0 = QCy * v12_7_0 + WQy * v12_7_1 + (VT)2.0 * oo2e * (v12_2_0 - rho_e * v12_2_1);
            const VT v12_16_1 = QCy * v12_7_1 + WQy * v12_7_2 + (VT)2.0 * oo2e * (v12_2_1 - rho_e * v12_2_2);
            const VT v13_16_0 = QCy * v13_7_0 + WQy * v13_7_1 + (VT)2.0 * oo2ze * v5_7_1 + (VT)2.0 * oo2e * (v13_2_0 - rho_e * v13_2_1);
            const VT v13_16_1 = QCy * v13_7_1 + WQy * v13_7_2 + (VT)2.0 * oo2ze * v5_7_2 + (VT)2.0 * oo2e * (v13_2_1 - rho_e * v13_2_2);
            const VT v14_16_0 = QCy * v14_7_0 + WQy * v14_7_1 + (VT)2.0 * oo2e * (v14_2_0 - rho_e * v14_2_1);
            const VT v14_16_1 = QCy * v14_7_1 + WQy * v14_7_2 + (VT)2.0 * oo2e * (v14_2_1 - rho_e * v14_2_2);
            const VT v15_16_0 = QCy * v15_7_0 + WQy * v15_7_1 + (VT)1.0 * oo2ze * v6_7_1 + (VT)2.0 * oo2e * (v15_2_0 - rho_e * v15_2_1);
            const VT v15_16_1 = QCy * v15_7_1 + WQy * v15_7_2 + (VT)1.0 * oo2ze * v6_7_2 + (VT)2.0 * oo2e * (v15_2_1 - rho_e * v15_2_2);
            const VT v16_16_0 = QCy * v16_7_0 + WQy * v16_7_1 + (VT)3.0 * oo2ze * v7_7_1 + (VT)2.0 * oo2e * (v16_2_0 - rho_e * v16_2_1);
            const VT v16_16_1 = QCy * v16_7_1 + WQy * v16_7_2 + (VT)3.0 * oo2ze * v7_7_2 + (VT)2.0 * oo2e * (v16_2_1 - rho_e * v16_2_2);
            const VT v17_16_0 = QCy * v17_7_0 + WQy * v17_7_1 + (VT)2.0 * oo2ze * v8_7_1 + (VT)2.0 * oo2e * (v17_2_0 - rho_e * v17_2_1);
            const VT v17_16_1 = QCy * v17_7_1 + WQy * v17_7_2 + (VT)2.0 * oo2ze * v8_7_2 + (VT)2.0 * oo2e * (v17_2_1 - rho_e * v17_2_2);
            const VT v18_16_0 = QCy * v18_7_0 + WQy * v18_7_1 + (VT)1.0 * oo2ze * v9_7_1 + (VT)2.0 * oo2e * (v18_2_0 - rho_e * v18_2_1);
            const VT v18_16_1 = QCy * v18_7_1 + WQy * v18_7_2 + (VT)1.0 * oo2ze * v9_7_2 + (VT)2.0 * oo2e * (v18_2_1 - rho_e * v18_2_2);
            const VT v19_16_0 = QCy * v19_7_0 + WQy * v19_7_1 + (VT)2.0 * oo2e * (v19_2_0 - rho_e * v19_2_1);
            const VT v19_16_1 = QCy * v19_7_1 + WQy * v19_7_2 + (VT)2.0 * oo2e * (v19_2_1 - rho_e * v19_2_2);
            const VT v20_16_0 = QCy * v20_7_0 + WQy * v20_7_1 + (VT)2.0 * oo2e * (v20_2_0 - rho_e * v20_2_1);
            const VT v20_16_1 = QCy * v20_7_1 + WQy * v20_7_2 + (VT)2.0 * oo2e * (v20_2_1 - rho_e * v20_2_2);
            const VT v21_16_0 = QCy * v21_7_0 + WQy * v21_7_1 + (VT)1.0 * oo2ze * v10_7_1 + (VT)2.0 * oo2e * (v21_2_0 - rho_e * v21_2_1);
            const VT v21_16_1 = QCy * v21_7_1 + WQy * v21_7_2 + (VT)1.0 * oo2ze * v10_7_2 + (VT)2.0 * oo2e * (v21_2_1 - rho_e * v21_2_2);
            const VT v22_16_0 = QCy * v22_7_0 + WQy * v22_7_1 + (VT)2.0 * oo2e * (v22_2_0 - rho_e * v22_2_1);
            const VT v22_16_1 = QCy * v22_7_1 + WQy * v22_7_2 + (VT)2.0 * oo2e * (v22_2_1 - rho_e * v22_2_2);
            const VT v23_16_0 = QCy * v23_7_0 + WQy * v23_7_1 + (VT)2.0 * oo2ze * v11_7_1 + (VT)2.0 * oo2e * (v23_2_0 - rho_e * v23_2_1);
            const VT v23_16_1 = QCy * v23_7_1 + WQy * v23_7_2 + (VT)2.0 * oo2ze * v11_7_2 + (VT)2.0 * oo2e * (v23_2_1 - rho_e * v23_2_2);
            const VT v24_16_0 = QCy * v24_7_0 + WQy * v24_7_1 + (VT)1.0 * oo2ze * v12_7_1 + (VT)2.0 * oo2e * (v24_2_0 - rho_e * v24_2_1);
            const VT v24_16_1 = QCy * v24_7_1 + WQy * v24_7_2 + (VT)1.0 * oo2ze * v12_7_2 + (VT)2.0 * oo2e * (v24_2_1 - rho_e * v24_2_2);
            const VT v25_16_0 = QCy * v25_7_0 + WQy * v25_7_1 + (VT)2.0 * oo2e * (v25_2_0 - rho_e * v25_2_1);
            const VT v25_16_1 = QCy * v25_7_1 + WQy * v25_7_2 + (VT)2.0 * oo2e * (v25_2_1 - rho_e * v25_2_2);
            const VT v26_16_0 = QCy * v26_7_0 + WQy * v26_7_1 + (VT)3.0 * oo2ze * v13_7_1 + (VT)2.0 * oo2e * (v26_2_0 - rho_e * v26_2_1);
            const VT v26_16_1 = QCy * v26_7_1 + WQy * v26_7_2 + (VT)3.0 * oo2ze * v13_7_2 + (VT)2.0 * oo2e * (v26_2_1 - rho_e * v26_2_2);
            const VT v27_16_0 = QCy * v27_7_0 + WQy * v27_7_1 + (VT)2.0 * oo2ze * v15_7_1 + (VT)2.0 * oo2e * (v27_2_0 - rho_e * v27_2_1);
            const VT v27_16_1 = QCy * v27_7_1 + WQy * v27_7_2 + (VT)2.0 * oo2ze * v15_7_2 + (VT)2.0 * oo2e * (v27_2_1 - rho_e * v27_2_2);
            const VT v28_16_0 = QCy * v28_7_0 + WQy * v28_7_1 + (VT)1.0 * oo2ze * v14_7_1 + (VT)2.0 * oo2e * (v28_2_0 - rho_e * v28_2_1);
            const VT v28_16_1 = QCy * v28_7_1 + WQy * v28_7_2 + (VT)1.0 * oo2ze * v14_7_2 + (VT)2.0 * oo2e * (v28_2_1 - rho_e * v28_2_2);
            const VT v29_16_0 = QCy * v29_7_0 + WQy * v29_7_1 + (VT)2.0 * oo2e * (v29_2_0 - rho_e * v29_2_1);
            const VT v29_16_1 = QCy * v29_7_1 + WQy * v29_7_2 + (VT)2.0 * oo2e * (v29_2_1 - rho_e * v29_2_2);
            const VT v30_16_0 = QCy * v30_7_0 + WQy * v30_7_1 + (VT)4.0 * oo2ze * v16_7_1 + (VT)2.0 * oo2e * (v30_2_0 - rho_e * v30_2_1);
            const VT v30_16_1 = QCy * v30_7_1 + WQy * v30_7_2 + (VT)4.0 * oo2ze * v16_7_2 + (VT)2.0 * oo2e * (v30_2_1 - rho_e * v30_2_2);
            const VT v31_16_0 = QCy * v31_7_0 + WQy * v31_7_1 + (VT)3.0 * oo2ze * v17_7_1 + (VT)2.0 * oo2e * (v31_2_0 - rho_e * v31_2_1);
            const VT v31_16_1 = QCy * v31_7_1 + WQy * v31_7_2 + (VT)3.0 * oo2ze * v17_7_2 + (VT)2.0 * oo2e * (v31_2_1 - rho_e * v31_2_2);
            const VT v32_16_0 = QCy * v32_7_0 + WQy * v32_7_1 + (VT)2.0 * oo2ze * v18_7_1 + (VT)2.0 * oo2e * (v32_2_0 - rho_e * v32_2_1);
            const VT v32_16_1 = QCy * v32_7_1 + WQy * v32_7_2 + (VT)2.0 * oo2ze * v18_7_2 + (VT)2.0 * oo2e * (v32_2_1 - rho_e * v32_2_2);
            const VT v33_16_0 = QCy * v33_7_0 + WQy * v33_7_1 + (VT)1.0 * oo2ze * v19_7_1 + (VT)2.0 * oo2e * (v33_2_0 - rho_e * v33_2_1);
            const VT v33_16_1 = QCy * v33_7_1 + WQy * v33_7_2 + (VT)1.0 * oo2ze * v19_7_2 + (VT)2.0 * oo2e * (v33_2_1 - rho_e * v33_2_2);
            const VT v34_16_0 = QCy * v34_7_0 + WQy * v34_7_1 + (VT)2.0 * oo2e * (v34_2_0 - rho_e * v34_2_1);
            const VT v34_16_1 = QCy * v34_7_1 + WQy * v34_7_2 + (VT)2.0 * oo2e * (v34_2_1 - rho_e * v34_2_2);
            const VT v1_17_1 = QCy * v1_8_1 + WQy * v1_8_2 + (VT)1.0 * oo2e * (v1_3_1 - rho_e * v1_3_2);
            const VT v2_17_1 = QCy * v2_8_1 + WQy * v2_8_2 + (VT)1.0 * oo2ze * v0_8_2 + (VT)1.0 * oo2e * (v2_3_1 - rho_e * v2_3_2);
            const VT v3_17_1 = QCy * v3_8_1 + WQy * v3_8_2 + (VT)1.0 * oo2e * (v3_3_1 - rho_e * v3_3_2);
            const VT v4_17_0 = QCy * v4_8_0 + WQy * v4_8_1 + (VT)1.0 * oo2e * (v4_3_0 - rho_e * v4_3_1);
            const VT v4_17_1 = QCy * v4_8_1 + WQy * v4_8_2 + (VT)1.0 * oo2e * (v4_3_1 - rho_e * v4_3_2);
            const VT v5_17_0 = QCy * v5_8_0 + WQy * v5_8_1 + (VT)1.0 * oo2ze * v1_8_1 + (VT)1.0 * oo2e * (v5_3_0 - rho_e * v5_3_1);
            const VT v5_17_1 = QCy * v5_8_1 + WQy * v5_8_2 + (VT)1.0 * oo2ze * v1_8_2 + (VT)1.0 * oo2e * (v5_3_1 - rho_e * v5_3_2);
            const VT v6_17_0 = QCy * v6_8_0 + WQy * v6_8_1 + (VT)1.0 * oo2e * (v6_3_0 - rho_e * v6_3_1);
            const VT v6_17_1 = QCy * v6_8_1 + WQy * v6_8_2 + (VT)1.0 * oo2e * (v6_3_1 - rho_e * v6_3_2);
            const VT v7_17_0 = QCy * v7_8_0 + WQy * v7_8_1 + (VT)2.0 * oo2ze * v2_8_1 + (VT)1.0 * oo2e * (v7_3_0 - rho_e * v7_3_1);
            const VT v7_17_1 = QCy * v7_8_1 + WQy * v7_8_2 + (VT)2.0 * oo2ze * v2_8_2 + (VT)1.0 * oo2e * (v7_3_1 - rho_e * v7_3_2);
            const VT v8_17_0 = QCy * v8_8_0 + WQy * v8_8_1 + (VT)1.0 * oo2ze * v3_8_1 + (VT)1.0 * oo2e * (v8_3_0 - rho_e * v8_3_1);
            const VT v8_17_1 = QCy * v8_8_1 + WQy * v8_8_2 + (VT)1.0 * oo2ze * v3_8_2 + (VT)1.0 * oo2e * (v8_3_1 - rho_e * v8_3_2);
            const VT v9_17_0 = QCy * v9_8_0 + WQy * v9_8_1 + (VT)1.0 * oo2e * (v9_3_0 - rho_e * v9_3_1);
            const VT v9_17_1 = QCy * v9_8_1 + WQy * v9_8_2 + (VT)1.0 * oo2e * (v9_3_1 - rho_e * v9_3_2);
            const VT v10_17_0 = QCy * v10_8_0 + WQy * v10_8_1 + (VT)1.0 * oo2e * (v10_3_0 - rho_e * v10_3_1);
            const VT v10_17_1 = QCy * v10_8_1 + WQy * v10_8_2 + (VT)1.0 * oo2e * (v10_3_1 - rho_e * v10_3_2);
            const VT v11_17_0 = QCy * v11_8_0 + WQy * v11_8_1 + (VT)1.0 * oo2ze * v4_8_1 + (VT)1.0 * oo2e * (v11_3_0 - rho_e * v11_3_1);
            const VT v11_17_1 = QCy * v11_8_1 + WQy * v11_8_2 + (VT)1.0 * oo2ze * v4_8_2 + (VT)1.0 * oo2e * (v11_3_1 - rho_e * v11_3_2);
            const VT v12_17_0 = QCy * v12_8_0 + WQy * v12_8_1 + (VT)1.0 * oo2e * (v12_3_0 - rho_e * v12_3_1);
            const VT v12_17_1 = QCy * v12_8_1 + WQy * v12_8_2 + (VT)1.0 * oo2e * (v12_3_1 - rho_e * v12_3_2);
            const VT v13_17_0 = QCy * v13_8_0 + WQy * v13_8_1 + (VT)2.0 * oo2ze * v5_8_1 + (VT)1.0 * oo2e * (v13_3_0 - rho_e * v13_3_1);
            const VT v13_17_1 = QCy * v13_8_1 + WQy * v13_8_2 + (VT)2.0 * oo2ze * v5_8_2 + (VT)1.0 * oo2e * (v13_3_1 - rho_e * v13_3_2);
            const VT v14_17_0 = QCy * v14_8_0 + WQy * v14_8_1 + (VT)1.0 * oo2e * (v14_3_0 - rho_e * v14_3_1);
            const VT v14_17_1 = QCy * v14_8_1 + WQy * v14_8_2 + (VT)1.0 * oo2e * (v14_3_1 - rho_e * v14_3_2);
            const VT v15_17_0 = QCy * v15_8_0 + WQy * v15_8_1 + (VT)1.0 * oo2ze * v6_8_1 + (VT)1.0 * oo2e * (v15_3_0 - rho_e * v15_3_1);
            const VT v15_17_1 = QCy * v15_8_1 + WQy * v15_8_2 + (VT)1.0 * oo2ze * v6_8_2 + (VT)1.0 * oo2e * (v15_3_1 - rho_e * v15_3_2);
            const VT v16_17_0 = QCy * v16_8_0 + WQy * v16_8_1 + (VT)3.0 * oo2ze * v7_8_1 + (VT)1.0 * oo2e * (v16_3_0 - rho_e * v16_3_1);
            const VT v16_17_1 = QCy * v16_8_1 + WQy * v16_8_2 + (VT)3.0 * oo2ze * v7_8_2 + (VT)1.0 * oo2e * (v16_3_1 - rho_e * v16_3_2);
            const VT v17_17_0 = QCy * v17_8_0 + WQy * v17_8_1 + (VT)2.0 * oo2ze * v8_8_1 + (VT)1.0 * oo2e * (v17_3_0 - rho_e * v17_3_1);
            const VT v17_17_1 = QCy * v17_8_1 + WQy * v17_8_2 + (VT)2.0 * oo2ze * v8_8_2 + (VT)1.0 * oo2e * (v17_3_1 - rho_e * v17_3_2);
            const VT v18_17_0 = QCy * v18_8_0 + WQy * v18_8_1 + (VT)1.0 * oo2ze * v9_8_1 + (VT)1.0 * oo2e * (v18_3_0 - rho_e * v18_3_1);
            const VT v18_17_1 = QCy * v18_8_1 + WQy * v18_8_2 + (VT)1.0 * oo2ze * v9_8_2 + (VT)1.0 * oo2e * (v18_3_1 - rho_e * v18_3_2);
            const VT v19_17_0 = QCy * v19_8_0 + WQy * v19_8_1 + (VT)1.0 * oo2e * (v19_3_0 - rho_e * v19_3_1);
            const VT v19_17_1 = QCy * v19_8_1 + WQy * v19_8_2 + (VT)1.0 * oo2e * (v19_3_1 - rho_e * v19_3_2);
            const VT v20_17_0 = QCy * v20_8_0 + WQy * v20_8_1 + (VT)1.0 * oo2e * (v20_3_0 - rho_e * v20_3_1);
            const VT v20_17_1 = QCy * v20_8_1 + WQy * v20_8_2 + (VT)1.0 * oo2e * (v20_3_1 - rho_e * v20_3_2);
            const VT v21_17_0 = QCy * v21_8_0 + WQy * v21_8_1 + (VT)1.0 * oo2ze * v10_8_1 + (VT)1.0 * oo2e * (v21_3_0 - rho_e * v21_3_1);
            const VT v21_17_1 = QCy * v21_8_1 + WQy * v21_8_2 + (VT)1.0 * oo2ze * v10_8_2 + (VT)1.0 * oo2e * (v21_3_1 - rho_e * v21_3_2);
            const VT v22_17_0 = QCy * v22_8_0 + WQy * v22_8_1 + (VT)1.0 * oo2e * (v22_3_0 - rho_e * v22_3_1);
            const VT v22_17_1 = QCy * v22_8_1 + WQy * v22_8_2 + (VT)1.0 * oo2e * (v22_3_1 - rho_e * v22_3_2);
            const VT v23_17_0 = QCy * v23_8_0 + WQy * v23_8_1 + (VT)2.0 * oo2ze * v11_8_1 + (VT)1.0 * oo2e * (v23_3_0 - rho_e * v23_3_1);
            const VT v23_17_1 = QCy * v23_8_1 + WQy * v23_8_2 + (VT)2.0 * oo2ze * v11_8_2 + (VT)1.0 * oo2e * (v23_3_1 - rho_e * v23_3_2);
            const VT v24_17_0 = QCy * v24_8_0 + WQy * v24_8_1 + (VT)1.0 * oo2ze * v12_8_1 + (VT)1.0 * oo2e * (v24_3_0 - rho_e * v24_3_1);
            const VT v24_17_1 = QCy * v24_8_1 + WQy * v24_8_2 + (VT)1.0 * oo2ze * v12_8_2 + (VT)1.0 * oo2e * (v24_3_1 - rho_e * v24_3_2);
            const VT v25_17_0 = QCy * v25_8_0 + WQy * v25_8_1 + (VT)1.0 * oo2e * (v25_3_0 - rho_e * v25_3_1);
            const VT v25_17_1 = QCy * v25_8_1 + WQy * v25_8_2 + (VT)1.0 * oo2e * (v25_3_1 - rho_e * v25_3_2);
            const VT v26_17_0 = QCy * v26_8_0 + WQy * v26_8_1 + (VT)3.0 * oo2ze * v13_8_1 + (VT)1.0 * oo2e * (v26_3_0 - rho_e * v26_3_1);
            const VT v26_17_1 = QCy * v26_8_1 + WQy * v26_8_2 + (VT)3.0 * oo2ze * v13_8_2 + (VT)1.0 * oo2e * (v26_3_1 - rho_e * v26_3_2);
            const VT v27_17_0 = QCy * v27_8_0 + WQy * v27_8_1 + (VT)2.0 * oo2ze * v15_8_1 + (VT)1.0 * oo2e * (v27_3_0 - rho_e * v27_3_1);
            const VT v27_17_1 = QCy * v27_8_1 + WQy * v27_8_2 + (VT)2.0 * oo2ze * v15_8_2 + (VT)1.0 * oo2e * (v27_3_1 - rho_e * v27_3_2);
            const VT v28_17_0 = QCy * v28_8_0 + WQy * v28_8_1 + (VT)1.0 * oo2ze * v14_8_1 + (VT)1.0 * oo2e * (v28_3_0 - rho_e * v28_3_1);
            const VT v28_17_1 = QCy * v28_8_1 + WQy * v28_8_2 + (VT)1.0 * oo2ze * v14_8_2 + (VT)1.0 * oo2e * (v28_3_1 - rho_e * v28_3_2);
            const VT v29_17_0 = QCy * v29_8_0 + WQy * v29_8_1 + (VT)1.0 * oo2e * (v29_3_0 - rho_e * v29_3_1);
            const VT v29_17_1 = QCy * v29_8_1 + WQy * v29_8_2 + (VT)1.0 * oo2e * (v29_3_1 - rho_e * v29_3_2);
            const VT v30_17_0 = QCy * v30_8_0 + WQy * v30_8_1 + (VT)4.0 * oo2ze * v16_8_1 + (VT)1.0 * oo2e * (v30_3_0 - rho_e * v30_3_1);
            const VT v30_17_1 = QCy * v30_8_1 + WQy * v30_8_2 + (VT)4.0 * oo2ze * v16_8_2 + (VT)1.0 * oo2e * (v30_3_1 - rho_e * v30_3_2);
            const VT v31_17_0 = QCy * v31_8_0 + WQy * v31_8_1 + (VT)3.0 * oo2ze * v17_8_1 + (VT)1.0 * oo2e * (v31_3_0 - rho_e * v31_3_1);
            const VT v31_17_1 = QCy * v31_8_1 + WQy * v31_8_2 + (VT)3.0 * oo2ze * v17_8_2 + (VT)1.0 * oo2e * (v31_3_1 - rho_e * v31_3_2);
            const VT v32_17_0 = QCy * v32_8_0 + WQy * v32_8_1 + (VT)2.0 * oo2ze * v18_8_1 + (VT)1.0 * oo2e * (v32_3_0 - rho_e * v32_3_1);
            const VT v32_17_1 = QCy * v32_8_1 + WQy * v32_8_2 + (VT)2.0 * oo2ze * v18_8_2 + (VT)1.0 * oo2e * (v32_3_1 - rho_e * v32_3_2);
            const VT v33_17_0 = QCy * v33_8_0 + WQy * v33_8_1 + (VT)1.0 * oo2ze * v19_8_1 + (VT)1.0 * oo2e * (v33_3_0 - rho_e * v33_3_1);
            const VT v33_17_1 = QCy * v33_8_1 + WQy * v33_8_2 + (VT)1.0 * oo2ze * v19_8_2 + (VT)1.0 * oo2e * (v33_3_1 - rho_e * v33_3_2);
            const VT v34_17_0 = QCy * v34_8_0 + WQy * v34_8_1 + (VT)1.0 * oo2e * (v34_3_0 - rho_e * v34_3_1);
            const VT v34_17_1 = QCy * v34_8_1 + WQy * v34_8_2 + (VT)1.0 * oo2e * (v34_3_1 - rho_e * v34_3_2);
            const VT v1_18_1 = QCz * v1_8_1 + WQz * v1_8_2 + (VT)1.0 * oo2e * (v1_2_1 - rho_e * v1_2_2);
            const VT v2_18_1 = QCz * v2_8_1 + WQz * v2_8_2 + (VT)1.0 * oo2e * (v2_2_1 - rho_e * v2_2_2);
            const VT v3_18_1 = QCz * v3_8_1 + WQz * v3_8_2 + (VT)1.0 * oo2ze * v0_8_2 + (VT)1.0 * oo2e * (v3_2_1 - rho_e * v3_2_2);
            const VT v4_18_0 = QCz * v4_8_0 + WQz * v4_8_1 + (VT)1.0 * oo2e * (v4_2_0 - rho_e * v4_2_1);
            const VT v4_18_1 = QCz * v4_8_1 + WQz * v4_8_2 + (VT)1.0 * oo2e * (v4_2_1 - rho_e * v4_2_2);
            const VT v5_18_0 = QCz * v5_8_0 + WQz * v5_8_1 + (VT)1.0 * oo2e * (v5_2_0 - rho_e * v5_2_1);
            const VT v5_18_1 = QCz * v5_8_1 + WQz * v5_8_2 + (VT)1.0 * oo2e * (v5_2_1 - rho_e * v5_2_2);
            const VT v6_18_0 = QCz * v6_8_0 + WQz * v6_8_1 + (VT)1.0 * oo2ze * v1_8_1 + (VT)1.0 * oo2e * (v6_2_0 - rho_e * v6_2_1);
            const VT v6_18_1 = QCz * v6_8_1 + WQz * v6_8_2 + (VT)1.0 * oo2ze * v1_8_2 + (VT)1.0 * oo2e * (v6_2_1 - rho_e * v6_2_2);
            const VT v7_18_0 = QCz * v7_8_0 + WQz * v7_8_1 + (VT)1.0 * oo2e * (v7_2_0 - rho_e * v7_2_1);
            const VT v7_18_1 = QCz * v7_8_1 + WQz * v7_8_2 + (VT)1.0 * oo2e * (v7_2_1 - rho_e * v7_2_2);
            const VT v8_18_0 = QCz * v8_8_0 + WQz * v8_8_1 + (VT)1.0 * oo2ze * v2_8_1 + (VT)1.0 * oo2e * (v8_2_0 - rho_e * v8_2_1);
            const VT v8_18_1 = QCz * v8_8_1 + WQz * v8_8_2 + (VT)1.0 * oo2ze * v2_8_2 + (VT)1.0 * oo2e * (v8_2_1 - rho_e * v8_2_2);
            const VT v9_18_0 = QCz * v9_8_0 + WQz * v9_8_1 + (VT)2.0 * oo2ze * v3_8_1 + (VT)1.0 * oo2e * (v9_2_0 - rho_e * v9_2_1);
            const VT v9_18_1 = QCz * v9_8_1 + WQz * v9_8_2 + (VT)2.0 * oo2ze * v3_8_2 + (VT)1.0 * oo2e * (v9_2_1 - rho_e * v9_2_2);
            const VT v10_18_0 = QCz * v10_8_0 + WQz * v10_8_1 + (VT)1.0 * oo2e * (v10_2_0 - rho_e * v10_2_1);
            const VT v10_18_1 = QCz * v10_8_1 + WQz * v10_8_2 + (VT)1.0 * oo2e * (v10_2_1 - rho_e * v10_2_2);
            const VT v11_18_0 = QCz * v11_8_0 + WQz * v11_8_1 + (VT)1.0 * oo2e * (v11_2_0 - rho_e * v11_2_1);
            const VT v11_18_1 = QCz * v11_8_1 + WQz * v11_8_2 + (VT)1.0 * oo2e * (v11_2_1 - rho_e * v11_2_2);
            const VT v12_18_0 = QCz * v12_8_0 + WQz * v12_8_1 + (VT)1.0 * oo2ze * v4_8_1 + (VT)1.0 * oo2e * (v12_2_0 - rho_e * v12_2_1);
            const VT v12_18_1 = QCz * v12_8_1 + WQz * v12_8_2 + (VT)1.0 * oo2ze * v4_8_2 + (VT)1.0 * oo2e * (v12_2_1 - rho_e * v12_2_2);
            const VT v13_18_0 = QCz * v13_8_0 + WQz * v13_8_1 + (VT)1.0 * oo2e * (v13_2_0 - rho_e * v13_2_1);
            const VT v13_18_1 = QCz * v13_8_1 + WQz * v13_8_2 + (VT)1.0 * oo2e * (v13_2_1 - rho_e * v13_2_2);
            const VT v14_18_0 = QCz * v14_8_0 + WQz * v14_8_1 + (VT)2.0 * oo2ze * v6_8_1 + (VT)1.0 * oo2e * (v14_2_0 - rho_e * v14_2_1);
            const VT v14_18_1 = QCz * v14_8_1 + WQz * v14_8_2 + (VT)2.0 * oo2ze * v6_8_2 + (VT)1.0 * oo2e * (v14_2_1 - rho_e * v14_2_2);
            const VT v15_18_0 = QCz * v15_8_0 + WQz * v15_8_1 + (VT)1.0 * oo2ze * v5_8_1 + (VT)1.0 * oo2e * (v15_2_0 - rho_e * v15_2_1);
            const VT v15_18_1 = QCz * v15_8_1 + WQz * v15_8_2 + (VT)1.0 * oo2ze * v5_8_2 + (VT)1.0 * oo2e * (v15_2_1 - rho_e * v15_2_2);
            const VT v16_18_0 = QCz * v16_8_0 + WQz * v16_8_1 + (VT)1.0 * oo2e * (v16_2_0 - rho_e * v16_2_1);
            const VT v16_18_1 = QCz * v16_8_1 + WQz * v16_8_2 + (VT)1.0 * oo2e * (v16_2_1 - rho_e * v16_2_2);
            const VT v17_18_0 = QCz * v17_8_0 + WQz * v17_8_1 + (VT)1.0 * oo2ze * v7_8_1 + (VT)1.0 * oo2e * (v17_2_0 - rho_e * v17_2_1);
            const VT v17_18_1 = QCz * v17_8_1 + WQz * v17_8_2 + (VT)1.0 * oo2ze * v7_8_2 + (VT)1.0 * oo2e * (v17_2_1 - rho_e * v17_2_2);
            const VT v18_18_0 = QCz * v18_8_0 + WQz * v18_8_1 + (VT)2.0 * oo2ze * v8_8_1 + (VT)1.0 * oo2e * (v18_2_0 - rho_e * v18_2_1);
            const VT v18_18_1 = QCz * v18_8_1 + WQz * v18_8_2 + (VT)2.0 * oo2ze * v8_8_2 + (VT)1.0 * oo2e * (v18_2_1 - rho_e * v18_2_2);
            const VT v19_18_0 = QCz * v19_8_0 + WQz * v19_8_1 + (VT)3.0 * oo2ze * v9_8_1 + (VT)1.0 * oo2e * (v19_2_0 - rho_e * v19_2_1);
            const VT v19_18_1 = QCz * v19_8_1 + WQz * v19_8_2 + (VT)3.0 * oo2ze * v9_8_2 + (VT)1.0 * oo2e * (v19_2_1 - rho_e * v19_2_2);
            const VT v20_18_0 = QCz * v20_8_0 + WQz * v20_8_1 + (VT)1.0 * oo2e * (v20_2_0 - rho_e * v20_2_1);
            const VT v20_18_1 = QCz * v20_8_1 + WQz * v20_8_2 + (VT)1.0 * oo2e * (v20_2_1 - rho_e * v20_2_2);
            const VT v21_18_0 = QCz * v21_8_0 + WQz * v21_8_1 + (VT)1.0 * oo2e * (v21_2_0 - rho_e * v21_2_1);
            const VT v21_18_1 = QCz * v21_8_1 + WQz * v21_8_2 + (VT)1.0 * oo2e * (v21_2_1 - rho_e * v21_2_2);
            const VT v22_18_0 = QCz * v22_8_0 + WQz * v22_8_1 + (VT)1.0 * oo2ze * v10_8_1 + (VT)1.0 * oo2e * (v22_2_0 - rho_e * v22_2_1);
            const VT v22_18_1 = QCz * v22_8_1 + WQz * v22_8_2 + (VT)1.0 * oo2ze * v10_8_2 + (VT)1.0 * oo2e * (v22_2_1 - rho_e * v22_2_2);
            const VT v23_18_0 = QCz * v23_8_0 + WQz * v23_8_1 + (VT)1.0 * oo2e * (v23_2_0 - rho_e * v23_2_1);
            const VT v23_18_1 = QCz * v23_8_1 + WQz * v23_8_2 + (VT)1.0 * oo2e * (v23_2_1 - rho_e * v23_2_2);
            const VT v24_18_0 = QCz * v24_8_0 + WQz * v24_8_1 + (VT)1.0 * oo2ze * v11_8_1 + (VT)1.0 * oo2e * (v24_2_0 - rho_e * v24_2_1);
            const VT v24_18_1 = QCz * v24_8_1 + WQz * v24_8_2 + (VT)1.0 * oo2ze * v11_8_2 + (VT)1.0 * oo2e * (v24_2_1 - rho_e * v24_2_2);
            const VT v25_18_0 = QCz * v25_8_0 + WQz * v25_8_1 + (VT)2.0 * oo2ze * v12_8_1 + (VT)1.0 * oo2e * (v25_2_0 - rho_e * v25_2_1);
            const VT v25_18_1 = QCz * v25_8_1 + WQz * v25_8_2 + (VT)2.0 * oo2ze * v12_8_2 + (VT)1.0 * oo2e * (v25_2_1 - rho_e * v25_2_2);
            const VT v26_18_0 = QCz * v26_8_0 + WQz * v26_8_1 + (VT)1.0 * oo2e * (v26_2_0 - rho_e * v26_2_1);
            const VT v26_18_1 = QCz * v26_8_1 + WQz * v26_8_2 + (VT)1.0 * oo2e * (v26_2_1 - rho_e * v26_2_2);
            const VT v27_18_0 = QCz * v27_8_0 + WQz * v27_8_1 + (VT)1.0 * oo2ze * v13_8_1 + (VT)1.0 * oo2e * (v27_2_0 - rho_e * v27_2_1);
            const VT v27_18_1 = QCz * v27_8_1 + WQz * v27_8_2 + (VT)1.0 * oo2ze * v13_8_2 + (VT)1.0 * oo2e * (v27_2_1 - rho_e * v27_2_2);
            const VT v28_18_0 = QCz * v28_8_0 + WQz * v28_8_1 + (VT)2.0 * oo2ze * v15_8_1 + (VT)1.0 * oo2e * (v28_2_0 - rho_e * v28_2_1);
            const VT v28_18_1 = QCz * v28_8_1 + WQz * v28_8_2 + (VT)2.0 * oo2ze * v15_8_2 + (VT)1.0 * oo2e * (v28_2_1 - rho_e * v28_2_2);
            const VT v29_18_0 = QCz * v29_8_0 + WQz * v29_8_1 + (VT)3.0 * oo2ze * v14_8_1 + (VT)1.0 * oo2e * (v29_2_0 - rho_e * v29_2_1);
            const VT v29_18_1 = QCz * v29_8_1 + WQz * v29_8_2 + (VT)3.0 * oo2ze * v14_8_2 + (VT)1.0 * oo2e * (v29_2_1 - rho_e * v29_2_2);
            const VT v30_18_0 = QCz * v30_8_0 + WQz * v30_8_1 + (VT)1.0 * oo2e * (v30_2_0 - rho_e * v30_2_1);
            const VT v30_18_1 = QCz * v30_8_1 + WQz * v30_8_2 + (VT)1.0 * oo2e * (v30_2_1 - rho_e * v30_2_2);
            const VT v31_18_0 = QCz * v31_8_0 + WQz * v31_8_1 + (VT)1.0 * oo2ze * v16_8_1 + (VT)1.0 * oo2e * (v31_2_0 - rho_e * v31_2_1);
            const VT v31_18_1 = QCz * v31_8_1 + WQz * v31_8_2 + (VT)1.0 * oo2ze * v16_8_2 + (VT)1.0 * oo2e * (v31_2_1 - rho_e * v31_2_2);
            const VT v32_18_0 = QCz * v32_8_0 + WQz * v32_8_1 + (VT)2.0 * oo2ze * v17_8_1 + (VT)1.0 * oo2e * (v32_2_0 - rho_e * v32_2_1);
            const VT v32_18_1 = QCz * v32_8_1 + WQz * v32_8_2 + (VT)2.0 * oo2ze * v17_8_2 + (VT)1.0 * oo2e * (v32_2_1 - rho_e * v32_2_2);
            const VT v33_18_0 = QCz * v33_8_0 + WQz * v33_8_1 + (VT)3.0 * oo2ze * v18_8_1 + (VT)1.0 * oo2e * (v33_2_0 - rho_e * v33_2_1);
            const VT v33_18_1 = QCz * v33_8_1 + WQz * v33_8_2 + (VT)3.0 * oo2ze * v18_8_2 + (VT)1.0 * oo2e * (v33_2_1 - rho_e * v33_2_2);
            const VT v34_18_0 = QCz * v34_8_0 + WQz * v34_8_1 + (VT)4.0 * oo2ze * v19_8_1 + (VT)1.0 * oo2e * (v34_2_0 - rho_e * v34_2_1);
            const VT v34_18_1 = QCz * v34_8_1 + WQz * v34_8_2 + (VT)4.0 * oo2ze * v19_8_2 + (VT)1.0 * oo2e * (v34_2_1 - rho_e * v34_2_2);
            const VT v1_19_1 = QCz * v1_9_1 + WQz * v1_9_2 + (VT)2.0 * oo2e * (v1_3_1 - rho_e * v1_3_2);
            const VT v2_19_1 = QCz * v2_9_1 + WQz * v2_9_2 + (VT)2.0 * oo2e * (v2_3_1 - rho_e * v2_3_2);
            const VT v3_19_1 = QCz * v3_9_1 + WQz * v3_9_2 + (VT)1.0 * oo2ze * v0_9_2 + (VT)2.0 * oo2e * (v3_3_1 - rho_e * v3_3_2);
            const VT v4_19_0 = QCz * v4_9_0 + WQz * v4_9_1 + (VT)2.0 * oo2e * (v4_3_0 - rho_e * v4_3_1);
            const VT v4_19_1 = QCz * v4_9_1 + WQz * v4_9_2 + (VT)2.0 * oo2e * (v4_3_1 - rho_e * v4_3_2);
            const VT v5_19_0 = QCz * v5_9_0 + WQz * v5_9_1 + (VT)2.0 * oo2e * (v5_3_0 - rho_e * v5_3_1);
            const VT v5_19_1 = QCz * v5_9_1 + WQz * v5_9_2 + (VT)2.0 * oo2e * (v5_3_1 - rho_e * v5_3_2);
            const VT v6_19_0 = QCz * v6_9_0 + WQz * v6_9_1 + (VT)1.0 * oo2ze * v1_9_1 + (VT)2.0 * oo2e * (v6_3_0 - rho_e * v6_3_1);
            const VT v6_19_1 = QCz * v6_9_1 + WQz * v6_9_2 + (VT)1.0 * oo2ze * v1_9_2 + (VT)2.0 * oo2e * (v6_3_1 - rho_e * v6_3_2);
            const VT v7_19_0 = QCz * v7_9_0 + WQz * v7_9_1 + (VT)2.0 * oo2e * (v7_3_0 - rho_e * v7_3_1);
            const VT v7_19_1 = QCz * v7_9_1 + WQz * v7_9_2 + (VT)2.0 * oo2e * (v7_3_1 - rho_e * v7_3_2);
            const VT v8_19_0 = QCz * v8_9_0 + WQz * v8_9_1 + (VT)1.0 * oo2ze * v2_9_1 + (VT)2.0 * oo2e * (v8_3_0 - rho_e * v8_3_1);
            const VT v8_19_1 = QCz * v8_9_1 + WQz * v8_9_2 + (VT)1.0 * oo2ze * v2_9_2 + (VT)2.0 * oo2e * (v8_3_1 - rho_e * v8_3_2);
            const VT v9_19_0 = QCz * v9_9_0 + WQz * v9_9_1 + (VT)2.0 * oo2ze * v3_9_1 + (VT)2.0 * oo2e * (v9_3_0 - rho_e * v9_3_1);
            const VT v9_19_1 = QCz * v9_9_1 + WQz * v9_9_2 + (VT)2.0 * oo2ze * v3_9_2 + (VT)2.0 * oo2e * (v9_3_1 - rho_e * v9_3_2);
            const VT v10_19_0 = QCz * v10_9_0 + WQz * v10_9_1 + (VT)2.0 * oo2e * (v10_3_0 - rho_e * v10_3_1);
            const VT v10_19_1 = QCz * v10_9_1 + WQz * v10_9_2 + (VT)2.0 * oo2e * (v10_3_1 - rho_e * v10_3_2);
            const VT v11_19_0 = QCz * v11_9_0 + WQz * v11_9_1 + (VT)2.0 * oo2e * (v11_3_0 - rho_e * v11_3_1);
            const VT v11_19_1 = QCz * v11_9_1 + WQz * v11_9_2 + (VT)2.0 * oo2e * (v11_3_1 - rho_e * v11_3_2);
            const VT v12_19_0 = QCz * v12_9_0 + WQz * v12_9_1 + (VT)1.0 * oo2ze * v4_9_1 + (VT)2.0 * oo2e * (v12_3_0 - rho_e * v12_3_1);
            const VT v12_19_1 = QCz * v12_9_1 + WQz * v12_9_2 + (VT)1.0 * oo2ze * v4_9_2 + (VT)2.0 * oo2e * (v12_3_1 - rho_e * v12_3_2);
            const VT v13_19_0 = QCz * v13_9_0 + WQz * v13_9_1 + (VT)2.0 * oo2e * (v13_3_0 - rho_e * v13_3_1);
            const VT v13_19_1 = QCz * v13_9_1 + WQz * v13_9_2 + (VT)2.0 * oo2e * (v13_3_1 - rho_e * v13_3_2);
            const VT v14_19_0 = QCz * v14_9_0 + WQz * v14_9_1 + (VT)2.0 * oo2ze * v6_9_1 + (VT)2.0 * oo2e * (v14_3_0 - rho_e * v14_3_1);
            const VT v14_19_1 = QCz * v14_9_1 + WQz * v14_9_2 + (VT)2.0 * oo2ze * v6_9_2 + (VT)2.0 * oo2e * (v14_3_1 - rho_e * v14_3_2);
            const VT v15_19_0 = QCz * v15_9_0 + WQz * v15_9_1 + (VT)1.0 * oo2ze * v5_9_1 + (VT)2.0 * oo2e * (v15_3_0 - rho_e * v15_3_1);
            const VT v15_19_1 = QCz * v15_9_1 + WQz * v15_9_2 + (VT)1.0 * oo2ze * v5_9_2 + (VT)2.0 * oo2e * (v15_3_1 - rho_e * v15_3_2);
            const VT v16_19_0 = QCz * v16_9_0 + WQz * v16_9_1 + (VT)2.0 * oo2e * (v16_3_0 - rho_e * v16_3_1);
            const VT v16_19_1 = QCz * v16_9_1 + WQz * v16_9_2 + (VT)2.0 * oo2e * (v16_3_1 - rho_e * v16_3_2);
            const VT v17_19_0 = QCz * v17_9_0 + WQz * v17_9_1 + (VT)1.0 * oo2ze * v7_9_1 + (VT)2.0 * oo2e * (v17_3_0 - rho_e * v17_3_1);
            const VT v17_19_1 = QCz * v17_9_1 + WQz * v17_9_2 + (VT)1.0 * oo2ze * v7_9_2 + (VT)2.0 * oo2e * (v17_3_1 - rho_e * v17_3_2);
            const VT v18_19_0 = QCz * v18_9_0 + WQz * v18_9_1 + (VT)2.0 * oo2ze * v8_9_1 + (VT)2.0 * oo2e * (v18_3_0 - rho_e * v18_3_1);
            const VT v18_19_1 = QCz * v18_9_1 + WQz * v18_9_2 + (VT)2.0 * oo2ze * v8_9_2 + (VT)2.0 * oo2e * (v18_3_1 - rho_e * v18_3_2);
            const VT v19_19_0 = QCz * v19_9_0 + WQz * v19_9_1 + (VT)3.0 * oo2ze * v9_9_1 + (VT)2.0 * oo2e * (v19_3_0 - rho_e * v19_3_1);
            const VT v19_19_1 = QCz * v19_9_1 + WQz * v19_9_2 + (VT)3.0 * oo2ze * v9_9_2 + (VT)2.0 * oo2e * (v19_3_1 - rho_e * v19_3_2);
            const VT v20_19_0 = QCz * v20_9_0 + WQz * v20_9_1 + (VT)2.0 * oo2e * (v20_3_0 - rho_e * v20_3_1);
            const VT v20_19_1 = QCz * v20_9_1 + WQz * v20_9_2 + (VT)2.0 * oo2e * (v20_3_1 - rho_e * v20_3_2);
            const VT v21_19_0 = QCz * v21_9_0 + WQz * v21_9_1 + (VT)2.0 * oo2e * (v21_3_0 - rho_e * v21_3_1);
            const VT v21_19_1 = QCz * v21_9_1 + WQz * v21_9_2 + (VT)2.0 * oo2e * (v21_3_1 - rho_e * v21_3_2);
            const VT v22_19_0 = QCz * v22_9_0 + WQz * v22_9_1 + (VT)1.0 * oo2ze * v10_9_1 + (VT)2.0 * oo2e * (v22_3_0 - rho_e * v22_3_1);
            const VT v22_19_1 = QCz * v22_9_1 + WQz * v22_9_2 + (VT)1.0 * oo2ze * v10_9_2 + (VT)2.0 * oo2e * (v22_3_1 - rho_e * v22_3_2);
            const VT v23_19_0 = QCz * v23_9_0 + WQz * v23_9_1 + (VT)2.0 * oo2e * (v23_3_0 - rho_e * v23_3_1);
            const VT v23_19_1 = QCz * v23_9_1 + WQz * v23_9_2 + (VT)2.0 * oo2e * (v23_3_1 - rho_e * v23_3_2);
            const VT v24_19_0 = QCz * v24_9_0 + WQz * v24_9_1 + (VT)1.0 * oo2ze * v11_9_1 + (VT)2.0 * oo2e * (v24_3_0 - rho_e * v24_3_1);
            const VT v24_19_1 = QCz * v24_9_1 + WQz * v24_9_2 + (VT)1.0 * oo2ze * v11_9_2 + (VT)2.0 * oo2e * (v24_3_1 - rho_e * v24_3_2);
            const VT v25_19_0 = QCz * v25_9_0 + WQz * v25_9_1 + (VT)2.0 * oo2ze * v12_9_1 + (VT)2.0 * oo2e * (v25_3_0 - rho_e * v25_3_1);
            const VT v25_19_1 = QCz * v25_9_1 + WQz * v25_9_2 + (VT)2.0 * oo2ze * v12_9_2 + (VT)2.0 * oo2e * (v25_3_1 - rho_e * v25_3_2);
            const VT v26_19_0 = QCz * v26_9_0 + WQz * v26_9_1 + (VT)2.0 * oo2e * (v26_3_0 - rho_e * v26_3_1);
            const VT v26_19_1 = QCz * v26_9_1 + WQz * v26_9_2 + (VT)2.0 * oo2e * (v26_3_1 - rho_e * v26_3_2);
            const VT v27_19_0 = QCz * v27_9_0 + WQz * v27_9_1 + (VT)1.0 * oo2ze * v13_9_1 + (VT)2.0 * oo2e * (v27_3_0 - rho_e * v27_3_1);
            const VT v27_19_1 = QCz * v27_9_1 + WQz * v27_9_2 + (VT)1.0 * oo2ze * v13_9_2 + (VT)2.0 * oo2e * (v27_3_1 - rho_e * v27_3_2);
            const VT v28_19_0 = QCz * v28_9_0 + WQz * v28_9_1 + (VT)2.0 * oo2ze * v15_9_1 + (VT)2.0 * oo2e * (v28_3_0 - rho_e * v28_3_1);
            const VT v28_19_1 = QCz * v28_9_1 + WQz * v28_9_2 + (VT)2.0 * oo2ze * v15_9_2 + (VT)2.0 * oo2e * (v28_3_1 - rho_e * v28_3_2);
            const VT v29_19_0 = QCz * v29_9_0 + WQz * v29_9_1 + (VT)3.0 * oo2ze * v14_9_1 + (VT)2.0 * oo2e * (v29_3_0 - rho_e * v29_3_1);
            const VT v29_19_1 = QCz * v29_9_1 + WQz * v29_9_2 + (VT)3.0 * oo2ze * v14_9_2 + (VT)2.0 * oo2e * (v29_3_1 - rho_e * v29_3_2);
            const VT v30_19_0 = QCz * v30_9_0 + WQz * v30_9_1 + (VT)2.0 * oo2e * (v30_3_0 - rho_e * v30_3_1);
            const VT v30_19_1 = QCz * v30_9_1 + WQz * v30_9_2 + (VT)2.0 * oo2e * (v30_3_1 - rho_e * v30_3_2);
            const VT v31_19_0 = QCz * v31_9_0 + WQz * v31_9_1 + (VT)1.0 * oo2ze * v16_9_1 + (VT)2.0 * oo2e * (v31_3_0 - rho_e * v31_3_1);
            const VT v31_19_1 = QCz * v31_9_1 + WQz * v31_9_2 + (VT)1.0 * oo2ze * v16_9_2 + (VT)2.0 * oo2e * (v31_3_1 - rho_e * v31_3_2);
            const VT v32_19_0 = QCz * v32_9_0 + WQz * v32_9_1 + (VT)2.0 * oo2ze * v17_9_1 + (VT)2.0 * oo2e * (v32_3_0 - rho_e * v32_3_1);
            const VT v32_19_1 = QCz * v32_9_1 + WQz * v32_9_2 + (VT)2.0 * oo2ze * v17_9_2 + (VT)2.0 * oo2e * (v32_3_1 - rho_e * v32_3_2);
            const VT v33_19_0 = QCz * v33_9_0 + WQz * v33_9_1 + (VT)3.0 * oo2ze * v18_9_1 + (VT)2.0 * oo2e * (v33_3_0 - rho_e * v33_3_1);
            const VT v33_19_1 = QCz * v33_9_1 + WQz * v33_9_2 + (VT)3.0 * oo2ze * v18_9_2 + (VT)2.0 * oo2e * (v33_3_1 - rho_e * v33_3_2);
            const VT v34_19_0 = QCz * v34_9_0 + WQz * v34_9_1 + (VT)4.0 * oo2ze * v19_9_1 + (VT)2.0 * oo2e * (v34_3_0 - rho_e * v34_3_1);
            const VT v34_19_1 = QCz * v34_9_1 + WQz * v34_9_2 + (VT)4.0 * oo2ze * v19_9_2 + (VT)2.0 * oo2e * (v34_3_1 - rho_e * v34_3_2);
            const VT v4_20_0 = QCx * v4_10_0 + WQx * v4_10_1 + (VT)2.0 * oo2ze * v1_10_1 + (VT)3.0 * oo2e * (v4_4_0 - rho_e * v4_4_1);
            const VT v5_20_0 = QCx * v5_10_0 + WQx * v5_10_1 + (VT)1.0 * oo2ze * v2_10_1 + (VT)3.0 * oo2e * (v5_4_0 - rho_e * v5_4_1);
            const VT v6_20_0 = QCx * v6_10_0 + WQx * v6_10_1 + (VT)1.0 * oo2ze * v3_10_1 + (VT)3.0 * oo2e * (v6_4_0 - rho_e * v6_4_1);
            const VT v7_20_0 = QCx * v7_10_0 + WQx * v7_10_1 + (VT)3.0 * oo2e * (v7_4_0 - rho_e * v7_4_1);
            const VT v8_20_0 = QCx * v8_10_0 + WQx * v8_10_1 + (VT)3.0 * oo2e * (v8_4_0 - rho_e * v8_4_1);
            const VT v9_20_0 = QCx * v9_10_0 + WQx * v9_10_1 + (VT)3.0 * oo2e * (v9_4_0 - rho_e * v9_4_1);
            const VT v10_20_0 = QCx * v10_10_0 + WQx * v10_10_1 + (VT)3.0 * oo2ze * v4_10_1 + (VT)3.0 * oo2e * (v10_4_0 - rho_e * v10_4_1);
            const VT v11_20_0 = QCx * v11_10_0 + WQx * v11_10_1 + (VT)2.0 * oo2ze * v5_10_1 + (VT)3.0 * oo2e * (v11_4_0 - rho_e * v11_4_1);
            const VT v12_20_0 = QCx * v12_10_0 + WQx * v12_10_1 + (VT)2.0 * oo2ze * v6_10_1 + (VT)3.0 * oo2e * (v12_4_0 - rho_e * v12_4_1);
            const VT v13_20_0 = QCx * v13_10_0 + WQx * v13_10_1 + (VT)1.0 * oo2ze * v7_10_1 + (VT)3.0 * oo2e * (v13_4_0 - rho_e * v13_4_1);
            const VT v14_20_0 = QCx * v14_10_0 + WQx * v14_10_1 + (VT)1.0 * oo2ze * v9_10_1 + (VT)3.0 * oo2e * (v14_4_0 - rho_e * v14_4_1);
            const VT v15_20_0 = QCx * v15_10_0 + WQx * v15_10_1 + (VT)1.0 * oo2ze * v8_10_1 + (VT)3.0 * oo2e * (v15_4_0 - rho_e * v15_4_1);
            const VT v16_20_0 = QCx * v16_10_0 + WQx * v16_10_1 + (VT)3.0 * oo2e * (v16_4_0 - rho_e * v16_4_1);
            const VT v17_20_0 = QCx * v17_10_0 + WQx * v17_10_1 + (VT)3.0 * oo2e * (v17_4_0 - rho_e * v17_4_1);
            const VT v18_20_0 = QCx * v18_10_0 + WQx * v18_10_1 + (VT)3.0 * oo2e * (v18_4_0 - rho_e * v18_4_1);
            const VT v19_20_0 = QCx * v19_10_0 + WQx * v19_10_1 + (VT)3.0 * oo2e * (v19_4_0 - rho_e * v19_4_1);
            const VT v20_20_0 = QCx * v20_10_0 + WQx * v20_10_1 + (VT)4.0 * oo2ze * v10_10_1 + (VT)3.0 * oo2e * (v20_4_0 - rho_e * v20_4_1);
            const VT v21_20_0 = QCx * v21_10_0 + WQx * v21_10_1 + (VT)3.0 * oo2ze * v11_10_1 + (VT)3.0 * oo2e * (v21_4_0 - rho_e * v21_4_1);
            const VT v22_20_0 = QCx * v22_10_0 + WQx * v22_10_1 + (VT)3.0 * oo2ze * v12_10_1 + (VT)3.0 * oo2e * (v22_4_0 - rho_e * v22_4_1);
            const VT v23_20_0 = QCx * v23_10_0 + WQx * v23_10_1 + (VT)2.0 * oo2ze * v13_10_1 + (VT)3.0 * oo2e * (v23_4_0 - rho_e * v23_4_1);
            const VT v24_20_0 = QCx * v24_10_0 + WQx * v24_10_1 + (VT)2.0 * oo2ze * v15_10_1 + (VT)3.0 * oo2e * (v24_4_0 - rho_e * v24_4_1);
            const VT v25_20_0 = QCx * v25_10_0 + WQx * v25_10_1 + (VT)2.0 * oo2ze * v14_10_1 + (VT)3.0 * oo2e * (v25_4_0 - rho_e * v25_4_1);
            const VT v26_20_0 = QCx * v26_10_0 + WQx * v26_10_1 + (VT)1.0 * oo2ze * v16_10_1 + (VT)3.0 * oo2e * (v26_4_0 - rho_e * v26_4_1);
            const VT v27_20_0 = QCx * v27_10_0 + WQx * v27_10_1 + (VT)1.0 * oo2ze * v17_10_1 + (VT)3.0 * oo2e * (v27_4_0 - rho_e * v27_4_1);
            const VT v28_20_0 = QCx * v28_10_0 + WQx * v28_10_1 + (VT)1.0 * oo2ze * v18_10_1 + (VT)3.0 * oo2e * (v28_4_0 - rho_e * v28_4_1);
            const VT v29_20_0 = QCx * v29_10_0 + WQx * v29_10_1 + (VT)1.0 * oo2ze * v19_10_1 + (VT)3.0 * oo2e * (v29_4_0 - rho_e * v29_4_1);
            const VT v30_20_0 = QCx * v30_10_0 + WQx * v30_10_1 + (VT)3.0 * oo2e * (v30_4_0 - rho_e * v30_4_1);
            const VT v31_20_0 = QCx * v31_10_0 + WQx * v31_10_1 + (VT)3.0 * oo2e * (v31_4_0 - rho_e * v31_4_1);
            const VT v32_20_0 = QCx * v32_10_0 + WQx * v32_10_1 + (VT)3.0 * oo2e * (v32_4_0 - rho_e * v32_4_1);
            const VT v33_20_0 = QCx * v33_10_0 + WQx * v33_10_1 + (VT)3.0 * oo2e * (v33_4_0 - rho_e * v33_4_1);
            const VT v34_20_0 = QCx * v34_10_0 + WQx * v34_10_1 + (VT)3.0 * oo2e * (v34_4_0 - rho_e * v34_4_1);
            const VT v4_21_0 = QCx * v4_11_0 + WQx * v4_11_1 + (VT)2.0 * oo2ze * v1_11_1 + (VT)2.0 * oo2e * (v4_5_0 - rho_e * v4_5_1);
            const VT v5_21_0 = QCx * v5_11_0 + WQx * v5_11_1 + (VT)1.0 * oo2ze * v2_11_1 + (VT)2.0 * oo2e * (v5_5_0 - rho_e * v5_5_1);
            const VT v6_21_0 = QCx * v6_11_0 + WQx * v6_11_1 + (VT)1.0 * oo2ze * v3_11_1 + (VT)2.0 * oo2e * (v6_5_0 - rho_e * v6_5_1);
            const VT v7_21_0 = QCx * v7_11_0 + WQx * v7_11_1 + (VT)2.0 * oo2e * (v7_5_0 - rho_e * v7_5_1);
            const VT v8_21_0 = QCx * v8_11_0 + WQx * v8_11_1 + (VT)2.0 * oo2e * (v8_5_0 - rho_e * v8_5_1);
            const VT v9_21_0 = QCx * v9_11_0 + WQx * v9_11_1 + (VT)2.0 * oo2e * (v9_5_0 - rho_e * v9_5_1);
            const VT v10_21_0 = QCx * v10_11_0 + WQx * v10_11_1 + (VT)3.0 * oo2ze * v4_11_1 + (VT)2.0 * oo2e * (v10_5_0 - rho_e * v10_5_1);
            const VT v11_21_0 = QCx * v11_11_0 + WQx * v11_11_1 + (VT)2.0 * oo2ze * v5_11_1 + (VT)2.0 * oo2e * (v11_5_0 - rho_e * v11_5_1);
            const VT v12_21_0 = QCx * v12_11_0 + WQx * v12_11_1 + (VT)2.0 * oo2ze * v6_11_1 + (VT)2.0 * oo2e * (v12_5_0 - rho_e * v12_5_1);
            const VT v13_21_0 = QCx * v13_11_0 + WQx * v13_11_1 + (VT)1.0 * oo2ze * v7_11_1 + (VT)2.0 * oo2e * (v13_5_0 - rho_e * v13_5_1);
            const VT v14_21_0 = QCx * v14_11_0 + WQx * v14_11_1 + (VT)1.0 * oo2ze * v9_11_1 + (VT)2.0 * oo2e * (v14_5_0 - rho_e * v14_5_1);
            const VT v15_21_0 = QCx * v15_11_0 + WQx * v15_11_1 + (VT)1.0 * oo2ze * v8_11_1 + (VT)2.0 * oo2e * (v15_5_0 - rho_e * v15_5_1);
            const VT v16_21_0 = QCx * v16_11_0 + WQx * v16_11_1 + (VT)2.0 * oo2e * (v16_5_0 - rho_e * v16_5_1);
            const VT v17_21_0 = QCx * v17_11_0 + WQx * v17_11_1 + (VT)2.0 * oo2e * (v17_5_0 - rho_e * v17_5_1);
            const VT v18_21_0 = QCx * v18_11_0 + WQx * v18_11_1 + (VT)2.0 * oo2e * (v18_5_0 - rho_e * v18_5_1);
            const VT v19_21_0 = QCx * v19_11_0 + WQx * v19_11_1 + (VT)2.0 * oo2e * (v19_5_0 - rho_e * v19_5_1);
            const VT v20_21_0 = QCx * v20_11_0 + WQx * v20_11_1 + (VT)4.0 * oo2ze * v10_11_1 + (VT)2.0 * oo2e * (v20_5_0 - rho_e * v20_5_1);
            const VT v21_21_0 = QCx * v21_11_0 + WQx * v21_11_1 + (VT)3.0 * oo2ze * v11_11_1 + (VT)2.0 * oo2e * (v21_5_0 - rho_e * v21_5_1);
            const VT v22_21_0 = QCx * v22_11_0 + WQx * v22_11_1 + (VT)3.0 * oo2ze * v12_11_1 + (VT)2.0 * oo2e * (v22_5_0 - rho_e * v22_5_1);
            const VT v23_21_0 = QCx * v23_11_0 + WQx * v23_11_1 + (VT)2.0 * oo2ze * v13_11_1 + (VT)2.0 * oo2e * (v23_5_0 - rho_e * v23_5_1);
            const VT v24_21_0 = QCx * v24_11_0 + WQx * v24_11_1 + (VT)2.0 * oo2ze * v15_11_1 + (VT)2.0 * oo2e * (v24_5_0 - rho_e * v24_5_1);
            const VT v25_21_0 = QCx * v25_11_0 + WQx * v25_11_1 + (VT)2.0 * oo2ze * v14_11_1 + (VT)2.0 * oo2e * (v25_5_0 - rho_e * v25_5_1);
            const VT v26_21_0 = QCx * v26_11_0 + WQx * v26_11_1 + (VT)1.0 * oo2ze * v16_11_1 + (VT)2.0 * oo2e * (v26_5_0 - rho_e * v26_5_1);
            const VT v27_21_0 = QCx * v27_11_0 + WQx * v27_11_1 + (VT)1.0 * oo2ze * v17_11_1 + (VT)2.0 * oo2e * (v27_5_0 - rho_e * v27_5_1);
            const VT v28_21_0 = QCx * v28_11_0 + WQx * v28_11_1 + (VT)1.0 * oo2ze * v18_11_1 + (VT)2.0 * oo2e * (v28_5_0 - rho_e * v28_5_1);
            const VT v29_21_0 = QCx * v29_11_0 + WQx * v29_11_1 + (VT)1.0 * oo2ze * v19_11_1 + (VT)2.0 * oo2e * (v29_5_0 - rho_e * v29_5_1);
            const VT v30_21_0 = QCx * v30_11_0 + WQx * v30_11_1 + (VT)2.0 * oo2e * (v30_5_0 - rho_e * v30_5_1);
            const VT v31_21_0 = QCx * v31_11_0 + WQx * v31_11_1 + (VT)2.0 * oo2e * (v31_5_0 - rho_e * v31_5_1);
            const VT v32_21_0 = QCx * v32_11_0 + WQx * v32_11_1 + (VT)2.0 * oo2e * (v32_5_0 - rho_e * v32_5_1);
            const VT v33_21_0 = QCx * v33_11_0 + WQx * v33_11_1 + (VT)2.0 * oo2e * (v33_5_0 - rho_e * v33_5_1);
            const VT v34_21_0 = QCx * v34_11_0 + WQx * v34_11_1 + (VT)2.0 * oo2e * (v34_5_0 - rho_e * v34_5_1);
            const VT v4_22_0 = QCx * v4_12_0 + WQx * v4_12_1 + (VT)2.0 * oo2ze * v1_12_1 + (VT)2.0 * oo2e * (v4_6_0 - rho_e * v4_6_1);
            const VT v5_22_0 = QCx * v5_12_0 + WQx * v5_12_1 + (VT)1.0 * oo2ze * v2_12_1 + (VT)2.0 * oo2e * (v5_6_0 - rho_e * v5_6_1);
            const VT v6_22_0 = QCx * v6_12_0 + WQx * v6_12_1 + (VT)1.0 * oo2ze * v3_12_1 + (VT)2.0 * oo2e * (v6_6_0 - rho_e * v6_6_1);
            const VT v7_22_0 = QCx * v7_12_0 + WQx * v7_12_1 + (VT)2.0 * oo2e * (v7_6_0 - rho_e * v7_6_1);
            const VT v8_22_0 = QCx * v8_12_0 + WQx * v8_12_1 + (VT)2.0 * oo2e * (v8_6_0 - rho_e * v8_6_1);
            const VT v9_22_0 = QCx * v9_12_0 + WQx * v9_12_1 + (VT)2.0 * oo2e * (v9_6_0 - rho_e * v9_6_1);
            const VT v10_22_0 = QCx * v10_12_0 + WQx * v10_12_1 + (VT)3.0 * oo2ze * v4_12_1 + (VT)2.0 * oo2e * (v10_6_0 - rho_e * v10_6_1);
            const VT v11_22_0 = QCx * v11_12_0 + WQx * v11_12_1 + (VT)2.0 * oo2ze * v5_12_1 + (VT)2.0 * oo2e * (v11_6_0 - rho_e * v11_6_1);
            const VT v12_22_0 = QCx * v12_12_0 + WQx * v12_12_1 + (VT)2.0 * oo2ze * v6_12_1 + (VT)2.0 * oo2e * (v12_6_0 - rho_e * v12_6_1);
            const VT v13_22_0 = QCx * v13_12_0 + WQx * v13_12_1 + (VT)1.0 * oo2ze * v7_12_1 + (VT)2.0 * oo2e * (v13_6_0 - rho_e * v13_6_1);
            const VT v14_22_0 = QCx * v14_12_0 + WQx * v14_12_1 + (VT)1.0 * oo2ze * v9_12_1 + (VT)2.0 * oo2e * (v14_6_0 - rho_e * v14_6_1);
            const VT v15_22_0 = QCx * v15_12_0 + WQx * v15_12_1 + (VT)1.0 * oo2ze * v8_12_1 + (VT)2.0 * oo2e * (v15_6_0 - rho_e * v15_6_1);
            const VT v16_22_0 = QCx * v16_12_0 + WQx * v16_12_1 + (VT)2.0 * oo2e * (v16_6_0 - rho_e * v16_6_1);
            const VT v17_22_0 = QCx * v17_12_0 + WQx * v17_12_1 + (VT)2.0 * oo2e * (v17_6_0 - rho_e * v17_6_1);
            const VT v18_22_0 = QCx * v18_12_0 + WQx * v18_12_1 + (VT)2.0 * oo2e * (v18_6_0 - rho_e * v18_6_1);
            const VT v19_22_0 = QCx * v19_12_0 + WQx * v19_12_1 + (VT)2.0 * oo2e * (v19_6_0 - rho_e * v19_6_1);
            const VT v20_22_0 = QCx * v20_12_0 + WQx * v20_12_1 + (VT)4.0 * oo2ze * v10_12_1 + (VT)2.0 * oo2e * (v20_6_0 - rho_e * v20_6_1);
            const VT v21_22_0 = QCx * v21_12_0 + WQx * v21_12_1 + (VT)3.0 * oo2ze * v11_12_1 + (VT)2.0 * oo2e * (v21_6_0 - rho_e * v21_6_1);
            const VT v22_22_0 = QCx * v22_12_0 + WQx * v22_12_1 + (VT)3.0 * oo2ze * v12_12_1 + (VT)2.0 * oo2e * (v22_6_0 - rho_e * v22_6_1);
            const VT v23_22_0 = QCx * v23_12_0 + WQx * v23_12_1 + (VT)2.0 * oo2ze * v13_12_1 + (VT)2.0 * oo2e * (v23_6_0 - rho_e * v23_6_1);
            const VT v24_22_0 = QCx * v24_12_0 + WQx * v24_12_1 + (VT)2.0 * oo2ze * v15_12_1 + (VT)2.0 * oo2e * (v24_6_0 - rho_e * v24_6_1);
            const VT v25_22_0 = QCx * v25_12_0 + WQx * v25_12_1 + (VT)2.0 * oo2ze * v14_12_1 + (VT)2.0 * oo2e * (v25_6_0 - rho_e * v25_6_1);
            const VT v26_22_0 = QCx * v26_12_0 + WQx * v26_12_1 + (VT)1.0 * oo2ze * v16_12_1 + (VT)2.0 * oo2e * (v26_6_0 - rho_e * v26_6_1);
            const VT v27_22_0 = QCx * v27_12_0 + WQx * v27_12_1 + (VT)1.0 * oo2ze * v17_12_1 + (VT)2.0 * oo2e * (v27_6_0 - rho_e * v27_6_1);
            const VT v28_22_0 = QCx * v28_12_0 + WQx * v28_12_1 + (VT)1.0 * oo2ze * v18_12_1 + (VT)2.0 * oo2e * (v28_6_0 - rho_e * v28_6_1);
            const VT v29_22_0 = QCx * v29_12_0 + WQx * v29_12_1 + (VT)1.0 * oo2ze * v19_12_1 + (VT)2.0 * oo2e * (v29_6_0 - rho_e * v29_6_1);
            const VT v30_22_0 = QCx * v30_12_0 + WQx * v30_12_1 + (VT)2.0 * oo2e * (v30_6_0 - rho_e * v30_6_1);
            const VT v31_22_0 = QCx * v31_12_0 + WQx * v31_12_1 + (VT)2.0 * oo2e * (v31_6_0 - rho_e * v31_6_1);
            const VT v32_22_0 = QCx * v32_12_0 + WQx * v32_12_1 + (VT)2.0 * oo2e * (v32_6_0 - rho_e * v32_6_1);
            const VT v33_22_0 = QCx * v33_12_0 + WQx * v33_12_1 + (VT)2.0 * oo2e * (v33_6_0 - rho_e * v33_6_1);
            const VT v34_22_0 = QCx * v34_12_0 + WQx * v34_12_1 + (VT)2.0 * oo2e * (v34_6_0 - rho_e * v34_6_1);
            const VT v4_23_0 = QCx * v4_13_0 + WQx * v4_13_1 + (VT)2.0 * oo2ze * v1_13_1 + (VT)1.0 * oo2e * (v4_7_0 - rho_e * v4_7_1);
            const VT v5_23_0 = QCx * v5_13_0 + WQx * v5_13_1 + (VT)1.0 * oo2ze * v2_13_1 + (VT)1.0 * oo2e * (v5_7_0 - rho_e * v5_7_1);
            const VT v6_23_0 = QCx * v6_13_0 + WQx * v6_13_1 + (VT)1.0 * oo2ze * v3_13_1 + (VT)1.0 * oo2e * (v6_7_0 - rho_e * v6_7_1);
            const VT v7_23_0 = QCx * v7_13_0 + WQx * v7_13_1 + (VT)1.0 * oo2e * (v7_7_0 - rho_e * v7_7_1);
            const VT v8_23_0 = QCx * v8_13_0 + WQx * v8_13_1 + (VT)1.0 * oo2e * (v8_7_0 - rho_e * v8_7_1);
            const VT v9_23_0 = QCx * v9_13_0 + WQx * v9_13_1 + (VT)1.0 * oo2e * (v9_7_0 - rho_e * v9_7_1);
            const VT v10_23_0 = QCx * v10_13_0 + WQx * v10_13_1 + (VT)3.0 * oo2ze * v4_13_1 + (VT)1.0 * oo2e * (v10_7_0 - rho_e * v10_7_1);
            const VT v11_23_0 = QCx * v11_13_0 + WQx * v11_13_1 + (VT)2.0 * oo2ze * v5_13_1 + (VT)1.0 * oo2e * (v11_7_0 - rho_e * v11_7_1);
            const VT v12_23_0 = QCx * v12_13_0 + WQx * v12_13_1 + (VT)2.0 * oo2ze * v6_13_1 + (VT)1.0 * oo2e * (v12_7_0 - rho_e * v12_7_1);
            const VT v13_23_0 = QCx * v13_13_0 + WQx * v13_13_1 + (VT)1.0 * oo2ze * v7_13_1 + (VT)1.0 * oo2e * (v13_7_0 - rho_e * v13_7_1);
            const VT v14_23_0 = QCx * v14_13_0 + WQx * v14_13_1 + (VT)1.0 * oo2ze * v9_13_1 + (VT)1.0 * oo2e * (v14_7_0 - rho_e * v14_7_1);
            const VT v15_23_0 = QCx * v15_13_0 + WQx * v15_13_1 + (VT)1.0 * oo2ze * v8_13_1 + (VT)1.0 * oo2e * (v15_7_0 - rho_e * v15_7_1);
            const VT v16_23_0 = QCx * v16_13_0 + WQx * v16_13_1 + (VT)1.0 * oo2e * (v16_7_0 - rho_e * v16_7_1);
            const VT v17_23_0 = QCx * v17_13_0 + WQx * v17_13_1 + (VT)1.0 * oo2e * (v17_7_0 - rho_e * v17_7_1);
            const VT v18_23_0 = QCx * v18_13_0 + WQx * v18_13_1 + (VT)1.0 * oo2e * (v18_7_0 - rho_e * v18_7_1);
            const VT v19_23_0 = QCx * v19_13_0 + WQx * v19_13_1 + (VT)1.0 * oo2e * (v19_7_0 - rho_e * v19_7_1);
            const VT v20_23_0 = QCx * v20_13_0 + WQx * v20_13_1 + (VT)4.0 * oo2ze * v10_13_1 + (VT)1.0 * oo2e * (v20_7_0 - rho_e * v20_7_1);
            const VT v21_23_0 = QCx * v21_13_0 + WQx * v21_13_1 + (VT)3.0 * oo2ze * v11_13_1 + (VT)1.0 * oo2e * (v21_7_0 - rho_e * v21_7_1);
            const VT v22_23_0 = QCx * v22_13_0 + WQx * v22_13_1 + (VT)3.0 * oo2ze * v12_13_1 + (VT)1.0 * oo2e * (v22_7_0 - rho_e * v22_7_1);
            const VT v23_23_0 = QCx * v23_13_0 + WQx * v23_13_1 + (VT)2.0 * oo2ze * v13_13_1 + (VT)1.0 * oo2e * (v23_7_0 - rho_e * v23_7_1);
            const VT v24_23_0 = QCx * v24_13_0 + WQx * v24_13_1 + (VT)2.0 * oo2ze * v15_13_1 + (VT)1.0 * oo2e * (v24_7_0 - rho_e * v24_7_1);
            const VT v25_23_0 = QCx * v25_13_0 + WQx * v25_13_1 + (VT)2.0 * oo2ze * v14_13_1 + (VT)1.0 * oo2e * (v25_7_0 - rho_e * v25_7_1);
            const VT v26_23_0 = QCx * v26_13_0 + WQx * v26_13_1 + (VT)1.0 * oo2ze * v16_13_1 + (VT)1.0 * oo2e * (v26_7_0 - rho_e * v26_7_1);
            const VT v27_23_0 = QCx * v27_13_0 + WQx * v27_13_1 + (VT)1.0 * oo2ze * v17_13_1 + (VT)1.0 * oo2e * (v27_7_0 - rho_e * v27_7_1);
            const VT v28_23_0 = QCx * v28_13_0 + WQx * v28_13_1 + (VT)1.0 * oo2ze * v18_13_1 + (VT)1.0 * oo2e * (v28_7_0 - rho_e * v28_7_1);
            const VT v29_23_0 = QCx * v29_13_0 + WQx * v29_13_1 + (VT)1.0 * oo2ze * v19_13_1 + (VT)1.0 * oo2e * (v29_7_0 - rho_e * v29_7_1);
            const VT v30_23_0 = QCx * v30_13_0 + WQx * v30_13_1 + (VT)1.0 * oo2e * (v30_7_0 - rho_e * v30_7_1);
            const VT v31_23_0 = QCx * v31_13_0 + WQx * v31_13_1 + (VT)1.0 * oo2e * (v31_7_0 - rho_e * v31_7_1);
            const VT v32_23_0 = QCx * v32_13_0 + WQx * v32_13_1 + (VT)1.0 * oo2e * (v32_7_0 - rho_e * v32_7_1);
            const VT v33_23_0 = QCx * v33_13_0 + WQx * v33_13_1 + (VT)1.0 * oo2e * (v33_7_0 - rho_e * v33_7_1);
            const VT v34_23_0 = QCx * v34_13_0 + WQx * v34_13_1 + (VT)1.0 * oo2e * (v34_7_0 - rho_e * v34_7_1);
            const VT v4_24_0 = QCx * v4_15_0 + WQx * v4_15_1 + (VT)2.0 * oo2ze * v1_15_1 + (VT)1.0 * oo2e * (v4_8_0 - rho_e * v4_8_1);
            const VT v5_24_0 = QCx * v5_15_0 + WQx * v5_15_1 + (VT)1.0 * oo2ze * v2_15_1 + (VT)1.0 * oo2e * (v5_8_0 - rho_e * v5_8_1);
            const VT v6_24_0 = QCx * v6_15_0 + WQx * v6_15_1 + (VT)1.0 * oo2ze * v3_15_1 + (VT)1.0 * oo2e * (v6_8_0 - rho_e * v6_8_1);
            const VT v7_24_0 = QCx * v7_15_0 + WQx * v7_15_1 + (VT)1.0 * oo2e * (v7_8_0 - rho_e * v7_8_1);
            const VT v8_24_0 = QCx * v8_15_0 + WQx * v8_15_1 + (VT)1.0 * oo2e * (v8_8_0 - rho_e * v8_8_1);
            const VT v9_24_0 = QCx * v9_15_0 + WQx * v9_15_1 + (VT)1.0 * oo2e * (v9_8_0 - rho_e * v9_8_1);
            const VT v10_24_0 = QCx * v10_15_0 + WQx * v10_15_1 + (VT)3.0 * oo2ze * v4_15_1 + (VT)1.0 * oo2e * (v10_8_0 - rho_e * v10_8_1);
            const VT v11_24_0 = QCx * v11_15_0 + WQx * v11_15_1 + (VT)2.0 * oo2ze * v5_15_1 + (VT)1.0 * oo2e * (v11_8_0 - rho_e * v11_8_1);
            const VT v12_24_0 = QCx * v12_15_0 + WQx * v12_15_1 + (VT)2.0 * oo2ze * v6_15_1 + (VT)1.0 * oo2e * (v12_8_0 - rho_e * v12_8_1);
            const VT v13_24_0 = QCx * v13_15_0 + WQx * v13_15_1 + (VT)1.0 * oo2ze * v7_15_1 + (VT)1.0 * oo2e * (v13_8_0 - rho_e * v13_8_1);
            const VT v14_24_0 = QCx * v14_15_0 + WQx * v14_15_1 + (VT)1.0 * oo2ze * v9_15_1 + (VT)1.0 * oo2e * (v14_8_0 - rho_e * v14_8_1);
            const VT v15_24_0 = QCx * v15_15_0 + WQx * v15_15_1 + (VT)1.0 * oo2ze * v8_15_1 + (VT)1.0 * oo2e * (v15_8_0 - rho_e * v15_8_1);
            const VT v16_24_0 = QCx * v16_15_0 + WQx * v16_15_1 + (VT)1.0 * oo2e * (v16_8_0 - rho_e * v16_8_1);
            const VT v17_24_0 = QCx * v17_15_0 + WQx * v17_15_1 + (VT)1.0 * oo2e * (v17_8_0 - rho_e * v17_8_1);
            const VT v18_24_0 = QCx * v18_15_0 + WQx * v18_15_1 + (VT)1.0 * oo2e * (v18_8_0 - rho_e * v18_8_1);
            const VT v19_24_0 = QCx * v19_15_0 + WQx * v19_15_1 + (VT)1.0 * oo2e * (v19_8_0 - rho_e * v19_8_1);
            const VT v20_24_0 = QCx * v20_15_0 + WQx * v20_15_1 + (VT)4.0 * oo2ze * v10_15_1 + (VT)1.0 * oo2e * (v20_8_0 - rho_e * v20_8_1);
            const VT v21_24_0 = QCx * v21_15_0 + WQx * v21_15_1 + (VT)3.0 * oo2ze * v11_15_1 + (VT)1.0 * oo2e * (v21_8_0 - rho_e * v21_8_1);
            const VT v22_24_0 = QCx * v22_15_0 + WQx * v22_15_1 + (VT)3.0 * oo2ze * v12_15_1 + (VT)1.0 * oo2e * (v22_8_0 - rho_e * v22_8_1);
            const VT v23_24_0 = QCx * v23_15_0 + WQx * v23_15_1 + (VT)2.0 * oo2ze * v13_15_1 + (VT)1.0 * oo2e * (v23_8_0 - rho_e * v23_8_1);
            const VT v24_24_0 = QCx * v24_15_0 + WQx * v24_15_1 + (VT)2.0 * oo2ze * v15_15_1 + (VT)1.0 * oo2e * (v24_8_0 - rho_e * v24_8_1);
            const VT v25_24_0 = QCx * v25_15_0 + WQx * v25_15_1 + (VT)2.0 * oo2ze * v14_15_1 + (VT)1.0 * oo2e * (v25_8_0 - rho_e * v25_8_1);
            const VT v26_24_0 = QCx * v26_15_0 + WQx * v26_15_1 + (VT)1.0 * oo2ze * v16_15_1 + (VT)1.0 * oo2e * (v26_8_0 - rho_e * v26_8_1);
            const VT v27_24_0 = QCx * v27_15_0 + WQx * v27_15_1 + (VT)1.0 * oo2ze * v17_15_1 + (VT)1.0 * oo2e * (v27_8_0 - rho_e * v27_8_1);
            const VT v28_24_0 = QCx * v28_15_0 + WQx * v28_15_1 + (VT)1.0 * oo2ze * v18_15_1 + (VT)1.0 * oo2e * (v28_8_0 - rho_e * v28_8_1);
            const VT v29_24_0 = QCx * v29_15_0 + WQx * v29_15_1 + (VT)1.0 * oo2ze * v19_15_1 + (VT)1.0 * oo2e * (v29_8_0 - rho_e * v29_8_1);
            const VT v30_24_0 = QCx * v30_15_0 + WQx * v30_15_1 + (VT)1.0 * oo2e * (v30_8_0 - rho_e * v30_8_1);
            const VT v31_24_0 = QCx * v31_15_0 + WQx * v31_15_1 + (VT)1.0 * oo2e * (v31_8_0 - rho_e * v31_8_1);
            const VT v32_24_0 = QCx * v32_15_0 + WQx * v32_15_1 + (VT)1.0 * oo2e * (v32_8_0 - rho_e * v32_8_1);
            const VT v33_24_0 = QCx * v33_15_0 + WQx * v33_15_1 + (VT)1.0 * oo2e * (v33_8_0 - rho_e * v33_8_1);
            const VT v34_24_0 = QCx * v34_15_0 + WQx * v34_15_1 + (VT)1.0 * oo2e * (v34_8_0 - rho_e * v34_8_1);
            const VT v4_25_0 = QCx * v4_14_0 + WQx * v4_14_1 + (VT)2.0 * oo2ze * v1_14_1 + (VT)1.0 * oo2e * (v4_9_0 - rho_e * v4_9_1);
            const VT v5_25_0 = QCx * v5_14_0 + WQx * v5_14_1 + (VT)1.0 * oo2ze * v2_14_1 + (VT)1.0 * oo2e * (v5_9_0 - rho_e * v5_9_1);
            const VT v6_25_0 = QCx * v6_14_0 + WQx * v6_14_1 + (VT)1.0 * oo2ze * v3_14_1 + (VT)1.0 * oo2e * (v6_9_0 - rho_e * v6_9_1);
            const VT v7_25_0 = QCx * v7_14_0 + WQx * v7_14_1 + (VT)1.0 * oo2e * (v7_9_0 - rho_e * v7_9_1);
            const VT v8_25_0 = QCx * v8_14_0 + WQx * v8_14_1 + (VT)1.0 * oo2e * (v8_9_0 - rho_e * v8_9_1);
            const VT v9_25_0 = QCx * v9_14_0 + WQx * v9_14_1 + (VT)1.0 * oo2e * (v9_9_0 - rho_e * v9_9_1);
            const VT v10_25_0 = QCx * v10_14_0 + WQx * v10_14_1 + (VT)3.0 * oo2ze * v4_14_1 + (VT)1.0 * oo2e * (v10_9_0 - rho_e * v10_9_1);
            const VT v11_25_0 = QCx * v11_14_0 + WQx * v11_14_1 + (VT)2.0 * oo2ze * v5_14_1 + (VT)1.0 * oo2e * (v11_9_0 - rho_e * v11_9_1);
            const VT v12_25_0 = QCx * v12_14_0 + WQx * v12_14_1 + (VT)2.0 * oo2ze * v6_14_1 + (VT)1.0 * oo2e * (v12_9_0 - rho_e * v12_9_1);
            const VT v13_25_0 = QCx * v13_14_0 + WQx * v13_14_1 + (VT)1.0 * oo2ze * v7_14_1 + (VT)1.0 * oo2e * (v13_9_0 - rho_e * v13_9_1);
            const VT v14_25_0 = QCx * v14_14_0 + WQx * v14_14_1 + (VT)1.0 * oo2ze * v9_14_1 + (VT)1.0 * oo2e * (v14_9_0 - rho_e * v14_9_1);
            const VT v15_25_0 = QCx * v15_14_0 + WQx * v15_14_1 + (VT)1.0 * oo2ze * v8_14_1 + (VT)1.0 * oo2e * (v15_9_0 - rho_e * v15_9_1);
            const VT v16_25_0 = QCx * v16_14_0 + WQx * v16_14_1 + (VT)1.0 * oo2e * (v16_9_0 - rho_e * v16_9_1);
            const VT v17_25_0 = QCx * v17_14_0 + WQx * v17_14_1 + (VT)1.0 * oo2e * (v17_9_0 - rho_e * v17_9_1);
            const VT v18_25_0 = QCx * v18_14_0 + WQx * v18_14_1 + (VT)1.0 * oo2e * (v18_9_0 - rho_e * v18_9_1);
            const VT v19_25_0 = QCx * v19_14_0 + WQx * v19_14_1 + (VT)1.0 * oo2e * (v19_9_0 - rho_e * v19_9_1);
            const VT v20_25_0 = QCx * v20_14_0 + WQx * v20_14_1 + (VT)4.0 * oo2ze * v10_14_1 + (VT)1.0 * oo2e * (v20_9_0 - rho_e * v20_9_1);
            const VT v21_25_0 = QCx * v21_14_0 + WQx * v21_14_1 + (VT)3.0 * oo2ze * v11_14_1 + (VT)1.0 * oo2e * (v21_9_0 - rho_e * v21_9_1);
            const VT v22_25_0 = QCx * v22_14_0 + WQx * v22_14_1 + (VT)3.0 * oo2ze * v12_14_1 + (VT)1.0 * oo2e * (v22_9_0 - rho_e * v22_9_1);
            const VT v23_25_0 = QCx * v23_14_0 + WQx * v23_14_1 + (VT)2.0 * oo2ze * v13_14_1 + (VT)1.0 * oo2e * (v23_9_0 - rho_e * v23_9_1);
            const VT v24_25_0 = QCx * v24_14_0 + WQx * v24_14_1 + (VT)2.0 * oo2ze * v15_14_1 + (VT)1.0 * oo2e * (v24_9_0 - rho_e * v24_9_1);
            const VT v25_25_0 = QCx * v25_14_0 + WQx * v25_14_1 + (VT)2.0 * oo2ze * v14_14_1 + (VT)1.0 * oo2e * (v25_9_0 - rho_e * v25_9_1);
            const VT v26_25_0 = QCx * v26_14_0 + WQx * v26_14_1 + (VT)1.0 * oo2ze * v16_14_1 + (VT)1.0 * oo2e * (v26_9_0 - rho_e * v26_9_1);
            const VT v27_25_0 = QCx * v27_14_0 + WQx * v27_14_1 + (VT)1.0 * oo2ze * v17_14_1 + (VT)1.0 * oo2e * (v27_9_0 - rho_e * v27_9_1);
            const VT v28_25_0 = QCx * v28_14_0 + WQx * v28_14_1 + (VT)1.0 * oo2ze * v18_14_1 + (VT)1.0 * oo2e * (v28_9_0 - rho_e * v28_9_1);
            const VT v29_25_0 = QCx * v29_14_0 + WQx * v29_14_1 + (VT)1.0 * oo2ze * v19_14_1 + (VT)1.0 * oo2e * (v29_9_0 - rho_e * v29_9_1);
            const VT v30_25_0 = QCx * v30_14_0 + WQx * v30_14_1 + (VT)1.0 * oo2e * (v30_9_0 - rho_e * v30_9_1);
            const VT v31_25_0 = QCx * v31_14_0 + WQx * v31_14_1 + (VT)1.0 * oo2e * (v31_9_0 - rho_e * v31_9_1);
            const VT v32_25_0 = QCx * v32_14_0 + WQx * v32_14_1 + (VT)1.0 * oo2e * (v32_9_0 - rho_e * v32_9_1);
            const VT v33_25_0 = QCx * v33_14_0 + WQx * v33_14_1 + (VT)1.0 * oo2e * (v33_9_0 - rho_e * v33_9_1);
            const VT v34_25_0 = QCx * v34_14_0 + WQx * v34_14_1 + (VT)1.0 * oo2e * (v34_9_0 - rho_e * v34_9_1);
            const VT v4_26_0 = QCy * v4_13_0 + WQy * v4_13_1 + (VT)2.0 * oo2e * (v4_5_0 - rho_e * v4_5_1);
            const VT v5_26_0 = QCy * v5_13_0 + WQy * v5_13_1 + (VT)1.0 * oo2ze * v1_13_1 + (VT)2.0 * oo2e * (v5_5_0 - rho_e * v5_5_1);
            const VT v6_26_0 = QCy * v6_13_0 + WQy * v6_13_1 + (VT)2.0 * oo2e * (v6_5_0 - rho_e * v6_5_1);
            const VT v7_26_0 = QCy * v7_13_0 + WQy * v7_13_1 + (VT)2.0 * oo2ze * v2_13_1 + (VT)2.0 * oo2e * (v7_5_0 - rho_e * v7_5_1);
            const VT v8_26_0 = QCy * v8_13_0 + WQy * v8_13_1 + (VT)1.0 * oo2ze * v3_13_1 + (VT)2.0 * oo2e * (v8_5_0 - rho_e * v8_5_1);
            const VT v9_26_0 = QCy * v9_13_0 + WQy * v9_13_1 + (VT)2.0 * oo2e * (v9_5_0 - rho_e * v9_5_1);
            const VT v10_26_0 = QCy * v10_13_0 + WQy * v10_13_1 + (VT)2.0 * oo2e * (v10_5_0 - rho_e * v10_5_1);
            const VT v11_26_0 = QCy * v11_13_0 + WQy * v11_13_1 + (VT)1.0 * oo2ze * v4_13_1 + (VT)2.0 * oo2e * (v11_5_0 - rho_e * v11_5_1);
            const VT v12_26_0 = QCy * v12_13_0 + WQy * v12_13_1 + (VT)2.0 * oo2e * (v12_5_0 - rho_e * v12_5_1);
            const VT v13_26_0 = QCy * v13_13_0 + WQy * v13_13_1 + (VT)2.0 * oo2ze * v5_13_1 + (VT)2.0 * oo2e * (v13_5_0 - rho_e * v13_5_1);
            const VT v14_26_0 = QCy * v14_13_0 + WQy * v14_13_1 + (VT)2.0 * oo2e * (v14_5_0 - rho_e * v14_5_1);
            const VT v15_26_0 = QCy * v15_13_0 + WQy * v15_13_1 + (VT)1.0 * oo2ze * v6_13_1 + (VT)2.0 * oo2e * (v15_5_0 - rho_e * v15_5_1);
            const VT v16_26_0 = QCy * v16_13_0 + WQy * v16_13_1 + (VT)3.0 * oo2ze * v7_13_1 + (VT)2.0 * oo2e * (v16_5_0 - rho_e * v16_5_1);
            const VT v17_26_0 = QCy * v17_13_0 + WQy * v17_13_1 + (VT)2.0 * oo2ze * v8_13_1 + (VT)2.0 * oo2e * (v17_5_0 - rho_e * v17_5_1);
            const VT v18_26_0 = QCy * v18_13_0 + WQy * v18_13_1 + (VT)1.0 * oo2ze * v9_13_1 + (VT)2.0 * oo2e * (v18_5_0 - rho_e * v18_5_1);
            const VT v19_26_0 = QCy * v19_13_0 + WQy * v19_13_1 + (VT)2.0 * oo2e * (v19_5_0 - rho_e * v19_5_1);
            const VT v20_26_0 = QCy * v20_13_0 + WQy * v20_13_1 + (VT)2.0 * oo2e * (v20_5_0 - rho_e * v20_5_1);
            const VT v21_26_0 = QCy * v21_13_0 + WQy * v21_13_1 + (VT)1.0 * oo2ze * v10_13_1 + (VT)2.0 * oo2e * (v21_5_0 - rho_e * v21_5_1);
            const VT v22_26_0 = QCy * v22_13_0 + WQy * v22_13_1 + (VT)2.0 * oo2e * (v22_5_0 - rho_e * v22_5_1);
            const VT v23_26_0 = QCy * v23_13_0 + WQy * v23_13_1 + (VT)2.0 * oo2ze * v11_13_1 + (VT)2.0 * oo2e * (v23_5_0 - rho_e * v23_5_1);
            const VT v24_26_0 = QCy * v24_13_0 + WQy * v24_13_1 + (VT)1.0 * oo2ze * v12_13_1 + (VT)2.0 * oo2e * (v24_5_0 - rho_e * v24_5_1);
            const VT v25_26_0 = QCy * v25_13_0 + WQy * v25_13_1 + (VT)2.0 * oo2e * (v25_5_0 - rho_e * v25_5_1);
            const VT v26_26_0 = QCy * v26_13_0 + WQy * v26_13_1 + (VT)3.0 * oo2ze * v13_13_1 + (VT)2.0 * oo2e * (v26_5_0 - rho_e * v26_5_1);
            const VT v27_26_0 = QCy * v27_13_0 + WQy * v27_13_1 + (VT)2.0 * oo2ze * v15_13_1 + (VT)2.0 * oo2e * (v27_5_0 - rho_e * v27_5_1);
            const VT v28_26_0 = QCy * v28_13_0 + WQy * v28_13_1 + (VT)1.0 * oo2ze * v14_13_1 + (VT)2.0 * oo2e * (v28_5_0 - rho_e * v28_5_1);
            const VT v29_26_0 = QCy * v29_13_0 + WQy * v29_13_1 + (VT)2.0 * oo2e * (v29_5_0 - rho_e * v29_5_1);
            const VT v30_26_0 = QCy * v30_13_0 + WQy * v30_13_1 + (VT)4.0 * oo2ze * v16_13_1 + (VT)2.0 * oo2e * (v30_5_0 - rho_e * v30_5_1);
            const VT v31_26_0 = QCy * v31_13_0 + WQy * v31_13_1 + (VT)3.0 * oo2ze * v17_13_1 + (VT)2.0 * oo2e * (v31_5_0 - rho_e * v31_5_1);
            const VT v32_26_0 = QCy * v32_13_0 + WQy * v32_13_1 + (VT)2.0 * oo2ze * v18_13_1 + (VT)2.0 * oo2e * (v32_5_0 - rho_e * v32_5_1);
            const VT v33_26_0 = QCy * v33_13_0 + WQy * v33_13_1 + (VT)1.0 * oo2ze * v19_13_1 + (VT)2.0 * oo2e * (v33_5_0 - rho_e * v33_5_1);
            const VT v34_26_0 = QCy * v34_13_0 + WQy * v34_13_1 + (VT)2.0 * oo2e * (v34_5_0 - rho_e * v34_5_1);
            const VT v4_27_0 = QCy * v4_15_0 + WQy * v4_15_1 + (VT)1.0 * oo2e * (v4_6_0 - rho_e * v4_6_1);
            const VT v5_27_0 = QCy * v5_15_0 + WQy * v5_15_1 + (VT)1.0 * oo2ze * v1_15_1 + (VT)1.0 * oo2e * (v5_6_0 - rho_e * v5_6_1);
            const VT v6_27_0 = QCy * v6_15_0 + WQy * v6_15_1 + (VT)1.0 * oo2e * (v6_6_0 - rho_e * v6_6_1);
            const VT v7_27_0 = QCy * v7_15_0 + WQy * v7_15_1 + (VT)2.0 * oo2ze * v2_15_1 + (VT)1.0 * oo2e * (v7_6_0 - rho_e * v7_6_1);
            const VT v8_27_0 = QCy * v8_15_0 + WQy * v8_15_1 + (VT)1.0 * oo2ze * v3_15_1 + (VT)1.0 * oo2e * (v8_6_0 - rho_e * v8_6_1);
            const VT v9_27_0 = QCy * v9_15_0 + WQy * v9_15_1 + (VT)1.0 * oo2e * (v9_6_0 - rho_e * v9_6_1);
            const VT v10_27_0 = QCy * v10_15_0 + WQy * v10_15_1 + (VT)1.0 * oo2e * (v10_6_0 - rho_e * v10_6_1);
            const VT v11_27_0 = QCy * v11_15_0 + WQy * v11_15_1 + (VT)1.0 * oo2ze * v4_15_1 + (VT)1.0 * oo2e * (v11_6_0 - rho_e * v11_6_1);
            const VT v12_27_0 = QCy * v12_15_0 + WQy * v12_15_1 + (VT)1.0 * oo2e * (v12_6_0 - rho_e * v12_6_1);
            const VT v13_27_0 = QCy * v13_15_0 + WQy * v13_15_1 + (VT)2.0 * oo2ze * v5_15_1 + (VT)1.0 * oo2e * (v13_6_0 - rho_e * v13_6_1);
            const VT v14_27_0 = QCy * v14_15_0 + WQy * v14_15_1 + (VT)1.0 * oo2e * (v14_6_0 - rho_e * v14_6_1);
            const VT v15_27_0 = QCy * v15_15_0 + WQy * v15_15_1 + (VT)1.0 * oo2ze * v6_15_1 + (VT)1.0 * oo2e * (v15_6_0 - rho_e * v15_6_1);
            const VT v16_27_0 = QCy * v16_15_0 + WQy * v16_15_1 + (VT)3.0 * oo2ze * v7_15_1 + (VT)1.0 * oo2e * (v16_6_0 - rho_e * v16_6_1);
            const VT v17_27_0 = QCy * v17_15_0 + WQy * v17_15_1 + (VT)2.0 * oo2ze * v8_15_1 + (VT)1.0 * oo2e * (v17_6_0 - rho_e * v17_6_1);
            const VT v18_27_0 = QCy * v18_15_0 + WQy * v18_15_1 + (VT)1.0 * oo2ze * v9_15_1 + (VT)1.0 * oo2e * (v18_6_0 - rho_e * v18_6_1);
            const VT v19_27_0 = QCy * v19_15_0 + WQy * v19_15_1 + (VT)1.0 * oo2e * (v19_6_0 - rho_e * v19_6_1);
            const VT v20_27_0 = QCy * v20_15_0 + WQy * v20_15_1 + (VT)1.0 * oo2e * (v20_6_0 - rho_e * v20_6_1);
            const VT v21_27_0 = QCy * v21_15_0 + WQy * v21_15_1 + (VT)1.0 * oo2ze * v10_15_1 + (VT)1.0 * oo2e * (v21_6_0 - rho_e * v21_6_1);
            const VT v22_27_0 = QCy * v22_15_0 + WQy * v22_15_1 + (VT)1.0 * oo2e * (v22_6_0 - rho_e * v22_6_1);
            const VT v23_27_0 = QCy * v23_15_0 + WQy * v23_15_1 + (VT)2.0 * oo2ze * v11_15_1 + (VT)1.0 * oo2e * (v23_6_0 - rho_e * v23_6_1);
            const VT v24_27_0 = QCy * v24_15_0 + WQy * v24_15_1 + (VT)1.0 * oo2ze * v12_15_1 + (VT)1.0 * oo2e * (v24_6_0 - rho_e * v24_6_1);
            const VT v25_27_0 = QCy * v25_15_0 + WQy * v25_15_1 + (VT)1.0 * oo2e * (v25_6_0 - rho_e * v25_6_1);
            const VT v26_27_0 = QCy * v26_15_0 + WQy * v26_15_1 + (VT)3.0 * oo2ze * v13_15_1 + (VT)1.0 * oo2e * (v26_6_0 - rho_e * v26_6_1);
            const VT v27_27_0 = QCy * v27_15_0 + WQy * v27_15_1 + (VT)2.0 * oo2ze * v15_15_1 + (VT)1.0 * oo2e * (v27_6_0 - rho_e * v27_6_1);
            const VT v28_27_0 = QCy * v28_15_0 + WQy * v28_15_1 + (VT)1.0 * oo2ze * v14_15_1 + (VT)1.0 * oo2e * (v28_6_0 - rho_e * v28_6_1);
            const VT v29_27_0 = QCy * v29_15_0 + WQy * v29_15_1 + (VT)1.0 * oo2e * (v29_6_0 - rho_e * v29_6_1);
            const VT v30_27_0 = QCy * v30_15_0 + WQy * v30_15_1 + (VT)4.0 * oo2ze * v16_15_1 + (VT)1.0 * oo2e * (v30_6_0 - rho_e * v30_6_1);
            const VT v31_27_0 = QCy * v31_15_0 + WQy * v31_15_1 + (VT)3.0 * oo2ze * v17_15_1 + (VT)1.0 * oo2e * (v31_6_0 - rho_e * v31_6_1);
            const VT v32_27_0 = QCy * v32_15_0 + WQy * v32_15_1 + (VT)2.0 * oo2ze * v18_15_1 + (VT)1.0 * oo2e * (v32_6_0 - rho_e * v32_6_1);
            const VT v33_27_0 = QCy * v33_15_0 + WQy * v33_15_1 + (VT)1.0 * oo2ze * v19_15_1 + (VT)1.0 * oo2e * (v33_6_0 - rho_e * v33_6_1);
            const VT v34_27_0 = QCy * v34_15_0 + WQy * v34_15_1 + (VT)1.0 * oo2e * (v34_6_0 - rho_e * v34_6_1);
            const VT v4_28_0 = QCz * v4_15_0 + WQz * v4_15_1 + (VT)1.0 * oo2e * (v4_5_0 - rho_e * v4_5_1);
            const VT v5_28_0 = QCz * v5_15_0 + WQz * v5_15_1 + (VT)1.0 * oo2e * (v5_5_0 - rho_e * v5_5_1);
            const VT v6_28_0 = QCz * v6_15_0 + WQz * v6_15_1 + (VT)1.0 * oo2ze * v1_15_1 + (VT)1.0 * oo2e * (v6_5_0 - rho_e * v6_5_1);
            const VT v7_28_0 = QCz * v7_15_0 + WQz * v7_15_1 + (VT)1.0 * oo2e * (v7_5_0 - rho_e * v7_5_1);
            const VT v8_28_0 = QCz * v8_15_0 + WQz * v8_15_1 + (VT)1.0 * oo2ze * v2_15_1 + (VT)1.0 * oo2e * (v8_5_0 - rho_e * v8_5_1);
            const VT v9_28_0 = QCz * v9_15_0 + WQz * v9_15_1 + (VT)2.0 * oo2ze * v3_15_1 + (VT)1.0 * oo2e * (v9_5_0 - rho_e * v9_5_1);
            const VT v10_28_0 = QCz * v10_15_0 + WQz * v10_15_1 + (VT)1.0 * oo2e * (v10_5_0 - rho_e * v10_5_1);
            const VT v11_28_0 = QCz * v11_15_0 + WQz * v11_15_1 + (VT)1.0 * oo2e * (v11_5_0 - rho_e * v11_5_1);
            const VT v12_28_0 = QCz * v12_15_0 + WQz * v12_15_1 + (VT)1.0 * oo2ze * v4_15_1 + (VT)1.0 * oo2e * (v12_5_0 - rho_e * v12_5_1);
            const VT v13_28_0 = QCz * v13_15_0 + WQz * v13_15_1 + (VT)1.0 * oo2e * (v13_5_0 - rho_e * v13_5_1);
            const VT v14_28_0 = QCz * v14_15_0 + WQz * v14_15_1 + (VT)2.0 * oo2ze * v6_15_1 + (VT)1.0 * oo2e * (v14_5_0 - rho_e * v14_5_1);
            const VT v15_28_0 = QCz * v15_15_0 + WQz * v15_15_1 + (VT)1.0 * oo2ze * v5_15_1 + (VT)1.0 * oo2e * (v15_5_0 - rho_e * v15_5_1);
            const VT v16_28_0 = QCz * v16_15_0 + WQz * v16_15_1 + (VT)1.0 * oo2e * (v16_5_0 - rho_e * v16_5_1);
            const VT v17_28_0 = QCz * v17_15_0 + WQz * v17_15_1 + (VT)1.0 * oo2ze * v7_15_1 + (VT)1.0 * oo2e * (v17_5_0 - rho_e * v17_5_1);
            const VT v18_28_0 = QCz * v18_15_0 + WQz * v18_15_1 + (VT)2.0 * oo2ze * v8_15_1 + (VT)1.0 * oo2e * (v18_5_0 - rho_e * v18_5_1);
            const VT v19_28_0 = QCz * v19_15_0 + WQz * v19_15_1 + (VT)3.0 * oo2ze * v9_15_1 + (VT)1.0 * oo2e * (v19_5_0 - rho_e * v19_5_1);
            const VT v20_28_0 = QCz * v20_15_0 + WQz * v20_15_1 + (VT)1.0 * oo2e * (v20_5_0 - rho_e * v20_5_1);
            const VT v21_28_0 = QCz * v21_15_0 + WQz * v21_15_1 + (VT)1.0 * oo2e * (v21_5_0 - rho_e * v21_5_1);
            const VT v22_28_0 = QCz * v22_15_0 + WQz * v22_15_1 + (VT)1.0 * oo2ze * v10_15_1 + (VT)1.0 * oo2e * (v22_5_0 - rho_e * v22_5_1);
            const VT v23_28_0 = QCz * v23_15_0 + WQz * v23_15_1 + (VT)1.0 * oo2e * (v23_5_0 - rho_e * v23_5_1);
            const VT v24_28_0 = QCz * v24_15_0 + WQz * v24_15_1 + (VT)1.0 * oo2ze * v11_15_1 + (VT)1.0 * oo2e * (v24_5_0 - rho_e * v24_5_1);
            const VT v25_28_0 = QCz * v25_15_0 + WQz * v25_15_1 + (VT)2.0 * oo2ze * v12_15_1 + (VT)1.0 * oo2e * (v25_5_0 - rho_e * v25_5_1);
            const VT v26_28_0 = QCz * v26_15_0 + WQz * v26_15_1 + (VT)1.0 * oo2e * (v26_5_0 - rho_e * v26_5_1);
            const VT v27_28_0 = QCz * v27_15_0 + WQz * v27_15_1 + (VT)1.0 * oo2ze * v13_15_1 + (VT)1.0 * oo2e * (v27_5_0 - rho_e * v27_5_1);
            const VT v28_28_0 = QCz * v28_15_0 + WQz * v28_15_1 + (VT)2.0 * oo2ze * v15_15_1 + (VT)1.0 * oo2e * (v28_5_0 - rho_e * v28_5_1);
            const VT v29_28_0 = QCz * v29_15_0 + WQz * v29_15_1 + (VT)3.0 * oo2ze * v14_15_1 + (VT)1.0 * oo2e * (v29_5_0 - rho_e * v29_5_1);
            const VT v30_28_0 = QCz * v30_15_0 + WQz * v30_15_1 + (VT)1.0 * oo2e * (v30_5_0 - rho_e * v30_5_1);
            const VT v31_28_0 = QCz * v31_15_0 + WQz * v31_15_1 + (VT)1.0 * oo2ze * v16_15_1 + (VT)1.0 * oo2e * (v31_5_0 - rho_e * v31_5_1);
            const VT v32_28_0 = QCz * v32_15_0 + WQz * v32_15_1 + (VT)2.0 * oo2ze * v17_15_1 + (VT)1.0 * oo2e * (v32_5_0 - rho_e * v32_5_1);
            const VT v33_28_0 = QCz * v33_15_0 + WQz * v33_15_1 + (VT)3.0 * oo2ze * v18_15_1 + (VT)1.0 * oo2e * (v33_5_0 - rho_e * v33_5_1);
            const VT v34_28_0 = QCz * v34_15_0 + WQz * v34_15_1 + (VT)4.0 * oo2ze * v19_15_1 + (VT)1.0 * oo2e * (v34_5_0 - rho_e * v34_5_1);
            const VT v4_29_0 = QCz * v4_14_0 + WQz * v4_14_1 + (VT)2.0 * oo2e * (v4_6_0 - rho_e * v4_6_1);
            const VT v5_29_0 = QCz * v5_14_0 + WQz * v5_14_1 + (VT)2.0 * oo2e * (v5_6_0 - rho_e * v5_6_1);
            const VT v6_29_0 = QCz * v6_14_0 + WQz * v6_14_1 + (VT)1.0 * oo2ze * v1_14_1 + (VT)2.0 * oo2e * (v6_6_0 - rho_e * v6_6_1);
            const VT v7_29_0 = QCz * v7_14_0 + WQz * v7_14_1 + (VT)2.0 * oo2e * (v7_6_0 - rho_e * v7_6_1);
            const VT v8_29_0 = QCz * v8_14_0 + WQz * v8_14_1 + (VT)1.0 * oo2ze * v2_14_1 + (VT)2.0 * oo2e * (v8_6_0 - rho_e * v8_6_1);
            const VT v9_29_0 = QCz * v9_14_0 + WQz * v9_14_1 + (VT)2.0 * oo2ze * v3_14_1 + (VT)2.0 * oo2e * (v9_6_0 - rho_e * v9_6_1);
            const VT v10_29_0 = QCz * v10_14_0 + WQz * v10_14_1 + (VT)2.0 * oo2e * (v10_6_0 - rho_e * v10_6_1);
            const VT v11_29_0 = QCz * v11_14_0 + WQz * v11_14_1 + (VT)2.0 * oo2e * (v11_6_0 - rho_e * v11_6_1);
            const VT v12_29_0 = QCz * v12_14_0 + WQz * v12_14_1 + (VT)1.0 * oo2ze * v4_14_1 + (VT)2.0 * oo2e * (v12_6_0 - rho_e * v12_6_1);
            const VT v13_29_0 = QCz * v13_14_0 + WQz * v13_14_1 + (VT)2.0 * oo2e * (v13_6_0 - rho_e * v13_6_1);
            const VT v14_29_0 = QCz * v14_14_0 + WQz * v14_14_1 + (VT)2.0 * oo2ze * v6_14_1 + (VT)2.0 * oo2e * (v14_6_0 - rho_e * v14_6_1);
            const VT v15_29_0 = QCz * v15_14_0 + WQz * v15_14_1 + (VT)1.0 * oo2ze * v5_14_1 + (VT)2.0 * oo2e * (v15_6_0 - rho_e * v15_6_1);
            const VT v16_29_0 = QCz * v16_14_0 + WQz * v16_14_1 + (VT)2.0 * oo2e * (v16_6_0 - rho_e * v16_6_1);
            const VT v17_29_0 = QCz * v17_14_0 + WQz * v17_14_1 + (VT)1.0 * oo2ze * v7_14_1 + (VT)2.0 * oo2e * (v17_6_0 - rho_e * v17_6_1);
            const VT v18_29_0 = QCz * v18_14_0 + WQz * v18_14_1 + (VT)2.0 * oo2ze * v8_14_1 + (VT)2.0 * oo2e * (v18_6_0 - rho_e * v18_6_1);
            const VT v19_29_0 = QCz * v19_14_0 + WQz * v19_14_1 + (VT)3.0 * oo2ze * v9_14_1 + (VT)2.0 * oo2e * (v19_6_0 - rho_e * v19_6_1);
            const VT v20_29_0 = QCz * v20_14_0 + WQz * v20_14_1 + (VT)2.0 * oo2e * (v20_6_0 - rho_e * v20_6_1);
            const VT v21_29_0 = QCz * v21_14_0 + WQz * v21_14_1 + (VT)2.0 * oo2e * (v21_6_0 - rho_e * v21_6_1);
            const VT v22_29_0 = QCz * v22_14_0 + WQz * v22_14_1 + (VT)1.0 * oo2ze * v10_14_1 + (VT)2.0 * oo2e * (v22_6_0 - rho_e * v22_6_1);
            const VT v23_29_0 = QCz * v23_14_0 + WQz * v23_14_1 + (VT)2.0 * oo2e * (v23_6_0 - rho_e * v23_6_1);
            const VT v24_29_0 = QCz * v24_14_0 + WQz * v24_14_1 + (VT)1.0 * oo2ze * v11_14_1 + (VT)2.0 * oo2e * (v24_6_0 - rho_e * v24_6_1);
            const VT v25_29_0 = QCz * v25_14_0 + WQz * v25_14_1 + (VT)2.0 * oo2ze * v12_14_1 + (VT)2.0 * oo2e * (v25_6_0 - rho_e * v25_6_1);
            const VT v26_29_0 = QCz * v26_14_0 + WQz * v26_14_1 + (VT)2.0 * oo2e * (v26_6_0 - rho_e * v26_6_1);
            const VT v27_29_0 = QCz * v27_14_0 + WQz * v27_14_1 + (VT)1.0 * oo2ze * v13_14_1 + (VT)2.0 * oo2e * (v27_6_0 - rho_e * v27_6_1);
            const VT v28_29_0 = QCz * v28_14_0 + WQz * v28_14_1 + (VT)2.0 * oo2ze * v15_14_1 + (VT)2.0 * oo2e * (v28_6_0 - rho_e * v28_6_1);
            const VT v29_29_0 = QCz * v29_14_0 + WQz * v29_14_1 + (VT)3.0 * oo2ze * v14_14_1 + (VT)2.0 * oo2e * (v29_6_0 - rho_e * v29_6_1);
            const VT v30_29_0 = QCz * v30_14_0 + WQz * v30_14_1 + (VT)2.0 * oo2e * (v30_6_0 - rho_e * v30_6_1);
            const VT v31_29_0 = QCz * v31_14_0 + WQz * v31_14_1 + (VT)1.0 * oo2ze * v16_14_1 + (VT)2.0 * oo2e * (v31_6_0 - rho_e * v31_6_1);
            const VT v32_29_0 = QCz * v32_14_0 + WQz * v32_14_1 + (VT)2.0 * oo2ze * v17_14_1 + (VT)2.0 * oo2e * (v32_6_0 - rho_e * v32_6_1);
            const VT v33_29_0 = QCz * v33_14_0 + WQz * v33_14_1 + (VT)3.0 * oo2ze * v18_14_1 + (VT)2.0 * oo2e * (v33_6_0 - rho_e * v33_6_1);
            const VT v34_29_0 = QCz * v34_14_0 + WQz * v34_14_1 + (VT)4.0 * oo2ze * v19_14_1 + (VT)2.0 * oo2e * (v34_6_0 - rho_e * v34_6_1);
            const VT v4_30_0 = QCy * v4_16_0 + WQy * v4_16_1 + (VT)3.0 * oo2e * (v4_7_0 - rho_e * v4_7_1);
            const VT v5_30_0 = QCy * v5_16_0 + WQy * v5_16_1 + (VT)1.0 * oo2ze * v1_16_1 + (VT)3.0 * oo2e * (v5_7_0 - rho_e * v5_7_1);
            const VT v6_30_0 = QCy * v6_16_0 + WQy * v6_16_1 + (VT)3.0 * oo2e * (v6_7_0 - rho_e * v6_7_1);
            const VT v7_30_0 = QCy * v7_16_0 + WQy * v7_16_1 + (VT)2.0 * oo2ze * v2_16_1 + (VT)3.0 * oo2e * (v7_7_0 - rho_e * v7_7_1);
            const VT v8_30_0 = QCy * v8_16_0 + WQy * v8_16_1 + (VT)1.0 * oo2ze * v3_16_1 + (VT)3.0 * oo2e * (v8_7_0 - rho_e * v8_7_1);
            const VT v9_30_0 = QCy * v9_16_0 + WQy * v9_16_1 + (VT)3.0 * oo2e * (v9_7_0 - rho_e * v9_7_1);
            const VT v10_30_0 = QCy * v10_16_0 + WQy * v10_16_1 + (VT)3.0 * oo2e * (v10_7_0 - rho_e * v10_7_1);
            const VT v11_30_0 = QCy * v11_16_0 + WQy * v11_16_1 + (VT)1.0 * oo2ze * v4_16_1 + (VT)3.0 * oo2e * (v11_7_0 - rho_e * v11_7_1);
            const VT v12_30_0 = QCy * v12_16_0 + WQy * v12_16_1 + (VT)3.0 * oo2e * (v12_7_0 - rho_e * v12_7_1);
            const VT v13_30_0 = QCy * v13_16_0 + WQy * v13_16_1 + (VT)2.0 * oo2ze * v5_16_1 + (VT)3.0 * oo2e * (v13_7_0 - rho_e * v13_7_1);
            const VT v14_30_0 = QCy * v14_16_0 + WQy * v14_16_1 + (VT)3.0 * oo2e * (v14_7_0 - rho_e * v14_7_1);
            const VT v15_30_0 = QCy * v15_16_0 + WQy * v15_16_1 + (VT)1.0 * oo2ze * v6_16_1 + (VT)3.0 * oo2e * (v15_7_0 - rho_e * v15_7_1);
            const VT v16_30_0 = QCy * v16_16_0 + WQy * v16_16_1 + (VT)3.0 * oo2ze * v7_16_1 + (VT)3.0 * oo2e * (v16_7_0 - rho_e * v16_7_1);
            const VT v17_30_0 = QCy * v17_16_0 + WQy * v17_16_1 + (VT)2.0 * oo2ze * v8_16_1 + (VT)3.0 * oo2e * (v17_7_0 - rho_e * v17_7_1);
            const VT v18_30_0 = QCy * v18_16_0 + WQy * v18_16_1 + (VT)1.0 * oo2ze * v9_16_1 + (VT)3.0 * oo2e * (v18_7_0 - rho_e * v18_7_1);
            const VT v19_30_0 = QCy * v19_16_0 + WQy * v19_16_1 + (VT)3.0 * oo2e * (v19_7_0 - rho_e * v19_7_1);
            const VT v20_30_0 = QCy * v20_16_0 + WQy * v20_16_1 + (VT)3.0 * oo2e * (v20_7_0 - rho_e * v20_7_1);
            const VT v21_30_0 = QCy * v21_16_0 + WQy * v21_16_1 + (VT)1.0 * oo2ze * v10_16_1 + (VT)3.0 * oo2e * (v21_7_0 - rho_e * v21_7_1);
            const VT v22_30_0 = QCy * v22_16_0 + WQy * v22_16_1 + (VT)3.0 * oo2e * (v22_7_0 - rho_e * v22_7_1);
            const VT v23_30_0 = QCy * v23_16_0 + WQy * v23_16_1 + (VT)2.0 * oo2ze * v11_16_1 + (VT)3.0 * oo2e * (v23_7_0 - rho_e * v23_7_1);
            const VT v24_30_0 = QCy * v24_16_0 + WQy * v24_16_1 + (VT)1.0 * oo2ze * v12_16_1 + (VT)3.0 * oo2e * (v24_7_0 - rho_e * v24_7_1);
            const VT v25_30_0 = QCy * v25_16_0 + WQy * v25_16_1 + (VT)3.0 * oo2e * (v25_7_0 - rho_e * v25_7_1);
            const VT v26_30_0 = QCy * v26_16_0 + WQy * v26_16_1 + (VT)3.0 * oo2ze * v13_16_1 + (VT)3.0 * oo2e * (v26_7_0 - rho_e * v26_7_1);
            const VT v27_30_0 = QCy * v27_16_0 + WQy * v27_16_1 + (VT)2.0 * oo2ze * v15_16_1 + (VT)3.0 * oo2e * (v27_7_0 - rho_e * v27_7_1);
            const VT v28_30_0 = QCy * v28_16_0 + WQy * v28_16_1 + (VT)1.0 * oo2ze * v14_16_1 + (VT)3.0 * oo2e * (v28_7_0 - rho_e * v28_7_1);
            const VT v29_30_0 = QCy * v29_16_0 + WQy * v29_16_1 + (VT)3.0 * oo2e * (v29_7_0 - rho_e * v29_7_1);
            const VT v30_30_0 = QCy * v30_16_0 + WQy * v30_16_1 + (VT)4.0 * oo2ze * v16_16_1 + (VT)3.0 * oo2e * (v30_7_0 - rho_e * v30_7_1);
            const VT v31_30_0 = QCy * v31_16_0 + WQy * v31_16_1 + (VT)3.0 * oo2ze * v17_16_1 + (VT)3.0 * oo2e * (v31_7_0 - rho_e * v31_7_1);
            const VT v32_30_0 = QCy * v32_16_0 + WQy * v32_16_1 + (VT)2.0 * oo2ze * v18_16_1 + (VT)3.0 * oo2e * (v32_7_0 - rho_e * v32_7_1);
            const VT v33_30_0 = QCy * v33_16_0 + WQy * v33_16_1 + (VT)1.0 * oo2ze * v19_16_1 + (VT)3.0 * oo2e * (v33_7_0 - rho_e * v33_7_1);
            const VT v34_30_0 = QCy * v34_16_0 + WQy * v34_16_1 + (VT)3.0 * oo2e * (v34_7_0 - rho_e * v34_7_1);
            const VT v4_31_0 = QCy * v4_17_0 + WQy * v4_17_1 + (VT)2.0 * oo2e * (v4_8_0 - rho_e * v4_8_1);
            const VT v5_31_0 = QCy * v5_17_0 + WQy * v5_17_1 + (VT)1.0 * oo2ze * v1_17_1 + (VT)2.0 * oo2e * (v5_8_0 - rho_e * v5_8_1);
            const VT v6_31_0 = QCy * v6_17_0 + WQy * v6_17_1 + (VT)2.0 * oo2e * (v6_8_0 - rho_e * v6_8_1);
            const VT v7_31_0 = QCy * v7_17_0 + WQy * v7_17_1 + (VT)2.0 * oo2ze * v2_17_1 + (VT)2.0 * oo2e * (v7_8_0 - rho_e * v7_8_1);
            const VT v8_31_0 = QCy * v8_17_0 + WQy * v8_17_1 + (VT)1.0 * oo2ze * v3_17_1 + (VT)2.0 * oo2e * (v8_8_0 - rho_e * v8_8_1);
            const VT v9_31_0 = QCy * v9_17_0 + WQy * v9_17_1 + (VT)2.0 * oo2e * (v9_8_0 - rho_e * v9_8_1);
            const VT v10_31_0 = QCy * v10_17_0 + WQy * v10_17_1 + (VT)2.0 * oo2e * (v10_8_0 - rho_e * v10_8_1);
            const VT v11_31_0 = QCy * v11_17_0 + WQy * v11_17_1 + (VT)1.0 * oo2ze * v4_17_1 + (VT)2.0 * oo2e * (v11_8_0 - rho_e * v11_8_1);
            const VT v12_31_0 = QCy * v12_17_0 + WQy * v12_17_1 + (VT)2.0 * oo2e * (v12_8_0 - rho_e * v12_8_1);
            const VT v13_31_0 = QCy * v13_17_0 + WQy * v13_17_1 + (VT)2.0 * oo2ze * v5_17_1 + (VT)2.0 * oo2e * (v13_8_0 - rho_e * v13_8_1);
            const VT v14_31_0 = QCy * v14_17_0 + WQy * v14_17_1 + (VT)2.0 * oo2e * (v14_8_0 - rho_e * v14_8_1);
            const VT v15_31_0 = QCy * v15_17_0 + WQy * v15_17_1 + (VT)1.0 * oo2ze * v6_17_1 + (VT)2.0 * oo2e * (v15_8_0 - rho_e * v15_8_1);
            const VT v16_31_0 = QCy * v16_17_0 + WQy * v16_17_1 + (VT)3.0 * oo2ze * v7_17_1 + (VT)2.0 * oo2e * (v16_8_0 - rho_e * v16_8_1);
            const VT v17_31_0 = QCy * v17_17_0 + WQy * v17_17_1 + (VT)2.0 * oo2ze * v8_17_1 + (VT)2.0 * oo2e * (v17_8_0 - rho_e * v17_8_1);
            const VT v18_31_0 = QCy * v18_17_0 + WQy * v18_17_1 + (VT)1.0 * oo2ze * v9_17_1 + (VT)2.0 * oo2e * (v18_8_0 - rho_e * v18_8_1);
            const VT v19_31_0 = QCy * v19_17_0 + WQy * v19_17_1 + (VT)2.0 * oo2e * (v19_8_0 - rho_e * v19_8_1);
            const VT v20_31_0 = QCy * v20_17_0 + WQy * v20_17_1 + (VT)2.0 * oo2e * (v20_8_0 - rho_e * v20_8_1);
            const VT v21_31_0 = QCy * v21_17_0 + WQy * v21_17_1 + (VT)1.0 * oo2ze * v10_17_1 + (VT)2.0 * oo2e * (v21_8_0 - rho_e * v21_8_1);
            const VT v22_31_0 = QCy * v22_17_0 + WQy * v22_17_1 + (VT)2.0 * oo2e * (v22_8_0 - rho_e * v22_8_1);
            const VT v23_31_0 = QCy * v23_17_0 + WQy * v23_17_1 + (VT)2.0 * oo2ze * v11_17_1 + (VT)2.0 * oo2e * (v23_8_0 - rho_e * v23_8_1);
            const VT v24_31_0 = QCy * v24_17_0 + WQy * v24_17_1 + (VT)1.0 * oo2ze * v12_17_1 + (VT)2.0 * oo2e * (v24_8_0 - rho_e * v24_8_1);
            const VT v25_31_0 = QCy * v25_17_0 + WQy * v25_17_1 + (VT)2.0 * oo2e * (v25_8_0 - rho_e * v25_8_1);
            const VT v26_31_0 = QCy * v26_17_0 + WQy * v26_17_1 + (VT)3.0 * oo2ze * v13_17_1 + (VT)2.0 * oo2e * (v26_8_0 - rho_e * v26_8_1);
            const VT v27_31_0 = QCy * v27_17_0 + WQy * v27_17_1 + (VT)2.0 * oo2ze * v15_17_1 + (VT)2.0 * oo2e * (v27_8_0 - rho_e * v27_8_1);
            const VT v28_31_0 = QCy * v28_17_0 + WQy * v28_17_1 + (VT)1.0 * oo2ze * v14_17_1 + (VT)2.0 * oo2e * (v28_8_0 - rho_e * v28_8_1);
            const VT v29_31_0 = QCy * v29_17_0 + WQy * v29_17_1 + (VT)2.0 * oo2e * (v29_8_0 - rho_e * v29_8_1);
            const VT v30_31_0 = QCy * v30_17_0 + WQy * v30_17_1 + (VT)4.0 * oo2ze * v16_17_1 + (VT)2.0 * oo2e * (v30_8_0 - rho_e * v30_8_1);
            const VT v31_31_0 = QCy * v31_17_0 + WQy * v31_17_1 + (VT)3.0 * oo2ze * v17_17_1 + (VT)2.0 * oo2e * (v31_8_0 - rho_e * v31_8_1);
            const VT v32_31_0 = QCy * v32_17_0 + WQy * v32_17_1 + (VT)2.0 * oo2ze * v18_17_1 + (VT)2.0 * oo2e * (v32_8_0 - rho_e * v32_8_1);
            const VT v33_31_0 = QCy * v33_17_0 + WQy * v33_17_1 + (VT)1.0 * oo2ze * v19_17_1 + (VT)2.0 * oo2e * (v33_8_0 - rho_e * v33_8_1);
            const VT v34_31_0 = QCy * v34_17_0 + WQy * v34_17_1 + (VT)2.0 * oo2e * (v34_8_0 - rho_e * v34_8_1);
            const VT v4_32_0 = QCy * v4_18_0 + WQy * v4_18_1 + (VT)1.0 * oo2e * (v4_9_0 - rho_e * v4_9_1);
            const VT v5_32_0 = QCy * v5_18_0 + WQy * v5_18_1 + (VT)1.0 * oo2ze * v1_18_1 + (VT)1.0 * oo2e * (v5_9_0 - rho_e * v5_9_1);
            const VT v6_32_0 = QCy * v6_18_0 + WQy * v6_18_1 + (VT)1.0 * oo2e * (v6_9_0 - rho_e * v6_9_1);
            const VT v7_32_0 = QCy * v7_18_0 + WQy * v7_18_1 + (VT)2.0 * oo2ze * v2_18_1 + (VT)1.0 * oo2e * (v7_9_0 - rho_e * v7_9_1);
            const VT v8_32_0 = QCy * v8_18_0 + WQy * v8_18_1 + (VT)1.0 * oo2ze * v3_18_1 + (VT)1.0 * oo2e * (v8_9_0 - rho_e * v8_9_1);
            const VT v9_32_0 = QCy * v9_18_0 + WQy * v9_18_1 + (VT)1.0 * oo2e * (v9_9_0 - rho_e * v9_9_1);
            const VT v10_32_0 = QCy * v10_18_0 + WQy * v10_18_1 + (VT)1.0 * oo2e * (v10_9_0 - rho_e * v10_9_1);
            const VT v11_32_0 = QCy * v11_18_0 + WQy * v11_18_1 + (VT)1.0 * oo2ze * v4_18_1 + (VT)1.0 * oo2e * (v11_9_0 - rho_e * v11_9_1);
            const VT v12_32_0 = QCy * v12_18_0 + WQy * v12_18_1 + (VT)1.0 * oo2e * (v12_9_0 - rho_e * v12_9_1);
            const VT v13_32_0 = QCy * v13_18_0 + WQy * v13_18_1 + (VT)2.0 * oo2ze * v5_18_1 + (VT)1.0 * oo2e * (v13_9_0 - rho_e * v13_9_1);
            const VT v14_32_0 = QCy * v14_18_0 + WQy * v14_18_1 + (VT)1.0 * oo2e * (v14_9_0 - rho_e * v14_9_1);
            const VT v15_32_0 = QCy * v15_18_0 + WQy * v15_18_1 + (VT)1.0 * oo2ze * v6_18_1 + (VT)1.0 * oo2e * (v15_9_0 - rho_e * v15_9_1);
            const VT v16_32_0 = QCy * v16_18_0 + WQy * v16_18_1 + (VT)3.0 * oo2ze * v7_18_1 + (VT)1.0 * oo2e * (v16_9_0 - rho_e * v16_9_1);
            const VT v17_32_0 = QCy * v17_18_0 + WQy * v17_18_1 + (VT)2.0 * oo2ze * v8_18_1 + (VT)1.0 * oo2e * (v17_9_0 - rho_e * v17_9_1);
            const VT v18_32_0 = QCy * v18_18_0 + WQy * v18_18_1 + (VT)1.0 * oo2ze * v9_18_1 + (VT)1.0 * oo2e * (v18_9_0 - rho_e * v18_9_1);
            const VT v19_32_0 = QCy * v19_18_0 + WQy * v19_18_1 + (VT)1.0 * oo2e * (v19_9_0 - rho_e * v19_9_1);
            const VT v20_32_0 = QCy * v20_18_0 + WQy * v20_18_1 + (VT)1.0 * oo2e * (v20_9_0 - rho_e * v20_9_1);
            const VT v21_32_0 = QCy * v21_18_0 + WQy * v21_18_1 + (VT)1.0 * oo2ze * v10_18_1 + (VT)1.0 * oo2e * (v21_9_0 - rho_e * v21_9_1);
            const VT v22_32_0 = QCy * v22_18_0 + WQy * v22_18_1 + (VT)1.0 * oo2e * (v22_9_0 - rho_e * v22_9_1);
            const VT v23_32_0 = QCy * v23_18_0 + WQy * v23_18_1 + (VT)2.0 * oo2ze * v11_18_1 + (VT)1.0 * oo2e * (v23_9_0 - rho_e * v23_9_1);
            const VT v24_32_0 = QCy * v24_18_0 + WQy * v24_18_1 + (VT)1.0 * oo2ze * v12_18_1 + (VT)1.0 * oo2e * (v24_9_0 - rho_e * v24_9_1);
            const VT v25_32_0 = QCy * v25_18_0 + WQy * v25_18_1 + (VT)1.0 * oo2e * (v25_9_0 - rho_e * v25_9_1);
            const VT v26_32_0 = QCy * v26_18_0 + WQy * v26_18_1 + (VT)3.0 * oo2ze * v13_18_1 + (VT)1.0 * oo2e * (v26_9_0 - rho_e * v26_9_1);
            const VT v27_32_0 = QCy * v27_18_0 + WQy * v27_18_1 + (VT)2.0 * oo2ze * v15_18_1 + (VT)1.0 * oo2e * (v27_9_0 - rho_e * v27_9_1);
            const VT v28_32_0 = QCy * v28_18_0 + WQy * v28_18_1 + (VT)1.0 * oo2ze * v14_18_1 + (VT)1.0 * oo2e * (v28_9_0 - rho_e * v28_9_1);
            const VT v29_32_0 = QCy * v29_18_0 + WQy * v29_18_1 + (VT)1.0 * oo2e * (v29_9_0 - rho_e * v29_9_1);
            const VT v30_32_0 = QCy * v30_18_0 + WQy * v30_18_1 + (VT)4.0 * oo2ze * v16_18_1 + (VT)1.0 * oo2e * (v30_9_0 - rho_e * v30_9_1);
            const VT v31_32_0 = QCy * v31_18_0 + WQy * v31_18_1 + (VT)3.0 * oo2ze * v17_18_1 + (VT)1.0 * oo2e * (v31_9_0 - rho_e * v31_9_1);
            const VT v32_32_0 = QCy * v32_18_0 + WQy * v32_18_1 + (VT)2.0 * oo2ze * v18_18_1 + (VT)1.0 * oo2e * (v32_9_0 - rho_e * v32_9_1);
            const VT v33_32_0 = QCy * v33_18_0 + WQy * v33_18_1 + (VT)1.0 * oo2ze * v19_18_1 + (VT)1.0 * oo2e * (v33_9_0 - rho_e * v33_9_1);
            const VT v34_32_0 = QCy * v34_18_0 + WQy * v34_18_1 + (VT)1.0 * oo2e * (v34_9_0 - rho_e * v34_9_1);
            const VT v4_33_0 = QCz * v4_18_0 + WQz * v4_18_1 + (VT)2.0 * oo2e * (v4_8_0 - rho_e * v4_8_1);
            const VT v5_33_0 = QCz * v5_18_0 + WQz * v5_18_1 + (VT)2.0 * oo2e * (v5_8_0 - rho_e * v5_8_1);
            const VT v6_33_0 = QCz * v6_18_0 + WQz * v6_18_1 + (VT)1.0 * oo2ze * v1_18_1 + (VT)2.0 * oo2e * (v6_8_0 - rho_e * v6_8_1);
            const VT v7_33_0 = QCz * v7_18_0 + WQz * v7_18_1 + (VT)2.0 * oo2e * (v7_8_0 - rho_e * v7_8_1);
            const VT v8_33_0 = QCz * v8_18_0 + WQz * v8_18_1 + (VT)1.0 * oo2ze * v2_18_1 + (VT)2.0 * oo2e * (v8_8_0 - rho_e * v8_8_1);
            const VT v9_33_0 = QCz * v9_18_0 + WQz * v9_18_1 + (VT)2.0 * oo2ze * v3_18_1 + (VT)2.0 * oo2e * (v9_8_0 - rho_e * v9_8_1);
            const VT v10_33_0 = QCz * v10_18_0 + WQz * v10_18_1 + (VT)2.0 * oo2e * (v10_8_0 - rho_e * v10_8_1);
            const VT v11_33_0 = QCz * v11_18_0 + WQz * v11_18_1 + (VT)2.0 * oo2e * (v11_8_0 - rho_e * v11_8_1);
            const VT v12_33_0 = QCz * v12_18_0 + WQz * v12_18_1 + (VT)1.0 * oo2ze * v4_18_1 + (VT)2.0 * oo2e * (v12_8_0 - rho_e * v12_8_1);
            const VT v13_33_0 = QCz * v13_18_0 + WQz * v13_18_1 + (VT)2.0 * oo2e * (v13_8_0 - rho_e * v13_8_1);
            const VT v14_33_0 = QCz * v14_18_0 + WQz * v14_18_1 + (VT)2.0 * oo2ze * v6_18_1 + (VT)2.0 * oo2e * (v14_8_0 - rho_e * v14_8_1);
            const VT v15_33_0 = QCz * v15_18_0 + WQz * v15_18_1 + (VT)1.0 * oo2ze * v5_18_1 + (VT)2.0 * oo2e * (v15_8_0 - rho_e * v15_8_1);
            const VT v16_33_0 = QCz * v16_18_0 + WQz * v16_18_1 + (VT)2.0 * oo2e * (v16_8_0 - rho_e * v16_8_1);
            const VT v17_33_0 = QCz * v17_18_0 + WQz * v17_18_1 + (VT)1.0 * oo2ze * v7_18_1 + (VT)2.0 * oo2e * (v17_8_0 - rho_e * v17_8_1);
            const VT v18_33_0 = QCz * v18_18_0 + WQz * v18_18_1 + (VT)2.0 * oo2ze * v8_18_1 + (VT)2.0 * oo2e * (v18_8_0 - rho_e * v18_8_1);
            const VT v19_33_0 = QCz * v19_18_0 + WQz * v19_18_1 + (VT)3.0 * oo2ze * v9_18_1 + (VT)2.0 * oo2e * (v19_8_0 - rho_e * v19_8_1);
            const VT v20_33_0 = QCz * v20_18_0 + WQz * v20_18_1 + (VT)2.0 * oo2e * (v20_8_0 - rho_e * v20_8_1);
            const VT v21_33_0 = QCz * v21_18_0 + WQz * v21_18_1 + (VT)2.0 * oo2e * (v21_8_0 - rho_e * v21_8_1);
            const VT v22_33_0 = QCz * v22_18_0 + WQz * v22_18_1 + (VT)1.0 * oo2ze * v10_18_1 + (VT)2.0 * oo2e * (v22_8_0 - rho_e * v22_8_1);
            const VT v23_33_0 = QCz * v23_18_0 + WQz * v23_18_1 + (VT)2.0 * oo2e * (v23_8_0 - rho_e * v23_8_1);
            const VT v24_33_0 = QCz * v24_18_0 + WQz * v24_18_1 + (VT)1.0 * oo2ze * v11_18_1 + (VT)2.0 * oo2e * (v24_8_0 - rho_e * v24_8_1);
            const VT v25_33_0 = QCz * v25_18_0 + WQz * v25_18_1 + (VT)2.0 * oo2ze * v12_18_1 + (VT)2.0 * oo2e * (v25_8_0 - rho_e * v25_8_1);
            const VT v26_33_0 = QCz * v26_18_0 + WQz * v26_18_1 + (VT)2.0 * oo2e * (v26_8_0 - rho_e * v26_8_1);
            const VT v27_33_0 = QCz * v27_18_0 + WQz * v27_18_1 + (VT)1.0 * oo2ze * v13_18_1 + (VT)2.0 * oo2e * (v27_8_0 - rho_e * v27_8_1);
            const VT v28_33_0 = QCz * v28_18_0 + WQz * v28_18_1 + (VT)2.0 * oo2ze * v15_18_1 + (VT)2.0 * oo2e * (v28_8_0 - rho_e * v28_8_1);
            const VT v29_33_0 = QCz * v29_18_0 + WQz * v29_18_1 + (VT)3.0 * oo2ze * v14_18_1 + (VT)2.0 * oo2e * (v29_8_0 - rho_e * v29_8_1);
            const VT v30_33_0 = QCz * v30_18_0 + WQz * v30_18_1 + (VT)2.0 * oo2e * (v30_8_0 - rho_e * v30_8_1);
            const VT v31_33_0 = QCz * v31_18_0 + WQz * v31_18_1 + (VT)1.0 * oo2ze * v16_18_1 + (VT)2.0 * oo2e * (v31_8_0 - rho_e * v31_8_1);
            const VT v32_33_0 = QCz * v32_18_0 + WQz * v32_18_1 + (VT)2.0 * oo2ze * v17_18_1 + (VT)2.0 * oo2e * (v32_8_0 - rho_e * v32_8_1);
            const VT v33_33_0 = QCz * v33_18_0 + WQz * v33_18_1 + (VT)3.0 * oo2ze * v18_18_1 + (VT)2.0 * oo2e * (v33_8_0 - rho_e * v33_8_1);
            const VT v34_33_0 = QCz * v34_18_0 + WQz * v34_18_1 + (VT)4.0 * oo2ze * v19_18_1 + (VT)2.0 * oo2e * (v34_8_0 - rho_e * v34_8_1);
            const VT v4_34_0 = QCz * v4_19_0 + WQz * v4_19_1 + (VT)3.0 * oo2e * (v4_9_0 - rho_e * v4_9_1);
            const VT v5_34_0 = QCz * v5_19_0 + WQz * v5_19_1 + (VT)3.0 * oo2e * (v5_9_0 - rho_e * v5_9_1);
            const VT v6_34_0 = QCz * v6_19_0 + WQz * v6_19_1 + (VT)1.0 * oo2ze * v1_19_1 + (VT)3.0 * oo2e * (v6_9_0 - rho_e * v6_9_1);
            const VT v7_34_0 = QCz * v7_19_0 + WQz * v7_19_1 + (VT)3.0 * oo2e * (v7_9_0 - rho_e * v7_9_1);
            const VT v8_34_0 = QCz * v8_19_0 + WQz * v8_19_1 + (VT)1.0 * oo2ze * v2_19_1 + (VT)3.0 * oo2e * (v8_9_0 - rho_e * v8_9_1);
            const VT v9_34_0 = QCz * v9_19_0 + WQz * v9_19_1 + (VT)2.0 * oo2ze * v3_19_1 + (VT)3.0 * oo2e * (v9_9_0 - rho_e * v9_9_1);
            const VT v10_34_0 = QCz * v10_19_0 + WQz * v10_19_1 + (VT)3.0 * oo2e * (v10_9_0 - rho_e * v10_9_1);
            const VT v11_34_0 = QCz * v11_19_0 + WQz * v11_19_1 + (VT)3.0 * oo2e * (v11_9_0 - rho_e * v11_9_1);
            const VT v12_34_0 = QCz * v12_19_0 + WQz * v12_19_1 + (VT)1.0 * oo2ze * v4_19_1 + (VT)3.0 * oo2e * (v12_9_0 - rho_e * v12_9_1);
            const VT v13_34_0 = QCz * v13_19_0 + WQz * v13_19_1 + (VT)3.0 * oo2e * (v13_9_0 - rho_e * v13_9_1);
            const VT v14_34_0 = QCz * v14_19_0 + WQz * v14_19_1 + (VT)2.0 * oo2ze * v6_19_1 + (VT)3.0 * oo2e * (v14_9_0 - rho_e * v14_9_1);
            const VT v15_34_0 = QCz * v15_19_0 + WQz * v15_19_1 + (VT)1.0 * oo2ze * v5_19_1 + (VT)3.0 * oo2e * (v15_9_0 - rho_e * v15_9_1);
            const VT v16_34_0 = QCz * v16_19_0 + WQz * v16_19_1 + (VT)3.0 * oo2e * (v16_9_0 - rho_e * v16_9_1);
            const VT v17_34_0 = QCz * v17_19_0 + WQz * v17_19_1 + (VT)1.0 * oo2ze * v7_19_1 + (VT)3.0 * oo2e * (v17_9_0 - rho_e * v17_9_1);
            const VT v18_34_0 = QCz * v18_19_0 + WQz * v18_19_1 + (VT)2.0 * oo2ze * v8_19_1 + (VT)3.0 * oo2e * (v18_9_0 - rho_e * v18_9_1);
            const VT v19_34_0 = QCz * v19_19_0 + WQz * v19_19_1 + (VT)3.0 * oo2ze * v9_19_1 + (VT)3.0 * oo2e * (v19_9_0 - rho_e * v19_9_1);
            const VT v20_34_0 = QCz * v20_19_0 + WQz * v20_19_1 + (VT)3.0 * oo2e * (v20_9_0 - rho_e * v20_9_1);
            const VT v21_34_0 = QCz * v21_19_0 + WQz * v21_19_1 + (VT)3.0 * oo2e * (v21_9_0 - rho_e * v21_9_1);
            const VT v22_34_0 = QCz * v22_19_0 + WQz * v22_19_1 + (VT)1.0 * oo2ze * v10_19_1 + (VT)3.0 * oo2e * (v22_9_0 - rho_e * v22_9_1);
            const VT v23_34_0 = QCz * v23_19_0 + WQz * v23_19_1 + (VT)3.0 * oo2e * (v23_9_0 - rho_e * v23_9_1);
            const VT v24_34_0 = QCz * v24_19_0 + WQz * v24_19_1 + (VT)1.0 * oo2ze * v11_19_1 + (VT)3.0 * oo2e * (v24_9_0 - rho_e * v24_9_1);
            const VT v25_34_0 = QCz * v25_19_0 + WQz * v25_19_1 + (VT)2.0 * oo2ze * v12_19_1 + (VT)3.0 * oo2e * (v25_9_0 - rho_e * v25_9_1);
            const VT v26_34_0 = QCz * v26_19_0 + WQz * v26_19_1 + (VT)3.0 * oo2e * (v26_9_0 - rho_e * v26_9_1);
            const VT v27_34_0 = QCz * v27_19_0 + WQz * v27_19_1 + (VT)1.0 * oo2ze * v13_19_1 + (VT)3.0 * oo2e * (v27_9_0 - rho_e * v27_9_1);
            const VT v28_34_0 = QCz * v28_19_0 + WQz * v28_19_1 + (VT)2.0 * oo2ze * v15_19_1 + (VT)3.0 * oo2e * (v28_9_0 - rho_e * v28_9_1);
            const VT v29_34_0 = QCz * v29_19_0 + WQz * v29_19_1 + (VT)3.0 * oo2ze * v14_19_1 + (VT)3.0 * oo2e * (v29_9_0 - rho_e * v29_9_1);
            const VT v30_34_0 = QCz * v30_19_0 + WQz * v30_19_1 + (VT)3.0 * oo2e * (v30_9_0 - rho_e * v30_9_1);
            const VT v31_34_0 = QCz * v31_19_0 + WQz * v31_19_1 + (VT)1.0 * oo2ze * v16_19_1 + (VT)3.0 * oo2e * (v31_9_0 - rho_e * v31_9_1);
            const VT v32_34_0 = QCz * v32_19_0 + WQz * v32_19_1 + (VT)2.0 * oo2ze * v17_19_1 + (VT)3.0 * oo2e * (v32_9_0 - rho_e * v32_9_1);
            const VT v33_34_0 = QCz * v33_19_0 + WQz * v33_19_1 + (VT)3.0 * oo2ze * v18_19_1 + (VT)3.0 * oo2e * (v33_9_0 - rho_e * v33_9_1);
            const VT v34_34_0 = QCz * v34_19_0 + WQz * v34_19_1 + (VT)4.0 * oo2ze * v19_19_1 + (VT)3.0 * oo2e * (v34_9_0 - rho_e * v34_9_1);
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
            acc[16] += (double)v4_20_0;
            acc[17] += (double)v4_21_0;
            acc[18] += (double)v4_22_0;
            acc[19] += (double)v4_23_0;
            acc[20] += (double)v4_24_0;
            acc[21] += (double)v4_25_0;
            acc[22] += (double)v4_26_0;
            acc[23] += (double)v4_27_0;
            acc[24] += (double)v4_28_0;
            acc[25] += (double)v4_29_0;
            acc[26] += (double)v4_30_0;
            acc[27] += (double)v4_31_0;
            acc[28] += (double)v4_32_0;
            acc[29] += (double)v4_33_0;
            acc[30] += (double)v4_34_0;
            acc[31] += (double)v5_4_0;
            acc[32] += (double)v5_5_0;
            acc[33] += (double)v5_6_0;
            acc[34] += (double)v5_7_0;
            acc[35] += (double)v5_8_0;
            acc[36] += (double)v5_9_0;
            acc[37] += (double)v5_10_0;
            acc[38] += (double)v5_11_0;
            acc[39] += (double)v5_12_0;
            acc[40] += (double)v5_13_0;
            acc[41] += (double)v5_14_0;
            acc[42] += (double)v5_15_0;
            acc[43] += (double)v5_16_0;
            acc[44] += (double)v5_17_0;
            acc[45] += (double)v5_18_0;
            acc[46] += (double)v5_19_0;
            acc[47] += (double)v5_20_0;
            acc[48] += (double)v5_21_0;
            acc[49] += (double)v5_22_0;
            acc[50] += (double)v5_23_0;
            acc[51] += (double)v5_24_0;
            acc[52] += (double)v5_25_0;
            acc[53] += (double)v5_26_0;
            acc[54] += (double)v5_27_0;
            acc[55] += (double)v5_28_0;
            acc[56] += (double)v5_29_0;
            acc[57] += (double)v5_30_0;
            acc[58] += (double)v5_31_0;
            acc[59] += (double)v5_32_0;
            acc[60] += (double)v5_33_0;
            acc[61] += (double)v5_34_0;
            acc[62] += (double)v6_4_0;
            acc[63] += (double)v6_5_0;
            acc[64] += (double)v6_6_0;
            acc[65] += (double)v6_7_0;
            acc[66] += (double)v6_8_0;
            acc[67] += (double)v6_9_0;
            acc[68] += (double)v6_10_0;
            acc[69] += (double)v6_11_0;
            acc[70] += (double)v6_12_0;
            acc[71] += (double)v6_13_0;
            acc[72] += (double)v6_14_0;
            acc[73] += (double)v6_15_0;
            acc[74] += (double)v6_16_0;
            acc[75] += (double)v6_17_0;
            acc[76] += (double)v6_18_0;
            acc[77] += (double)v6_19_0;
            acc[78] += (double)v6_20_0;
            acc[79] += (double)v6_21_0;
            acc[80] += (double)v6_22_0;
            acc[81] += (double)v6_23_0;
            acc[82] += (double)v6_24_0;
            acc[83] += (double)v6_25_0;
            acc[84] += (double)v6_26_0;
            acc[85] += (double)v6_27_0;
            acc[86] += (double)v6_28_0;
            acc[87] += (double)v6_29_0;
            acc[88] += (double)v6_30_0;
            acc[89] += (double)v6_31_0;
            acc[90] += (double)v6_32_0;
            acc[91] += (double)v6_33_0;
            acc[92] += (double)v6_34_0;
            acc[93] += (double)v7_4_0;
            acc[94] += (double)v7_5_0;
            acc[95] += (double)v7_6_0;
            acc[96] += (double)v7_7_0;
            acc[97] += (double)v7_8_0;
            acc[98] += (double)v7_9_0;
            acc[99] += (double)v7_10_0;
            acc[100] += (double)v7_11_0;
            acc[101] += (double)v7_12_0;
            acc[102] += (double)v7_13_0;
            acc[103] += (double)v7_14_0;
            acc[104] += (double)v7_15_0;
            acc[105] += (double)v7_16_0;
            acc[106] += (double)v7_17_0;
            acc[107] += (double)v7_18_0;
            acc[108] += (double)v7_19_0;
            acc[109] += (double)v7_20_0;
            acc[110] += (double)v7_21_0;
            acc[111] += (double)v7_22_0;
            acc[112] += (double)v7_23_0;
            acc[113] += (double)v7_24_0;
            acc[114] += (double)v7_25_0;
            acc[115] += (double)v7_26_0;
            acc[116] += (double)v7_27_0;
            acc[117] += (double)v7_28_0;
            acc[118] += (double)v7_29_0;
            acc[119] += (double)v7_30_0;
            acc[120] += (double)v7_31_0;
            acc[121] += (double)v7_32_0;
            acc[122] += (double)v7_33_0;
            acc[123] += (double)v7_34_0;
            acc[124] += (double)v8_4_0;
            acc[125] += (double)v8_5_0;
            acc[126] += (double)v8_6_0;
            acc[127] += (double)v8_7_0;
            acc[128] += (double)v8_8_0;
            acc[129] += (double)v8_9_0;
            acc[130] += (double)v8_10_0;
            acc[131] += (double)v8_11_0;
            acc[132] += (double)v8_12_0;
            acc[133] += (double)v8_13_0;
            acc[134] += (double)v8_14_0;
            acc[135] += (double)v8_15_0;
            acc[136] += (double)v8_16_0;
            acc[137] += (double)v8_17_0;
            acc[138] += (double)v8_18_0;
            acc[139] += (double)v8_19_0;
            acc[140] += (double)v8_20_0;
            acc[141] += (double)v8_21_0;
            acc[142] += (double)v8_22_0;
            acc[143] += (double)v8_23_0;
            acc[144] += (double)v8_24_0;
            acc[145] += (double)v8_25_0;
            acc[146] += (double)v8_26_0;
            acc[147] += (double)v8_27_0;
            acc[148] += (double)v8_28_0;
            acc[149] += (double)v8_29_0;
            acc[150] += (double)v8_30_0;
            acc[151] += (double)v8_31_0;
            acc[152] += (double)v8_32_0;
            acc[153] += (double)v8_33_0;
            acc[154] += (double)v8_34_0;
            acc[155] += (double)v9_4_0;
            acc[156] += (double)v9_5_0;
            acc[157] += (double)v9_6_0;
            acc[158] += (double)v9_7_0;
            acc[159] += (double)v9_8_0;
            acc[160] += (double)v9_9_0;
            acc[161] += (double)v9_10_0;
            acc[162] += (double)v9_11_0;
            acc[163] += (double)v9_12_0;
            acc[164] += (double)v9_13_0;
            acc[165] += (double)v9_14_0;
            acc[166] += (double)v9_15_0;
            acc[167] += (double)v9_16_0;
            acc[168] += (double)v9_17_0;
            acc[169] += (double)v9_18_0;
            acc[170] += (double)v9_19_0;
            acc[171] += (double)v9_20_0;
            acc[172] += (double)v9_21_0;
            acc[173] += (double)v9_22_0;
            acc[174] += (double)v9_23_0;
            acc[175] += (double)v9_24_0;
            acc[176] += (double)v9_25_0;
            acc[177] += (double)v9_26_0;
            acc[178] += (double)v9_27_0;
            acc[179] += (double)v9_28_0;
            acc[180] += (double)v9_29_0;
            acc[181] += (double)v9_30_0;
            acc[182] += (double)v9_31_0;
            acc[183] += (double)v9_32_0;
            acc[184] += (double)v9_33_0;
            acc[185] += (double)v9_34_0;
            acc[186] += (double)v10_4_0;
            acc[187] += (double)v10_5_0;
            acc[188] += (double)v10_6_0;
            acc[189] += (double)v10_7_0;
            acc[190] += (double)v10_8_0;
            acc[191] += (double)v10_9_0;
            acc[192] += (double)v10_10_0;
            acc[193] += (double)v10_11_0;
            acc[194] += (double)v10_12_0;
            acc[195] += (double)v10_13_0;
            acc[196] += (double)v10_14_0;
            acc[197] += (double)v10_15_0;
            acc[198] += (double)v10_16_0;
            acc[199] += (double)v10_17_0;
            acc[200] += (double)v10_18_0;
            acc[201] += (double)v10_19_0;
            acc[202] += (double)v10_20_0;
            acc[203] += (double)v10_21_0;
            acc[204] += (double)v10_22_0;
            acc[205] += (double)v10_23_0;
            acc[206] += (double)v10_24_0;
            acc[207] += (double)v10_25_0;
            acc[208] += (double)v10_26_0;
            acc[209] += (double)v10_27_0;
            acc[210] += (double)v10_28_0;
            acc[211] += (double)v10_29_0;
            acc[212] += (double)v10_30_0;
            acc[213] += (double)v10_31_0;
            acc[214] += (double)v10_32_0;
            acc[215] += (double)v10_33_0;
            acc[216] += (double)v10_34_0;
            acc[217] += (double)v11_4_0;
            acc[218] += (double)v11_5_0;
            acc[219] += (double)v11_6_0;
            acc[220] += (double)v11_7_0;
            acc[221] += (double)v11_8_0;
            acc[222] += (double)v11_9_0;
            acc[223] += (double)v11_10_0;
            acc[224] += (double)v11_11_0;
            acc[225] += (double)v11_12_0;
            acc[226] += (double)v11_13_0;
            acc[227] += (double)v11_14_0;
            acc[228] += (double)v11_15_0;
            acc[229] += (double)v11_16_0;
            acc[230] += (double)v11_17_0;
            acc[231] += (double)v11_18_0;
            acc[232] += (double)v11_19_0;
            acc[233] += (double)v11_20_0;
            acc[234] += (double)v11_21_0;
            acc[235] += (double)v11_22_0;
            acc[236] += (double)v11_23_0;
            acc[237] += (double)v11_24_0;
            acc[238] += (double)v11_25_0;
            acc[239] += (double)v11_26_0;
            acc[240] += (double)v11_27_0;
            acc[241] += (double)v11_28_0;
            acc[242] += (double)v11_29_0;
            acc[243] += (double)v11_30_0;
            acc[244] += (double)v11_31_0;
            acc[245] += (double)v11_32_0;
            acc[246] += (double)v11_33_0;
            acc[247] += (double)v11_34_0;
            acc[248] += (double)v12_4_0;
            acc[249] += (double)v12_5_0;
            acc[250] += (double)v12_6_0;
            acc[251] += (double)v12_7_0;
            acc[252] += (double)v12_8_0;
            acc[253] += (double)v12_9_0;
            acc[254] += (double)v12_10_0;
            acc[255] += (double)v12_11_0;
            acc[256] += (double)v12_12_0;
            acc[257] += (double)v12_13_0;
            acc[258] += (double)v12_14_0;
            acc[259] += (double)v12_15_0;
            acc[260] += (double)v12_16_0;
            acc[261] += (double)v12_17_0;
            acc[262] += (double)v12_18_0;
            acc[263] += (double)v12_19_0;
            acc[264] += (double)v12_20_0;
            acc[265] += (double)v12_21_0;
            acc[266] += (double)v12_22_0;
            acc[267] += (double)v12_23_0;
            acc[268] += (double)v12_24_0;
            acc[269] += (double)v12_25_0;
            acc[270] += (double)v12_26_0;
            acc[271] += (double)v12_27_0;
            acc[272] += (double)v12_28_0;
            acc[273] += (double)v12_29_0;
            acc[274] += (double)v12_30_0;
            acc[275] += (double)v12_31_0;
            acc[276] += (double)v12_32_0;
            acc[277] += (double)v12_33_0;
            acc[278] += (double)v12_34_0;
            acc[279] += (double)v13_4_0;
            acc[280] += (double)v13_5_0;
            acc[281] += (double)v13_6_0;
            acc[282] += (double)v13_7_0;
            acc[283] += (double)v13_8_0;
            acc[284] += (double)v13_9_0;
            acc[285] += (double)v13_10_0;
            acc[286] += (double)v13_11_0;
            acc[287] += (double)v13_12_0;
            acc[288] += (double)v13_13_0;
            acc[289] += (double)v13_14_0;
            acc[290] += (double)v13_15_0;
            acc[291] += (double)v13_16_0;
            acc[292] += (double)v13_17_0;
            acc[293] += (double)v13_18_0;
            acc[294] += (double)v13_19_0;
            acc[295] += (double)v13_20_0;
            acc[296] += (double)v13_21_0;
            acc[297] += (double)v13_22_0;
            acc[298] += (double)v13_23_0;
            acc[299] += (double)v13_24_0;
            acc[300] += (double)v13_25_0;
            acc[301] += (double)v13_26_0;
            acc[302] += (double)v13_27_0;
            acc[303] += (double)v13_28_0;
            acc[304] += (double)v13_29_0;
            acc[305] += (double)v13_30_0;
            acc[306] += (double)v13_31_0;
            acc[307] += (double)v13_32_0;
            acc[308] += (double)v13_33_0;
            acc[309] += (double)v13_34_0;
            acc[310] += (double)v14_4_0;
            acc[311] += (double)v14_5_0;
            acc[312] += (double)v14_6_0;
            acc[313] += (double)v14_7_0;
            acc[314] += (double)v14_8_0;
            acc[315] += (double)v14_9_0;
            acc[316] += (double)v14_10_0;
            acc[317] += (double)v14_11_0;
            acc[318] += (double)v14_12_0;
            acc[319] += (double)v14_13_0;
            acc[320] += (double)v14_14_0;
            acc[321] += (double)v14_15_0;
            acc[322] += (double)v14_16_0;
            acc[323] += (double)v14_17_0;
            acc[324] += (double)v14_18_0;
            acc[325] += (double)v14_19_0;
            acc[326] += (double)v14_20_0;
            acc[327] += (double)v14_21_0;
            acc[328] += (double)v14_22_0;
            acc[329] += (double)v14_23_0;
            acc[330] += (double)v14_24_0;
            acc[331] += (double)v14_25_0;
            acc[332] += (double)v14_26_0;
            acc[333] += (double)v14_27_0;
            acc[334] += (double)v14_28_0;
            acc[335] += (double)v14_29_0;
            acc[336] += (double)v14_30_0;
            acc[337] += (double)v14_31_0;
            acc[338] += (double)v14_32_0;
            acc[339] += (double)v14_33_0;
            acc[340] += (double)v14_34_0;
            acc[341] += (double)v15_4_0;
            acc[342] += (double)v15_5_0;
            acc[343] += (double)v15_6_0;
            acc[344] += (double)v15_7_0;
            acc[345] += (double)v15_8_0;
            acc[346] += (double)v15_9_0;
            acc[347] += (double)v15_10_0;
            acc[348] += (double)v15_11_0;
            acc[349] += (double)v15_12_0;
            acc[350] += (double)v15_13_0;
            acc[351] += (double)v15_14_0;
            acc[352] += (double)v15_15_0;
            acc[353] += (double)v15_16_0;
            acc[354] += (double)v15_17_0;
            acc[355] += (double)v15_18_0;
            acc[356] += (double)v15_19_0;
            acc[357] += (double)v15_20_0;
            acc[358] += (double)v15_21_0;
            acc[359] += (double)v15_22_0;
            acc[360] += (double)v15_23_0;
            acc[361] += (double)v15_24_0;
            acc[362] += (double)v15_25_0;
            acc[363] += (double)v15_26_0;
            acc[364] += (double)v15_27_0;
            acc[365] += (double)v15_28_0;
            acc[366] += (double)v15_29_0;
            acc[367] += (double)v15_30_0;
            acc[368] += (double)v15_31_0;
            acc[369] += (double)v15_32_0;
            acc[370] += (double)v15_33_0;
            acc[371] += (double)v15_34_0;
            acc[372] += (double)v16_4_0;
            acc[373] += (double)v16_5_0;
            acc[374] += (double)v16_6_0;
            acc[375] += (double)v16_7_0;
            acc[376] += (double)v16_8_0;
            acc[377] += (double)v16_9_0;
            acc[378] += (double)v16_10_0;
            acc[379] += (double)v16_11_0;
            acc[380] += (double)v16_12_0;
            acc[381] += (double)v16_13_0;
            acc[382] += (double)v16_14_0;
            acc[383] += (double)v16_15_0;
            acc[384] += (double)v16_16_0;
            acc[385] += (double)v16_17_0;
            acc[386] += (double)v16_18_0;
            acc[387] += (double)v16_19_0;
            acc[388] += (double)v16_20_0;
            acc[389] += (double)v16_21_0;
            acc[390] += (double)v16_22_0;
            acc[391] += (double)v16_23_0;
            acc[392] += (double)v16_24_0;
            acc[393] += (double)v16_25_0;
            acc[394] += (double)v16_26_0;
            acc[395] += (double)v16_27_0;
            acc[396] += (double)v16_28_0;
            acc[397] += (double)v16_29_0;
            acc[398] += (double)v16_30_0;
            acc[399] += (double)v16_31_0;
            acc[400] += (double)v16_32_0;
            acc[401] += (double)v16_33_0;
            acc[402] += (double)v16_34_0;
            acc[403] += (double)v17_4_0;
            acc[404] += (double)v17_5_0;
            acc[405] += (double)v17_6_0;
            acc[406] += (double)v17_7_0;
            acc[407] += (double)v17_8_0;
            acc[408] += (double)v17_9_0;
            acc[409] += (double)v17_10_0;
            acc[410] += (double)v17_11_0;
            acc[411] += (double)v17_12_0;
            acc[412] += (double)v17_13_0;
            acc[413] += (double)v17_14_0;
            acc[414] += (double)v17_15_0;
            acc[415] += (double)v17_16_0;
            acc[416] += (double)v17_17_0;
            acc[417] += (double)v17_18_0;
            acc[418] += (double)v17_19_0;
            acc[419] += (double)v17_20_0;
            acc[420] += (double)v17_21_0;
            acc[421] += (double)v17_22_0;
            acc[422] += (double)v17_23_0;
            acc[423] += (double)v17_24_0;
            acc[424] += (double)v17_25_0;
            acc[425] += (double)v17_26_0;
            acc[426] += (double)v17_27_0;
            acc[427] += (double)v17_28_0;
            acc[428] += (double)v17_29_0;
            acc[429] += (double)v17_30_0;
            acc[430] += (double)v17_31_0;
            acc[431] += (double)v17_32_0;
            acc[432] += (double)v17_33_0;
            acc[433] += (double)v17_34_0;
            acc[434] += (double)v18_4_0;
            acc[435] += (double)v18_5_0;
            acc[436] += (double)v18_6_0;
            acc[437] += (double)v18_7_0;
            acc[438] += (double)v18_8_0;
            acc[439] += (double)v18_9_0;
            acc[440] += (double)v18_10_0;
            acc[441] += (double)v18_11_0;
            acc[442] += (double)v18_12_0;
            acc[443] += (double)v18_13_0;
            acc[444] += (double)v18_14_0;
            acc[445] += (double)v18_15_0;
            acc[446] += (double)v18_16_0;
            acc[447] += (double)v18_17_0;
            acc[448] += (double)v18_18_0;
            acc[449] += (double)v18_19_0;
            acc[450] += (double)v18_20_0;
            acc[451] += (double)v18_21_0;
            acc[452] += (double)v18_22_0;
            acc[453] += (double)v18_23_0;
            acc[454] += (double)v18_24_0;
            acc[455] += (double)v18_25_0;
            acc[456] += (double)v18_26_0;
            acc[457] += (double)v18_27_0;
            acc[458] += (double)v18_28_0;
            acc[459] += (double)v18_29_0;
            acc[460] += (double)v18_30_0;
            acc[461] += (double)v18_31_0;
            acc[462] += (double)v18_32_0;
            acc[463] += (double)v18_33_0;
            acc[464] += (double)v18_34_0;
            acc[465] += (double)v19_4_0;
            acc[466] += (double)v19_5_0;
            acc[467] += (double)v19_6_0;
            acc[468] += (double)v19_7_0;
            acc[469] += (double)v19_8_0;
            acc[470] += (double)v19_9_0;
            acc[471] += (double)v19_10_0;
            acc[472] += (double)v19_11_0;
            acc[473] += (double)v19_12_0;
            acc[474] += (double)v19_13_0;
            acc[475] += (double)v19_14_0;
            acc[476] += (double)v19_15_0;
            acc[477] += (double)v19_16_0;
            acc[478] += (double)v19_17_0;
            acc[479] += (double)v19_18_0;
            acc[480] += (double)v19_19_0;
            acc[481] += (double)v19_20_0;
            acc[482] += (double)v19_21_0;
            acc[483] += (double)v19_22_0;
            acc[484] += (double)v19_23_0;
            acc[485] += (double)v19_24_0;
            acc[486] += (double)v19_25_0;
            acc[487] += (double)v19_26_0;
            acc[488] += (double)v19_27_0;
            acc[489] += (double)v19_28_0;
            acc[490] += (double)v19_29_0;
            acc[491] += (double)v19_30_0;
            acc[492] += (double)v19_31_0;
            acc[493] += (double)v19_32_0;
            acc[494] += (double)v19_33_0;
            acc[495] += (double)v19_34_0;
            acc[496] += (double)v20_4_0;
            acc[497] += (double)v20_5_0;
            acc[498] += (double)v20_6_0;
            acc[499] += (double)v20_7_0;
            acc[500] += (double)v20_8_0;
            acc[501] += (double)v20_9_0;
            acc[502] += (double)v20_10_0;
            acc[503] += (double)v20_11_0;
            acc[504] += (double)v20_12_0;
            acc[505] += (double)v20_13_0;
            acc[506] += (double)v20_14_0;
            acc[507] += (double)v20_15_0;
            acc[508] += (double)v20_16_0;
            acc[509] += (double)v20_17_0;
            acc[510] += (double)v20_18_0;
            acc[511] += (double)v20_19_0;
            acc[512] += (double)v20_20_0;
            acc[513] += (double)v20_21_0;
            acc[514] += (double)v20_22_0;
            acc[515] += (double)v20_23_0;
            acc[516] += (double)v20_24_0;
            acc[517] += (double)v20_25_0;
            acc[518] += (double)v20_26_0;
            acc[519] += (double)v20_27_0;
            acc[520] += (double)v20_28_0;
            acc[521] += (double)v20_29_0;
            acc[522] += (double)v20_30_0;
            acc[523] += (double)v20_31_0;
            acc[524] += (double)v20_32_0;
            acc[525] += (double)v20_33_0;
            acc[526] += (double)v20_34_0;
            acc[527] += (double)v21_4_0;
            acc[528] += (double)v21_5_0;
            acc[529] += (double)v21_6_0;
            acc[530] += (double)v21_7_0;
            acc[531] += (double)v21_8_0;
            acc[532] += (double)v21_9_0;
            acc[533] += (double)v21_10_0;
            acc[534] += (double)v21_11_0;
            acc[535] += (double)v21_12_0;
            acc[536] += (double)v21_13_0;
            acc[537] += (double)v21_14_0;
            acc[538] += (double)v21_15_0;
            acc[539] += (double)v21_16_0;
            acc[540] += (double)v21_17_0;
            acc[541] += (double)v21_18_0;
            acc[542] += (double)v21_19_0;
            acc[543] += (double)v21_20_0;
            acc[544] += (double)v21_21_0;
            acc[545] += (double)v21_22_0;
            acc[546] += (double)v21_23_0;
            acc[547] += (double)v21_24_0;
            acc[548] += (double)v21_25_0;
            acc[549] += (double)v21_26_0;
            acc[550] += (double)v21_27_0;
            acc[551] += (double)v21_28_0;
            acc[552] += (double)v21_29_0;
            acc[553] += (double)v21_30_0;
            acc[554] += (double)v21_31_0;
            acc[555] += (double)v21_32_0;
            acc[556] += (double)v21_33_0;
            acc[557] += (double)v21_34_0;
            acc[558] += (double)v22_4_0;
            acc[559] += (double)v22_5_0;
            acc[560] += (double)v22_6_0;
            acc[561] += (double)v22_7_0;
            acc[562] += (double)v22_8_0;
            acc[563] += (double)v22_9_0;
            acc[564] += (double)v22_10_0;
            acc[565] += (double)v22_11_0;
            acc[566] += (double)v22_12_0;
            acc[567] += (double)v22_13_0;
            acc[568] += (double)v22_14_0;
            acc[569] += (double)v22_15_0;
            acc[570] += (double)v22_16_0;
            acc[571] += (double)v22_17_0;
            acc[572] += (double)v22_18_0;
            acc[573] += (double)v22_19_0;
            acc[574] += (double)v22_20_0;
            acc[575] += (double)v22_21_0;
            acc[576] += (double)v22_22_0;
            acc[577] += (double)v22_23_0;
            acc[578] += (double)v22_24_0;
            acc[579] += (double)v22_25_0;
            acc[580] += (double)v22_26_0;
            acc[581] += (double)v22_27_0;
            acc[582] += (double)v22_28_0;
            acc[583] += (double)v22_29_0;
            acc[584] += (double)v22_30_0;
            acc[585] += (double)v22_31_0;
            acc[586] += (double)v22_32_0;
            acc[587] += (double)v22_33_0;
            acc[588] += (double)v22_34_0;
            acc[589] += (double)v23_4_0;
            acc[590] += (double)v23_5_0;
            acc[591] += (double)v23_6_0;
            acc[592] += (double)v23_7_0;
            acc[593] += (double)v23_8_0;
            acc[594] += (double)v23_9_0;
            acc[595] += (double)v23_10_0;
            acc[596] += (double)v23_11_0;
            acc[597] += (double)v23_12_0;
            acc[598] += (double)v23_13_0;
            acc[599] += (double)v23_14_0;
            acc[600] += (double)v23_15_0;
            acc[601] += (double)v23_16_0;
            acc[602] += (double)v23_17_0;
            acc[603] += (double)v23_18_0;
            acc[604] += (double)v23_19_0;
            acc[605] += (double)v23_20_0;
            acc[606] += (double)v23_21_0;
            acc[607] += (double)v23_22_0;
            acc[608] += (double)v23_23_0;
            acc[609] += (double)v23_24_0;
            acc[610] += (double)v23_25_0;
            acc[611] += (double)v23_26_0;
            acc[612] += (double)v23_27_0;
            acc[613] += (double)v23_28_0;
            acc[614] += (double)v23_29_0;
            acc[615] += (double)v23_30_0;
            acc[616] += (double)v23_31_0;
            acc[617] += (double)v23_32_0;
            acc[618] += (double)v23_33_0;
            acc[619] += (double)v23_34_0;
            acc[620] += (double)v24_4_0;
            acc[621] += (double)v24_5_0;
            acc[622] += (double)v24_6_0;
            acc[623] += (double)v24_7_0;
            acc[624] += (double)v24_8_0;
            acc[625] += (double)v24_9_0;
            acc[626] += (double)v24_10_0;
            acc[627] += (double)v24_11_0;
            acc[628] += (double)v24_12_0;
            acc[629] += (double)v24_13_0;
            acc[630] += (double)v24_14_0;
            acc[631] += (double)v24_15_0;
            acc[632] += (double)v24_16_0;
            acc[633] += (double)v24_17_0;
            acc[634] += (double)v24_18_0;
            acc[635] += (double)v24_19_0;
            acc[636] += (double)v24_20_0;
            acc[637] += (double)v24_21_0;
            acc[638] += (double)v24_22_0;
            acc[639] += (double)v24_23_0;
            acc[640] += (double)v24_24_0;
            acc[641] += (double)v24_25_0;
            acc[642] += (double)v24_26_0;
            acc[643] += (double)v24_27_0;
            acc[644] += (double)v24_28_0;
            acc[645] += (double)v24_29_0;
            acc[646] += (double)v24_30_0;
            acc[647] += (double)v24_31_0;
            acc[648] += (double)v24_32_0;
            acc[649] += (double)v24_33_0;
            acc[650] += (double)v24_34_0;
            acc[651] += (double)v25_4_0;
            acc[652] += (double)v25_5_0;
            acc[653] += (double)v25_6_0;
            acc[654] += (double)v25_7_0;
            acc[655] += (double)v25_8_0;
            acc[656] += (double)v25_9_0;
            acc[657] += (double)v25_10_0;
            acc[658] += (double)v25_11_0;
            acc[659] += (double)v25_12_0;
            acc[660] += (double)v25_13_0;
            acc[661] += (double)v25_14_0;
            acc[662] += (double)v25_15_0;
            acc[663] += (double)v25_16_0;
            acc[664] += (double)v25_17_0;
            acc[665] += (double)v25_18_0;
            acc[666] += (double)v25_19_0;
            acc[667] += (double)v25_20_0;
            acc[668] += (double)v25_21_0;
            acc[669] += (double)v25_22_0;
            acc[670] += (double)v25_23_0;
            acc[671] += (double)v25_24_0;
            acc[672] += (double)v25_25_0;
            acc[673] += (double)v25_26_0;
            acc[674] += (double)v25_27_0;
            acc[675] += (double)v25_28_0;
            acc[676] += (double)v25_29_0;
            acc[677] += (double)v25_30_0;
            acc[678] += (double)v25_31_0;
            acc[679] += (double)v25_32_0;
            acc[680] += (double)v25_33_0;
            acc[681] += (double)v25_34_0;
            acc[682] += (double)v26_4_0;
            acc[683] += (double)v26_5_0;
            acc[684] += (double)v26_6_0;
            acc[685] += (double)v26_7_0;
            acc[686] += (double)v26_8_0;
            acc[687] += (double)v26_9_0;
            acc[688] += (double)v26_10_0;
            acc[689] += (double)v26_11_0;
            acc[690] += (double)v26_12_0;
            acc[691] += (double)v26_13_0;
            acc[692] += (double)v26_14_0;
            acc[693] += (double)v26_15_0;
            acc[694] += (double)v26_16_0;
            acc[695] += (double)v26_17_0;
            acc[696] += (double)v26_18_0;
            acc[697] += (double)v26_19_0;
            acc[698] += (double)v26_20_0;
            acc[699] += (double)v26_21_0;
            acc[700] += (double)v26_22_0;
            acc[701] += (double)v26_23_0;
            acc[702] += (double)v26_24_0;
            acc[703] += (double)v26_25_0;
            acc[704] += (double)v26_26_0;
            acc[705] += (double)v26_27_0;
            acc[706] += (double)v26_28_0;
            acc[707] += (double)v26_29_0;
            acc[708] += (double)v26_30_0;
            acc[709] += (double)v26_31_0;
            acc[710] += (double)v26_32_0;
            acc[711] += (double)v26_33_0;
            acc[712] += (double)v26_34_0;
            acc[713] += (double)v27_4_0;
            acc[714] += (double)v27_5_0;
            acc[715] += (double)v27_6_0;
            acc[716] += (double)v27_7_0;
            acc[717] += (double)v27_8_0;
            acc[718] += (double)v27_9_0;
            acc[719] += (double)v27_10_0;
            acc[720] += (double)v27_11_0;
            acc[721] += (double)v27_12_0;
            acc[722] += (double)v27_13_0;
            acc[723] += (double)v27_14_0;
            acc[724] += (double)v27_15_0;
            acc[725] += (double)v27_16_0;
            acc[726] += (double)v27_17_0;
            acc[727] += (double)v27_18_0;
            acc[728] += (double)v27_19_0;
            acc[729] += (double)v27_20_0;
            acc[730] += (double)v27_21_0;
            acc[731] += (double)v27_22_0;
            acc[732] += (double)v27_23_0;
            acc[733] += (double)v27_24_0;
            acc[734] += (double)v27_25_0;
            acc[735] += (double)v27_26_0;
            acc[736] += (double)v27_27_0;
            acc[737] += (double)v27_28_0;
            acc[738] += (double)v27_29_0;
            acc[739] += (double)v27_30_0;
            acc[740] += (double)v27_31_0;
            acc[741] += (double)v27_32_0;
            acc[742] += (double)v27_33_0;
            acc[743] += (double)v27_34_0;
            acc[744] += (double)v28_4_0;
            acc[745] += (double)v28_5_0;
            acc[746] += (double)v28_6_0;
            acc[747] += (double)v28_7_0;
            acc[748] += (double)v28_8_0;
            acc[749] += (double)v28_9_0;
            acc[750] += (double)v28_10_0;
            acc[751] += (double)v28_11_0;
            acc[752] += (double)v28_12_0;
            acc[753] += (double)v28_13_0;
            acc[754] += (double)v28_14_0;
            acc[755] += (double)v28_15_0;
            acc[756] += (double)v28_16_0;
            acc[757] += (double)v28_17_0;
            acc[758] += (double)v28_18_0;
            acc[759] += (double)v28_19_0;
            acc[760] += (double)v28_20_0;
            acc[761] += (double)v28_21_0;
            acc[762] += (double)v28_22_0;
            acc[763] += (double)v28_23_0;
            acc[764] += (double)v28_24_0;
            acc[765] += (double)v28_25_0;
            acc[766] += (double)v28_26_0;
            acc[767] += (double)v28_27_0;
            acc[768] += (double)v28_28_0;
            acc[769] += (double)v28_29_0;
            acc[770] += (double)v28_30_0;
            acc[771] += (double)v28_31_0;
            acc[772] += (double)v28_32_0;
            acc[773] += (double)v28_33_0;
            acc[774] += (double)v28_34_0;
            acc[775] += (double)v29_4_0;
            acc[776] += (double)v29_5_0;
            acc[777] += (double)v29_6_0;
            acc[778] += (double)v29_7_0;
            acc[779] += (double)v29_8_0;
            acc[780] += (double)v29_9_0;
            acc[781] += (double)v29_10_0;
            acc[782] += (double)v29_11_0;
            acc[783] += (double)v29_12_0;
            acc[784] += (double)v29_13_0;
            acc[785] += (double)v29_14_0;
            acc[786] += (double)v29_15_0;
            acc[787] += (double)v29_16_0;
            acc[788] += (double)v29_17_0;
            acc[789] += (double)v29_18_0;
            acc[790] += (double)v29_19_0;
            acc[791] += (double)v29_20_0;
            acc[792] += (double)v29_21_0;
            acc[793] += (double)v29_22_0;
            acc[794] += (double)v29_23_0;
            acc[795] += (double)v29_24_0;
            acc[796] += (double)v29_25_0;
            acc[797] += (double)v29_26_0;
            acc[798] += (double)v29_27_0;
            acc[799] += (double)v29_28_0;
            acc[800] += (double)v29_29_0;
            acc[801] += (double)v29_30_0;
            acc[802] += (double)v29_31_0;
            acc[803] += (double)v29_32_0;
            acc[804] += (double)v29_33_0;
            acc[805] += (double)v29_34_0;
            acc[806] += (double)v30_4_0;
            acc[807] += (double)v30_5_0;
            acc[808] += (double)v30_6_0;
            acc[809] += (double)v30_7_0;
            acc[810] += (double)v30_8_0;
            acc[811] += (double)v30_9_0;
            acc[812] += (double)v30_10_0;
            acc[813] += (double)v30_11_0;
            acc[814] += (double)v30_12_0;
            acc[815] += (double)v30_13_0;
            acc[816] += (double)v30_14_0;
            acc[817] += (double)v30_15_0;
            acc[818] += (double)v30_16_0;
            acc[819] += (double)v30_17_0;
            acc[820] += (double)v30_18_0;
            acc[821] += (double)v30_19_0;
            acc[822] += (double)v30_20_0;
            acc[823] += (double)v30_21_0;
            acc[824] += (double)v30_22_0;
            acc[825] += (double)v30_23_0;
            acc[826] += (double)v30_24_0;
            acc[827] += (double)v30_25_0;
            acc[828] += (double)v30_26_0;
            acc[829] += (double)v30_27_0;
            acc[830] += (double)v30_28_0;
            acc[831] += (double)v30_29_0;
            acc[832] += (double)v30_30_0;
            acc[833] += (double)v30_31_0;
            acc[834] += (double)v30_32_0;
            acc[835] += (double)v30_33_0;
            acc[836] += (double)v30_34_0;
            acc[837] += (double)v31_4_0;
            acc[838] += (double)v31_5_0;
            acc[839] += (double)v31_6_0;
            acc[840] += (double)v31_7_0;
            acc[841] += (double)v31_8_0;
            acc[842] += (double)v31_9_0;
            acc[843] += (double)v31_10_0;
            acc[844] += (double)v31_11_0;
            acc[845] += (double)v31_12_0;
            acc[846] += (double)v31_13_0;
            acc[847] += (double)v31_14_0;
            acc[848] += (double)v31_15_0;
            acc[849] += (double)v31_16_0;
            acc[850] += (double)v31_17_0;
            acc[851] += (double)v31_18_0;
            acc[852] += (double)v31_19_0;
            acc[853] += (double)v31_20_0;
            acc[854] += (double)v31_21_0;
            acc[855] += (double)v31_22_0;
            acc[856] += (double)v31_23_0;
            acc[857] += (double)v31_24_0;
            acc[858] += (double)v31_25_0;
            acc[859] += (double)v31_26_0;
            acc[860] += (double)v31_27_0;
            acc[861] += (double)v31_28_0;
            acc[862] += (double)v31_29_0;
            acc[863] += (double)v31_30_0;
            acc[864] += (double)v31_31_0;
            acc[865] += (double)v31_32_0;
            acc[866] += (double)v31_33_0;
            acc[867] += (double)v31_34_0;
            acc[868] += (double)v32_4_0;
            acc[869] += (double)v32_5_0;
            acc[870] += (double)v32_6_0;
            acc[871] += (double)v32_7_0;
            acc[872] += (double)v32_8_0;
            acc[873] += (double)v32_9_0;
            acc[874] += (double)v32_10_0;
            acc[875] += (double)v32_11_0;
            acc[876] += (double)v32_12_0;
            acc[877] += (double)v32_13_0;
            acc[878] += (double)v32_14_0;
            acc[879] += (double)v32_15_0;
            acc[880] += (double)v32_16_0;
            acc[881] += (double)v32_17_0;
            acc[882] += (double)v32_18_0;
            acc[883] += (double)v32_19_0;
            acc[884] += (double)v32_20_0;
            acc[885] += (double)v32_21_0;
            acc[886] += (double)v32_22_0;
            acc[887] += (double)v32_23_0;
            acc[888] += (double)v32_24_0;
            acc[889] += (double)v32_25_0;
            acc[890] += (double)v32_26_0;
            acc[891] += (double)v32_27_0;
            acc[892] += (double)v32_28_0;
            acc[893] += (double)v32_29_0;
            acc[894] += (double)v32_30_0;
            acc[895] += (double)v32_31_0;
            acc[896] += (double)v32_32_0;
            acc[897] += (double)v32_33_0;
            acc[898] += (double)v32_34_0;
            acc[899] += (double)v33_4_0;
            acc[900] += (double)v33_5_0;
            acc[901] += (double)v33_6_0;
            acc[902] += (double)v33_7_0;
            acc[903] += (double)v33_8_0;
            acc[904] += (double)v33_9_0;
            acc[905] += (double)v33_10_0;
            acc[906] += (double)v33_11_0;
            acc[907] += (double)v33_12_0;
            acc[908] += (double)v33_13_0;
            acc[909] += (double)v33_14_0;
            acc[910] += (double)v33_15_0;
            acc[911] += (double)v33_16_0;
            acc[912] += (double)v33_17_0;
            acc[913] += (double)v33_18_0;
            acc[914] += (double)v33_19_0;
            acc[915] += (double)v33_20_0;
            acc[916] += (double)v33_21_0;
            acc[917] += (double)v33_22_0;
            acc[918] += (double)v33_23_0;
            acc[919] += (double)v33_24_0;
            acc[920] += (double)v33_25_0;
            acc[921] += (double)v33_26_0;
            acc[922] += (double)v33_27_0;
            acc[923] += (double)v33_28_0;
            acc[924] += (double)v33_29_0;
            acc[925] += (double)v33_30_0;
            acc[926] += (double)v33_31_0;
            acc[927] += (double)v33_32_0;
            acc[928] += (double)v33_33_0;
            acc[929] += (double)v33_34_0;
            acc[930] += (double)v34_4_0;
            acc[931] += (double)v34_5_0;
            acc[932] += (double)v34_6_0;
            acc[933] += (double)v34_7_0;
            acc[934] += (double)v34_8_0;
            acc[935] += (double)v34_9_0;
            acc[936] += (double)v34_10_0;
            acc[937] += (double)v34_11_0;
            acc[938] += (double)v34_12_0;
            acc[939] += (double)v34_13_0;
            acc[940] += (double)v34_14_0;
            acc[941] += (double)v34_15_0;
            acc[942] += (double)v34_16_0;
            acc[943] += (double)v34_17_0;
            acc[944] += (double)v34_18_0;
            acc[945] += (double)v34_19_0;
            acc[946] += (double)v34_20_0;
            acc[947] += (double)v34_21_0;
            acc[948] += (double)v34_22_0;
            acc[949] += (double)v34_23_0;
            acc[950] += (double)v34_24_0;
            acc[951] += (double)v34_25_0;
            acc[952] += (double)v34_26_0;
            acc[953] += (double)v34_27_0;
            acc[954] += (double)v34_28_0;
            acc[955] += (double)v34_29_0;
            acc[956] += (double)v34_30_0;
            acc[957] += (double)v34_31_0;
            acc[958] += (double)v34_32_0;
            acc[959] += (double)v34_33_0;
            acc[960] += (double)v34_34_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[1296] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_dddd(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h10_1_20 = acc[512] + ABx * acc[202];
    const double h4_1_20 = acc[202] + ABx * acc[16];
    const double h4_4_20 = h10_1_20 + ABx * h4_1_20;
    const double h10_1_10 = acc[502] + ABx * acc[192];
    const double h4_1_10 = acc[192] + ABx * acc[6];
    const double h4_4_10 = h10_1_10 + ABx * h4_1_10;
    const double k4_4_10_1 = h4_4_20 + CDx * h4_4_10;
    const double h10_1_4 = acc[496] + ABx * acc[186];
    const double h4_1_4 = acc[186] + ABx * acc[0];
    const double h4_4_4 = h10_1_4 + ABx * h4_1_4;
    const double k4_4_4_1 = h4_4_10 + CDx * h4_4_4;
    const double k4_4_4_4 = k4_4_10_1 + CDx * k4_4_4_1;
    const double h10_1_21 = acc[513] + ABx * acc[203];
    const double h4_1_21 = acc[203] + ABx * acc[17];
    const double h4_4_21 = h10_1_21 + ABx * h4_1_21;
    const double k4_4_10_2 = h4_4_21 + CDy * h4_4_10;
    const double h10_1_11 = acc[503] + ABx * acc[193];
    const double h4_1_11 = acc[193] + ABx * acc[7];
    const double h4_4_11 = h10_1_11 + ABx * h4_1_11;
    const double k4_4_4_2 = h4_4_11 + CDy * h4_4_4;
    const double k4_4_4_5 = k4_4_10_2 + CDx * k4_4_4_2;
    const double h10_1_22 = acc[514] + ABx * acc[204];
    const double h4_1_22 = acc[204] + ABx * acc[18];
    const double h4_4_22 = h10_1_22 + ABx * h4_1_22;
    const double k4_4_10_3 = h4_4_22 + CDz * h4_4_10;
    const double h10_1_12 = acc[504] + ABx * acc[194];
    const double h4_1_12 = acc[194] + ABx * acc[8];
    const double h4_4_12 = h10_1_12 + ABx * h4_1_12;
    const double k4_4_4_3 = h4_4_12 + CDz * h4_4_4;
    const double k4_4_4_6 = k4_4_10_3 + CDx * k4_4_4_3;
    const double h10_1_23 = acc[515] + ABx * acc[205];
    const double h4_1_23 = acc[205] + ABx * acc[19];
    const double h4_4_23 = h10_1_23 + ABx * h4_1_23;
    const double k4_4_11_2 = h4_4_23 + CDy * h4_4_11;
    const double k4_4_4_7 = k4_4_11_2 + CDy * k4_4_4_2;
    const double h10_1_24 = acc[516] + ABx * acc[206];
    const double h4_1_24 = acc[206] + ABx * acc[20];
    const double h4_4_24 = h10_1_24 + ABx * h4_1_24;
    const double k4_4_11_3 = h4_4_24 + CDz * h4_4_11;
    const double k4_4_4_8 = k4_4_11_3 + CDy * k4_4_4_3;
    const double h10_1_25 = acc[517] + ABx * acc[207];
    const double h4_1_25 = acc[207] + ABx * acc[21];
    const double h4_4_25 = h10_1_25 + ABx * h4_1_25;
    const double k4_4_12_3 = h4_4_25 + CDz * h4_4_12;
    const double k4_4_4_9 = k4_4_12_3 + CDz * k4_4_4_3;
    const double k4_4_11_1 = h4_4_21 + CDx * h4_4_11;
    const double h10_1_5 = acc[497] + ABx * acc[187];
    const double h4_1_5 = acc[187] + ABx * acc[1];
    const double h4_4_5 = h10_1_5 + ABx * h4_1_5;
    const double k4_4_5_1 = h4_4_11 + CDx * h4_4_5;
    const double k4_4_5_4 = k4_4_11_1 + CDx * k4_4_5_1;
    const double h10_1_13 = acc[505] + ABx * acc[195];
    const double h4_1_13 = acc[195] + ABx * acc[9];
    const double h4_4_13 = h10_1_13 + ABx * h4_1_13;
    const double k4_4_5_2 = h4_4_13 + CDy * h4_4_5;
    const double k4_4_5_5 = k4_4_11_2 + CDx * k4_4_5_2;
    const double h10_1_15 = acc[507] + ABx * acc[197];
    const double h4_1_15 = acc[197] + ABx * acc[11];
    const double h4_4_15 = h10_1_15 + ABx * h4_1_15;
    const double k4_4_5_3 = h4_4_15 + CDz * h4_4_5;
    const double k4_4_5_6 = k4_4_11_3 + CDx * k4_4_5_3;
    const double h10_1_26 = acc[518] + ABx * acc[208];
    const double h4_1_26 = acc[208] + ABx * acc[22];
    const double h4_4_26 = h10_1_26 + ABx * h4_1_26;
    const double k4_4_13_2 = h4_4_26 + CDy * h4_4_13;
    const double k4_4_5_7 = k4_4_13_2 + CDy * k4_4_5_2;
    const double h10_1_27 = acc[519] + ABx * acc[209];
    const double h4_1_27 = acc[209] + ABx * acc[23];
    const double h4_4_27 = h10_1_27 + ABx * h4_1_27;
    const double k4_4_13_3 = h4_4_27 + CDz * h4_4_13;
    const double k4_4_5_8 = k4_4_13_3 + CDy * k4_4_5_3;
    const double h10_1_28 = acc[520] + ABx * acc[210];
    const double h4_1_28 = acc[210] + ABx * acc[24];
    const double h4_4_28 = h10_1_28 + ABx * h4_1_28;
    const double k4_4_15_3 = h4_4_28 + CDz * h4_4_15;
    const double k4_4_5_9 = k4_4_15_3 + CDz * k4_4_5_3;
    const double k4_4_12_1 = h4_4_22 + CDx * h4_4_12;
    const double h10_1_6 = acc[498] + ABx * acc[188];
    const double h4_1_6 = acc[188] + ABx * acc[2];
    const double h4_4_6 = h10_1_6 + ABx * h4_1_6;
    const double k4_4_6_1 = h4_4_12 + CDx * h4_4_6;
    const double k4_4_6_4 = k4_4_12_1 + CDx * k4_4_6_1;
    const double k4_4_12_2 = h4_4_24 + CDy * h4_4_12;
    const double k4_4_6_2 = h4_4_15 + CDy * h4_4_6;
    const double k4_4_6_5 = k4_4_12_2 + CDx * k4_4_6_2;
    const double h10_1_14 = acc[506] + ABx * acc[196];
    const double h4_1_14 = acc[196] + ABx * acc[10];
    const double h4_4_14 = h10_1_14 + ABx * h4_1_14;
    const double k4_4_6_3 = h4_4_14 + CDz * h4_4_6;
    const double k4_4_6_6 = k4_4_12_3 + CDx * k4_4_6_3;
    const double k4_4_15_2 = h4_4_27 + CDy * h4_4_15;
    const double k4_4_6_7 = k4_4_15_2 + CDy * k4_4_6_2;
    const double k4_4_6_8 = k4_4_15_3 + CDy * k4_4_6_3;
    const double h10_1_29 = acc[521] + ABx * acc[211];
    const double h4_1_29 = acc[211] + ABx * acc[25];
    const double h4_4_29 = h10_1_29 + ABx * h4_1_29;
    const double k4_4_14_3 = h4_4_29 + CDz * h4_4_14;
    const double k4_4_6_9 = k4_4_14_3 + CDz * k4_4_6_3;
    const double k4_4_13_1 = h4_4_23 + CDx * h4_4_13;
    const double h10_1_7 = acc[499] + ABx * acc[189];
    const double h4_1_7 = acc[189] + ABx * acc[3];
    const double h4_4_7 = h10_1_7 + ABx * h4_1_7;
    const double k4_4_7_1 = h4_4_13 + CDx * h4_4_7;
    const double k4_4_7_4 = k4_4_13_1 + CDx * k4_4_7_1;
    const double h10_1_16 = acc[508] + ABx * acc[198];
    const double h4_1_16 = acc[198] + ABx * acc[12];
    const double h4_4_16 = h10_1_16 + ABx * h4_1_16;
    const double k4_4_7_2 = h4_4_16 + CDy * h4_4_7;
    const double k4_4_7_5 = k4_4_13_2 + CDx * k4_4_7_2;
    const double h10_1_17 = acc[509] + ABx * acc[199];
    const double h4_1_17 = acc[199] + ABx * acc[13];
    const double h4_4_17 = h10_1_17 + ABx * h4_1_17;
    const double k4_4_7_3 = h4_4_17 + CDz * h4_4_7;
    const double k4_4_7_6 = k4_4_13_3 + CDx * k4_4_7_3;
    const double h10_1_30 = acc[522] + ABx * acc[212];
    const double h4_1_30 = acc[212] + ABx * acc[26];
    const double h4_4_30 = h10_1_30 + ABx * h4_1_30;
    const double k4_4_16_2 = h4_4_30 + CDy * h4_4_16;
    const double k4_4_7_7 = k4_4_16_2 + CDy * k4_4_7_2;
    const double h10_1_31 = acc[523] + ABx * acc[213];
    const double h4_1_31 = acc[213] + ABx * acc[27];
    const double h4_4_31 = h10_1_31 + ABx * h4_1_31;
    const double k4_4_16_3 = h4_4_31 + CDz * h4_4_16;
    const double k4_4_7_8 = k4_4_16_3 + CDy * k4_4_7_3;
    const double h10_1_32 = acc[524] + ABx * acc[214];
    const double h4_1_32 = acc[214] + ABx * acc[28];
    const double h4_4_32 = h10_1_32 + ABx * h4_1_32;
    const double k4_4_17_3 = h4_4_32 + CDz * h4_4_17;
    const double k4_4_7_9 = k4_4_17_3 + CDz * k4_4_7_3;
    const double k4_4_15_1 = h4_4_24 + CDx * h4_4_15;
    const double h10_1_8 = acc[500] + ABx * acc[190];
    const double h4_1_8 = acc[190] + ABx * acc[4];
    const double h4_4_8 = h10_1_8 + ABx * h4_1_8;
    const double k4_4_8_1 = h4_4_15 + CDx * h4_4_8;
    const double k4_4_8_4 = k4_4_15_1 + CDx * k4_4_8_1;
    const double k4_4_8_2 = h4_4_17 + CDy * h4_4_8;
    const double k4_4_8_5 = k4_4_15_2 + CDx * k4_4_8_2;
    const double h10_1_18 = acc[510] + ABx * acc[200];
    const double h4_1_18 = acc[200] + ABx * acc[14];
    const double h4_4_18 = h10_1_18 + ABx * h4_1_18;
    const double k4_4_8_3 = h4_4_18 + CDz * h4_4_8;
    const double k4_4_8_6 = k4_4_15_3 + CDx * k4_4_8_3;
    const double k4_4_17_2 = h4_4_31 + CDy * h4_4_17;
    const double k4_4_8_7 = k4_4_17_2 + CDy * k4_4_8_2;
    const double k4_4_8_8 = k4_4_17_3 + CDy * k4_4_8_3;
    const double h10_1_33 = acc[525] + ABx * acc[215];
    const double h4_1_33 = acc[215] + ABx * acc[29];
    const double h4_4_33 = h10_1_33 + ABx * h4_1_33;
    const double k4_4_18_3 = h4_4_33 + CDz * h4_4_18;
    const double k4_4_8_9 = k4_4_18_3 + CDz * k4_4_8_3;
    const double k4_4_14_1 = h4_4_25 + CDx * h4_4_14;
    const double h10_1_9 = acc[501] + ABx * acc[191];
    const double h4_1_9 = acc[191] + ABx * acc[5];
    const double h4_4_9 = h10_1_9 + ABx * h4_1_9;
    const double k4_4_9_1 = h4_4_14 + CDx * h4_4_9;
    const double k4_4_9_4 = k4_4_14_1 + CDx * k4_4_9_1;
    const double k4_4_14_2 = h4_4_28 + CDy * h4_4_14;
    const double k4_4_9_2 = h4_4_18 + CDy * h4_4_9;
    const double k4_4_9_5 = k4_4_14_2 + CDx * k4_4_9_2;
    const double h10_1_19 = acc[511] + ABx * acc[201];
    const double h4_1_19 = acc[201] + ABx * acc[15];
    const double h4_4_19 = h10_1_19 + ABx * h4_1_19;
    const double k4_4_9_3 = h4_4_19 + CDz * h4_4_9;
    const double k4_4_9_6 = k4_4_14_3 + CDx * k4_4_9_3;
    const double k4_4_18_2 = h4_4_32 + CDy * h4_4_18;
    const double k4_4_9_7 = k4_4_18_2 + CDy * k4_4_9_2;
    const double k4_4_9_8 = k4_4_18_3 + CDy * k4_4_9_3;
    const double h10_1_34 = acc[526] + ABx * acc[216];
    const double h4_1_34 = acc[216] + ABx * acc[30];
    const double h4_4_34 = h10_1_34 + ABx * h4_1_34;
    const double k4_4_19_3 = h4_4_34 + CDz * h4_4_19;
    const double k4_4_9_9 = k4_4_19_3 + CDz * k4_4_9_3;
    const double h10_2_20 = acc[543] + ABy * acc[202];
    const double h4_2_20 = acc[233] + ABy * acc[16];
    const double h4_5_20 = h10_2_20 + ABx * h4_2_20;
    const double h10_2_10 = acc[533] + ABy * acc[192];
    const double h4_2_10 = acc[223] + ABy * acc[6];
    const double h4_5_10 = h10_2_10 + ABx * h4_2_10;
    const double k4_5_10_1 = h4_5_20 + CDx * h4_5_10;
    const double h10_2_4 = acc[527] + ABy * acc[186];
    const double h4_2_4 = acc[217] + ABy * acc[0];
    const double h4_5_4 = h10_2_4 + ABx * h4_2_4;
    const double k4_5_4_1 = h4_5_10 + CDx * h4_5_4;
    const double k4_5_4_4 = k4_5_10_1 + CDx * k4_5_4_1;
    const double h10_2_21 = acc[544] + ABy * acc[203];
    const double h4_2_21 = acc[234] + ABy * acc[17];
    const double h4_5_21 = h10_2_21 + ABx * h4_2_21;
    const double k4_5_10_2 = h4_5_21 + CDy * h4_5_10;
    const double h10_2_11 = acc[534] + ABy * acc[193];
    const double h4_2_11 = acc[224] + ABy * acc[7];
    const double h4_5_11 = h10_2_11 + ABx * h4_2_11;
    const double k4_5_4_2 = h4_5_11 + CDy * h4_5_4;
    const double k4_5_4_5 = k4_5_10_2 + CDx * k4_5_4_2;
    const double h10_2_22 = acc[545] + ABy * acc[204];
    const double h4_2_22 = acc[235] + ABy * acc[18];
    const double h4_5_22 = h10_2_22 + ABx * h4_2_22;
    const double k4_5_10_3 = h4_5_22 + CDz * h4_5_10;
    const double h10_2_12 = acc[535] + ABy * acc[194];
    const double h4_2_12 = acc[225] + ABy * acc[8];
    const double h4_5_12 = h10_2_12 + ABx * h4_2_12;
    const double k4_5_4_3 = h4_5_12 + CDz * h4_5_4;
    const double k4_5_4_6 = k4_5_10_3 + CDx * k4_5_4_3;
    const double h10_2_23 = acc[546] + ABy * acc[205];
    const double h4_2_23 = acc[236] + ABy * acc[19];
    const double h4_5_23 = h10_2_23 + ABx * h4_2_23;
    const double k4_5_11_2 = h4_5_23 + CDy * h4_5_11;
    const double k4_5_4_7 = k4_5_11_2 + CDy * k4_5_4_2;
    const double h10_2_24 = acc[547] + ABy * acc[206];
    const double h4_2_24 = acc[237] + ABy * acc[20];
    const double h4_5_24 = h10_2_24 + ABx * h4_2_24;
    const double k4_5_11_3 = h4_5_24 + CDz * h4_5_11;
    const double k4_5_4_8 = k4_5_11_3 + CDy * k4_5_4_3;
    const double h10_2_25 = acc[548] + ABy * acc[207];
    const double h4_2_25 = acc[238] + ABy * acc[21];
    const double h4_5_25 = h10_2_25 + ABx * h4_2_25;
    const double k4_5_12_3 = h4_5_25 + CDz * h4_5_12;
    const double k4_5_4_9 = k4_5_12_3 + CDz * k4_5_4_3;
    const double k4_5_11_1 = h4_5_21 + CDx * h4_5_11;
    const double h10_2_5 = acc[528] + ABy * acc[187];
    const double h4_2_5 = acc[218] + ABy * acc[1];
    const double h4_5_5 = h10_2_5 + ABx * h4_2_5;
    const double k4_5_5_1 = h4_5_11 + CDx * h4_5_5;
    const double k4_5_5_4 = k4_5_11_1 + CDx * k4_5_5_1;
    const double h10_2_13 = acc[536] + ABy * acc[195];
    const double h4_2_13 = acc[226] + ABy * acc[9];
    const double h4_5_13 = h10_2_13 + ABx * h4_2_13;
    const double k4_5_5_2 = h4_5_13 + CDy * h4_5_5;
    const double k4_5_5_5 = k4_5_11_2 + CDx * k4_5_5_2;
    const double h10_2_15 = acc[538] + ABy * acc[197];
    const double h4_2_15 = acc[228] + ABy * acc[11];
    const double h4_5_15 = h10_2_15 + ABx * h4_2_15;
    const double k4_5_5_3 = h4_5_15 + CDz * h4_5_5;
    const double k4_5_5_6 = k4_5_11_3 + CDx * k4_5_5_3;
    const double h10_2_26 = acc[549] + ABy * acc[208];
    const double h4_2_26 = acc[239] + ABy * acc[22];
    const double h4_5_26 = h10_2_26 + ABx * h4_2_26;
    const double k4_5_13_2 = h4_5_26 + CDy * h4_5_13;
    const double k4_5_5_7 = k4_5_13_2 + CDy * k4_5_5_2;
    const double h10_2_27 = acc[550] + ABy * acc[209];
    const double h4_2_27 = acc[240] + ABy * acc[23];
    const double h4_5_27 = h10_2_27 + ABx * h4_2_27;
    const double k4_5_13_3 = h4_5_27 + CDz * h4_5_13;
    const double k4_5_5_8 = k4_5_13_3 + CDy * k4_5_5_3;
    const double h10_2_28 = acc[551] + ABy * acc[210];
    const double h4_2_28 = acc[241] + ABy * acc[24];
    const double h4_5_28 = h10_2_28 + ABx * h4_2_28;
    const double k4_5_15_3 = h4_5_28 + CDz * h4_5_15;
    const double k4_5_5_9 = k4_5_15_3 + CDz * k4_5_5_3;
    const double k4_5_12_1 = h4_5_22 + CDx * h4_5_12;
    const double h10_2_6 = acc[529] + ABy * acc[188];
    const double h4_2_6 = acc[219] + ABy * acc[2];
    const double h4_5_6 = h10_2_6 + ABx * h4_2_6;
    const double k4_5_6_1 = h4_5_12 + CDx * h4_5_6;
    const double k4_5_6_4 = k4_5_12_1 + CDx * k4_5_6_1;
    const double k4_5_12_2 = h4_5_24 + CDy * h4_5_12;
    const double k4_5_6_2 = h4_5_15 + CDy * h4_5_6;
    const double k4_5_6_5 = k4_5_12_2 + CDx * k4_5_6_2;
    const double h10_2_14 = acc[537] + ABy * acc[196];
    const double h4_2_14 = acc[227] + ABy * acc[10];
    const double h4_5_14 = h10_2_14 + ABx * h4_2_14;
    const double k4_5_6_3 = h4_5_14 + CDz * h4_5_6;
    const double k4_5_6_6 = k4_5_12_3 + CDx * k4_5_6_3;
    const double k4_5_15_2 = h4_5_27 + CDy * h4_5_15;
    const double k4_5_6_7 = k4_5_15_2 + CDy * k4_5_6_2;
    const double k4_5_6_8 = k4_5_15_3 + CDy * k4_5_6_3;
    const double h10_2_29 = acc[552] + ABy * acc[211];
    const double h4_2_29 = acc[242] + ABy * acc[25];
    const double h4_5_29 = h10_2_29 + ABx * h4_2_29;
    const double k4_5_14_3 = h4_5_29 + CDz * h4_5_14;
    const double k4_5_6_9 = k4_5_14_3 + CDz * k4_5_6_3;
    const double k4_5_13_1 = h4_5_23 + CDx * h4_5_13;
    const double h10_2_7 = acc[530] + ABy * acc[189];
    const double h4_2_7 = acc[220] + ABy * acc[3];
    const double h4_5_7 = h10_2_7 + ABx * h4_2_7;
    const double k4_5_7_1 = h4_5_13 + CDx * h4_5_7;
    const double k4_5_7_4 = k4_5_13_1 + CDx * k4_5_7_1;
    const double h10_2_16 = acc[539] + ABy * acc[198];
    const double h4_2_16 = acc[229] + ABy * acc[12];
    const double h4_5_16 = h10_2_16 + ABx * h4_2_16;
    const double k4_5_7_2 = h4_5_16 + CDy * h4_5_7;
    const double k4_5_7_5 = k4_5_13_2 + CDx * k4_5_7_2;
    const double h10_2_17 = acc[540] + ABy * acc[199];
    const double h4_2_17 = acc[230] + ABy * acc[13];
    const double h4_5_17 = h10_2_17 + ABx * h4_2_17;
    const double k4_5_7_3 = h4_5_17 + CDz * h4_5_7;
    const double k4_5_7_6 = k4_5_13_3 + CDx * k4_5_7_3;
    const double h10_2_30 = acc[553] + ABy * acc[212];
    const double h4_2_30 = acc[243] + ABy * acc[26];
    const double h4_5_30 = h10_2_30 + ABx * h4_2_30;
    const double k4_5_16_2 = h4_5_30 + CDy * h4_5_16;
    const double k4_5_7_7 = k4_5_16_2 + CDy * k4_5_7_2;
    const double h10_2_31 = acc[554] + ABy * acc[213];
    const double h4_2_31 = acc[244] + ABy * acc[27];
    const double h4_5_31 = h10_2_31 + ABx * h4_2_31;
    const double k4_5_16_3 = h4_5_31 + CDz * h4_5_16;
    const double k4_5_7_8 = k4_5_16_3 + CDy * k4_5_7_3;
    const double h10_2_32 = acc[555] + ABy * acc[214];
    const double h4_2_32 = acc[245] + ABy * acc[28];
    const double h4_5_32 = h10_2_32 + ABx * h4_2_32;
    const double k4_5_17_3 = h4_5_32 + CDz * h4_5_17;
    const double k4_5_7_9 = k4_5_17_3 + CDz * k4_5_7_3;
    const double k4_5_15_1 = h4_5_24 + CDx * h4_5_15;
    const double h10_2_8 = acc[531] + ABy * acc[190];
    const double h4_2_8 = acc[221] + ABy * acc[4];
    const double h4_5_8 = h10_2_8 + ABx * h4_2_8;
    const double k4_5_8_1 = h4_5_15 + CDx * h4_5_8;
    const double k4_5_8_4 = k4_5_15_1 + CDx * k4_5_8_1;
    const double k4_5_8_2 = h4_5_17 + CDy * h4_5_8;
    const double k4_5_8_5 = k4_5_15_2 + CDx * k4_5_8_2;
    const double h10_2_18 = acc[541] + ABy * acc[200];
    const double h4_2_18 = acc[231] + ABy * acc[14];
    const double h4_5_18 = h10_2_18 + ABx * h4_2_18;
    const double k4_5_8_3 = h4_5_18 + CDz * h4_5_8;
    const double k4_5_8_6 = k4_5_15_3 + CDx * k4_5_8_3;
    const double k4_5_17_2 = h4_5_31 + CDy * h4_5_17;
    const double k4_5_8_7 = k4_5_17_2 + CDy * k4_5_8_2;
    const double k4_5_8_8 = k4_5_17_3 + CDy * k4_5_8_3;
    const double h10_2_33 = acc[556] + ABy * acc[215];
    const double h4_2_33 = acc[246] + ABy * acc[29];
    const double h4_5_33 = h10_2_33 + ABx * h4_2_33;
    const double k4_5_18_3 = h4_5_33 + CDz * h4_5_18;
    const double k4_5_8_9 = k4_5_18_3 + CDz * k4_5_8_3;
    const double k4_5_14_1 = h4_5_25 + CDx * h4_5_14;
    const double h10_2_9 = acc[532] + ABy * acc[191];
    const double h4_2_9 = acc[222] + ABy * acc[5];
    const double h4_5_9 = h10_2_9 + ABx * h4_2_9;
    const double k4_5_9_1 = h4_5_14 + CDx * h4_5_9;
    const double k4_5_9_4 = k4_5_14_1 + CDx * k4_5_9_1;
    const double k4_5_14_2 = h4_5_28 + CDy * h4_5_14;
    const double k4_5_9_2 = h4_5_18 + CDy * h4_5_9;
    const double k4_5_9_5 = k4_5_14_2 + CDx * k4_5_9_2;
    const double h10_2_19 = acc[542] + ABy * acc[201];
    const double h4_2_19 = acc[232] + ABy * acc[15];
    const double h4_5_19 = h10_2_19 + ABx * h4_2_19;
    const double k4_5_9_3 = h4_5_19 + CDz * h4_5_9;
    const double k4_5_9_6 = k4_5_14_3 + CDx * k4_5_9_3;
    const double k4_5_18_2 = h4_5_32 + CDy * h4_5_18;
    const double k4_5_9_7 = k4_5_18_2 + CDy * k4_5_9_2;
    const double k4_5_9_8 = k4_5_18_3 + CDy * k4_5_9_3;
    const double h10_2_34 = acc[557] + ABy * acc[216];
    const double h4_2_34 = acc[247] + ABy * acc[30];
    const double h4_5_34 = h10_2_34 + ABx * h4_2_34;
    const double k4_5_19_3 = h4_5_34 + CDz * h4_5_19;
    const double k4_5_9_9 = k4_5_19_3 + CDz * k4_5_9_3;
    const double h10_3_20 = acc[574] + ABz * acc[202];
    const double h4_3_20 = acc[264] + ABz * acc[16];
    const double h4_6_20 = h10_3_20 + ABx * h4_3_20;
    const double h10_3_10 = acc[564] + ABz * acc[192];
    const double h4_3_10 = acc[254] + ABz * acc[6];
    const double h4_6_10 = h10_3_10 + ABx * h4_3_10;
    const double k4_6_10_1 = h4_6_20 + CDx * h4_6_10;
    const double h10_3_4 = acc[558] + ABz * acc[186];
    const double h4_3_4 = acc[248] + ABz * acc[0];
    const double h4_6_4 = h10_3_4 + ABx * h4_3_4;
    const double k4_6_4_1 = h4_6_10 + CDx * h4_6_4;
    const double k4_6_4_4 = k4_6_10_1 + CDx * k4_6_4_1;
    const double h10_3_21 = acc[575] + ABz * acc[203];
    const double h4_3_21 = acc[265] + ABz * acc[17];
    const double h4_6_21 = h10_3_21 + ABx * h4_3_21;
    const double k4_6_10_2 = h4_6_21 + CDy * h4_6_10;
    const double h10_3_11 = acc[565] + ABz * acc[193];
    const double h4_3_11 = acc[255] + ABz * acc[7];
    const double h4_6_11 = h10_3_11 + ABx * h4_3_11;
    const double k4_6_4_2 = h4_6_11 + CDy * h4_6_4;
    const double k4_6_4_5 = k4_6_10_2 + CDx * k4_6_4_2;
    const double h10_3_22 = acc[576] + ABz * acc[204];
    const double h4_3_22 = acc[266] + ABz * acc[18];
    const double h4_6_22 = h10_3_22 + ABx * h4_3_22;
    const double k4_6_10_3 = h4_6_22 + CDz * h4_6_10;
    const double h10_3_12 = acc[566] + ABz * acc[194];
    const double h4_3_12 = acc[256] + ABz * acc[8];
    const double h4_6_12 = h10_3_12 + ABx * h4_3_12;
    const double k4_6_4_3 = h4_6_12 + CDz * h4_6_4;
    const double k4_6_4_6 = k4_6_10_3 + CDx * k4_6_4_3;
    const double h10_3_23 = acc[577] + ABz * acc[205];
    const double h4_3_23 = acc[267] + ABz * acc[19];
    const double h4_6_23 = h10_3_23 + ABx * h4_3_23;
    const double k4_6_11_2 = h4_6_23 + CDy * h4_6_11;
    const double k4_6_4_7 = k4_6_11_2 + CDy * k4_6_4_2;
    const double h10_3_24 = acc[578] + ABz * acc[206];
    const double h4_3_24 = acc[268] + ABz * acc[20];
    const double h4_6_24 = h10_3_24 + ABx * h4_3_24;
    const double k4_6_11_3 = h4_6_24 + CDz * h4_6_11;
    const double k4_6_4_8 = k4_6_11_3 + CDy * k4_6_4_3;
    const double h10_3_25 = acc[579] + ABz * acc[207];
    const double h4_3_25 = acc[269] + ABz * acc[21];
    const double h4_6_25 = h10_3_25 + ABx * h4_3_25;
    const double k4_6_12_3 = h4_6_25 + CDz * h4_6_12;
    const double k4_6_4_9 = k4_6_12_3 + CDz * k4_6_4_3;
    const double k4_6_11_1 = h4_6_21 + CDx * h4_6_11;
    const double h10_3_5 = acc[559] + ABz * acc[187];
    const double h4_3_5 = acc[249] + ABz * acc[1];
    const double h4_6_5 = h10_3_5 + ABx * h4_3_5;
    const double k4_6_5_1 = h4_6_11 + CDx * h4_6_5;
    const double k4_6_5_4 = k4_6_11_1 + CDx * k4_6_5_1;
    const double h10_3_13 = acc[567] + ABz * acc[195];
    const double h4_3_13 = acc[257] + ABz * acc[9];
    const double h4_6_13 = h10_3_13 + ABx * h4_3_13;
    const double k4_6_5_2 = h4_6_13 + CDy * h4_6_5;
    const double k4_6_5_5 = k4_6_11_2 + CDx * k4_6_5_2;
    const double h10_3_15 = acc[569] + ABz * acc[197];
    const double h4_3_15 = acc[259] + ABz * acc[11];
    const double h4_6_15 = h10_3_15 + ABx * h4_3_15;
    const double k4_6_5_3 = h4_6_15 + CDz * h4_6_5;
    const double k4_6_5_6 = k4_6_11_3 + CDx * k4_6_5_3;
    const double h10_3_26 = acc[580] + ABz * acc[208];
    const double h4_3_26 = acc[270] + ABz * acc[22];
    const double h4_6_26 = h10_3_26 + ABx * h4_3_26;
    const double k4_6_13_2 = h4_6_26 + CDy * h4_6_13;
    const double k4_6_5_7 = k4_6_13_2 + CDy * k4_6_5_2;
    const double h10_3_27 = acc[581] + ABz * acc[209];
    const double h4_3_27 = acc[271] + ABz * acc[23];
    const double h4_6_27 = h10_3_27 + ABx * h4_3_27;
    const double k4_6_13_3 = h4_6_27 + CDz * h4_6_13;
    const double k4_6_5_8 = k4_6_13_3 + CDy * k4_6_5_3;
    const double h10_3_28 = acc[582] + ABz * acc[210];
    const double h4_3_28 = acc[272] + ABz * acc[24];
    const double h4_6_28 = h10_3_28 + ABx * h4_3_28;
    const double k4_6_15_3 = h4_6_28 + CDz * h4_6_15;
    const double k4_6_5_9 = k4_6_15_3 + CDz * k4_6_5_3;
    const double k4_6_12_1 = h4_6_22 + CDx * h4_6_12;
    const double h10_3_6 = acc[560] + ABz * acc[188];
    const double h4_3_6 = acc[250] + ABz * acc[2];
    const double h4_6_6 = h10_3_6 + ABx * h4_3_6;
    const double k4_6_6_1 = h4_6_12 + CDx * h4_6_6;
    const double k4_6_6_4 = k4_6_12_1 + CDx * k4_6_6_1;
    const double k4_6_12_2 = h4_6_24 + CDy * h4_6_12;
    const double k4_6_6_2 = h4_6_15 + CDy * h4_6_6;
    const double k4_6_6_5 = k4_6_12_2 + CDx * k4_6_6_2;
    const double h10_3_14 = acc[568] + ABz * acc[196];
    const double h4_3_14 = acc[258] + ABz * acc[10];
    const double h4_6_14 = h10_3_14 + ABx * h4_3_14;
    const double k4_6_6_3 = h4_6_14 + CDz * h4_6_6;
    const double k4_6_6_6 = k4_6_12_3 + CDx * k4_6_6_3;
    const double k4_6_15_2 = h4_6_27 + CDy * h4_6_15;
    const double k4_6_6_7 = k4_6_15_2 + CDy * k4_6_6_2;
    const double k4_6_6_8 = k4_6_15_3 + CDy * k4_6_6_3;
    const double h10_3_29 = acc[583] + ABz * acc[211];
    const double h4_3_29 = acc[273] + ABz * acc[25];
    const double h4_6_29 = h10_3_29 + ABx * h4_3_29;
    const double k4_6_14_3 = h4_6_29 + CDz * h4_6_14;
    const double k4_6_6_9 = k4_6_14_3 + CDz * k4_6_6_3;
    const double k4_6_13_1 = h4_6_23 + CDx * h4_6_13;
    const double h10_3_7 = acc[561] + ABz * acc[189];
    const double h4_3_7 = acc[251] + ABz * acc[3];
    const double h4_6_7 = h10_3_7 + ABx * h4_3_7;
    const double k4_6_7_1 = h4_6_13 + CDx * h4_6_7;
    const double k4_6_7_4 = k4_6_13_1 + CDx * k4_6_7_1;
    const double h10_3_16 = acc[570] + ABz * acc[198];
    const double h4_3_16 = acc[260] + ABz * acc[12];
    const double h4_6_16 = h10_3_16 + ABx * h4_3_16;
    const double k4_6_7_2 = h4_6_16 + CDy * h4_6_7;
    const double k4_6_7_5 = k4_6_13_2 + CDx * k4_6_7_2;
    const double h10_3_17 = acc[571] + ABz * acc[199];
    const double h4_3_17 = acc[261] + ABz * acc[13];
    const double h4_6_17 = h10_3_17 + ABx * h4_3_17;
    const double k4_6_7_3 = h4_6_17 + CDz * h4_6_7;
    const double k4_6_7_6 = k4_6_13_3 + CDx * k4_6_7_3;
    const double h10_3_30 = acc[584] + ABz * acc[212];
    const double h4_3_30 = acc[274] + ABz * acc[26];
    const double h4_6_30 = h10_3_30 + ABx * h4_3_30;
    const double k4_6_16_2 = h4_6_30 + CDy * h4_6_16;
    const double k4_6_7_7 = k4_6_16_2 + CDy * k4_6_7_2;
    const double h10_3_31 = acc[585] + ABz * acc[213];
    const double h4_3_31 = acc[275] + ABz * acc[27];
    const double h4_6_31 = h10_3_31 + ABx * h4_3_31;
    const double k4_6_16_3 = h4_6_31 + CDz * h4_6_16;
    const double k4_6_7_8 = k4_6_16_3 + CDy * k4_6_7_3;
    const double h10_3_32 = acc[586] + ABz * acc[214];
    const double h4_3_32 = acc[276] + ABz * acc[28];
    const double h4_6_32 = h10_3_32 + ABx * h4_3_32;
    const double k4_6_17_3 = h4_6_32 + CDz * h4_6_17;
    const double k4_6_7_9 = k4_6_17_3 + CDz * k4_6_7_3;
    const double k4_6_15_1 = h4_6_24 + CDx * h4_6_15;
    const double h10_3_8 = acc[562] + ABz * acc[190];
    const double h4_3_8 = acc[252] + ABz * acc[4];
    const double h4_6_8 = h10_3_8 + ABx * h4_3_8;
    const double k4_6_8_1 = h4_6_15 + CDx * h4_6_8;
    const double k4_6_8_4 = k4_6_15_1 + CDx * k4_6_8_1;
    const double k4_6_8_2 = h4_6_17 + CDy * h4_6_8;
    const double k4_6_8_5 = k4_6_15_2 + CDx * k4_6_8_2;
    const double h10_3_18 = acc[572] + ABz * acc[200];
    const double h4_3_18 = acc[262] + ABz * acc[14];
    const double h4_6_18 = h10_3_18 + ABx * h4_3_18;
    const double k4_6_8_3 = h4_6_18 + CDz * h4_6_8;
    const double k4_6_8_6 = k4_6_15_3 + CDx * k4_6_8_3;
    const double k4_6_17_2 = h4_6_31 + CDy * h4_6_17;
    const double k4_6_8_7 = k4_6_17_2 + CDy * k4_6_8_2;
    const double k4_6_8_8 = k4_6_17_3 + CDy * k4_6_8_3;
    const double h10_3_33 = acc[587] + ABz * acc[215];
    const double h4_3_33 = acc[277] + ABz * acc[29];
    const double h4_6_33 = h10_3_33 + ABx * h4_3_33;
    const double k4_6_18_3 = h4_6_33 + CDz * h4_6_18;
    const double k4_6_8_9 = k4_6_18_3 + CDz * k4_6_8_3;
    const double k4_6_14_1 = h4_6_25 + CDx * h4_6_14;
    const double h10_3_9 = acc[563] + ABz * acc[191];
    const double h4_3_9 = acc[253] + ABz * acc[5];
    const double h4_6_9 = h10_3_9 + ABx * h4_3_9;
    const double k4_6_9_1 = h4_6_14 + CDx * h4_6_9;
    const double k4_6_9_4 = k4_6_14_1 + CDx * k4_6_9_1;
    const double k4_6_14_2 = h4_6_28 + CDy * h4_6_14;
    const double k4_6_9_2 = h4_6_18 + CDy * h4_6_9;
    const double k4_6_9_5 = k4_6_14_2 + CDx * k4_6_9_2;
    const double h10_3_19 = acc[573] + ABz * acc[201];
    const double h4_3_19 = acc[263] + ABz * acc[15];
    const double h4_6_19 = h10_3_19 + ABx * h4_3_19;
    const double k4_6_9_3 = h4_6_19 + CDz * h4_6_9;
    const double k4_6_9_6 = k4_6_14_3 + CDx * k4_6_9_3;
    const double k4_6_18_2 = h4_6_32 + CDy * h4_6_18;
    const double k4_6_9_7 = k4_6_18_2 + CDy * k4_6_9_2;
    const double k4_6_9_8 = k4_6_18_3 + CDy * k4_6_9_3;
    const double h10_3_34 = acc[588] + ABz * acc[216];
    const double h4_3_34 = acc[278] + ABz * acc[30];
    const double h4_6_34 = h10_3_34 + ABx * h4_3_34;
    const double k4_6_19_3 = h4_6_34 + CDz * h4_6_19;
    const double k4_6_9_9 = k4_6_19_3 + CDz * k4_6_9_3;
    const double h11_2_20 = acc[605] + ABy * acc[233];
    const double h4_7_20 = h11_2_20 + ABy * h4_2_20;
    const double h11_2_10 = acc[595] + ABy * acc[223];
    const double h4_7_10 = h11_2_10 + ABy * h4_2_10;
    const double k4_7_10_1 = h4_7_20 + CDx * h4_7_10;
    const double h11_2_4 = acc[589] + ABy * acc[217];
    const double h4_7_4 = h11_2_4 + ABy * h4_2_4;
    const double k4_7_4_1 = h4_7_10 + CDx * h4_7_4;
    const double k4_7_4_4 = k4_7_10_1 + CDx * k4_7_4_1;
    const double h11_2_21 = acc[606] + ABy * acc[234];
    const double h4_7_21 = h11_2_21 + ABy * h4_2_21;
    const double k4_7_10_2 = h4_7_21 + CDy * h4_7_10;
    const double h11_2_11 = acc[596] + ABy * acc[224];
    const double h4_7_11 = h11_2_11 + ABy * h4_2_11;
    const double k4_7_4_2 = h4_7_11 + CDy * h4_7_4;
    const double k4_7_4_5 = k4_7_10_2 + CDx * k4_7_4_2;
    const double h11_2_22 = acc[607] + ABy * acc[235];
    const double h4_7_22 = h11_2_22 + ABy * h4_2_22;
    const double k4_7_10_3 = h4_7_22 + CDz * h4_7_10;
    const double h11_2_12 = acc[597] + ABy * acc[225];
    const double h4_7_12 = h11_2_12 + ABy * h4_2_12;
    const double k4_7_4_3 = h4_7_12 + CDz * h4_7_4;
    const double k4_7_4_6 = k4_7_10_3 + CDx * k4_7_4_3;
    const double h11_2_23 = acc[608] + ABy * acc[236];
    const double h4_7_23 = h11_2_23 + ABy * h4_2_23;
    const double k4_7_11_2 = h4_7_23 + CDy * h4_7_11;
    const double k4_7_4_7 = k4_7_11_2 + CDy * k4_7_4_2;
    const double h11_2_24 = acc[609] + ABy * acc[237];
    const double h4_7_24 = h11_2_24 + ABy * h4_2_24;
    const double k4_7_11_3 = h4_7_24 + CDz * h4_7_11;
    const double k4_7_4_8 = k4_7_11_3 + CDy * k4_7_4_3;
    const double h11_2_25 = acc[610] + ABy * acc[238];
    const double h4_7_25 = h11_2_25 + ABy * h4_2_25;
    const double k4_7_12_3 = h4_7_25 + CDz * h4_7_12;
    const double k4_7_4_9 = k4_7_12_3 + CDz * k4_7_4_3;
    const double k4_7_11_1 = h4_7_21 + CDx * h4_7_11;
    const double h11_2_5 = acc[590] + ABy * acc[218];
    const double h4_7_5 = h11_2_5 + ABy * h4_2_5;
    const double k4_7_5_1 = h4_7_11 + CDx * h4_7_5;
    const double k4_7_5_4 = k4_7_11_1 + CDx * k4_7_5_1;
    const double h11_2_13 = acc[598] + ABy * acc[226];
    const double h4_7_13 = h11_2_13 + ABy * h4_2_13;
    const double k4_7_5_2 = h4_7_13 + CDy * h4_7_5;
    const double k4_7_5_5 = k4_7_11_2 + CDx * k4_7_5_2;
    const double h11_2_15 = acc[600] + ABy * acc[228];
    const double h4_7_15 = h11_2_15 + ABy * h4_2_15;
    const double k4_7_5_3 = h4_7_15 + CDz * h4_7_5;
    const double k4_7_5_6 = k4_7_11_3 + CDx * k4_7_5_3;
    const double h11_2_26 = acc[611] + ABy * acc[239];
    const double h4_7_26 = h11_2_26 + ABy * h4_2_26;
    const double k4_7_13_2 = h4_7_26 + CDy * h4_7_13;
    const double k4_7_5_7 = k4_7_13_2 + CDy * k4_7_5_2;
    const double h11_2_27 = acc[612] + ABy * acc[240];
    const double h4_7_27 = h11_2_27 + ABy * h4_2_27;
    const double k4_7_13_3 = h4_7_27 + CDz * h4_7_13;
    const double k4_7_5_8 = k4_7_13_3 + CDy * k4_7_5_3;
    const double h11_2_28 = acc[613] + ABy * acc[241];
    const double h4_7_28 = h11_2_28 + ABy * h4_2_28;
    const double k4_7_15_3 = h4_7_28 + CDz * h4_7_15;
    const double k4_7_5_9 = k4_7_15_3 + CDz * k4_7_5_3;
    const double k4_7_12_1 = h4_7_22 + CDx * h4_7_12;
    const double h11_2_6 = acc[591] + ABy * acc[219];
    const double h4_7_6 = h11_2_6 + ABy * h4_2_6;
    const double k4_7_6_1 = h4_7_12 + CDx * h4_7_6;
    const double k4_7_6_4 = k4_7_12_1 + CDx * k4_7_6_1;
    const double k4_7_12_2 = h4_7_24 + CDy * h4_7_12;
    const double k4_7_6_2 = h4_7_15 + CDy * h4_7_6;
    const double k4_7_6_5 = k4_7_12_2 + CDx * k4_7_6_2;
    const double h11_2_14 = acc[599] + ABy * acc[227];
    const double h4_7_14 = h11_2_14 + ABy * h4_2_14;
    const double k4_7_6_3 = h4_7_14 + CDz * h4_7_6;
    const double k4_7_6_6 = k4_7_12_3 + CDx * k4_7_6_3;
    const double k4_7_15_2 = h4_7_27 + CDy * h4_7_15;
    const double k4_7_6_7 = k4_7_15_2 + CDy * k4_7_6_2;
    const double k4_7_6_8 = k4_7_15_3 + CDy * k4_7_6_3;
    const double h11_2_29 = acc[614] + ABy * acc[242];
    const double h4_7_29 = h11_2_29 + ABy * h4_2_29;
    const double k4_7_14_3 = h4_7_29 + CDz * h4_7_14;
    const double k4_7_6_9 = k4_7_14_3 + CDz * k4_7_6_3;
    const double k4_7_13_1 = h4_7_23 + CDx * h4_7_13;
    const double h11_2_7 = acc[592] + ABy * acc[220];
    const double h4_7_7 = h11_2_7 + ABy * h4_2_7;
    const double k4_7_7_1 = h4_7_13 + CDx * h4_7_7;
    const double k4_7_7_4 = k4_7_13_1 + CDx * k4_7_7_1;
    const double h11_2_16 = acc[601] + ABy * acc[229];
    const double h4_7_16 = h11_2_16 + ABy * h4_2_16;
    const double k4_7_7_2 = h4_7_16 + CDy * h4_7_7;
    const double k4_7_7_5 = k4_7_13_2 + CDx * k4_7_7_2;
    const double h11_2_17 = acc[602] + ABy * acc[230];
    const double h4_7_17 = h11_2_17 + ABy * h4_2_17;
    const double k4_7_7_3 = h4_7_17 + CDz * h4_7_7;
    const double k4_7_7_6 = k4_7_13_3 + CDx * k4_7_7_3;
    const double h11_2_30 = acc[615] + ABy * acc[243];
    const double h4_7_30 = h11_2_30 + ABy * h4_2_30;
    const double k4_7_16_2 = h4_7_30 + CDy * h4_7_16;
    const double k4_7_7_7 = k4_7_16_2 + CDy * k4_7_7_2;
    const double h11_2_31 = acc[616] + ABy * acc[244];
    const double h4_7_31 = h11_2_31 + ABy * h4_2_31;
    const double k4_7_16_3 = h4_7_31 + CDz * h4_7_16;
    const double k4_7_7_8 = k4_7_16_3 + CDy * k4_7_7_3;
    const double h11_2_32 = acc[617] + ABy * acc[245];
    const double h4_7_32 = h11_2_32 + ABy * h4_2_32;
    const double k4_7_17_3 = h4_7_32 + CDz * h4_7_17;
    const double k4_7_7_9 = k4_7_17_3 + CDz * k4_7_7_3;
    const double k4_7_15_1 = h4_7_24 + CDx * h4_7_15;
    const double h11_2_8 = acc[593] + ABy * acc[221];
    const double h4_7_8 = h11_2_8 + ABy * h4_2_8;
    const double k4_7_8_1 = h4_7_15 + CDx * h4_7_8;
    const double k4_7_8_4 = k4_7_15_1 + CDx * k4_7_8_1;
    const double k4_7_8_2 = h4_7_17 + CDy * h4_7_8;
    const double k4_7_8_5 = k4_7_15_2 + CDx * k4_7_8_2;
    const double h11_2_18 = acc[603] + ABy * acc[231];
    const double h4_7_18 = h11_2_18 + ABy * h4_2_18;
    const double k4_7_8_3 = h4_7_18 + CDz * h4_7_8;
    const double k4_7_8_6 = k4_7_15_3 + CDx * k4_7_8_3;
    const double k4_7_17_2 = h4_7_31 + CDy * h4_7_17;
    const double k4_7_8_7 = k4_7_17_2 + CDy * k4_7_8_2;
    const double k4_7_8_8 = k4_7_17_3 + CDy * k4_7_8_3;
    const double h11_2_33 = acc[618] + ABy * acc[246];
    const double h4_7_33 = h11_2_33 + ABy * h4_2_33;
    const double k4_7_18_3 = h4_7_33 + CDz * h4_7_18;
    const double k4_7_8_9 = k4_7_18_3 + CDz * k4_7_8_3;
    const double k4_7_14_1 = h4_7_25 + CDx * h4_7_14;
    const double h11_2_9 = acc[594] + ABy * acc[222];
    const double h4_7_9 = h11_2_9 + ABy * h4_2_9;
    const double k4_7_9_1 = h4_7_14 + CDx * h4_7_9;
    const double k4_7_9_4 = k4_7_14_1 + CDx * k4_7_9_1;
    const double k4_7_14_2 = h4_7_28 + CDy * h4_7_14;
    const double k4_7_9_2 = h4_7_18 + CDy * h4_7_9;
    const double k4_7_9_5 = k4_7_14_2 + CDx * k4_7_9_2;
    const double h11_2_19 = acc[604] + ABy * acc[232];
    const double h4_7_19 = h11_2_19 + ABy * h4_2_19;
    const double k4_7_9_3 = h4_7_19 + CDz * h4_7_9;
    const double k4_7_9_6 = k4_7_14_3 + CDx * k4_7_9_3;
    const double k4_7_18_2 = h4_7_32 + CDy * h4_7_18;
    const double k4_7_9_7 = k4_7_18_2 + CDy * k4_7_9_2;
    const double k4_7_9_8 = k4_7_18_3 + CDy * k4_7_9_3;
    const double h11_2_34 = acc[619] + ABy * acc[247];
    const double h4_7_34 = h11_2_34 + ABy * h4_2_34;
    const double k4_7_19_3 = h4_7_34 + CDz * h4_7_19;
    const double k4_7_9_9 = k4_7_19_3 + CDz * k4_7_9_3;
    const double h11_3_20 = acc[636] + ABz * acc[233];
    const double h4_8_20 = h11_3_20 + ABy * h4_3_20;
    const double h11_3_10 = acc[626] + ABz * acc[223];
    const double h4_8_10 = h11_3_10 + ABy * h4_3_10;
    const double k4_8_10_1 = h4_8_20 + CDx * h4_8_10;
    const double h11_3_4 = acc[620] + ABz * acc[217];
    const double h4_8_4 = h11_3_4 + ABy * h4_3_4;
    const double k4_8_4_1 = h4_8_10 + CDx * h4_8_4;
    const double k4_8_4_4 = k4_8_10_1 + CDx * k4_8_4_1;
    const double h11_3_21 = acc[637] + ABz * acc[234];
    const double h4_8_21 = h11_3_21 + ABy * h4_3_21;
    const double k4_8_10_2 = h4_8_21 + CDy * h4_8_10;
    const double h11_3_11 = acc[627] + ABz * acc[224];
    const double h4_8_11 = h11_3_11 + ABy * h4_3_11;
    const double k4_8_4_2 = h4_8_11 + CDy * h4_8_4;
    const double k4_8_4_5 = k4_8_10_2 + CDx * k4_8_4_2;
    const double h11_3_22 = acc[638] + ABz * acc[235];
    const double h4_8_22 = h11_3_22 + ABy * h4_3_22;
    const double k4_8_10_3 = h4_8_22 + CDz * h4_8_10;
    const double h11_3_12 = acc[628] + ABz * acc[225];
    const double h4_8_12 = h11_3_12 + ABy * h4_3_12;
    const double k4_8_4_3 = h4_8_12 + CDz * h4_8_4;
    const double k4_8_4_6 = k4_8_10_3 + CDx * k4_8_4_3;
    const double h11_3_23 = acc[639] + ABz * acc[236];
    const double h4_8_23 = h11_3_23 + ABy * h4_3_23;
    const double k4_8_11_2 = h4_8_23 + CDy * h4_8_11;
    const double k4_8_4_7 = k4_8_11_2 + CDy * k4_8_4_2;
    const double h11_3_24 = acc[640] + ABz * acc[237];
    const double h4_8_24 = h11_3_24 + ABy * h4_3_24;
    const double k4_8_11_3 = h4_8_24 + CDz * h4_8_11;
    const double k4_8_4_8 = k4_8_11_3 + CDy * k4_8_4_3;
    const double h11_3_25 = acc[641] + ABz * acc[238];
    const double h4_8_25 = h11_3_25 + ABy * h4_3_25;
    const double k4_8_12_3 = h4_8_25 + CDz * h4_8_12;
    const double k4_8_4_9 = k4_8_12_3 + CDz * k4_8_4_3;
    const double k4_8_11_1 = h4_8_21 + CDx * h4_8_11;
    const double h11_3_5 = acc[621] + ABz * acc[218];
    const double h4_8_5 = h11_3_5 + ABy * h4_3_5;
    const double k4_8_5_1 = h4_8_11 + CDx * h4_8_5;
    const double k4_8_5_4 = k4_8_11_1 + CDx * k4_8_5_1;
    const double h11_3_13 = acc[629] + ABz * acc[226];
    const double h4_8_13 = h11_3_13 + ABy * h4_3_13;
    const double k4_8_5_2 = h4_8_13 + CDy * h4_8_5;
    const double k4_8_5_5 = k4_8_11_2 + CDx * k4_8_5_2;
    const double h11_3_15 = acc[631] + ABz * acc[228];
    const double h4_8_15 = h11_3_15 + ABy * h4_3_15;
    const double k4_8_5_3 = h4_8_15 + CDz * h4_8_5;
    const double k4_8_5_6 = k4_8_11_3 + CDx * k4_8_5_3;
    const double h11_3_26 = acc[642] + ABz * acc[239];
    const double h4_8_26 = h11_3_26 + ABy * h4_3_26;
    const double k4_8_13_2 = h4_8_26 + CDy * h4_8_13;
    const double k4_8_5_7 = k4_8_13_2 + CDy * k4_8_5_2;
    const double h11_3_27 = acc[643] + ABz * acc[240];
    const double h4_8_27 = h11_3_27 + ABy * h4_3_27;
    const double k4_8_13_3 = h4_8_27 + CDz * h4_8_13;
    const double k4_8_5_8 = k4_8_13_3 + CDy * k4_8_5_3;
    const double h11_3_28 = acc[644] + ABz * acc[241];
    const double h4_8_28 = h11_3_28 + ABy * h4_3_28;
    const double k4_8_15_3 = h4_8_28 + CDz * h4_8_15;
    const double k4_8_5_9 = k4_8_15_3 + CDz * k4_8_5_3;
    const double k4_8_12_1 = h4_8_22 + CDx * h4_8_12;
    const double h11_3_6 = acc[622] + ABz * acc[219];
    const double h4_8_6 = h11_3_6 + ABy * h4_3_6;
    const double k4_8_6_1 = h4_8_12 + CDx * h4_8_6;
    const double k4_8_6_4 = k4_8_12_1 + CDx * k4_8_6_1;
    const double k4_8_12_2 = h4_8_24 + CDy * h4_8_12;
    const double k4_8_6_2 = h4_8_15 + CDy * h4_8_6;
    const double k4_8_6_5 = k4_8_12_2 + CDx * k4_8_6_2;
    const double h11_3_14 = acc[630] + ABz * acc[227];
    const double h4_8_14 = h11_3_14 + ABy * h4_3_14;
    const double k4_8_6_3 = h4_8_14 + CDz * h4_8_6;
    const double k4_8_6_6 = k4_8_12_3 + CDx * k4_8_6_3;
    const double k4_8_15_2 = h4_8_27 + CDy * h4_8_15;
    const double k4_8_6_7 = k4_8_15_2 + CDy * k4_8_6_2;
    const double k4_8_6_8 = k4_8_15_3 + CDy * k4_8_6_3;
    const double h11_3_29 = acc[645] + ABz * acc[242];
    const double h4_8_29 = h11_3_29 + ABy * h4_3_29;
    const double k4_8_14_3 = h4_8_29 + CDz * h4_8_14;
    const double k4_8_6_9 = k4_8_14_3 + CDz * k4_8_6_3;
    const double k4_8_13_1 = h4_8_23 + CDx * h4_8_13;
    const double h11_3_7 = acc[623] + ABz * acc[220];
    const double h4_8_7 = h11_3_7 + ABy * h4_3_7;
    const double k4_8_7_1 = h4_8_13 + CDx * h4_8_7;
    const double k4_8_7_4 = k4_8_13_1 + CDx * k4_8_7_1;
    const double h11_3_16 = acc[632] + ABz * acc[229];
    const double h4_8_16 = h11_3_16 + ABy * h4_3_16;
    const double k4_8_7_2 = h4_8_16 + CDy * h4_8_7;
    const double k4_8_7_5 = k4_8_13_2 + CDx * k4_8_7_2;
    const double h11_3_17 = acc[633] + ABz * acc[230];
    const double h4_8_17 = h11_3_17 + ABy * h4_3_17;
    const double k4_8_7_3 = h4_8_17 + CDz * h4_8_7;
    const double k4_8_7_6 = k4_8_13_3 + CDx * k4_8_7_3;
    const double h11_3_30 = acc[646] + ABz * acc[243];
    const double h4_8_30 = h11_3_30 + ABy * h4_3_30;
    const double k4_8_16_2 = h4_8_30 + CDy * h4_8_16;
    const double k4_8_7_7 = k4_8_16_2 + CDy * k4_8_7_2;
    const double h11_3_31 = acc[647] + ABz * acc[244];
    const double h4_8_31 = h11_3_31 + ABy * h4_3_31;
    const double k4_8_16_3 = h4_8_31 + CDz * h4_8_16;
    const double k4_8_7_8 = k4_8_16_3 + CDy * k4_8_7_3;
    const double h11_3_32 = acc[648] + ABz * acc[245];
    const double h4_8_32 = h11_3_32 + ABy * h4_3_32;
    const double k4_8_17_3 = h4_8_32 + CDz * h4_8_17;
    const double k4_8_7_9 = k4_8_17_3 + CDz * k4_8_7_3;
    const double k4_8_15_1 = h4_8_24 + CDx * h4_8_15;
    const double h11_3_8 = acc[624] + ABz * acc[221];
    const double h4_8_8 = h11_3_8 + ABy * h4_3_8;
    const double k4_8_8_1 = h4_8_15 + CDx * h4_8_8;
    const double k4_8_8_4 = k4_8_15_1 + CDx * k4_8_8_1;
    const double k4_8_8_2 = h4_8_17 + CDy * h4_8_8;
    const double k4_8_8_5 = k4_8_15_2 + CDx * k4_8_8_2;
    const double h11_3_18 = acc[634] + ABz * acc[231];
    const double h4_8_18 = h11_3_18 + ABy * h4_3_18;
    const double k4_8_8_3 = h4_8_18 + CDz * h4_8_8;
    const double k4_8_8_6 = k4_8_15_3 + CDx * k4_8_8_3;
    const double k4_8_17_2 = h4_8_31 + CDy * h4_8_17;
    const double k4_8_8_7 = k4_8_17_2 + CDy * k4_8_8_2;
    const double k4_8_8_8 = k4_8_17_3 + CDy * k4_8_8_3;
    const double h11_3_33 = acc[649] + ABz * acc[246];
    const double h4_8_33 = h11_3_33 + ABy * h4_3_33;
    const double k4_8_18_3 = h4_8_33 + CDz * h4_8_18;
    const double k4_8_8_9 = k4_8_18_3 + CDz * k4_8_8_3;
    const double k4_8_14_1 = h4_8_25 + CDx * h4_8_14;
    const double h11_3_9 = acc[625] + ABz * acc[222];
    const double h4_8_9 = h11_3_9 + ABy * h4_3_9;
    const double k4_8_9_1 = h4_8_14 + CDx * h4_8_9;
    const double k4_8_9_4 = k4_8_14_1 + CDx * k4_8_9_1;
    const double k4_8_14_2 = h4_8_28 + CDy * h4_8_14;
    const double k4_8_9_2 = h4_8_18 + CDy * h4_8_9;
    const double k4_8_9_5 = k4_8_14_2 + CDx * k4_8_9_2;
    const double h11_3_19 = acc[635] + ABz * acc[232];
    const double h4_8_19 = h11_3_19 + ABy * h4_3_19;
    const double k4_8_9_3 = h4_8_19 + CDz * h4_8_9;
    const double k4_8_9_6 = k4_8_14_3 + CDx * k4_8_9_3;
    const double k4_8_18_2 = h4_8_32 + CDy * h4_8_18;
    const double k4_8_9_7 = k4_8_18_2 + CDy * k4_8_9_2;
    const double k4_8_9_8 = k4_8_18_3 + CDy * k4_8_9_3;
    const double h11_3_34 = acc[650] + ABz * acc[247];
    const double h4_8_34 = h11_3_34 + ABy * h4_3_34;
    const double k4_8_19_3 = h4_8_34 + CDz * h4_8_19;
    const double k4_8_9_9 = k4_8_19_3 + CDz * k4_8_9_3;
    const double h12_3_20 = acc[667] + ABz * acc[264];
    const double h4_9_20 = h12_3_20 + ABz * h4_3_20;
    const double h12_3_10 = acc[657] + ABz * acc[254];
    const double h4_9_10 = h12_3_10 + ABz * h4_3_10;
    const double k4_9_10_1 = h4_9_20 + CDx * h4_9_10;
    const double h12_3_4 = acc[651] + ABz * acc[248];
    const double h4_9_4 = h12_3_4 + ABz * h4_3_4;
    const double k4_9_4_1 = h4_9_10 + CDx * h4_9_4;
    const double k4_9_4_4 = k4_9_10_1 + CDx * k4_9_4_1;
    const double h12_3_21 = acc[668] + ABz * acc[265];
    const double h4_9_21 = h12_3_21 + ABz * h4_3_21;
    const double k4_9_10_2 = h4_9_21 + CDy * h4_9_10;
    const double h12_3_11 = acc[658] + ABz * acc[255];
    const double h4_9_11 = h12_3_11 + ABz * h4_3_11;
    const double k4_9_4_2 = h4_9_11 + CDy * h4_9_4;
    const double k4_9_4_5 = k4_9_10_2 + CDx * k4_9_4_2;
    const double h12_3_22 = acc[669] + ABz * acc[266];
    const double h4_9_22 = h12_3_22 + ABz * h4_3_22;
    const double k4_9_10_3 = h4_9_22 + CDz * h4_9_10;
    const double h12_3_12 = acc[659] + ABz * acc[256];
    const double h4_9_12 = h12_3_12 + ABz * h4_3_12;
    const double k4_9_4_3 = h4_9_12 + CDz * h4_9_4;
    const double k4_9_4_6 = k4_9_10_3 + CDx * k4_9_4_3;
    const double h12_3_23 = acc[670] + ABz * acc[267];
    const double h4_9_23 = h12_3_23 + ABz * h4_3_23;
    const double k4_9_11_2 = h4_9_23 + CDy * h4_9_11;
    const double k4_9_4_7 = k4_9_11_2 + CDy * k4_9_4_2;
    const double h12_3_24 = acc[671] + ABz * acc[268];
    const double h4_9_24 = h12_3_24 + ABz * h4_3_24;
    const double k4_9_11_3 = h4_9_24 + CDz * h4_9_11;
    const double k4_9_4_8 = k4_9_11_3 + CDy * k4_9_4_3;
    const double h12_3_25 = acc[672] + ABz * acc[269];
    const double h4_9_25 = h12_3_25 + ABz * h4_3_25;
    const double k4_9_12_3 = h4_9_25 + CDz * h4_9_12;
    const double k4_9_4_9 = k4_9_12_3 + CDz * k4_9_4_3;
    const double k4_9_11_1 = h4_9_21 + CDx * h4_9_11;
    const double h12_3_5 = acc[652] + ABz * acc[249];
    const double h4_9_5 = h12_3_5 + ABz * h4_3_5;
    const double k4_9_5_1 = h4_9_11 + CDx * h4_9_5;
    const double k4_9_5_4 = k4_9_11_1 + CDx * k4_9_5_1;
    const double h12_3_13 = acc[660] + ABz * acc[257];
    const double h4_9_13 = h12_3_13 + ABz * h4_3_13;
    const double k4_9_5_2 = h4_9_13 + CDy * h4_9_5;
    const double k4_9_5_5 = k4_9_11_2 + CDx * k4_9_5_2;
    const double h12_3_15 = acc[662] + ABz * acc[259];
    const double h4_9_15 = h12_3_15 + ABz * h4_3_15;
    const double k4_9_5_3 = h4_9_15 + CDz * h4_9_5;
    const double k4_9_5_6 = k4_9_11_3 + CDx * k4_9_5_3;
    const double h12_3_26 = acc[673] + ABz * acc[270];
    const double h4_9_26 = h12_3_26 + ABz * h4_3_26;
    const double k4_9_13_2 = h4_9_26 + CDy * h4_9_13;
    const double k4_9_5_7 = k4_9_13_2 + CDy * k4_9_5_2;
    const double h12_3_27 = acc[674] + ABz * acc[271];
    const double h4_9_27 = h12_3_27 + ABz * h4_3_27;
    const double k4_9_13_3 = h4_9_27 + CDz * h4_9_13;
    const double k4_9_5_8 = k4_9_13_3 + CDy * k4_9_5_3;
    const double h12_3_28 = acc[675] + ABz * acc[272];
    const double h4_9_28 = h12_3_28 + ABz * h4_3_28;
    const double k4_9_15_3 = h4_9_28 + CDz * h4_9_15;
    const double k4_9_5_9 = k4_9_15_3 + CDz * k4_9_5_3;
    const double k4_9_12_1 = h4_9_22 + CDx * h4_9_12;
    const double h12_3_6 = acc[653] + ABz * acc[250];
    const double h4_9_6 = h12_3_6 + ABz * h4_3_6;
    const double k4_9_6_1 = h4_9_12 + CDx * h4_9_6;
    const double k4_9_6_4 = k4_9_12_1 + CDx * k4_9_6_1;
    const double k4_9_12_2 = h4_9_24 + CDy * h4_9_12;
    const double k4_9_6_2 = h4_9_15 + CDy * h4_9_6;
    const double k4_9_6_5 = k4_9_12_2 + CDx * k4_9_6_2;
    const double h12_3_14 = acc[661] + ABz * acc[258];
    const double h4_9_14 = h12_3_14 + ABz * h4_3_14;
    const double k4_9_6_3 = h4_9_14 + CDz * h4_9_6;
    const double k4_9_6_6 = k4_9_12_3 + CDx * k4_9_6_3;
    const double k4_9_15_2 = h4_9_27 + CDy * h4_9_15;
    const double k4_9_6_7 = k4_9_15_2 + CDy * k4_9_6_2;
    const double k4_9_6_8 = k4_9_15_3 + CDy * k4_9_6_3;
    const double h12_3_29 = acc[676] + ABz * acc[273];
    const double h4_9_29 = h12_3_29 + ABz * h4_3_29;
    const double k4_9_14_3 = h4_9_29 + CDz * h4_9_14;
    const double k4_9_6_9 = k4_9_14_3 + CDz * k4_9_6_3;
    const double k4_9_13_1 = h4_9_23 + CDx * h4_9_13;
    const double h12_3_7 = acc[654] + ABz * acc[251];
    const double h4_9_7 = h12_3_7 + ABz * h4_3_7;
    const double k4_9_7_1 = h4_9_13 + CDx * h4_9_7;
    const double k4_9_7_4 = k4_9_13_1 + CDx * k4_9_7_1;
    const double h12_3_16 = acc[663] + ABz * acc[260];
    const double h4_9_16 = h12_3_16 + ABz * h4_3_16;
    const double k4_9_7_2 = h4_9_16 + CDy * h4_9_7;
    const double k4_9_7_5 = k4_9_13_2 + CDx * k4_9_7_2;
    const double h12_3_17 = acc[664] + ABz * acc[261];
    const double h4_9_17 = h12_3_17 + ABz * h4_3_17;
    const double k4_9_7_3 = h4_9_17 + CDz * h4_9_7;
    const double k4_9_7_6 = k4_9_13_3 + CDx * k4_9_7_3;
    const double h12_3_30 = acc[677] + ABz * acc[274];
    const double h4_9_30 = h12_3_30 + ABz * h4_3_30;
    const double k4_9_16_2 = h4_9_30 + CDy * h4_9_16;
    const double k4_9_7_7 = k4_9_16_2 + CDy * k4_9_7_2;
    const double h12_3_31 = acc[678] + ABz * acc[275];
    const double h4_9_31 = h12_3_31 + ABz * h4_3_31;
    const double k4_9_16_3 = h4_9_31 + CDz * h4_9_16;
    const double k4_9_7_8 = k4_9_16_3 + CDy * k4_9_7_3;
    const double h12_3_32 = acc[679] + ABz * acc[276];
    const double h4_9_32 = h12_3_32 + ABz * h4_3_32;
    const double k4_9_17_3 = h4_9_32 + CDz * h4_9_17;
    const double k4_9_7_9 = k4_9_17_3 + CDz * k4_9_7_3;
    const double k4_9_15_1 = h4_9_24 + CDx * h4_9_15;
    const double h12_3_8 = acc[655] + ABz * acc[252];
    const double h4_9_8 = h12_3_8 + ABz * h4_3_8;
    const double k4_9_8_1 = h4_9_15 + CDx * h4_9_8;
    const double k4_9_8_4 = k4_9_15_1 + CDx * k4_9_8_1;
    const double k4_9_8_2 = h4_9_17 + CDy * h4_9_8;
    const double k4_9_8_5 = k4_9_15_2 + CDx * k4_9_8_2;
    const double h12_3_18 = acc[665] + ABz * acc[262];
    const double h4_9_18 = h12_3_18 + ABz * h4_3_18;
    const double k4_9_8_3 = h4_9_18 + CDz * h4_9_8;
    const double k4_9_8_6 = k4_9_15_3 + CDx * k4_9_8_3;
    const double k4_9_17_2 = h4_9_31 + CDy * h4_9_17;
    const double k4_9_8_7 = k4_9_17_2 + CDy * k4_9_8_2;
    const double k4_9_8_8 = k4_9_17_3 + CDy * k4_9_8_3;
    const double h12_3_33 = acc[680] + ABz * acc[277];
    const double h4_9_33 = h12_3_33 + ABz * h4_3_33;
    const double k4_9_18_3 = h4_9_33 + CDz * h4_9_18;
    const double k4_9_8_9 = k4_9_18_3 + CDz * k4_9_8_3;
    const double k4_9_14_1 = h4_9_25 + CDx * h4_9_14;
    const double h12_3_9 = acc[656] + ABz * acc[253];
    const double h4_9_9 = h12_3_9 + ABz * h4_3_9;
    const double k4_9_9_1 = h4_9_14 + CDx * h4_9_9;
    const double k4_9_9_4 = k4_9_14_1 + CDx * k4_9_9_1;
    const double k4_9_14_2 = h4_9_28 + CDy * h4_9_14;
    const double k4_9_9_2 = h4_9_18 + CDy * h4_9_9;
    const double k4_9_9_5 = k4_9_14_2 + CDx * k4_9_9_2;
    const double h12_3_19 = acc[666] + ABz * acc[263];
    const double h4_9_19 = h12_3_19 + ABz * h4_3_19;
    const double k4_9_9_3 = h4_9_19 + CDz * h4_9_9;
    const double k4_9_9_6 = k4_9_14_3 + CDx * k4_9_9_3;
    const double k4_9_18_2 = h4_9_32 + CDy * h4_9_18;
    const double k4_9_9_7 = k4_9_18_2 + CDy * k4_9_9_2;
    const double k4_9_9_8 = k4_9_18_3 + CDy * k4_9_9_3;
    const double h12_3_34 = acc[681] + ABz * acc[278];
    const double h4_9_34 = h12_3_34 + ABz * h4_3_34;
    const double k4_9_19_3 = h4_9_34 + CDz * h4_9_19;
    const double k4_9_9_9 = k4_9_19_3 + CDz * k4_9_9_3;
    const double h11_1_20 = acc[543] + ABx * acc[233];
    const double h5_1_20 = acc[233] + ABx * acc[47];
    const double h5_4_20 = h11_1_20 + ABx * h5_1_20;
    const double h11_1_10 = acc[533] + ABx * acc[223];
    const double h5_1_10 = acc[223] + ABx * acc[37];
    const double h5_4_10 = h11_1_10 + ABx * h5_1_10;
    const double k5_4_10_1 = h5_4_20 + CDx * h5_4_10;
    const double h11_1_4 = acc[527] + ABx * acc[217];
    const double h5_1_4 = acc[217] + ABx * acc[31];
    const double h5_4_4 = h11_1_4 + ABx * h5_1_4;
    const double k5_4_4_1 = h5_4_10 + CDx * h5_4_4;
    const double k5_4_4_4 = k5_4_10_1 + CDx * k5_4_4_1;
    const double h11_1_21 = acc[544] + ABx * acc[234];
    const double h5_1_21 = acc[234] + ABx * acc[48];
    const double h5_4_21 = h11_1_21 + ABx * h5_1_21;
    const double k5_4_10_2 = h5_4_21 + CDy * h5_4_10;
    const double h11_1_11 = acc[534] + ABx * acc[224];
    const double h5_1_11 = acc[224] + ABx * acc[38];
    const double h5_4_11 = h11_1_11 + ABx * h5_1_11;
    const double k5_4_4_2 = h5_4_11 + CDy * h5_4_4;
    const double k5_4_4_5 = k5_4_10_2 + CDx * k5_4_4_2;
    const double h11_1_22 = acc[545] + ABx * acc[235];
    const double h5_1_22 = acc[235] + ABx * acc[49];
    const double h5_4_22 = h11_1_22 + ABx * h5_1_22;
    const double k5_4_10_3 = h5_4_22 + CDz * h5_4_10;
    const double h11_1_12 = acc[535] + ABx * acc[225];
    const double h5_1_12 = acc[225] + ABx * acc[39];
    const double h5_4_12 = h11_1_12 + ABx * h5_1_12;
    const double k5_4_4_3 = h5_4_12 + CDz * h5_4_4;
    const double k5_4_4_6 = k5_4_10_3 + CDx * k5_4_4_3;
    const double h11_1_23 = acc[546] + ABx * acc[236];
    const double h5_1_23 = acc[236] + ABx * acc[50];
    const double h5_4_23 = h11_1_23 + ABx * h5_1_23;
    const double k5_4_11_2 = h5_4_23 + CDy * h5_4_11;
    const double k5_4_4_7 = k5_4_11_2 + CDy * k5_4_4_2;
    const double h11_1_24 = acc[547] + ABx * acc[237];
    const double h5_1_24 = acc[237] + ABx * acc[51];
    const double h5_4_24 = h11_1_24 + ABx * h5_1_24;
    const double k5_4_11_3 = h5_4_24 + CDz * h5_4_11;
    const double k5_4_4_8 = k5_4_11_3 + CDy * k5_4_4_3;
    const double h11_1_25 = acc[548] + ABx * acc[238];
    const double h5_1_25 = acc[238] + ABx * acc[52];
    const double h5_4_25 = h11_1_25 + ABx * h5_1_25;
    const double k5_4_12_3 = h5_4_25 + CDz * h5_4_12;
    const double k5_4_4_9 = k5_4_12_3 + CDz * k5_4_4_3;
    const double k5_4_11_1 = h5_4_21 + CDx * h5_4_11;
    const double h11_1_5 = acc[528] + ABx * acc[218];
    const double h5_1_5 = acc[218] + ABx * acc[32];
    const double h5_4_5 = h11_1_5 + ABx * h5_1_5;
    const double k5_4_5_1 = h5_4_11 + CDx * h5_4_5;
    const double k5_4_5_4 = k5_4_11_1 + CDx * k5_4_5_1;
    const double h11_1_13 = acc[536] + ABx * acc[226];
    const double h5_1_13 = acc[226] + ABx * acc[40];
    const double h5_4_13 = h11_1_13 + ABx * h5_1_13;
    const double k5_4_5_2 = h5_4_13 + CDy * h5_4_5;
    const double k5_4_5_5 = k5_4_11_2 + CDx * k5_4_5_2;
    const double h11_1_15 = acc[538] + ABx * acc[228];
    const double h5_1_15 = acc[228] + ABx * acc[42];
    const double h5_4_15 = h11_1_15 + ABx * h5_1_15;
    const double k5_4_5_3 = h5_4_15 + CDz * h5_4_5;
    const double k5_4_5_6 = k5_4_11_3 + CDx * k5_4_5_3;
    const double h11_1_26 = acc[549] + ABx * acc[239];
    const double h5_1_26 = acc[239] + ABx * acc[53];
    const double h5_4_26 = h11_1_26 + ABx * h5_1_26;
    const double k5_4_13_2 = h5_4_26 + CDy * h5_4_13;
    const double k5_4_5_7 = k5_4_13_2 + CDy * k5_4_5_2;
    const double h11_1_27 = acc[550] + ABx * acc[240];
    const double h5_1_27 = acc[240] + ABx * acc[54];
    const double h5_4_27 = h11_1_27 + ABx * h5_1_27;
    const double k5_4_13_3 = h5_4_27 + CDz * h5_4_13;
    const double k5_4_5_8 = k5_4_13_3 + CDy * k5_4_5_3;
    const double h11_1_28 = acc[551] + ABx * acc[241];
    const double h5_1_28 = acc[241] + ABx * acc[55];
    const double h5_4_28 = h11_1_28 + ABx * h5_1_28;
    const double k5_4_15_3 = h5_4_28 + CDz * h5_4_15;
    const double k5_4_5_9 = k5_4_15_3 + CDz * k5_4_5_3;
    const double k5_4_12_1 = h5_4_22 + CDx * h5_4_12;
    const double h11_1_6 = acc[529] + ABx * acc[219];
    const double h5_1_6 = acc[219] + ABx * acc[33];
    const double h5_4_6 = h11_1_6 + ABx * h5_1_6;
    const double k5_4_6_1 = h5_4_12 + CDx * h5_4_6;
    const double k5_4_6_4 = k5_4_12_1 + CDx * k5_4_6_1;
    const double k5_4_12_2 = h5_4_24 + CDy * h5_4_12;
    const double k5_4_6_2 = h5_4_15 + CDy * h5_4_6;
    const double k5_4_6_5 = k5_4_12_2 + CDx * k5_4_6_2;
    const double h11_1_14 = acc[537] + ABx * acc[227];
    const double h5_1_14 = acc[227] + ABx * acc[41];
    const double h5_4_14 = h11_1_14 + ABx * h5_1_14;
    const double k5_4_6_3 = h5_4_14 + CDz * h5_4_6;
    const double k5_4_6_6 = k5_4_12_3 + CDx * k5_4_6_3;
    const double k5_4_15_2 = h5_4_27 + CDy * h5_4_15;
    const double k5_4_6_7 = k5_4_15_2 + CDy * k5_4_6_2;
    const double k5_4_6_8 = k5_4_15_3 + CDy * k5_4_6_3;
    const double h11_1_29 = acc[552] + ABx * acc[242];
    const double h5_1_29 = acc[242] + ABx * acc[56];
    const double h5_4_29 = h11_1_29 + ABx * h5_1_29;
    const double k5_4_14_3 = h5_4_29 + CDz * h5_4_14;
    const double k5_4_6_9 = k5_4_14_3 + CDz * k5_4_6_3;
    const double k5_4_13_1 = h5_4_23 + CDx * h5_4_13;
    const double h11_1_7 = acc[530] + ABx * acc[220];
    const double h5_1_7 = acc[220] + ABx * acc[34];
    const double h5_4_7 = h11_1_7 + ABx * h5_1_7;
    const double k5_4_7_1 = h5_4_13 + CDx * h5_4_7;
    const double k5_4_7_4 = k5_4_13_1 + CDx * k5_4_7_1;
    const double h11_1_16 = acc[539] + ABx * acc[229];
    const double h5_1_16 = acc[229] + ABx * acc[43];
    const double h5_4_16 = h11_1_16 + ABx * h5_1_16;
    const double k5_4_7_2 = h5_4_16 + CDy * h5_4_7;
    const double k5_4_7_5 = k5_4_13_2 + CDx * k5_4_7_2;
    const double h11_1_17 = acc[540] + ABx * acc[230];
    const double h5_1_17 = acc[230] + ABx * acc[44];
    const double h5_4_17 = h11_1_17 + ABx * h5_1_17;
    const double k5_4_7_3 = h5_4_17 + CDz * h5_4_7;
    const double k5_4_7_6 = k5_4_13_3 + CDx * k5_4_7_3;
    const double h11_1_30 = acc[553] + ABx * acc[243];
    const double h5_1_30 = acc[243] + ABx * acc[57];
    const double h5_4_30 = h11_1_30 + ABx * h5_1_30;
    const double k5_4_16_2 = h5_4_30 + CDy * h5_4_16;
    const double k5_4_7_7 = k5_4_16_2 + CDy * k5_4_7_2;
    const double h11_1_31 = acc[554] + ABx * acc[244];
    const double h5_1_31 = acc[244] + ABx * acc[58];
    const double h5_4_31 = h11_1_31 + ABx * h5_1_31;
    const double k5_4_16_3 = h5_4_31 + CDz * h5_4_16;
    const double k5_4_7_8 = k5_4_16_3 + CDy * k5_4_7_3;
    const double h11_1_32 = acc[555] + ABx * acc[245];
    const double h5_1_32 = acc[245] + ABx * acc[59];
    const double h5_4_32 = h11_1_32 + ABx * h5_1_32;
    const double k5_4_17_3 = h5_4_32 + CDz * h5_4_17;
    const double k5_4_7_9 = k5_4_17_3 + CDz * k5_4_7_3;
    const double k5_4_15_1 = h5_4_24 + CDx * h5_4_15;
    const double h11_1_8 = acc[531] + ABx * acc[221];
    const double h5_1_8 = acc[221] + ABx * acc[35];
    const double h5_4_8 = h11_1_8 + ABx * h5_1_8;
    const double k5_4_8_1 = h5_4_15 + CDx * h5_4_8;
    const double k5_4_8_4 = k5_4_15_1 + CDx * k5_4_8_1;
    const double k5_4_8_2 = h5_4_17 + CDy * h5_4_8;
    const double k5_4_8_5 = k5_4_15_2 + CDx * k5_4_8_2;
    const double h11_1_18 = acc[541] + ABx * acc[231];
    const double h5_1_18 = acc[231] + ABx * acc[45];
    const double h5_4_18 = h11_1_18 + ABx * h5_1_18;
    const double k5_4_8_3 = h5_4_18 + CDz * h5_4_8;
    const double k5_4_8_6 = k5_4_15_3 + CDx * k5_4_8_3;
    const double k5_4_17_2 = h5_4_31 + CDy * h5_4_17;
    const double k5_4_8_7 = k5_4_17_2 + CDy * k5_4_8_2;
    const double k5_4_8_8 = k5_4_17_3 + CDy * k5_4_8_3;
    const double h11_1_33 = acc[556] + ABx * acc[246];
    const double h5_1_33 = acc[246] + ABx * acc[60];
    const double h5_4_33 = h11_1_33 + ABx * h5_1_33;
    const double k5_4_18_3 = h5_4_33 + CDz * h5_4_18;
    const double k5_4_8_9 = k5_4_18_3 + CDz * k5_4_8_3;
    const double k5_4_14_1 = h5_4_25 + CDx * h5_4_14;
    const double h11_1_9 = acc[532] + ABx * acc[222];
    const double h5_1_9 = acc[222] + ABx * acc[36];
    const double h5_4_9 = h11_1_9 + ABx * h5_1_9;
    const double k5_4_9_1 = h5_4_14 + CDx * h5_4_9;
    const double k5_4_9_4 = k5_4_14_1 + CDx * k5_4_9_1;
    const double k5_4_14_2 = h5_4_28 + CDy * h5_4_14;
    const double k5_4_9_2 = h5_4_18 + CDy * h5_4_9;
    const double k5_4_9_5 = k5_4_14_2 + CDx * k5_4_9_2;
    const double h11_1_19 = acc[542] + ABx * acc[232];
    const double h5_1_19 = acc[232] + ABx * acc[46];
    const double h5_4_19 = h11_1_19 + ABx * h5_1_19;
    const double k5_4_9_3 = h5_4_19 + CDz * h5_4_9;
    const double k5_4_9_6 = k5_4_14_3 + CDx * k5_4_9_3;
    const double k5_4_18_2 = h5_4_32 + CDy * h5_4_18;
    const double k5_4_9_7 = k5_4_18_2 + CDy * k5_4_9_2;
    const double k5_4_9_8 = k5_4_18_3 + CDy * k5_4_9_3;
    const double h11_1_34 = acc[557] + ABx * acc[247];
    const double h5_1_34 = acc[247] + ABx * acc[61];
    const double h5_4_34 = h11_1_34 + ABx * h5_1_34;
    const double k5_4_19_3 = h5_4_34 + CDz * h5_4_19;
    const double k5_4_9_9 = k5_4_19_3 + CDz * k5_4_9_3;
    const double h5_2_20 = acc[295] + ABy * acc[47];
    const double h5_5_20 = h11_2_20 + ABx * h5_2_20;
    const double h5_2_10 = acc[285] + ABy * acc[37];
    const double h5_5_10 = h11_2_10 + ABx * h5_2_10;
    const double k5_5_10_1 = h5_5_20 + CDx * h5_5_10;
    const double h5_2_4 = acc[279] + ABy * acc[31];
    const double h5_5_4 = h11_2_4 + ABx * h5_2_4;
    const double k5_5_4_1 = h5_5_10 + CDx * h5_5_4;
    const double k5_5_4_4 = k5_5_10_1 + CDx * k5_5_4_1;
    const double h5_2_21 = acc[296] + ABy * acc[48];
    const double h5_5_21 = h11_2_21 + ABx * h5_2_21;
    const double k5_5_10_2 = h5_5_21 + CDy * h5_5_10;
    const double h5_2_11 = acc[286] + ABy * acc[38];
    const double h5_5_11 = h11_2_11 + ABx * h5_2_11;
    const double k5_5_4_2 = h5_5_11 + CDy * h5_5_4;
    const double k5_5_4_5 = k5_5_10_2 + CDx * k5_5_4_2;
    const double h5_2_22 = acc[297] + ABy * acc[49];
    const double h5_5_22 = h11_2_22 + ABx * h5_2_22;
    const double k5_5_10_3 = h5_5_22 + CDz * h5_5_10;
    const double h5_2_12 = acc[287] + ABy * acc[39];
    const double h5_5_12 = h11_2_12 + ABx * h5_2_12;
    const double k5_5_4_3 = h5_5_12 + CDz * h5_5_4;
    const double k5_5_4_6 = k5_5_10_3 + CDx * k5_5_4_3;
    const double h5_2_23 = acc[298] + ABy * acc[50];
    const double h5_5_23 = h11_2_23 + ABx * h5_2_23;
    const double k5_5_11_2 = h5_5_23 + CDy * h5_5_11;
    const double k5_5_4_7 = k5_5_11_2 + CDy * k5_5_4_2;
    const double h5_2_24 = acc[299] + ABy * acc[51];
    const double h5_5_24 = h11_2_24 + ABx * h5_2_24;
    const double k5_5_11_3 = h5_5_24 + CDz * h5_5_11;
    const double k5_5_4_8 = k5_5_11_3 + CDy * k5_5_4_3;
    const double h5_2_25 = acc[300] + ABy * acc[52];
    const double h5_5_25 = h11_2_25 + ABx * h5_2_25;
    const double k5_5_12_3 = h5_5_25 + CDz * h5_5_12;
    const double k5_5_4_9 = k5_5_12_3 + CDz * k5_5_4_3;
    const double k5_5_11_1 = h5_5_21 + CDx * h5_5_11;
    const double h5_2_5 = acc[280] + ABy * acc[32];
    const double h5_5_5 = h11_2_5 + ABx * h5_2_5;
    const double k5_5_5_1 = h5_5_11 + CDx * h5_5_5;
    const double k5_5_5_4 = k5_5_11_1 + CDx * k5_5_5_1;
    const double h5_2_13 = acc[288] + ABy * acc[40];
    const double h5_5_13 = h11_2_13 + ABx * h5_2_13;
    const double k5_5_5_2 = h5_5_13 + CDy * h5_5_5;
    const double k5_5_5_5 = k5_5_11_2 + CDx * k5_5_5_2;
    const double h5_2_15 = acc[290] + ABy * acc[42];
    const double h5_5_15 = h11_2_15 + ABx * h5_2_15;
    const double k5_5_5_3 = h5_5_15 + CDz * h5_5_5;
    const double k5_5_5_6 = k5_5_11_3 + CDx * k5_5_5_3;
    const double h5_2_26 = acc[301] + ABy * acc[53];
    const double h5_5_26 = h11_2_26 + ABx * h5_2_26;
    const double k5_5_13_2 = h5_5_26 + CDy * h5_5_13;
    const double k5_5_5_7 = k5_5_13_2 + CDy * k5_5_5_2;
    const double h5_2_27 = acc[302] + ABy * acc[54];
    const double h5_5_27 = h11_2_27 + ABx * h5_2_27;
    const double k5_5_13_3 = h5_5_27 + CDz * h5_5_13;
    const double k5_5_5_8 = k5_5_13_3 + CDy * k5_5_5_3;
    const double h5_2_28 = acc[303] + ABy * acc[55];
    const double h5_5_28 = h11_2_28 + ABx * h5_2_28;
    const double k5_5_15_3 = h5_5_28 + CDz * h5_5_15;
    const double k5_5_5_9 = k5_5_15_3 + CDz * k5_5_5_3;
    const double k5_5_12_1 = h5_5_22 + CDx * h5_5_12;
    const double h5_2_6 = acc[281] + ABy * acc[33];
    const double h5_5_6 = h11_2_6 + ABx * h5_2_6;
    const double k5_5_6_1 = h5_5_12 + CDx * h5_5_6;
    const double k5_5_6_4 = k5_5_12_1 + CDx * k5_5_6_1;
    const double k5_5_12_2 = h5_5_24 + CDy * h5_5_12;
    const double k5_5_6_2 = h5_5_15 + CDy * h5_5_6;
    const double k5_5_6_5 = k5_5_12_2 + CDx * k5_5_6_2;
    const double h5_2_14 = acc[289] + ABy * acc[41];
    const double h5_5_14 = h11_2_14 + ABx * h5_2_14;
    const double k5_5_6_3 = h5_5_14 + CDz * h5_5_6;
    const double k5_5_6_6 = k5_5_12_3 + CDx * k5_5_6_3;
    const double k5_5_15_2 = h5_5_27 + CDy * h5_5_15;
    const double k5_5_6_7 = k5_5_15_2 + CDy * k5_5_6_2;
    const double k5_5_6_8 = k5_5_15_3 + CDy * k5_5_6_3;
    const double h5_2_29 = acc[304] + ABy * acc[56];
    const double h5_5_29 = h11_2_29 + ABx * h5_2_29;
    const double k5_5_14_3 = h5_5_29 + CDz * h5_5_14;
    const double k5_5_6_9 = k5_5_14_3 + CDz * k5_5_6_3;
    const double k5_5_13_1 = h5_5_23 + CDx * h5_5_13;
    const double h5_2_7 = acc[282] + ABy * acc[34];
    const double h5_5_7 = h11_2_7 + ABx * h5_2_7;
    const double k5_5_7_1 = h5_5_13 + CDx * h5_5_7;
    const double k5_5_7_4 = k5_5_13_1 + CDx * k5_5_7_1;
    const double h5_2_16 = acc[291] + ABy * acc[43];
    const double h5_5_16 = h11_2_16 + ABx * h5_2_16;
    const double k5_5_7_2 = h5_5_16 + CDy * h5_5_7;
    const double k5_5_7_5 = k5_5_13_2 + CDx * k5_5_7_2;
    const double h5_2_17 = acc[292] + ABy * acc[44];
    const double h5_5_17 = h11_2_17 + ABx * h5_2_17;
    const double k5_5_7_3 = h5_5_17 + CDz * h5_5_7;
    const double k5_5_7_6 = k5_5_13_3 + CDx * k5_5_7_3;
    const double h5_2_30 = acc[305] + ABy * acc[57];
    const double h5_5_30 = h11_2_30 + ABx * h5_2_30;
    const double k5_5_16_2 = h5_5_30 + CDy * h5_5_16;
    const double k5_5_7_7 = k5_5_16_2 + CDy * k5_5_7_2;
    const double h5_2_31 = acc[306] + ABy * acc[58];
    const double h5_5_31 = h11_2_31 + ABx * h5_2_31;
    const double k5_5_16_3 = h5_5_31 + CDz * h5_5_16;
    const double k5_5_7_8 = k5_5_16_3 + CDy * k5_5_7_3;
    const double h5_2_32 = acc[307] + ABy * acc[59];
    const double h5_5_32 = h11_2_32 + ABx * h5_2_32;
    const double k5_5_17_3 = h5_5_32 + CDz * h5_5_17;
    const double k5_5_7_9 = k5_5_17_3 + CDz * k5_5_7_3;
    const double k5_5_15_1 = h5_5_24 + CDx * h5_5_15;
    const double h5_2_8 = acc[283] + ABy * acc[35];
    const double h5_5_8 = h11_2_8 + ABx * h5_2_8;
    const double k5_5_8_1 = h5_5_15 + CDx * h5_5_8;
    const double k5_5_8_4 = k5_5_15_1 + CDx * k5_5_8_1;
    const double k5_5_8_2 = h5_5_17 + CDy * h5_5_8;
    const double k5_5_8_5 = k5_5_15_2 + CDx * k5_5_8_2;
    const double h5_2_18 = acc[293] + ABy * acc[45];
    const double h5_5_18 = h11_2_18 + ABx * h5_2_18;
    const double k5_5_8_3 = h5_5_18 + CDz * h5_5_8;
    const double k5_5_8_6 = k5_5_15_3 + CDx * k5_5_8_3;
    const double k5_5_17_2 = h5_5_31 + CDy * h5_5_17;
    const double k5_5_8_7 = k5_5_17_2 + CDy * k5_5_8_2;
    const double k5_5_8_8 = k5_5_17_3 + CDy * k5_5_8_3;
    const double h5_2_33 = acc[308] + ABy * acc[60];
    const double h5_5_33 = h11_2_33 + ABx * h5_2_33;
    const double k5_5_18_3 = h5_5_33 + CDz * h5_5_18;
    const double k5_5_8_9 = k5_5_18_3 + CDz * k5_5_8_3;
    const double k5_5_14_1 = h5_5_25 + CDx * h5_5_14;
    const double h5_2_9 = acc[284] + ABy * acc[36];
    const double h5_5_9 = h11_2_9 + ABx * h5_2_9;
    const double k5_5_9_1 = h5_5_14 + CDx * h5_5_9;
    const double k5_5_9_4 = k5_5_14_1 + CDx * k5_5_9_1;
    const double k5_5_14_2 = h5_5_28 + CDy * h5_5_14;
    const double k5_5_9_2 = h5_5_18 + CDy * h5_5_9;
    const double k5_5_9_5 = k5_5_14_2 + CDx * k5_5_9_2;
    const double h5_2_19 = acc[294] + ABy * acc[46];
    const double h5_5_19 = h11_2_19 + ABx * h5_2_19;
    const double k5_5_9_3 = h5_5_19 + CDz * h5_5_9;
    const double k5_5_9_6 = k5_5_14_3 + CDx * k5_5_9_3;
    const double k5_5_18_2 = h5_5_32 + CDy * h5_5_18;
    const double k5_5_9_7 = k5_5_18_2 + CDy * k5_5_9_2;
    const double k5_5_9_8 = k5_5_18_3 + CDy * k5_5_9_3;
    const double h5_2_34 = acc[309] + ABy * acc[61];
    const double h5_5_34 = h11_2_34 + ABx * h5_2_34;
    const double k5_5_19_3 = h5_5_34 + CDz * h5_5_19;
    const double k5_5_9_9 = k5_5_19_3 + CDz * k5_5_9_3;
    const double h5_3_20 = acc[357] + ABz * acc[47];
    const double h5_6_20 = h11_3_20 + ABx * h5_3_20;
    const double h5_3_10 = acc[347] + ABz * acc[37];
    const double h5_6_10 = h11_3_10 + ABx * h5_3_10;
    const double k5_6_10_1 = h5_6_20 + CDx * h5_6_10;
    const double h5_3_4 = acc[341] + ABz * acc[31];
    const double h5_6_4 = h11_3_4 + ABx * h5_3_4;
    const double k5_6_4_1 = h5_6_10 + CDx * h5_6_4;
    const double k5_6_4_4 = k5_6_10_1 + CDx * k5_6_4_1;
    const double h5_3_21 = acc[358] + ABz * acc[48];
    const double h5_6_21 = h11_3_21 + ABx * h5_3_21;
    const double k5_6_10_2 = h5_6_21 + CDy * h5_6_10;
    const double h5_3_11 = acc[348] + ABz * acc[38];
    const double h5_6_11 = h11_3_11 + ABx * h5_3_11;
    const double k5_6_4_2 = h5_6_11 + CDy * h5_6_4;
    const double k5_6_4_5 = k5_6_10_2 + CDx * k5_6_4_2;
    const double h5_3_22 = acc[359] + ABz * acc[49];
    const double h5_6_22 = h11_3_22 + ABx * h5_3_22;
    const double k5_6_10_3 = h5_6_22 + CDz * h5_6_10;
    const double h5_3_12 = acc[349] + ABz * acc[39];
    const double h5_6_12 = h11_3_12 + ABx * h5_3_12;
    const double k5_6_4_3 = h5_6_12 + CDz * h5_6_4;
    const double k5_6_4_6 = k5_6_10_3 + CDx * k5_6_4_3;
    const double h5_3_23 = acc[360] + ABz * acc[50];
    const double h5_6_23 = h11_3_23 + ABx * h5_3_23;
    const double k5_6_11_2 = h5_6_23 + CDy * h5_6_11;
    const double k5_6_4_7 = k5_6_11_2 + CDy * k5_6_4_2;
    const double h5_3_24 = acc[361] + ABz * acc[51];
    const double h5_6_24 = h11_3_24 + ABx * h5_3_24;
    const double k5_6_11_3 = h5_6_24 + CDz * h5_6_11;
    const double k5_6_4_8 = k5_6_11_3 + CDy * k5_6_4_3;
    const double h5_3_25 = acc[362] + ABz * acc[52];
    const double h5_6_25 = h11_3_25 + ABx * h5_3_25;
    const double k5_6_12_3 = h5_6_25 + CDz * h5_6_12;
    const double k5_6_4_9 = k5_6_12_3 + CDz * k5_6_4_3;
    const double k5_6_11_1 = h5_6_21 + CDx * h5_6_11;
    const double h5_3_5 = acc[342] + ABz * acc[32];
    const double h5_6_5 = h11_3_5 + ABx * h5_3_5;
    const double k5_6_5_1 = h5_6_11 + CDx * h5_6_5;
    const double k5_6_5_4 = k5_6_11_1 + CDx * k5_6_5_1;
    const double h5_3_13 = acc[350] + ABz * acc[40];
    const double h5_6_13 = h11_3_13 + ABx * h5_3_13;
    const double k5_6_5_2 = h5_6_13 + CDy * h5_6_5;
    const double k5_6_5_5 = k5_6_11_2 + CDx * k5_6_5_2;
    const double h5_3_15 = acc[352] + ABz * acc[42];
    const double h5_6_15 = h11_3_15 + ABx * h5_3_15;
    const double k5_6_5_3 = h5_6_15 + CDz * h5_6_5;
    const double k5_6_5_6 = k5_6_11_3 + CDx * k5_6_5_3;
    const double h5_3_26 = acc[363] + ABz * acc[53];
    const double h5_6_26 = h11_3_26 + ABx * h5_3_26;
    const double k5_6_13_2 = h5_6_26 + CDy * h5_6_13;
    const double k5_6_5_7 = k5_6_13_2 + CDy * k5_6_5_2;
    const double h5_3_27 = acc[364] + ABz * acc[54];
    const double h5_6_27 = h11_3_27 + ABx * h5_3_27;
    const double k5_6_13_3 = h5_6_27 + CDz * h5_6_13;
    const double k5_6_5_8 = k5_6_13_3 + CDy * k5_6_5_3;
    const double h5_3_28 = acc[365] + ABz * acc[55];
    const double h5_6_28 = h11_3_28 + ABx * h5_3_28;
    const double k5_6_15_3 = h5_6_28 + CDz * h5_6_15;
    const double k5_6_5_9 = k5_6_15_3 + CDz * k5_6_5_3;
    const double k5_6_12_1 = h5_6_22 + CDx * h5_6_12;
    const double h5_3_6 = acc[343] + ABz * acc[33];
    const double h5_6_6 = h11_3_6 + ABx * h5_3_6;
    const double k5_6_6_1 = h5_6_12 + CDx * h5_6_6;
    const double k5_6_6_4 = k5_6_12_1 + CDx * k5_6_6_1;
    const double k5_6_12_2 = h5_6_24 + CDy * h5_6_12;
    const double k5_6_6_2 = h5_6_15 + CDy * h5_6_6;
    const double k5_6_6_5 = k5_6_12_2 + CDx * k5_6_6_2;
    const double h5_3_14 = acc[351] + ABz * acc[41];
    const double h5_6_14 = h11_3_14 + ABx * h5_3_14;
    const double k5_6_6_3 = h5_6_14 + CDz * h5_6_6;
    const double k5_6_6_6 = k5_6_12_3 + CDx * k5_6_6_3;
    const double k5_6_15_2 = h5_6_27 + CDy * h5_6_15;
    const double k5_6_6_7 = k5_6_15_2 + CDy * k5_6_6_2;
    const double k5_6_6_8 = k5_6_15_3 + CDy * k5_6_6_3;
    const double h5_3_29 = acc[366] + ABz * acc[56];
    const double h5_6_29 = h11_3_29 + ABx * h5_3_29;
    const double k5_6_14_3 = h5_6_29 + CDz * h5_6_14;
    const double k5_6_6_9 = k5_6_14_3 + CDz * k5_6_6_3;
    const double k5_6_13_1 = h5_6_23 + CDx * h5_6_13;
    const double h5_3_7 = acc[344] + ABz * acc[34];
    const double h5_6_7 = h11_3_7 + ABx * h5_3_7;
    const double k5_6_7_1 = h5_6_13 + CDx * h5_6_7;
    const double k5_6_7_4 = k5_6_13_1 + CDx * k5_6_7_1;
    const double h5_3_16 = acc[353] + ABz * acc[43];
    const double h5_6_16 = h11_3_16 + ABx * h5_3_16;
    const double k5_6_7_2 = h5_6_16 + CDy * h5_6_7;
    const double k5_6_7_5 = k5_6_13_2 + CDx * k5_6_7_2;
    const double h5_3_17 = acc[354] + ABz * acc[44];
    const double h5_6_17 = h11_3_17 + ABx * h5_3_17;
    const double k5_6_7_3 = h5_6_17 + CDz * h5_6_7;
    const double k5_6_7_6 = k5_6_13_3 + CDx * k5_6_7_3;
    const double h5_3_30 = acc[367] + ABz * acc[57];
    const double h5_6_30 = h11_3_30 + ABx * h5_3_30;
    const double k5_6_16_2 = h5_6_30 + CDy * h5_6_16;
    const double k5_6_7_7 = k5_6_16_2 + CDy * k5_6_7_2;
    const double h5_3_31 = acc[368] + ABz * acc[58];
    const double h5_6_31 = h11_3_31 + ABx * h5_3_31;
    const double k5_6_16_3 = h5_6_31 + CDz * h5_6_16;
    const double k5_6_7_8 = k5_6_16_3 + CDy * k5_6_7_3;
    const double h5_3_32 = acc[369] + ABz * acc[59];
    const double h5_6_32 = h11_3_32 + ABx * h5_3_32;
    const double k5_6_17_3 = h5_6_32 + CDz * h5_6_17;
    const double k5_6_7_9 = k5_6_17_3 + CDz * k5_6_7_3;
    const double k5_6_15_1 = h5_6_24 + CDx * h5_6_15;
    const double h5_3_8 = acc[345] + ABz * acc[35];
    const double h5_6_8 = h11_3_8 + ABx * h5_3_8;
    const double k5_6_8_1 = h5_6_15 + CDx * h5_6_8;
    const double k5_6_8_4 = k5_6_15_1 + CDx * k5_6_8_1;
    const double k5_6_8_2 = h5_6_17 + CDy * h5_6_8;
    const double k5_6_8_5 = k5_6_15_2 + CDx * k5_6_8_2;
    const double h5_3_18 = acc[355] + ABz * acc[45];
    const double h5_6_18 = h11_3_18 + ABx * h5_3_18;
    const double k5_6_8_3 = h5_6_18 + CDz * h5_6_8;
    const double k5_6_8_6 = k5_6_15_3 + CDx * k5_6_8_3;
    const double k5_6_17_2 = h5_6_31 + CDy * h5_6_17;
    const double k5_6_8_7 = k5_6_17_2 + CDy * k5_6_8_2;
    const double k5_6_8_8 = k5_6_17_3 + CDy * k5_6_8_3;
    const double h5_3_33 = acc[370] + ABz * acc[60];
    const double h5_6_33 = h11_3_33 + ABx * h5_3_33;
    const double k5_6_18_3 = h5_6_33 + CDz * h5_6_18;
    const double k5_6_8_9 = k5_6_18_3 + CDz * k5_6_8_3;
    const double k5_6_14_1 = h5_6_25 + CDx * h5_6_14;
    const double h5_3_9 = acc[346] + ABz * acc[36];
    const double h5_6_9 = h11_3_9 + ABx * h5_3_9;
    const double k5_6_9_1 = h5_6_14 + CDx * h5_6_9;
    const double k5_6_9_4 = k5_6_14_1 + CDx * k5_6_9_1;
    const double k5_6_14_2 = h5_6_28 + CDy * h5_6_14;
    const double k5_6_9_2 = h5_6_18 + CDy * h5_6_9;
    const double k5_6_9_5 = k5_6_14_2 + CDx * k5_6_9_2;
    const double h5_3_19 = acc[356] + ABz * acc[46];
    const double h5_6_19 = h11_3_19 + ABx * h5_3_19;
    const double k5_6_9_3 = h5_6_19 + CDz * h5_6_9;
    const double k5_6_9_6 = k5_6_14_3 + CDx * k5_6_9_3;
    const double k5_6_18_2 = h5_6_32 + CDy * h5_6_18;
    const double k5_6_9_7 = k5_6_18_2 + CDy * k5_6_9_2;
    const double k5_6_9_8 = k5_6_18_3 + CDy * k5_6_9_3;
    const double h5_3_34 = acc[371] + ABz * acc[61];
    const double h5_6_34 = h11_3_34 + ABx * h5_3_34;
    const double k5_6_19_3 = h5_6_34 + CDz * h5_6_19;
    const double k5_6_9_9 = k5_6_19_3 + CDz * k5_6_9_3;
    const double h13_2_20 = acc[698] + ABy * acc[295];
    const double h5_7_20 = h13_2_20 + ABy * h5_2_20;
    const double h13_2_10 = acc[688] + ABy * acc[285];
    const double h5_7_10 = h13_2_10 + ABy * h5_2_10;
    const double k5_7_10_1 = h5_7_20 + CDx * h5_7_10;
    const double h13_2_4 = acc[682] + ABy * acc[279];
    const double h5_7_4 = h13_2_4 + ABy * h5_2_4;
    const double k5_7_4_1 = h5_7_10 + CDx * h5_7_4;
    const double k5_7_4_4 = k5_7_10_1 + CDx * k5_7_4_1;
    const double h13_2_21 = acc[699] + ABy * acc[296];
    const double h5_7_21 = h13_2_21 + ABy * h5_2_21;
    const double k5_7_10_2 = h5_7_21 + CDy * h5_7_10;
    const double h13_2_11 = acc[689] + ABy * acc[286];
    const double h5_7_11 = h13_2_11 + ABy * h5_2_11;
    const double k5_7_4_2 = h5_7_11 + CDy * h5_7_4;
    const double k5_7_4_5 = k5_7_10_2 + CDx * k5_7_4_2;
    const double h13_2_22 = acc[700] + ABy * acc[297];
    const double h5_7_22 = h13_2_22 + ABy * h5_2_22;
    const double k5_7_10_3 = h5_7_22 + CDz * h5_7_10;
    const double h13_2_12 = acc[690] + ABy * acc[287];
    const double h5_7_12 = h13_2_12 + ABy * h5_2_12;
    const double k5_7_4_3 = h5_7_12 + CDz * h5_7_4;
    const double k5_7_4_6 = k5_7_10_3 + CDx * k5_7_4_3;
    const double h13_2_23 = acc[701] + ABy * acc[298];
    const double h5_7_23 = h13_2_23 + ABy * h5_2_23;
    const double k5_7_11_2 = h5_7_23 + CDy * h5_7_11;
    const double k5_7_4_7 = k5_7_11_2 + CDy * k5_7_4_2;
    const double h13_2_24 = acc[702] + ABy * acc[299];
    const double h5_7_24 = h13_2_24 + ABy * h5_2_24;
    const double k5_7_11_3 = h5_7_24 + CDz * h5_7_11;
    const double k5_7_4_8 = k5_7_11_3 + CDy * k5_7_4_3;
    const double h13_2_25 = acc[703] + ABy * acc[300];
    const double h5_7_25 = h13_2_25 + ABy * h5_2_25;
    const double k5_7_12_3 = h5_7_25 + CDz * h5_7_12;
    const double k5_7_4_9 = k5_7_12_3 + CDz * k5_7_4_3;
    const double k5_7_11_1 = h5_7_21 + CDx * h5_7_11;
    const double h13_2_5 = acc[683] + ABy * acc[280];
    const double h5_7_5 = h13_2_5 + ABy * h5_2_5;
    const double k5_7_5_1 = h5_7_11 + CDx * h5_7_5;
    const double k5_7_5_4 = k5_7_11_1 + CDx * k5_7_5_1;
    const double h13_2_13 = acc[691] + ABy * acc[288];
    const double h5_7_13 = h13_2_13 + ABy * h5_2_13;
    const double k5_7_5_2 = h5_7_13 + CDy * h5_7_5;
    const double k5_7_5_5 = k5_7_11_2 + CDx * k5_7_5_2;
    const double h13_2_15 = acc[693] + ABy * acc[290];
    const double h5_7_15 = h13_2_15 + ABy * h5_2_15;
    const double k5_7_5_3 = h5_7_15 + CDz * h5_7_5;
    const double k5_7_5_6 = k5_7_11_3 + CDx * k5_7_5_3;
    const double h13_2_26 = acc[704] + ABy * acc[301];
    const double h5_7_26 = h13_2_26 + ABy * h5_2_26;
    const double k5_7_13_2 = h5_7_26 + CDy * h5_7_13;
    const double k5_7_5_7 = k5_7_13_2 + CDy * k5_7_5_2;
    const double h13_2_27 = acc[705] + ABy * acc[302];
    const double h5_7_27 = h13_2_27 + ABy * h5_2_27;
    const double k5_7_13_3 = h5_7_27 + CDz * h5_7_13;
    const double k5_7_5_8 = k5_7_13_3 + CDy * k5_7_5_3;
    const double h13_2_28 = acc[706] + ABy * acc[303];
    const double h5_7_28 = h13_2_28 + ABy * h5_2_28;
    const double k5_7_15_3 = h5_7_28 + CDz * h5_7_15;
    const double k5_7_5_9 = k5_7_15_3 + CDz * k5_7_5_3;
    const double k5_7_12_1 = h5_7_22 + CDx * h5_7_12;
    const double h13_2_6 = acc[684] + ABy * acc[281];
    const double h5_7_6 = h13_2_6 + ABy * h5_2_6;
    const double k5_7_6_1 = h5_7_12 + CDx * h5_7_6;
    const double k5_7_6_4 = k5_7_12_1 + CDx * k5_7_6_1;
    const double k5_7_12_2 = h5_7_24 + CDy * h5_7_12;
    const double k5_7_6_2 = h5_7_15 + CDy * h5_7_6;
    const double k5_7_6_5 = k5_7_12_2 + CDx * k5_7_6_2;
    const double h13_2_14 = acc[692] + ABy * acc[289];
    const double h5_7_14 = h13_2_14 + ABy * h5_2_14;
    const double k5_7_6_3 = h5_7_14 + CDz * h5_7_6;
    const double k5_7_6_6 = k5_7_12_3 + CDx * k5_7_6_3;
    const double k5_7_15_2 = h5_7_27 + CDy * h5_7_15;
    const double k5_7_6_7 = k5_7_15_2 + CDy * k5_7_6_2;
    const double k5_7_6_8 = k5_7_15_3 + CDy * k5_7_6_3;
    const double h13_2_29 = acc[707] + ABy * acc[304];
    const double h5_7_29 = h13_2_29 + ABy * h5_2_29;
    const double k5_7_14_3 = h5_7_29 + CDz * h5_7_14;
    const double k5_7_6_9 = k5_7_14_3 + CDz * k5_7_6_3;
    const double k5_7_13_1 = h5_7_23 + CDx * h5_7_13;
    const double h13_2_7 = acc[685] + ABy * acc[282];
    const double h5_7_7 = h13_2_7 + ABy * h5_2_7;
    const double k5_7_7_1 = h5_7_13 + CDx * h5_7_7;
    const double k5_7_7_4 = k5_7_13_1 + CDx * k5_7_7_1;
    const double h13_2_16 = acc[694] + ABy * acc[291];
    const double h5_7_16 = h13_2_16 + ABy * h5_2_16;
    const double k5_7_7_2 = h5_7_16 + CDy * h5_7_7;
    const double k5_7_7_5 = k5_7_13_2 + CDx * k5_7_7_2;
    const double h13_2_17 = acc[695] + ABy * acc[292];
    const double h5_7_17 = h13_2_17 + ABy * h5_2_17;
    const double k5_7_7_3 = h5_7_17 + CDz * h5_7_7;
    const double k5_7_7_6 = k5_7_13_3 + CDx * k5_7_7_3;
    const double h13_2_30 = acc[708] + ABy * acc[305];
    const double h5_7_30 = h13_2_30 + ABy * h5_2_30;
    const double k5_7_16_2 = h5_7_30 + CDy * h5_7_16;
    const double k5_7_7_7 = k5_7_16_2 + CDy * k5_7_7_2;
    const double h13_2_31 = acc[709] + ABy * acc[306];
    const double h5_7_31 = h13_2_31 + ABy * h5_2_31;
    const double k5_7_16_3 = h5_7_31 + CDz * h5_7_16;
    const double k5_7_7_8 = k5_7_16_3 + CDy * k5_7_7_3;
    const double h13_2_32 = acc[710] + ABy * acc[307];
    const double h5_7_32 = h13_2_32 + ABy * h5_2_32;
    const double k5_7_17_3 = h5_7_32 + CDz * h5_7_17;
    const double k5_7_7_9 = k5_7_17_3 + CDz * k5_7_7_3;
    const double k5_7_15_1 = h5_7_24 + CDx * h5_7_15;
    const double h13_2_8 = acc[686] + ABy * acc[283];
    const double h5_7_8 = h13_2_8 + ABy * h5_2_8;
    const double k5_7_8_1 = h5_7_15 + CDx * h5_7_8;
    const double k5_7_8_4 = k5_7_15_1 + CDx * k5_7_8_1;
    const double k5_7_8_2 = h5_7_17 + CDy * h5_7_8;
    const double k5_7_8_5 = k5_7_15_2 + CDx * k5_7_8_2;
    const double h13_2_18 = acc[696] + ABy * acc[293];
    const double h5_7_18 = h13_2_18 + ABy * h5_2_18;
    const double k5_7_8_3 = h5_7_18 + CDz * h5_7_8;
    const double k5_7_8_6 = k5_7_15_3 + CDx * k5_7_8_3;
    const double k5_7_17_2 = h5_7_31 + CDy * h5_7_17;
    const double k5_7_8_7 = k5_7_17_2 + CDy * k5_7_8_2;
    const double k5_7_8_8 = k5_7_17_3 + CDy * k5_7_8_3;
    const double h13_2_33 = acc[711] + ABy * acc[308];
    const double h5_7_33 = h13_2_33 + ABy * h5_2_33;
    const double k5_7_18_3 = h5_7_33 + CDz * h5_7_18;
    const double k5_7_8_9 = k5_7_18_3 + CDz * k5_7_8_3;
    const double k5_7_14_1 = h5_7_25 + CDx * h5_7_14;
    const double h13_2_9 = acc[687] + ABy * acc[284];
    const double h5_7_9 = h13_2_9 + ABy * h5_2_9;
    const double k5_7_9_1 = h5_7_14 + CDx * h5_7_9;
    const double k5_7_9_4 = k5_7_14_1 + CDx * k5_7_9_1;
    const double k5_7_14_2 = h5_7_28 + CDy * h5_7_14;
    const double k5_7_9_2 = h5_7_18 + CDy * h5_7_9;
    const double k5_7_9_5 = k5_7_14_2 + CDx * k5_7_9_2;
    const double h13_2_19 = acc[697] + ABy * acc[294];
    const double h5_7_19 = h13_2_19 + ABy * h5_2_19;
    const double k5_7_9_3 = h5_7_19 + CDz * h5_7_9;
    const double k5_7_9_6 = k5_7_14_3 + CDx * k5_7_9_3;
    const double k5_7_18_2 = h5_7_32 + CDy * h5_7_18;
    const double k5_7_9_7 = k5_7_18_2 + CDy * k5_7_9_2;
    const double k5_7_9_8 = k5_7_18_3 + CDy * k5_7_9_3;
    const double h13_2_34 = acc[712] + ABy * acc[309];
    const double h5_7_34 = h13_2_34 + ABy * h5_2_34;
    const double k5_7_19_3 = h5_7_34 + CDz * h5_7_19;
    const double k5_7_9_9 = k5_7_19_3 + CDz * k5_7_9_3;
    const double h13_3_20 = acc[729] + ABz * acc[295];
    const double h5_8_20 = h13_3_20 + ABy * h5_3_20;
    const double h13_3_10 = acc[719] + ABz * acc[285];
    const double h5_8_10 = h13_3_10 + ABy * h5_3_10;
    const double k5_8_10_1 = h5_8_20 + CDx * h5_8_10;
    const double h13_3_4 = acc[713] + ABz * acc[279];
    const double h5_8_4 = h13_3_4 + ABy * h5_3_4;
    const double k5_8_4_1 = h5_8_10 + CDx * h5_8_4;
    const double k5_8_4_4 = k5_8_10_1 + CDx * k5_8_4_1;
    const double h13_3_21 = acc[730] + ABz * acc[296];
    const double h5_8_21 = h13_3_21 + ABy * h5_3_21;
    const double k5_8_10_2 = h5_8_21 + CDy * h5_8_10;
    const double h13_3_11 = acc[720] + ABz * acc[286];
    const double h5_8_11 = h13_3_11 + ABy * h5_3_11;
    const double k5_8_4_2 = h5_8_11 + CDy * h5_8_4;
    const double k5_8_4_5 = k5_8_10_2 + CDx * k5_8_4_2;
    const double h13_3_22 = acc[731] + ABz * acc[297];
    const double h5_8_22 = h13_3_22 + ABy * h5_3_22;
    const double k5_8_10_3 = h5_8_22 + CDz * h5_8_10;
    const double h13_3_12 = acc[721] + ABz * acc[287];
    const double h5_8_12 = h13_3_12 + ABy * h5_3_12;
    const double k5_8_4_3 = h5_8_12 + CDz * h5_8_4;
    const double k5_8_4_6 = k5_8_10_3 + CDx * k5_8_4_3;
    const double h13_3_23 = acc[732] + ABz * acc[298];
    const double h5_8_23 = h13_3_23 + ABy * h5_3_23;
    const double k5_8_11_2 = h5_8_23 + CDy * h5_8_11;
    const double k5_8_4_7 = k5_8_11_2 + CDy * k5_8_4_2;
    const double h13_3_24 = acc[733] + ABz * acc[299];
    const double h5_8_24 = h13_3_24 + ABy * h5_3_24;
    const double k5_8_11_3 = h5_8_24 + CDz * h5_8_11;
    const double k5_8_4_8 = k5_8_11_3 + CDy * k5_8_4_3;
    const double h13_3_25 = acc[734] + ABz * acc[300];
    const double h5_8_25 = h13_3_25 + ABy * h5_3_25;
    const double k5_8_12_3 = h5_8_25 + CDz * h5_8_12;
    const double k5_8_4_9 = k5_8_12_3 + CDz * k5_8_4_3;
    const double k5_8_11_1 = h5_8_21 + CDx * h5_8_11;
    const double h13_3_5 = acc[714] + ABz * acc[280];
    const double h5_8_5 = h13_3_5 + ABy * h5_3_5;
    const double k5_8_5_1 = h5_8_11 + CDx * h5_8_5;
    const double k5_8_5_4 = k5_8_11_1 + CDx * k5_8_5_1;
    const double h13_3_13 = acc[722] + ABz * acc[288];
    const double h5_8_13 = h13_3_13 + ABy * h5_3_13;
    const double k5_8_5_2 = h5_8_13 + CDy * h5_8_5;
    const double k5_8_5_5 = k5_8_11_2 + CDx * k5_8_5_2;
    const double h13_3_15 = acc[724] + ABz * acc[290];
    const double h5_8_15 = h13_3_15 + ABy * h5_3_15;
    const double k5_8_5_3 = h5_8_15 + CDz * h5_8_5;
    const double k5_8_5_6 = k5_8_11_3 + CDx * k5_8_5_3;
    const double h13_3_26 = acc[735] + ABz * acc[301];
    const double h5_8_26 = h13_3_26 + ABy * h5_3_26;
    const double k5_8_13_2 = h5_8_26 + CDy * h5_8_13;
    const double k5_8_5_7 = k5_8_13_2 + CDy * k5_8_5_2;
    const double h13_3_27 = acc[736] + ABz * acc[302];
    const double h5_8_27 = h13_3_27 + ABy * h5_3_27;
    const double k5_8_13_3 = h5_8_27 + CDz * h5_8_13;
    const double k5_8_5_8 = k5_8_13_3 + CDy * k5_8_5_3;
    const double h13_3_28 = acc[737] + ABz * acc[303];
    const double h5_8_28 = h13_3_28 + ABy * h5_3_28;
    const double k5_8_15_3 = h5_8_28 + CDz * h5_8_15;
    const double k5_8_5_9 = k5_8_15_3 + CDz * k5_8_5_3;
    const double k5_8_12_1 = h5_8_22 + CDx * h5_8_12;
    const double h13_3_6 = acc[715] + ABz * acc[281];
    const double h5_8_6 = h13_3_6 + ABy * h5_3_6;
    const double k5_8_6_1 = h5_8_12 + CDx * h5_8_6;
    const double k5_8_6_4 = k5_8_12_1 + CDx * k5_8_6_1;
    const double k5_8_12_2 = h5_8_24 + CDy * h5_8_12;
    const double k5_8_6_2 = h5_8_15 + CDy * h5_8_6;
    const double k5_8_6_5 = k5_8_12_2 + CDx * k5_8_6_2;
    const double h13_3_14 = acc[723] + ABz * acc[289];
    const double h5_8_14 = h13_3_14 + ABy * h5_3_14;
    const double k5_8_6_3 = h5_8_14 + CDz * h5_8_6;
    const double k5_8_6_6 = k5_8_12_3 + CDx * k5_8_6_3;
    const double k5_8_15_2 = h5_8_27 + CDy * h5_8_15;
    const double k5_8_6_7 = k5_8_15_2 + CDy * k5_8_6_2;
    const double k5_8_6_8 = k5_8_15_3 + CDy * k5_8_6_3;
    const double h13_3_29 = acc[738] + ABz * acc[304];
    const double h5_8_29 = h13_3_29 + ABy * h5_3_29;
    const double k5_8_14_3 = h5_8_29 + CDz * h5_8_14;
    const double k5_8_6_9 = k5_8_14_3 + CDz * k5_8_6_3;
    const double k5_8_13_1 = h5_8_23 + CDx * h5_8_13;
    const double h13_3_7 = acc[716] + ABz * acc[282];
    const double h5_8_7 = h13_3_7 + ABy * h5_3_7;
    const double k5_8_7_1 = h5_8_13 + CDx * h5_8_7;
    const double k5_8_7_4 = k5_8_13_1 + CDx * k5_8_7_1;
    const double h13_3_16 = acc[725] + ABz * acc[291];
    const double h5_8_16 = h13_3_16 + ABy * h5_3_16;
    const double k5_8_7_2 = h5_8_16 + CDy * h5_8_7;
    const double k5_8_7_5 = k5_8_13_2 + CDx * k5_8_7_2;
    const double h13_3_17 = acc[726] + ABz * acc[292];
    const double h5_8_17 = h13_3_17 + ABy * h5_3_17;
    const double k5_8_7_3 = h5_8_17 + CDz * h5_8_7;
    const double k5_8_7_6 = k5_8_13_3 + CDx * k5_8_7_3;
    const double h13_3_30 = acc[739] + ABz * acc[305];
    const double h5_8_30 = h13_3_30 + ABy * h5_3_30;
    const double k5_8_16_2 = h5_8_30 + CDy * h5_8_16;
    const double k5_8_7_7 = k5_8_16_2 + CDy * k5_8_7_2;
    const double h13_3_31 = acc[740] + ABz * acc[306];
    const double h5_8_31 = h13_3_31 + ABy * h5_3_31;
    const double k5_8_16_3 = h5_8_31 + CDz * h5_8_16;
    const double k5_8_7_8 = k5_8_16_3 + CDy * k5_8_7_3;
    const double h13_3_32 = acc[741] + ABz * acc[307];
    const double h5_8_32 = h13_3_32 + ABy * h5_3_32;
    const double k5_8_17_3 = h5_8_32 + CDz * h5_8_17;
    const double k5_8_7_9 = k5_8_17_3 + CDz * k5_8_7_3;
    const double k5_8_15_1 = h5_8_24 + CDx * h5_8_15;
    const double h13_3_8 = acc[717] + ABz * acc[283];
    const double h5_8_8 = h13_3_8 + ABy * h5_3_8;
    const double k5_8_8_1 = h5_8_15 + CDx * h5_8_8;
    const double k5_8_8_4 = k5_8_15_1 + CDx * k5_8_8_1;
    const double k5_8_8_2 = h5_8_17 + CDy * h5_8_8;
    const double k5_8_8_5 = k5_8_15_2 + CDx * k5_8_8_2;
    const double h13_3_18 = acc[727] + ABz * acc[293];
    const double h5_8_18 = h13_3_18 + ABy * h5_3_18;
    const double k5_8_8_3 = h5_8_18 + CDz * h5_8_8;
    const double k5_8_8_6 = k5_8_15_3 + CDx * k5_8_8_3;
    const double k5_8_17_2 = h5_8_31 + CDy * h5_8_17;
    const double k5_8_8_7 = k5_8_17_2 + CDy * k5_8_8_2;
    const double k5_8_8_8 = k5_8_17_3 + CDy * k5_8_8_3;
    const double h13_3_33 = acc[742] + ABz * acc[308];
    const double h5_8_33 = h13_3_33 + ABy * h5_3_33;
    const double k5_8_18_3 = h5_8_33 + CDz * h5_8_18;
    const double k5_8_8_9 = k5_8_18_3 + CDz * k5_8_8_3;
    const double k5_8_14_1 = h5_8_25 + CDx * h5_8_14;
    const double h13_3_9 = acc[718] + ABz * acc[284];
    const double h5_8_9 = h13_3_9 + ABy * h5_3_9;
    const double k5_8_9_1 = h5_8_14 + CDx * h5_8_9;
    const double k5_8_9_4 = k5_8_14_1 + CDx * k5_8_9_1;
    const double k5_8_14_2 = h5_8_28 + CDy * h5_8_14;
    const double k5_8_9_2 = h5_8_18 + CDy * h5_8_9;
    const double k5_8_9_5 = k5_8_14_2 + CDx * k5_8_9_2;
    const double h13_3_19 = acc[728] + ABz * acc[294];
    const double h5_8_19 = h13_3_19 + ABy * h5_3_19;
    const double k5_8_9_3 = h5_8_19 + CDz * h5_8_9;
    const double k5_8_9_6 = k5_8_14_3 + CDx * k5_8_9_3;
    const double k5_8_18_2 = h5_8_32 + CDy * h5_8_18;
    const double k5_8_9_7 = k5_8_18_2 + CDy * k5_8_9_2;
    const double k5_8_9_8 = k5_8_18_3 + CDy * k5_8_9_3;
    const double h13_3_34 = acc[743] + ABz * acc[309];
    const double h5_8_34 = h13_3_34 + ABy * h5_3_34;
    const double k5_8_19_3 = h5_8_34 + CDz * h5_8_19;
    const double k5_8_9_9 = k5_8_19_3 + CDz * k5_8_9_3;
    const double h15_3_20 = acc[760] + ABz * acc[357];
    const double h5_9_20 = h15_3_20 + ABz * h5_3_20;
    const double h15_3_10 = acc[750] + ABz * acc[347];
    const double h5_9_10 = h15_3_10 + ABz * h5_3_10;
    const double k5_9_10_1 = h5_9_20 + CDx * h5_9_10;
    const double h15_3_4 = acc[744] + ABz * acc[341];
    const double h5_9_4 = h15_3_4 + ABz * h5_3_4;
    const double k5_9_4_1 = h5_9_10 + CDx * h5_9_4;
    const double k5_9_4_4 = k5_9_10_1 + CDx * k5_9_4_1;
    const double h15_3_21 = acc[761] + ABz * acc[358];
    const double h5_9_21 = h15_3_21 + ABz * h5_3_21;
    const double k5_9_10_2 = h5_9_21 + CDy * h5_9_10;
    const double h15_3_11 = acc[751] + ABz * acc[348];
    const double h5_9_11 = h15_3_11 + ABz * h5_3_11;
    const double k5_9_4_2 = h5_9_11 + CDy * h5_9_4;
    const double k5_9_4_5 = k5_9_10_2 + CDx * k5_9_4_2;
    const double h15_3_22 = acc[762] + ABz * acc[359];
    const double h5_9_22 = h15_3_22 + ABz * h5_3_22;
    const double k5_9_10_3 = h5_9_22 + CDz * h5_9_10;
    const double h15_3_12 = acc[752] + ABz * acc[349];
    const double h5_9_12 = h15_3_12 + ABz * h5_3_12;
    const double k5_9_4_3 = h5_9_12 + CDz * h5_9_4;
    const double k5_9_4_6 = k5_9_10_3 + CDx * k5_9_4_3;
    const double h15_3_23 = acc[763] + ABz * acc[360];
    const double h5_9_23 = h15_3_23 + ABz * h5_3_23;
    const double k5_9_11_2 = h5_9_23 + CDy * h5_9_11;
    const double k5_9_4_7 = k5_9_11_2 + CDy * k5_9_4_2;
    const double h15_3_24 = acc[764] + ABz * acc[361];
    const double h5_9_24 = h15_3_24 + ABz * h5_3_24;
    const double k5_9_11_3 = h5_9_24 + CDz * h5_9_11;
    const double k5_9_4_8 = k5_9_11_3 + CDy * k5_9_4_3;
    const double h15_3_25 = acc[765] + ABz * acc[362];
    const double h5_9_25 = h15_3_25 + ABz * h5_3_25;
    const double k5_9_12_3 = h5_9_25 + CDz * h5_9_12;
    const double k5_9_4_9 = k5_9_12_3 + CDz * k5_9_4_3;
    const double k5_9_11_1 = h5_9_21 + CDx * h5_9_11;
    const double h15_3_5 = acc[745] + ABz * acc[342];
    const double h5_9_5 = h15_3_5 + ABz * h5_3_5;
    const double k5_9_5_1 = h5_9_11 + CDx * h5_9_5;
    const double k5_9_5_4 = k5_9_11_1 + CDx * k5_9_5_1;
    const double h15_3_13 = acc[753] + ABz * acc[350];
    const double h5_9_13 = h15_3_13 + ABz * h5_3_13;
    const double k5_9_5_2 = h5_9_13 + CDy * h5_9_5;
    const double k5_9_5_5 = k5_9_11_2 + CDx * k5_9_5_2;
    const double h15_3_15 = acc[755] + ABz * acc[352];
    const double h5_9_15 = h15_3_15 + ABz * h5_3_15;
    const double k5_9_5_3 = h5_9_15 + CDz * h5_9_5;
    const double k5_9_5_6 = k5_9_11_3 + CDx * k5_9_5_3;
    const double h15_3_26 = acc[766] + ABz * acc[363];
    const double h5_9_26 = h15_3_26 + ABz * h5_3_26;
    const double k5_9_13_2 = h5_9_26 + CDy * h5_9_13;
    const double k5_9_5_7 = k5_9_13_2 + CDy * k5_9_5_2;
    const double h15_3_27 = acc[767] + ABz * acc[364];
    const double h5_9_27 = h15_3_27 + ABz * h5_3_27;
    const double k5_9_13_3 = h5_9_27 + CDz * h5_9_13;
    const double k5_9_5_8 = k5_9_13_3 + CDy * k5_9_5_3;
    const double h15_3_28 = acc[768] + ABz * acc[365];
    const double h5_9_28 = h15_3_28 + ABz * h5_3_28;
    const double k5_9_15_3 = h5_9_28 + CDz * h5_9_15;
    const double k5_9_5_9 = k5_9_15_3 + CDz * k5_9_5_3;
    const double k5_9_12_1 = h5_9_22 + CDx * h5_9_12;
    const double h15_3_6 = acc[746] + ABz * acc[343];
    const double h5_9_6 = h15_3_6 + ABz * h5_3_6;
    const double k5_9_6_1 = h5_9_12 + CDx * h5_9_6;
    const double k5_9_6_4 = k5_9_12_1 + CDx * k5_9_6_1;
    const double k5_9_12_2 = h5_9_24 + CDy * h5_9_12;
    const double k5_9_6_2 = h5_9_15 + CDy * h5_9_6;
    const double k5_9_6_5 = k5_9_12_2 + CDx * k5_9_6_2;
    const double h15_3_14 = acc[754] + ABz * acc[351];
    const double h5_9_14 = h15_3_14 + ABz * h5_3_14;
    const double k5_9_6_3 = h5_9_14 + CDz * h5_9_6;
    const double k5_9_6_6 = k5_9_12_3 + CDx * k5_9_6_3;
    const double k5_9_15_2 = h5_9_27 + CDy * h5_9_15;
    const double k5_9_6_7 = k5_9_15_2 + CDy * k5_9_6_2;
    const double k5_9_6_8 = k5_9_15_3 + CDy * k5_9_6_3;
    const double h15_3_29 = acc[769] + ABz * acc[366];
    const double h5_9_29 = h15_3_29 + ABz * h5_3_29;
    const double k5_9_14_3 = h5_9_29 + CDz * h5_9_14;
    const double k5_9_6_9 = k5_9_14_3 + CDz * k5_9_6_3;
    const double k5_9_13_1 = h5_9_23 + CDx * h5_9_13;
    const double h15_3_7 = acc[747] + ABz * acc[344];
    const double h5_9_7 = h15_3_7 + ABz * h5_3_7;
    const double k5_9_7_1 = h5_9_13 + CDx * h5_9_7;
    const double k5_9_7_4 = k5_9_13_1 + CDx * k5_9_7_1;
    const double h15_3_16 = acc[756] + ABz * acc[353];
    const double h5_9_16 = h15_3_16 + ABz * h5_3_16;
    const double k5_9_7_2 = h5_9_16 + CDy * h5_9_7;
    const double k5_9_7_5 = k5_9_13_2 + CDx * k5_9_7_2;
    const double h15_3_17 = acc[757] + ABz * acc[354];
    const double h5_9_17 = h15_3_17 + ABz * h5_3_17;
    const double k5_9_7_3 = h5_9_17 + CDz * h5_9_7;
    const double k5_9_7_6 = k5_9_13_3 + CDx * k5_9_7_3;
    const double h15_3_30 = acc[770] + ABz * acc[367];
    const double h5_9_30 = h15_3_30 + ABz * h5_3_30;
    const double k5_9_16_2 = h5_9_30 + CDy * h5_9_16;
    const double k5_9_7_7 = k5_9_16_2 + CDy * k5_9_7_2;
    const double h15_3_31 = acc[771] + ABz * acc[368];
    const double h5_9_31 = h15_3_31 + ABz * h5_3_31;
    const double k5_9_16_3 = h5_9_31 + CDz * h5_9_16;
    const double k5_9_7_8 = k5_9_16_3 + CDy * k5_9_7_3;
    const double h15_3_32 = acc[772] + ABz * acc[369];
    const double h5_9_32 = h15_3_32 + ABz * h5_3_32;
    const double k5_9_17_3 = h5_9_32 + CDz * h5_9_17;
    const double k5_9_7_9 = k5_9_17_3 + CDz * k5_9_7_3;
    const double k5_9_15_1 = h5_9_24 + CDx * h5_9_15;
    const double h15_3_8 = acc[748] + ABz * acc[345];
    const double h5_9_8 = h15_3_8 + ABz * h5_3_8;
    const double k5_9_8_1 = h5_9_15 + CDx * h5_9_8;
    const double k5_9_8_4 = k5_9_15_1 + CDx * k5_9_8_1;
    const double k5_9_8_2 = h5_9_17 + CDy * h5_9_8;
    const double k5_9_8_5 = k5_9_15_2 + CDx * k5_9_8_2;
    const double h15_3_18 = acc[758] + ABz * acc[355];
    const double h5_9_18 = h15_3_18 + ABz * h5_3_18;
    const double k5_9_8_3 = h5_9_18 + CDz * h5_9_8;
    const double k5_9_8_6 = k5_9_15_3 + CDx * k5_9_8_3;
    const double k5_9_17_2 = h5_9_31 + CDy * h5_9_17;
    const double k5_9_8_7 = k5_9_17_2 + CDy * k5_9_8_2;
    const double k5_9_8_8 = k5_9_17_3 + CDy * k5_9_8_3;
    const double h15_3_33 = acc[773] + ABz * acc[370];
    const double h5_9_33 = h15_3_33 + ABz * h5_3_33;
    const double k5_9_18_3 = h5_9_33 + CDz * h5_9_18;
    const double k5_9_8_9 = k5_9_18_3 + CDz * k5_9_8_3;
    const double k5_9_14_1 = h5_9_25 + CDx * h5_9_14;
    const double h15_3_9 = acc[749] + ABz * acc[346];
    const double h5_9_9 = h15_3_9 + ABz * h5_3_9;
    const double k5_9_9_1 = h5_9_14 + CDx * h5_9_9;
    const double k5_9_9_4 = k5_9_14_1 + CDx * k5_9_9_1;
    const double k5_9_14_2 = h5_9_28 + CDy * h5_9_14;
    const double k5_9_9_2 = h5_9_18 + CDy * h5_9_9;
    const double k5_9_9_5 = k5_9_14_2 + CDx * k5_9_9_2;
    const double h15_3_19 = acc[759] + ABz * acc[356];
    const double h5_9_19 = h15_3_19 + ABz * h5_3_19;
    const double k5_9_9_3 = h5_9_19 + CDz * h5_9_9;
    const double k5_9_9_6 = k5_9_14_3 + CDx * k5_9_9_3;
    const double k5_9_18_2 = h5_9_32 + CDy * h5_9_18;
    const double k5_9_9_7 = k5_9_18_2 + CDy * k5_9_9_2;
    const double k5_9_9_8 = k5_9_18_3 + CDy * k5_9_9_3;
    const double h15_3_34 = acc[774] + ABz * acc[371];
    const double h5_9_34 = h15_3_34 + ABz * h5_3_34;
    const double k5_9_19_3 = h5_9_34 + CDz * h5_9_19;
    const double k5_9_9_9 = k5_9_19_3 + CDz * k5_9_9_3;
    const double h12_1_20 = acc[574] + ABx * acc[264];
    const double h6_1_20 = acc[264] + ABx * acc[78];
    const double h6_4_20 = h12_1_20 + ABx * h6_1_20;
    const double h12_1_10 = acc[564] + ABx * acc[254];
    const double h6_1_10 = acc[254] + ABx * acc[68];
    const double h6_4_10 = h12_1_10 + ABx * h6_1_10;
    const double k6_4_10_1 = h6_4_20 + CDx * h6_4_10;
    const double h12_1_4 = acc[558] + ABx * acc[248];
    const double h6_1_4 = acc[248] + ABx * acc[62];
    const double h6_4_4 = h12_1_4 + ABx * h6_1_4;
    const double k6_4_4_1 = h6_4_10 + CDx * h6_4_4;
    const double k6_4_4_4 = k6_4_10_1 + CDx * k6_4_4_1;
    const double h12_1_21 = acc[575] + ABx * acc[265];
    const double h6_1_21 = acc[265] + ABx * acc[79];
    const double h6_4_21 = h12_1_21 + ABx * h6_1_21;
    const double k6_4_10_2 = h6_4_21 + CDy * h6_4_10;
    const double h12_1_11 = acc[565] + ABx * acc[255];
    const double h6_1_11 = acc[255] + ABx * acc[69];
    const double h6_4_11 = h12_1_11 + ABx * h6_1_11;
    const double k6_4_4_2 = h6_4_11 + CDy * h6_4_4;
    const double k6_4_4_5 = k6_4_10_2 + CDx * k6_4_4_2;
    const double h12_1_22 = acc[576] + ABx * acc[266];
    const double h6_1_22 = acc[266] + ABx * acc[80];
    const double h6_4_22 = h12_1_22 + ABx * h6_1_22;
    const double k6_4_10_3 = h6_4_22 + CDz * h6_4_10;
    const double h12_1_12 = acc[566] + ABx * acc[256];
    const double h6_1_12 = acc[256] + ABx * acc[70];
    const double h6_4_12 = h12_1_12 + ABx * h6_1_12;
    const double k6_4_4_3 = h6_4_12 + CDz * h6_4_4;
    const double k6_4_4_6 = k6_4_10_3 + CDx * k6_4_4_3;
    const double h12_1_23 = acc[577] + ABx * acc[267];
    const double h6_1_23 = acc[267] + ABx * acc[81];
    const double h6_4_23 = h12_1_23 + ABx * h6_1_23;
    const double k6_4_11_2 = h6_4_23 + CDy * h6_4_11;
    const double k6_4_4_7 = k6_4_11_2 + CDy * k6_4_4_2;
    const double h12_1_24 = acc[578] + ABx * acc[268];
    const double h6_1_24 = acc[268] + ABx * acc[82];
    const double h6_4_24 = h12_1_24 + ABx * h6_1_24;
    const double k6_4_11_3 = h6_4_24 + CDz * h6_4_11;
    const double k6_4_4_8 = k6_4_11_3 + CDy * k6_4_4_3;
    const double h12_1_25 = acc[579] + ABx * acc[269];
    const double h6_1_25 = acc[269] + ABx * acc[83];
    const double h6_4_25 = h12_1_25 + ABx * h6_1_25;
    const double k6_4_12_3 = h6_4_25 + CDz * h6_4_12;
    const double k6_4_4_9 = k6_4_12_3 + CDz * k6_4_4_3;
    const double k6_4_11_1 = h6_4_21 + CDx * h6_4_11;
    const double h12_1_5 = acc[559] + ABx * acc[249];
    const double h6_1_5 = acc[249] + ABx * acc[63];
    const double h6_4_5 = h12_1_5 + ABx * h6_1_5;
    const double k6_4_5_1 = h6_4_11 + CDx * h6_4_5;
    const double k6_4_5_4 = k6_4_11_1 + CDx * k6_4_5_1;
    const double h12_1_13 = acc[567] + ABx * acc[257];
    const double h6_1_13 = acc[257] + ABx * acc[71];
    const double h6_4_13 = h12_1_13 + ABx * h6_1_13;
    const double k6_4_5_2 = h6_4_13 + CDy * h6_4_5;
    const double k6_4_5_5 = k6_4_11_2 + CDx * k6_4_5_2;
    const double h12_1_15 = acc[569] + ABx * acc[259];
    const double h6_1_15 = acc[259] + ABx * acc[73];
    const double h6_4_15 = h12_1_15 + ABx * h6_1_15;
    const double k6_4_5_3 = h6_4_15 + CDz * h6_4_5;
    const double k6_4_5_6 = k6_4_11_3 + CDx * k6_4_5_3;
    const double h12_1_26 = acc[580] + ABx * acc[270];
    const double h6_1_26 = acc[270] + ABx * acc[84];
    const double h6_4_26 = h12_1_26 + ABx * h6_1_26;
    const double k6_4_13_2 = h6_4_26 + CDy * h6_4_13;
    const double k6_4_5_7 = k6_4_13_2 + CDy * k6_4_5_2;
    const double h12_1_27 = acc[581] + ABx * acc[271];
    const double h6_1_27 = acc[271] + ABx * acc[85];
    const double h6_4_27 = h12_1_27 + ABx * h6_1_27;
    const double k6_4_13_3 = h6_4_27 + CDz * h6_4_13;
    const double k6_4_5_8 = k6_4_13_3 + CDy * k6_4_5_3;
    const double h12_1_28 = acc[582] + ABx * acc[272];
    const double h6_1_28 = acc[272] + ABx * acc[86];
    const double h6_4_28 = h12_1_28 + ABx * h6_1_28;
    const double k6_4_15_3 = h6_4_28 + CDz * h6_4_15;
    const double k6_4_5_9 = k6_4_15_3 + CDz * k6_4_5_3;
    const double k6_4_12_1 = h6_4_22 + CDx * h6_4_12;
    const double h12_1_6 = acc[560] + ABx * acc[250];
    const double h6_1_6 = acc[250] + ABx * acc[64];
    const double h6_4_6 = h12_1_6 + ABx * h6_1_6;
    const double k6_4_6_1 = h6_4_12 + CDx * h6_4_6;
    const double k6_4_6_4 = k6_4_12_1 + CDx * k6_4_6_1;
    const double k6_4_12_2 = h6_4_24 + CDy * h6_4_12;
    const double k6_4_6_2 = h6_4_15 + CDy * h6_4_6;
    const double k6_4_6_5 = k6_4_12_2 + CDx * k6_4_6_2;
    const double h12_1_14 = acc[568] + ABx * acc[258];
    const double h6_1_14 = acc[258] + ABx * acc[72];
    const double h6_4_14 = h12_1_14 + ABx * h6_1_14;
    const double k6_4_6_3 = h6_4_14 + CDz * h6_4_6;
    const double k6_4_6_6 = k6_4_12_3 + CDx * k6_4_6_3;
    const double k6_4_15_2 = h6_4_27 + CDy * h6_4_15;
    const double k6_4_6_7 = k6_4_15_2 + CDy * k6_4_6_2;
    const double k6_4_6_8 = k6_4_15_3 + CDy * k6_4_6_3;
    const double h12_1_29 = acc[583] + ABx * acc[273];
    const double h6_1_29 = acc[273] + ABx * acc[87];
    const double h6_4_29 = h12_1_29 + ABx * h6_1_29;
    const double k6_4_14_3 = h6_4_29 + CDz * h6_4_14;
    const double k6_4_6_9 = k6_4_14_3 + CDz * k6_4_6_3;
    const double k6_4_13_1 = h6_4_23 + CDx * h6_4_13;
    const double h12_1_7 = acc[561] + ABx * acc[251];
    const double h6_1_7 = acc[251] + ABx * acc[65];
    const double h6_4_7 = h12_1_7 + ABx * h6_1_7;
    const double k6_4_7_1 = h6_4_13 + CDx * h6_4_7;
    const double k6_4_7_4 = k6_4_13_1 + CDx * k6_4_7_1;
    const double h12_1_16 = acc[570] + ABx * acc[260];
    const double h6_1_16 = acc[260] + ABx * acc[74];
    const double h6_4_16 = h12_1_16 + ABx * h6_1_16;
    const double k6_4_7_2 = h6_4_16 + CDy * h6_4_7;
    const double k6_4_7_5 = k6_4_13_2 + CDx * k6_4_7_2;
    const double h12_1_17 = acc[571] + ABx * acc[261];
    const double h6_1_17 = acc[261] + ABx * acc[75];
    const double h6_4_17 = h12_1_17 + ABx * h6_1_17;
    const double k6_4_7_3 = h6_4_17 + CDz * h6_4_7;
    const double k6_4_7_6 = k6_4_13_3 + CDx * k6_4_7_3;
    const double h12_1_30 = acc[584] + ABx * acc[274];
    const double h6_1_30 = acc[274] + ABx * acc[88];
    const double h6_4_30 = h12_1_30 + ABx * h6_1_30;
    const double k6_4_16_2 = h6_4_30 + CDy * h6_4_16;
    const double k6_4_7_7 = k6_4_16_2 + CDy * k6_4_7_2;
    const double h12_1_31 = acc[585] + ABx * acc[275];
    const double h6_1_31 = acc[275] + ABx * acc[89];
    const double h6_4_31 = h12_1_31 + ABx * h6_1_31;
    const double k6_4_16_3 = h6_4_31 + CDz * h6_4_16;
    const double k6_4_7_8 = k6_4_16_3 + CDy * k6_4_7_3;
    const double h12_1_32 = acc[586] + ABx * acc[276];
    const double h6_1_32 = acc[276] + ABx * acc[90];
    const double h6_4_32 = h12_1_32 + ABx * h6_1_32;
    const double k6_4_17_3 = h6_4_32 + CDz * h6_4_17;
    const double k6_4_7_9 = k6_4_17_3 + CDz * k6_4_7_3;
    const double k6_4_15_1 = h6_4_24 + CDx * h6_4_15;
    const double h12_1_8 = acc[562] + ABx * acc[252];
    const double h6_1_8 = acc[252] + ABx * acc[66];
    const double h6_4_8 = h12_1_8 + ABx * h6_1_8;
    const double k6_4_8_1 = h6_4_15 + CDx * h6_4_8;
    const double k6_4_8_4 = k6_4_15_1 + CDx * k6_4_8_1;
    const double k6_4_8_2 = h6_4_17 + CDy * h6_4_8;
    const double k6_4_8_5 = k6_4_15_2 + CDx * k6_4_8_2;
    const double h12_1_18 = acc[572] + ABx * acc[262];
    const double h6_1_18 = acc[262] + ABx * acc[76];
    const double h6_4_18 = h12_1_18 + ABx * h6_1_18;
    const double k6_4_8_3 = h6_4_18 + CDz * h6_4_8;
    const double k6_4_8_6 = k6_4_15_3 + CDx * k6_4_8_3;
    const double k6_4_17_2 = h6_4_31 + CDy * h6_4_17;
    const double k6_4_8_7 = k6_4_17_2 + CDy * k6_4_8_2;
    const double k6_4_8_8 = k6_4_17_3 + CDy * k6_4_8_3;
    const double h12_1_33 = acc[587] + ABx * acc[277];
    const double h6_1_33 = acc[277] + ABx * acc[91];
    const double h6_4_33 = h12_1_33 + ABx * h6_1_33;
    const double k6_4_18_3 = h6_4_33 + CDz * h6_4_18;
    const double k6_4_8_9 = k6_4_18_3 + CDz * k6_4_8_3;
    const double k6_4_14_1 = h6_4_25 + CDx * h6_4_14;
    const double h12_1_9 = acc[563] + ABx * acc[253];
    const double h6_1_9 = acc[253] + ABx * acc[67];
    const double h6_4_9 = h12_1_9 + ABx * h6_1_9;
    const double k6_4_9_1 = h6_4_14 + CDx * h6_4_9;
    const double k6_4_9_4 = k6_4_14_1 + CDx * k6_4_9_1;
    const double k6_4_14_2 = h6_4_28 + CDy * h6_4_14;
    const double k6_4_9_2 = h6_4_18 + CDy * h6_4_9;
    const double k6_4_9_5 = k6_4_14_2 + CDx * k6_4_9_2;
    const double h12_1_19 = acc[573] + ABx * acc[263];
    const double h6_1_19 = acc[263] + ABx * acc[77];
    const double h6_4_19 = h12_1_19 + ABx * h6_1_19;
    const double k6_4_9_3 = h6_4_19 + CDz * h6_4_9;
    const double k6_4_9_6 = k6_4_14_3 + CDx * k6_4_9_3;
    const double k6_4_18_2 = h6_4_32 + CDy * h6_4_18;
    const double k6_4_9_7 = k6_4_18_2 + CDy * k6_4_9_2;
    const double k6_4_9_8 = k6_4_18_3 + CDy * k6_4_9_3;
    const double h12_1_34 = acc[588] + ABx * acc[278];
    const double h6_1_34 = acc[278] + ABx * acc[92];
    const double h6_4_34 = h12_1_34 + ABx * h6_1_34;
    const double k6_4_19_3 = h6_4_34 + CDz * h6_4_19;
    const double k6_4_9_9 = k6_4_19_3 + CDz * k6_4_9_3;
    const double h12_2_20 = acc[636] + ABy * acc[264];
    const double h6_2_20 = acc[357] + ABy * acc[78];
    const double h6_5_20 = h12_2_20 + ABx * h6_2_20;
    const double h12_2_10 = acc[626] + ABy * acc[254];
    const double h6_2_10 = acc[347] + ABy * acc[68];
    const double h6_5_10 = h12_2_10 + ABx * h6_2_10;
    const double k6_5_10_1 = h6_5_20 + CDx * h6_5_10;
    const double h12_2_4 = acc[620] + ABy * acc[248];
    const double h6_2_4 = acc[341] + ABy * acc[62];
    const double h6_5_4 = h12_2_4 + ABx * h6_2_4;
    const double k6_5_4_1 = h6_5_10 + CDx * h6_5_4;
    const double k6_5_4_4 = k6_5_10_1 + CDx * k6_5_4_1;
    const double h12_2_21 = acc[637] + ABy * acc[265];
    const double h6_2_21 = acc[358] + ABy * acc[79];
    const double h6_5_21 = h12_2_21 + ABx * h6_2_21;
    const double k6_5_10_2 = h6_5_21 + CDy * h6_5_10;
    const double h12_2_11 = acc[627] + ABy * acc[255];
    const double h6_2_11 = acc[348] + ABy * acc[69];
    const double h6_5_11 = h12_2_11 + ABx * h6_2_11;
    const double k6_5_4_2 = h6_5_11 + CDy * h6_5_4;
    const double k6_5_4_5 = k6_5_10_2 + CDx * k6_5_4_2;
    const double h12_2_22 = acc[638] + ABy * acc[266];
    const double h6_2_22 = acc[359] + ABy * acc[80];
    const double h6_5_22 = h12_2_22 + ABx * h6_2_22;
    const double k6_5_10_3 = h6_5_22 + CDz * h6_5_10;
    const double h12_2_12 = acc[628] + ABy * acc[256];
    const double h6_2_12 = acc[349] + ABy * acc[70];
    const double h6_5_12 = h12_2_12 + ABx * h6_2_12;
    const double k6_5_4_3 = h6_5_12 + CDz * h6_5_4;
    const double k6_5_4_6 = k6_5_10_3 + CDx * k6_5_4_3;
    const double h12_2_23 = acc[639] + ABy * acc[267];
    const double h6_2_23 = acc[360] + ABy * acc[81];
    const double h6_5_23 = h12_2_23 + ABx * h6_2_23;
    const double k6_5_11_2 = h6_5_23 + CDy * h6_5_11;
    const double k6_5_4_7 = k6_5_11_2 + CDy * k6_5_4_2;
    const double h12_2_24 = acc[640] + ABy * acc[268];
    const double h6_2_24 = acc[361] + ABy * acc[82];
    const double h6_5_24 = h12_2_24 + ABx * h6_2_24;
    const double k6_5_11_3 = h6_5_24 + CDz * h6_5_11;
    const double k6_5_4_8 = k6_5_11_3 + CDy * k6_5_4_3;
    const double h12_2_25 = acc[641] + ABy * acc[269];
    const double h6_2_25 = acc[362] + ABy * acc[83];
    const double h6_5_25 = h12_2_25 + ABx * h6_2_25;
    const double k6_5_12_3 = h6_5_25 + CDz * h6_5_12;
    const double k6_5_4_9 = k6_5_12_3 + CDz * k6_5_4_3;
    const double k6_5_11_1 = h6_5_21 + CDx * h6_5_11;
    const double h12_2_5 = acc[621] + ABy * acc[249];
    const double h6_2_5 = acc[342] + ABy * acc[63];
    const double h6_5_5 = h12_2_5 + ABx * h6_2_5;
    const double k6_5_5_1 = h6_5_11 + CDx * h6_5_5;
    const double k6_5_5_4 = k6_5_11_1 + CDx * k6_5_5_1;
    const double h12_2_13 = acc[629] + ABy * acc[257];
    const double h6_2_13 = acc[350] + ABy * acc[71];
    const double h6_5_13 = h12_2_13 + ABx * h6_2_13;
    const double k6_5_5_2 = h6_5_13 + CDy * h6_5_5;
    const double k6_5_5_5 = k6_5_11_2 + CDx * k6_5_5_2;
    const double h12_2_15 = acc[631] + ABy * acc[259];
    const double h6_2_15 = acc[352] + ABy * acc[73];
    const double h6_5_15 = h12_2_15 + ABx * h6_2_15;
    const double k6_5_5_3 = h6_5_15 + CDz * h6_5_5;
    const double k6_5_5_6 = k6_5_11_3 + CDx * k6_5_5_3;
    const double h12_2_26 = acc[642] + ABy * acc[270];
    const double h6_2_26 = acc[363] + ABy * acc[84];
    const double h6_5_26 = h12_2_26 + ABx * h6_2_26;
    const double k6_5_13_2 = h6_5_26 + CDy * h6_5_13;
    const double k6_5_5_7 = k6_5_13_2 + CDy * k6_5_5_2;
    const double h12_2_27 = acc[643] + ABy * acc[271];
    const double h6_2_27 = acc[364] + ABy * acc[85];
    const double h6_5_27 = h12_2_27 + ABx * h6_2_27;
    const double k6_5_13_3 = h6_5_27 + CDz * h6_5_13;
    const double k6_5_5_8 = k6_5_13_3 + CDy * k6_5_5_3;
    const double h12_2_28 = acc[644] + ABy * acc[272];
    const double h6_2_28 = acc[365] + ABy * acc[86];
    const double h6_5_28 = h12_2_28 + ABx * h6_2_28;
    const double k6_5_15_3 = h6_5_28 + CDz * h6_5_15;
    const double k6_5_5_9 = k6_5_15_3 + CDz * k6_5_5_3;
    const double k6_5_12_1 = h6_5_22 + CDx * h6_5_12;
    const double h12_2_6 = acc[622] + ABy * acc[250];
    const double h6_2_6 = acc[343] + ABy * acc[64];
    const double h6_5_6 = h12_2_6 + ABx * h6_2_6;
    const double k6_5_6_1 = h6_5_12 + CDx * h6_5_6;
    const double k6_5_6_4 = k6_5_12_1 + CDx * k6_5_6_1;
    const double k6_5_12_2 = h6_5_24 + CDy * h6_5_12;
    const double k6_5_6_2 = h6_5_15 + CDy * h6_5_6;
    const double k6_5_6_5 = k6_5_12_2 + CDx * k6_5_6_2;
    const double h12_2_14 = acc[630] + ABy * acc[258];
    const double h6_2_14 = acc[351] + ABy * acc[72];
    const double h6_5_14 = h12_2_14 + ABx * h6_2_14;
    const double k6_5_6_3 = h6_5_14 + CDz * h6_5_6;
    const double k6_5_6_6 = k6_5_12_3 + CDx * k6_5_6_3;
    const double k6_5_15_2 = h6_5_27 + CDy * h6_5_15;
    const double k6_5_6_7 = k6_5_15_2 + CDy * k6_5_6_2;
    const double k6_5_6_8 = k6_5_15_3 + CDy * k6_5_6_3;
    const double h12_2_29 = acc[645] + ABy * acc[273];
    const double h6_2_29 = acc[366] + ABy * acc[87];
    const double h6_5_29 = h12_2_29 + ABx * h6_2_29;
    const double k6_5_14_3 = h6_5_29 + CDz * h6_5_14;
    const double k6_5_6_9 = k6_5_14_3 + CDz * k6_5_6_3;
    const double k6_5_13_1 = h6_5_23 + CDx * h6_5_13;
    const double h12_2_7 = acc[623] + ABy * acc[251];
    const double h6_2_7 = acc[344] + ABy * acc[65];
    const double h6_5_7 = h12_2_7 + ABx * h6_2_7;
    const double k6_5_7_1 = h6_5_13 + CDx * h6_5_7;
    const double k6_5_7_4 = k6_5_13_1 + CDx * k6_5_7_1;
    const double h12_2_16 = acc[632] + ABy * acc[260];
    const double h6_2_16 = acc[353] + ABy * acc[74];
    const double h6_5_16 = h12_2_16 + ABx * h6_2_16;
    const double k6_5_7_2 = h6_5_16 + CDy * h6_5_7;
    const double k6_5_7_5 = k6_5_13_2 + CDx * k6_5_7_2;
    const double h12_2_17 = acc[633] + ABy * acc[261];
    const double h6_2_17 = acc[354] + ABy * acc[75];
    const double h6_5_17 = h12_2_17 + ABx * h6_2_17;
    const double k6_5_7_3 = h6_5_17 + CDz * h6_5_7;
    const double k6_5_7_6 = k6_5_13_3 + CDx * k6_5_7_3;
    const double h12_2_30 = acc[646] + ABy * acc[274];
    const double h6_2_30 = acc[367] + ABy * acc[88];
    const double h6_5_30 = h12_2_30 + ABx * h6_2_30;
    const double k6_5_16_2 = h6_5_30 + CDy * h6_5_16;
    const double k6_5_7_7 = k6_5_16_2 + CDy * k6_5_7_2;
    const double h12_2_31 = acc[647] + ABy * acc[275];
    const double h6_2_31 = acc[368] + ABy * acc[89];
    const double h6_5_31 = h12_2_31 + ABx * h6_2_31;
    const double k6_5_16_3 = h6_5_31 + CDz * h6_5_16;
    const double k6_5_7_8 = k6_5_16_3 + CDy * k6_5_7_3;
    const double h12_2_32 = acc[648] + ABy * acc[276];
    const double h6_2_32 = acc[369] + ABy * acc[90];
    const double h6_5_32 = h12_2_32 + ABx * h6_2_32;
    const double k6_5_17_3 = h6_5_32 + CDz * h6_5_17;
    const double k6_5_7_9 = k6_5_17_3 + CDz * k6_5_7_3;
    const double k6_5_15_1 = h6_5_24 + CDx * h6_5_15;
    const double h12_2_8 = acc[624] + ABy * acc[252];
    const double h6_2_8 = acc[345] + ABy * acc[66];
    const double h6_5_8 = h12_2_8 + ABx * h6_2_8;
    const double k6_5_8_1 = h6_5_15 + CDx * h6_5_8;
    const double k6_5_8_4 = k6_5_15_1 + CDx * k6_5_8_1;
    const double k6_5_8_2 = h6_5_17 + CDy * h6_5_8;
    const double k6_5_8_5 = k6_5_15_2 + CDx * k6_5_8_2;
    const double h12_2_18 = acc[634] + ABy * acc[262];
    const double h6_2_18 = acc[355] + ABy * acc[76];
    const double h6_5_18 = h12_2_18 + ABx * h6_2_18;
    const double k6_5_8_3 = h6_5_18 + CDz * h6_5_8;
    const double k6_5_8_6 = k6_5_15_3 + CDx * k6_5_8_3;
    const double k6_5_17_2 = h6_5_31 + CDy * h6_5_17;
    const double k6_5_8_7 = k6_5_17_2 + CDy * k6_5_8_2;
    const double k6_5_8_8 = k6_5_17_3 + CDy * k6_5_8_3;
    const double h12_2_33 = acc[649] + ABy * acc[277];
    const double h6_2_33 = acc[370] + ABy * acc[91];
    const double h6_5_33 = h12_2_33 + ABx * h6_2_33;
    const double k6_5_18_3 = h6_5_33 + CDz * h6_5_18;
    const double k6_5_8_9 = k6_5_18_3 + CDz * k6_5_8_3;
    const double k6_5_14_1 = h6_5_25 + CDx * h6_5_14;
    const double h12_2_9 = acc[625] + ABy * acc[253];
    const double h6_2_9 = acc[346] + ABy * acc[67];
    const double h6_5_9 = h12_2_9 + ABx * h6_2_9;
    const double k6_5_9_1 = h6_5_14 + CDx * h6_5_9;
    const double k6_5_9_4 = k6_5_14_1 + CDx * k6_5_9_1;
    const double k6_5_14_2 = h6_5_28 + CDy * h6_5_14;
    const double k6_5_9_2 = h6_5_18 + CDy * h6_5_9;
    const double k6_5_9_5 = k6_5_14_2 + CDx * k6_5_9_2;
    const double h12_2_19 = acc[635] + ABy * acc[263];
    const double h6_2_19 = acc[356] + ABy * acc[77];
    const double h6_5_19 = h12_2_19 + ABx * h6_2_19;
    const double k6_5_9_3 = h6_5_19 + CDz * h6_5_9;
    const double k6_5_9_6 = k6_5_14_3 + CDx * k6_5_9_3;
    const double k6_5_18_2 = h6_5_32 + CDy * h6_5_18;
    const double k6_5_9_7 = k6_5_18_2 + CDy * k6_5_9_2;
    const double k6_5_9_8 = k6_5_18_3 + CDy * k6_5_9_3;
    const double h12_2_34 = acc[650] + ABy * acc[278];
    const double h6_2_34 = acc[371] + ABy * acc[92];
    const double h6_5_34 = h12_2_34 + ABx * h6_2_34;
    const double k6_5_19_3 = h6_5_34 + CDz * h6_5_19;
    const double k6_5_9_9 = k6_5_19_3 + CDz * k6_5_9_3;
    const double h6_3_20 = acc[326] + ABz * acc[78];
    const double h6_6_20 = h12_3_20 + ABx * h6_3_20;
    const double h6_3_10 = acc[316] + ABz * acc[68];
    const double h6_6_10 = h12_3_10 + ABx * h6_3_10;
    const double k6_6_10_1 = h6_6_20 + CDx * h6_6_10;
    const double h6_3_4 = acc[310] + ABz * acc[62];
    const double h6_6_4 = h12_3_4 + ABx * h6_3_4;
    const double k6_6_4_1 = h6_6_10 + CDx * h6_6_4;
    const double k6_6_4_4 = k6_6_10_1 + CDx * k6_6_4_1;
    const double h6_3_21 = acc[327] + ABz * acc[79];
    const double h6_6_21 = h12_3_21 + ABx * h6_3_21;
    const double k6_6_10_2 = h6_6_21 + CDy * h6_6_10;
    const double h6_3_11 = acc[317] + ABz * acc[69];
    const double h6_6_11 = h12_3_11 + ABx * h6_3_11;
    const double k6_6_4_2 = h6_6_11 + CDy * h6_6_4;
    const double k6_6_4_5 = k6_6_10_2 + CDx * k6_6_4_2;
    const double h6_3_22 = acc[328] + ABz * acc[80];
    const double h6_6_22 = h12_3_22 + ABx * h6_3_22;
    const double k6_6_10_3 = h6_6_22 + CDz * h6_6_10;
    const double h6_3_12 = acc[318] + ABz * acc[70];
    const double h6_6_12 = h12_3_12 + ABx * h6_3_12;
    const double k6_6_4_3 = h6_6_12 + CDz * h6_6_4;
    const double k6_6_4_6 = k6_6_10_3 + CDx * k6_6_4_3;
    const double h6_3_23 = acc[329] + ABz * acc[81];
    const double h6_6_23 = h12_3_23 + ABx * h6_3_23;
    const double k6_6_11_2 = h6_6_23 + CDy * h6_6_11;
    const double k6_6_4_7 = k6_6_11_2 + CDy * k6_6_4_2;
    const double h6_3_24 = acc[330] + ABz * acc[82];
    const double h6_6_24 = h12_3_24 + ABx * h6_3_24;
    const double k6_6_11_3 = h6_6_24 + CDz * h6_6_11;
    const double k6_6_4_8 = k6_6_11_3 + CDy * k6_6_4_3;
    const double h6_3_25 = acc[331] + ABz * acc[83];
    const double h6_6_25 = h12_3_25 + ABx * h6_3_25;
    const double k6_6_12_3 = h6_6_25 + CDz * h6_6_12;
    const double k6_6_4_9 = k6_6_12_3 + CDz * k6_6_4_3;
    const double k6_6_11_1 = h6_6_21 + CDx * h6_6_11;
    const double h6_3_5 = acc[311] + ABz * acc[63];
    const double h6_6_5 = h12_3_5 + ABx * h6_3_5;
    const double k6_6_5_1 = h6_6_11 + CDx * h6_6_5;
    const double k6_6_5_4 = k6_6_11_1 + CDx * k6_6_5_1;
    const double h6_3_13 = acc[319] + ABz * acc[71];
    const double h6_6_13 = h12_3_13 + ABx * h6_3_13;
    const double k6_6_5_2 = h6_6_13 + CDy * h6_6_5;
    const double k6_6_5_5 = k6_6_11_2 + CDx * k6_6_5_2;
    const double h6_3_15 = acc[321] + ABz * acc[73];
    const double h6_6_15 = h12_3_15 + ABx * h6_3_15;
    const double k6_6_5_3 = h6_6_15 + CDz * h6_6_5;
    const double k6_6_5_6 = k6_6_11_3 + CDx * k6_6_5_3;
    const double h6_3_26 = acc[332] + ABz * acc[84];
    const double h6_6_26 = h12_3_26 + ABx * h6_3_26;
    const double k6_6_13_2 = h6_6_26 + CDy * h6_6_13;
    const double k6_6_5_7 = k6_6_13_2 + CDy * k6_6_5_2;
    const double h6_3_27 = acc[333] + ABz * acc[85];
    const double h6_6_27 = h12_3_27 + ABx * h6_3_27;
    const double k6_6_13_3 = h6_6_27 + CDz * h6_6_13;
    const double k6_6_5_8 = k6_6_13_3 + CDy * k6_6_5_3;
    const double h6_3_28 = acc[334] + ABz * acc[86];
    const double h6_6_28 = h12_3_28 + ABx * h6_3_28;
    const double k6_6_15_3 = h6_6_28 + CDz * h6_6_15;
    const double k6_6_5_9 = k6_6_15_3 + CDz * k6_6_5_3;
    const double k6_6_12_1 = h6_6_22 + CDx * h6_6_12;
    const double h6_3_6 = acc[312] + ABz * acc[64];
    const double h6_6_6 = h12_3_6 + ABx * h6_3_6;
    const double k6_6_6_1 = h6_6_12 + CDx * h6_6_6;
    const double k6_6_6_4 = k6_6_12_1 + CDx * k6_6_6_1;
    const double k6_6_12_2 = h6_6_24 + CDy * h6_6_12;
    const double k6_6_6_2 = h6_6_15 + CDy * h6_6_6;
    const double k6_6_6_5 = k6_6_12_2 + CDx * k6_6_6_2;
    const double h6_3_14 = acc[320] + ABz * acc[72];
    const double h6_6_14 = h12_3_14 + ABx * h6_3_14;
    const double k6_6_6_3 = h6_6_14 + CDz * h6_6_6;
    const double k6_6_6_6 = k6_6_12_3 + CDx * k6_6_6_3;
    const double k6_6_15_2 = h6_6_27 + CDy * h6_6_15;
    const double k6_6_6_7 = k6_6_15_2 + CDy * k6_6_6_2;
    const double k6_6_6_8 = k6_6_15_3 + CDy * k6_6_6_3;
    const double h6_3_29 = acc[335] + ABz * acc[87];
    const double h6_6_29 = h12_3_29 + ABx * h6_3_29;
    const double k6_6_14_3 = h6_6_29 + CDz * h6_6_14;
    const double k6_6_6_9 = k6_6_14_3 + CDz * k6_6_6_3;
    const double k6_6_13_1 = h6_6_23 + CDx * h6_6_13;
    const double h6_3_7 = acc[313] + ABz * acc[65];
    const double h6_6_7 = h12_3_7 + ABx * h6_3_7;
    const double k6_6_7_1 = h6_6_13 + CDx * h6_6_7;
    const double k6_6_7_4 = k6_6_13_1 + CDx * k6_6_7_1;
    const double h6_3_16 = acc[322] + ABz * acc[74];
    const double h6_6_16 = h12_3_16 + ABx * h6_3_16;
    const double k6_6_7_2 = h6_6_16 + CDy * h6_6_7;
    const double k6_6_7_5 = k6_6_13_2 + CDx * k6_6_7_2;
    const double h6_3_17 = acc[323] + ABz * acc[75];
    const double h6_6_17 = h12_3_17 + ABx * h6_3_17;
    const double k6_6_7_3 = h6_6_17 + CDz * h6_6_7;
    const double k6_6_7_6 = k6_6_13_3 + CDx * k6_6_7_3;
    const double h6_3_30 = acc[336] + ABz * acc[88];
    const double h6_6_30 = h12_3_30 + ABx * h6_3_30;
    const double k6_6_16_2 = h6_6_30 + CDy * h6_6_16;
    const double k6_6_7_7 = k6_6_16_2 + CDy * k6_6_7_2;
    const double h6_3_31 = acc[337] + ABz * acc[89];
    const double h6_6_31 = h12_3_31 + ABx * h6_3_31;
    const double k6_6_16_3 = h6_6_31 + CDz * h6_6_16;
    const double k6_6_7_8 = k6_6_16_3 + CDy * k6_6_7_3;
    const double h6_3_32 = acc[338] + ABz * acc[90];
    const double h6_6_32 = h12_3_32 + ABx * h6_3_32;
    const double k6_6_17_3 = h6_6_32 + CDz * h6_6_17;
    const double k6_6_7_9 = k6_6_17_3 + CDz * k6_6_7_3;
    const double k6_6_15_1 = h6_6_24 + CDx * h6_6_15;
    const double h6_3_8 = acc[314] + ABz * acc[66];
    const double h6_6_8 = h12_3_8 + ABx * h6_3_8;
    const double k6_6_8_1 = h6_6_15 + CDx * h6_6_8;
    const double k6_6_8_4 = k6_6_15_1 + CDx * k6_6_8_1;
    const double k6_6_8_2 = h6_6_17 + CDy * h6_6_8;
    const double k6_6_8_5 = k6_6_15_2 + CDx * k6_6_8_2;
    const double h6_3_18 = acc[324] + ABz * acc[76];
    const double h6_6_18 = h12_3_18 + ABx * h6_3_18;
    const double k6_6_8_3 = h6_6_18 + CDz * h6_6_8;
    const double k6_6_8_6 = k6_6_15_3 + CDx * k6_6_8_3;
    const double k6_6_17_2 = h6_6_31 + CDy * h6_6_17;
    const double k6_6_8_7 = k6_6_17_2 + CDy * k6_6_8_2;
    const double k6_6_8_8 = k6_6_17_3 + CDy * k6_6_8_3;
    const double h6_3_33 = acc[339] + ABz * acc[91];
    const double h6_6_33 = h12_3_33 + ABx * h6_3_33;
    const double k6_6_18_3 = h6_6_33 + CDz * h6_6_18;
    const double k6_6_8_9 = k6_6_18_3 + CDz * k6_6_8_3;
    const double k6_6_14_1 = h6_6_25 + CDx * h6_6_14;
    const double h6_3_9 = acc[315] + ABz * acc[67];
    const double h6_6_9 = h12_3_9 + ABx * h6_3_9;
    const double k6_6_9_1 = h6_6_14 + CDx * h6_6_9;
    const double k6_6_9_4 = k6_6_14_1 + CDx * k6_6_9_1;
    const double k6_6_14_2 = h6_6_28 + CDy * h6_6_14;
    const double k6_6_9_2 = h6_6_18 + CDy * h6_6_9;
    const double k6_6_9_5 = k6_6_14_2 + CDx * k6_6_9_2;
    const double h6_3_19 = acc[325] + ABz * acc[77];
    const double h6_6_19 = h12_3_19 + ABx * h6_3_19;
    const double k6_6_9_3 = h6_6_19 + CDz * h6_6_9;
    const double k6_6_9_6 = k6_6_14_3 + CDx * k6_6_9_3;
    const double k6_6_18_2 = h6_6_32 + CDy * h6_6_18;
    const double k6_6_9_7 = k6_6_18_2 + CDy * k6_6_9_2;
    const double k6_6_9_8 = k6_6_18_3 + CDy * k6_6_9_3;
    const double h6_3_34 = acc[340] + ABz * acc[92];
    const double h6_6_34 = h12_3_34 + ABx * h6_3_34;
    const double k6_6_19_3 = h6_6_34 + CDz * h6_6_19;
    const double k6_6_9_9 = k6_6_19_3 + CDz * k6_6_9_3;
    const double h15_2_20 = acc[729] + ABy * acc[357];
    const double h6_7_20 = h15_2_20 + ABy * h6_2_20;
    const double h15_2_10 = acc[719] + ABy * acc[347];
    const double h6_7_10 = h15_2_10 + ABy * h6_2_10;
    const double k6_7_10_1 = h6_7_20 + CDx * h6_7_10;
    const double h15_2_4 = acc[713] + ABy * acc[341];
    const double h6_7_4 = h15_2_4 + ABy * h6_2_4;
    const double k6_7_4_1 = h6_7_10 + CDx * h6_7_4;
    const double k6_7_4_4 = k6_7_10_1 + CDx * k6_7_4_1;
    const double h15_2_21 = acc[730] + ABy * acc[358];
    const double h6_7_21 = h15_2_21 + ABy * h6_2_21;
    const double k6_7_10_2 = h6_7_21 + CDy * h6_7_10;
    const double h15_2_11 = acc[720] + ABy * acc[348];
    const double h6_7_11 = h15_2_11 + ABy * h6_2_11;
    const double k6_7_4_2 = h6_7_11 + CDy * h6_7_4;
    const double k6_7_4_5 = k6_7_10_2 + CDx * k6_7_4_2;
    const double h15_2_22 = acc[731] + ABy * acc[359];
    const double h6_7_22 = h15_2_22 + ABy * h6_2_22;
    const double k6_7_10_3 = h6_7_22 + CDz * h6_7_10;
    const double h15_2_12 = acc[721] + ABy * acc[349];
    const double h6_7_12 = h15_2_12 + ABy * h6_2_12;
    const double k6_7_4_3 = h6_7_12 + CDz * h6_7_4;
    const double k6_7_4_6 = k6_7_10_3 + CDx * k6_7_4_3;
    const double h15_2_23 = acc[732] + ABy * acc[360];
    const double h6_7_23 = h15_2_23 + ABy * h6_2_23;
    const double k6_7_11_2 = h6_7_23 + CDy * h6_7_11;
    const double k6_7_4_7 = k6_7_11_2 + CDy * k6_7_4_2;
    const double h15_2_24 = acc[733] + ABy * acc[361];
    const double h6_7_24 = h15_2_24 + ABy * h6_2_24;
    const double k6_7_11_3 = h6_7_24 + CDz * h6_7_11;
    const double k6_7_4_8 = k6_7_11_3 + CDy * k6_7_4_3;
    const double h15_2_25 = acc[734] + ABy * acc[362];
    const double h6_7_25 = h15_2_25 + ABy * h6_2_25;
    const double k6_7_12_3 = h6_7_25 + CDz * h6_7_12;
    const double k6_7_4_9 = k6_7_12_3 + CDz * k6_7_4_3;
    const double k6_7_11_1 = h6_7_21 + CDx * h6_7_11;
    const double h15_2_5 = acc[714] + ABy * acc[342];
    const double h6_7_5 = h15_2_5 + ABy * h6_2_5;
    const double k6_7_5_1 = h6_7_11 + CDx * h6_7_5;
    const double k6_7_5_4 = k6_7_11_1 + CDx * k6_7_5_1;
    const double h15_2_13 = acc[722] + ABy * acc[350];
    const double h6_7_13 = h15_2_13 + ABy * h6_2_13;
    const double k6_7_5_2 = h6_7_13 + CDy * h6_7_5;
    const double k6_7_5_5 = k6_7_11_2 + CDx * k6_7_5_2;
    const double h15_2_15 = acc[724] + ABy * acc[352];
    const double h6_7_15 = h15_2_15 + ABy * h6_2_15;
    const double k6_7_5_3 = h6_7_15 + CDz * h6_7_5;
    const double k6_7_5_6 = k6_7_11_3 + CDx * k6_7_5_3;
    const double h15_2_26 = acc[735] + ABy * acc[363];
    const double h6_7_26 = h15_2_26 + ABy * h6_2_26;
    const double k6_7_13_2 = h6_7_26 + CDy * h6_7_13;
    const double k6_7_5_7 = k6_7_13_2 + CDy * k6_7_5_2;
    const double h15_2_27 = acc[736] + ABy * acc[364];
    const double h6_7_27 = h15_2_27 + ABy * h6_2_27;
    const double k6_7_13_3 = h6_7_27 + CDz * h6_7_13;
    const double k6_7_5_8 = k6_7_13_3 + CDy * k6_7_5_3;
    const double h15_2_28 = acc[737] + ABy * acc[365];
    const double h6_7_28 = h15_2_28 + ABy * h6_2_28;
    const double k6_7_15_3 = h6_7_28 + CDz * h6_7_15;
    const double k6_7_5_9 = k6_7_15_3 + CDz * k6_7_5_3;
    const double k6_7_12_1 = h6_7_22 + CDx * h6_7_12;
    const double h15_2_6 = acc[715] + ABy * acc[343];
    const double h6_7_6 = h15_2_6 + ABy * h6_2_6;
    const double k6_7_6_1 = h6_7_12 + CDx * h6_7_6;
    const double k6_7_6_4 = k6_7_12_1 + CDx * k6_7_6_1;
    const double k6_7_12_2 = h6_7_24 + CDy * h6_7_12;
    const double k6_7_6_2 = h6_7_15 + CDy * h6_7_6;
    const double k6_7_6_5 = k6_7_12_2 + CDx * k6_7_6_2;
    const double h15_2_14 = acc[723] + ABy * acc[351];
    const double h6_7_14 = h15_2_14 + ABy * h6_2_14;
    const double k6_7_6_3 = h6_7_14 + CDz * h6_7_6;
    const double k6_7_6_6 = k6_7_12_3 + CDx * k6_7_6_3;
    const double k6_7_15_2 = h6_7_27 + CDy * h6_7_15;
    const double k6_7_6_7 = k6_7_15_2 + CDy * k6_7_6_2;
    const double k6_7_6_8 = k6_7_15_3 + CDy * k6_7_6_3;
    const double h15_2_29 = acc[738] + ABy * acc[366];
    const double h6_7_29 = h15_2_29 + ABy * h6_2_29;
    const double k6_7_14_3 = h6_7_29 + CDz * h6_7_14;
    const double k6_7_6_9 = k6_7_14_3 + CDz * k6_7_6_3;
    const double k6_7_13_1 = h6_7_23 + CDx * h6_7_13;
    const double h15_2_7 = acc[716] + ABy * acc[344];
    const double h6_7_7 = h15_2_7 + ABy * h6_2_7;
    const double k6_7_7_1 = h6_7_13 + CDx * h6_7_7;
    const double k6_7_7_4 = k6_7_13_1 + CDx * k6_7_7_1;
    const double h15_2_16 = acc[725] + ABy * acc[353];
    const double h6_7_16 = h15_2_16 + ABy * h6_2_16;
    const double k6_7_7_2 = h6_7_16 + CDy * h6_7_7;
    const double k6_7_7_5 = k6_7_13_2 + CDx * k6_7_7_2;
    const double h15_2_17 = acc[726] + ABy * acc[354];
    const double h6_7_17 = h15_2_17 + ABy * h6_2_17;
    const double k6_7_7_3 = h6_7_17 + CDz * h6_7_7;
    const double k6_7_7_6 = k6_7_13_3 + CDx * k6_7_7_3;
    const double h15_2_30 = acc[739] + ABy * acc[367];
    const double h6_7_30 = h15_2_30 + ABy * h6_2_30;
    const double k6_7_16_2 = h6_7_30 + CDy * h6_7_16;
    const double k6_7_7_7 = k6_7_16_2 + CDy * k6_7_7_2;
    const double h15_2_31 = acc[740] + ABy * acc[368];
    const double h6_7_31 = h15_2_31 + ABy * h6_2_31;
    const double k6_7_16_3 = h6_7_31 + CDz * h6_7_16;
    const double k6_7_7_8 = k6_7_16_3 + CDy * k6_7_7_3;
    const double h15_2_32 = acc[741] + ABy * acc[369];
    const double h6_7_32 = h15_2_32 + ABy * h6_2_32;
    const double k6_7_17_3 = h6_7_32 + CDz * h6_7_17;
    const double k6_7_7_9 = k6_7_17_3 + CDz * k6_7_7_3;
    const double k6_7_15_1 = h6_7_24 + CDx * h6_7_15;
    const double h15_2_8 = acc[717] + ABy * acc[345];
    const double h6_7_8 = h15_2_8 + ABy * h6_2_8;
    const double k6_7_8_1 = h6_7_15 + CDx * h6_7_8;
    const double k6_7_8_4 = k6_7_15_1 + CDx * k6_7_8_1;
    const double k6_7_8_2 = h6_7_17 + CDy * h6_7_8;
    const double k6_7_8_5 = k6_7_15_2 + CDx * k6_7_8_2;
    const double h15_2_18 = acc[727] + ABy * acc[355];
    const double h6_7_18 = h15_2_18 + ABy * h6_2_18;
    const double k6_7_8_3 = h6_7_18 + CDz * h6_7_8;
    const double k6_7_8_6 = k6_7_15_3 + CDx * k6_7_8_3;
    const double k6_7_17_2 = h6_7_31 + CDy * h6_7_17;
    const double k6_7_8_7 = k6_7_17_2 + CDy * k6_7_8_2;
    const double k6_7_8_8 = k6_7_17_3 + CDy * k6_7_8_3;
    const double h15_2_33 = acc[742] + ABy * acc[370];
    const double h6_7_33 = h15_2_33 + ABy * h6_2_33;
    const double k6_7_18_3 = h6_7_33 + CDz * h6_7_18;
    const double k6_7_8_9 = k6_7_18_3 + CDz * k6_7_8_3;
    const double k6_7_14_1 = h6_7_25 + CDx * h6_7_14;
    const double h15_2_9 = acc[718] + ABy * acc[346];
    const double h6_7_9 = h15_2_9 + ABy * h6_2_9;
    const double k6_7_9_1 = h6_7_14 + CDx * h6_7_9;
    const double k6_7_9_4 = k6_7_14_1 + CDx * k6_7_9_1;
    const double k6_7_14_2 = h6_7_28 + CDy * h6_7_14;
    const double k6_7_9_2 = h6_7_18 + CDy * h6_7_9;
    const double k6_7_9_5 = k6_7_14_2 + CDx * k6_7_9_2;
    const double h15_2_19 = acc[728] + ABy * acc[356];
    const double h6_7_19 = h15_2_19 + ABy * h6_2_19;
    const double k6_7_9_3 = h6_7_19 + CDz * h6_7_9;
    const double k6_7_9_6 = k6_7_14_3 + CDx * k6_7_9_3;
    const double k6_7_18_2 = h6_7_32 + CDy * h6_7_18;
    const double k6_7_9_7 = k6_7_18_2 + CDy * k6_7_9_2;
    const double k6_7_9_8 = k6_7_18_3 + CDy * k6_7_9_3;
    const double h15_2_34 = acc[743] + ABy * acc[371];
    const double h6_7_34 = h15_2_34 + ABy * h6_2_34;
    const double k6_7_19_3 = h6_7_34 + CDz * h6_7_19;
    const double k6_7_9_9 = k6_7_19_3 + CDz * k6_7_9_3;
    const double h6_8_20 = h15_3_20 + ABy * h6_3_20;
    const double h6_8_10 = h15_3_10 + ABy * h6_3_10;
    const double k6_8_10_1 = h6_8_20 + CDx * h6_8_10;
    const double h6_8_4 = h15_3_4 + ABy * h6_3_4;
    const double k6_8_4_1 = h6_8_10 + CDx * h6_8_4;
    const double k6_8_4_4 = k6_8_10_1 + CDx * k6_8_4_1;
    const double h6_8_21 = h15_3_21 + ABy * h6_3_21;
    const double k6_8_10_2 = h6_8_21 + CDy * h6_8_10;
    const double h6_8_11 = h15_3_11 + ABy * h6_3_11;
    const double k6_8_4_2 = h6_8_11 + CDy * h6_8_4;
    const double k6_8_4_5 = k6_8_10_2 + CDx * k6_8_4_2;
    const double h6_8_22 = h15_3_22 + ABy * h6_3_22;
    const double k6_8_10_3 = h6_8_22 + CDz * h6_8_10;
    const double h6_8_12 = h15_3_12 + ABy * h6_3_12;
    const double k6_8_4_3 = h6_8_12 + CDz * h6_8_4;
    const double k6_8_4_6 = k6_8_10_3 + CDx * k6_8_4_3;
    const double h6_8_23 = h15_3_23 + ABy * h6_3_23;
    const double k6_8_11_2 = h6_8_23 + CDy * h6_8_11;
    const double k6_8_4_7 = k6_8_11_2 + CDy * k6_8_4_2;
    const double h6_8_24 = h15_3_24 + ABy * h6_3_24;
    const double k6_8_11_3 = h6_8_24 + CDz * h6_8_11;
    const double k6_8_4_8 = k6_8_11_3 + CDy * k6_8_4_3;
    const double h6_8_25 = h15_3_25 + ABy * h6_3_25;
    const double k6_8_12_3 = h6_8_25 + CDz * h6_8_12;
    const double k6_8_4_9 = k6_8_12_3 + CDz * k6_8_4_3;
    const double k6_8_11_1 = h6_8_21 + CDx * h6_8_11;
    const double h6_8_5 = h15_3_5 + ABy * h6_3_5;
    const double k6_8_5_1 = h6_8_11 + CDx * h6_8_5;
    const double k6_8_5_4 = k6_8_11_1 + CDx * k6_8_5_1;
    const double h6_8_13 = h15_3_13 + ABy * h6_3_13;
    const double k6_8_5_2 = h6_8_13 + CDy * h6_8_5;
    const double k6_8_5_5 = k6_8_11_2 + CDx * k6_8_5_2;
    const double h6_8_15 = h15_3_15 + ABy * h6_3_15;
    const double k6_8_5_3 = h6_8_15 + CDz * h6_8_5;
    const double k6_8_5_6 = k6_8_11_3 + CDx * k6_8_5_3;
    const double h6_8_26 = h15_3_26 + ABy * h6_3_26;
    const double k6_8_13_2 = h6_8_26 + CDy * h6_8_13;
    const double k6_8_5_7 = k6_8_13_2 + CDy * k6_8_5_2;
    const double h6_8_27 = h15_3_27 + ABy * h6_3_27;
    const double k6_8_13_3 = h6_8_27 + CDz * h6_8_13;
    const double k6_8_5_8 = k6_8_13_3 + CDy * k6_8_5_3;
    const double h6_8_28 = h15_3_28 + ABy * h6_3_28;
    const double k6_8_15_3 = h6_8_28 + CDz * h6_8_15;
    const double k6_8_5_9 = k6_8_15_3 + CDz * k6_8_5_3;
    const double k6_8_12_1 = h6_8_22 + CDx * h6_8_12;
    const double h6_8_6 = h15_3_6 + ABy * h6_3_6;
    const double k6_8_6_1 = h6_8_12 + CDx * h6_8_6;
    const double k6_8_6_4 = k6_8_12_1 + CDx * k6_8_6_1;
    const double k6_8_12_2 = h6_8_24 + CDy * h6_8_12;
    const double k6_8_6_2 = h6_8_15 + CDy * h6_8_6;
    const double k6_8_6_5 = k6_8_12_2 + CDx * k6_8_6_2;
    const double h6_8_14 = h15_3_14 + ABy * h6_3_14;
    const double k6_8_6_3 = h6_8_14 + CDz * h6_8_6;
    const double k6_8_6_6 = k6_8_12_3 + CDx * k6_8_6_3;
    const double k6_8_15_2 = h6_8_27 + CDy * h6_8_15;
    const double k6_8_6_7 = k6_8_15_2 + CDy * k6_8_6_2;
    const double k6_8_6_8 = k6_8_15_3 + CDy * k6_8_6_3;
    const double h6_8_29 = h15_3_29 + ABy * h6_3_29;
    const double k6_8_14_3 = h6_8_29 + CDz * h6_8_14;
    const double k6_8_6_9 = k6_8_14_3 + CDz * k6_8_6_3;
    const double k6_8_13_1 = h6_8_23 + CDx * h6_8_13;
    const double h6_8_7 = h15_3_7 + ABy * h6_3_7;
    const double k6_8_7_1 = h6_8_13 + CDx * h6_8_7;
    const double k6_8_7_4 = k6_8_13_1 + CDx * k6_8_7_1;
    const double h6_8_16 = h15_3_16 + ABy * h6_3_16;
    const double k6_8_7_2 = h6_8_16 + CDy * h6_8_7;
    const double k6_8_7_5 = k6_8_13_2 + CDx * k6_8_7_2;
    const double h6_8_17 = h15_3_17 + ABy * h6_3_17;
    const double k6_8_7_3 = h6_8_17 + CDz * h6_8_7;
    const double k6_8_7_6 = k6_8_13_3 + CDx * k6_8_7_3;
    const double h6_8_30 = h15_3_30 + ABy * h6_3_30;
    const double k6_8_16_2 = h6_8_30 + CDy * h6_8_16;
    const double k6_8_7_7 = k6_8_16_2 + CDy * k6_8_7_2;
    const double h6_8_31 = h15_3_31 + ABy * h6_3_31;
    const double k6_8_16_3 = h6_8_31 + CDz * h6_8_16;
    const double k6_8_7_8 = k6_8_16_3 + CDy * k6_8_7_3;
    const double h6_8_32 = h15_3_32 + ABy * h6_3_32;
    const double k6_8_17_3 = h6_8_32 + CDz * h6_8_17;
    const double k6_8_7_9 = k6_8_17_3 + CDz * k6_8_7_3;
    const double k6_8_15_1 = h6_8_24 + CDx * h6_8_15;
    const double h6_8_8 = h15_3_8 + ABy * h6_3_8;
    const double k6_8_8_1 = h6_8_15 + CDx * h6_8_8;
    const double k6_8_8_4 = k6_8_15_1 + CDx * k6_8_8_1;
    const double k6_8_8_2 = h6_8_17 + CDy * h6_8_8;
    const double k6_8_8_5 = k6_8_15_2 + CDx * k6_8_8_2;
    const double h6_8_18 = h15_3_18 + ABy * h6_3_18;
    const double k6_8_8_3 = h6_8_18 + CDz * h6_8_8;
    const double k6_8_8_6 = k6_8_15_3 + CDx * k6_8_8_3;
    const double k6_8_17_2 = h6_8_31 + CDy * h6_8_17;
    const double k6_8_8_7 = k6_8_17_2 + CDy * k6_8_8_2;
    const double k6_8_8_8 = k6_8_17_3 + CDy * k6_8_8_3;
    const double h6_8_33 = h15_3_33 + ABy * h6_3_33;
    const double k6_8_18_3 = h6_8_33 + CDz * h6_8_18;
    const double k6_8_8_9 = k6_8_18_3 + CDz * k6_8_8_3;
    const double k6_8_14_1 = h6_8_25 + CDx * h6_8_14;
    const double h6_8_9 = h15_3_9 + ABy * h6_3_9;
    const double k6_8_9_1 = h6_8_14 + CDx * h6_8_9;
    const double k6_8_9_4 = k6_8_14_1 + CDx * k6_8_9_1;
    const double k6_8_14_2 = h6_8_28 + CDy * h6_8_14;
    const double k6_8_9_2 = h6_8_18 + CDy * h6_8_9;
    const double k6_8_9_5 = k6_8_14_2 + CDx * k6_8_9_2;
    const double h6_8_19 = h15_3_19 + ABy * h6_3_19;
    const double k6_8_9_3 = h6_8_19 + CDz * h6_8_9;
    const double k6_8_9_6 = k6_8_14_3 + CDx * k6_8_9_3;
    const double k6_8_18_2 = h6_8_32 + CDy * h6_8_18;
    const double k6_8_9_7 = k6_8_18_2 + CDy * k6_8_9_2;
    const double k6_8_9_8 = k6_8_18_3 + CDy * k6_8_9_3;
    const double h6_8_34 = h15_3_34 + ABy * h6_3_34;
    const double k6_8_19_3 = h6_8_34 + CDz * h6_8_19;
    const double k6_8_9_9 = k6_8_19_3 + CDz * k6_8_9_3;
    const double h14_3_20 = acc[791] + ABz * acc[326];
    const double h6_9_20 = h14_3_20 + ABz * h6_3_20;
    const double h14_3_10 = acc[781] + ABz * acc[316];
    const double h6_9_10 = h14_3_10 + ABz * h6_3_10;
    const double k6_9_10_1 = h6_9_20 + CDx * h6_9_10;
    const double h14_3_4 = acc[775] + ABz * acc[310];
    const double h6_9_4 = h14_3_4 + ABz * h6_3_4;
    const double k6_9_4_1 = h6_9_10 + CDx * h6_9_4;
    const double k6_9_4_4 = k6_9_10_1 + CDx * k6_9_4_1;
    const double h14_3_21 = acc[792] + ABz * acc[327];
    const double h6_9_21 = h14_3_21 + ABz * h6_3_21;
    const double k6_9_10_2 = h6_9_21 + CDy * h6_9_10;
    const double h14_3_11 = acc[782] + ABz * acc[317];
    const double h6_9_11 = h14_3_11 + ABz * h6_3_11;
    const double k6_9_4_2 = h6_9_11 + CDy * h6_9_4;
    const double k6_9_4_5 = k6_9_10_2 + CDx * k6_9_4_2;
    const double h14_3_22 = acc[793] + ABz * acc[328];
    const double h6_9_22 = h14_3_22 + ABz * h6_3_22;
    const double k6_9_10_3 = h6_9_22 + CDz * h6_9_10;
    const double h14_3_12 = acc[783] + ABz * acc[318];
    const double h6_9_12 = h14_3_12 + ABz * h6_3_12;
    const double k6_9_4_3 = h6_9_12 + CDz * h6_9_4;
    const double k6_9_4_6 = k6_9_10_3 + CDx * k6_9_4_3;
    const double h14_3_23 = acc[794] + ABz * acc[329];
    const double h6_9_23 = h14_3_23 + ABz * h6_3_23;
    const double k6_9_11_2 = h6_9_23 + CDy * h6_9_11;
    const double k6_9_4_7 = k6_9_11_2 + CDy * k6_9_4_2;
    const double h14_3_24 = acc[795] + ABz * acc[330];
    const double h6_9_24 = h14_3_24 + ABz * h6_3_24;
    const double k6_9_11_3 = h6_9_24 + CDz * h6_9_11;
    const double k6_9_4_8 = k6_9_11_3 + CDy * k6_9_4_3;
    const double h14_3_25 = acc[796] + ABz * acc[331];
    const double h6_9_25 = h14_3_25 + ABz * h6_3_25;
    const double k6_9_12_3 = h6_9_25 + CDz * h6_9_12;
    const double k6_9_4_9 = k6_9_12_3 + CDz * k6_9_4_3;
    const double k6_9_11_1 = h6_9_21 + CDx * h6_9_11;
    const double h14_3_5 = acc[776] + ABz * acc[311];
    const double h6_9_5 = h14_3_5 + ABz * h6_3_5;
    const double k6_9_5_1 = h6_9_11 + CDx * h6_9_5;
    const double k6_9_5_4 = k6_9_11_1 + CDx * k6_9_5_1;
    const double h14_3_13 = acc[784] + ABz * acc[319];
    const double h6_9_13 = h14_3_13 + ABz * h6_3_13;
    const double k6_9_5_2 = h6_9_13 + CDy * h6_9_5;
    const double k6_9_5_5 = k6_9_11_2 + CDx * k6_9_5_2;
    const double h14_3_15 = acc[786] + ABz * acc[321];
    const double h6_9_15 = h14_3_15 + ABz * h6_3_15;
    const double k6_9_5_3 = h6_9_15 + CDz * h6_9_5;
    const double k6_9_5_6 = k6_9_11_3 + CDx * k6_9_5_3;
    const double h14_3_26 = acc[797] + ABz * acc[332];
    const double h6_9_26 = h14_3_26 + ABz * h6_3_26;
    const double k6_9_13_2 = h6_9_26 + CDy * h6_9_13;
    const double k6_9_5_7 = k6_9_13_2 + CDy * k6_9_5_2;
    const double h14_3_27 = acc[798] + ABz * acc[333];
    const double h6_9_27 = h14_3_27 + ABz * h6_3_27;
    const double k6_9_13_3 = h6_9_27 + CDz * h6_9_13;
    const double k6_9_5_8 = k6_9_13_3 + CDy * k6_9_5_3;
    const double h14_3_28 = acc[799] + ABz * acc[334];
    const double h6_9_28 = h14_3_28 + ABz * h6_3_28;
    const double k6_9_15_3 = h6_9_28 + CDz * h6_9_15;
    const double k6_9_5_9 = k6_9_15_3 + CDz * k6_9_5_3;
    const double k6_9_12_1 = h6_9_22 + CDx * h6_9_12;
    const double h14_3_6 = acc[777] + ABz * acc[312];
    const double h6_9_6 = h14_3_6 + ABz * h6_3_6;
    const double k6_9_6_1 = h6_9_12 + CDx * h6_9_6;
    const double k6_9_6_4 = k6_9_12_1 + CDx * k6_9_6_1;
    const double k6_9_12_2 = h6_9_24 + CDy * h6_9_12;
    const double k6_9_6_2 = h6_9_15 + CDy * h6_9_6;
    const double k6_9_6_5 = k6_9_12_2 + CDx * k6_9_6_2;
    const double h14_3_14 = acc[785] + ABz * acc[320];
    const double h6_9_14 = h14_3_14 + ABz * h6_3_14;
    const double k6_9_6_3 = h6_9_14 + CDz * h6_9_6;
    const double k6_9_6_6 = k6_9_12_3 + CDx * k6_9_6_3;
    const double k6_9_15_2 = h6_9_27 + CDy * h6_9_15;
    const double k6_9_6_7 = k6_9_15_2 + CDy * k6_9_6_2;
    const double k6_9_6_8 = k6_9_15_3 + CDy * k6_9_6_3;
    const double h14_3_29 = acc[800] + ABz * acc[335];
    const double h6_9_29 = h14_3_29 + ABz * h6_3_29;
    const double k6_9_14_3 = h6_9_29 + CDz * h6_9_14;
    const double k6_9_6_9 = k6_9_14_3 + CDz * k6_9_6_3;
    const double k6_9_13_1 = h6_9_23 + CDx * h6_9_13;
    const double h14_3_7 = acc[778] + ABz * acc[313];
    const double h6_9_7 = h14_3_7 + ABz * h6_3_7;
    const double k6_9_7_1 = h6_9_13 + CDx * h6_9_7;
    const double k6_9_7_4 = k6_9_13_1 + CDx * k6_9_7_1;
    const double h14_3_16 = acc[787] + ABz * acc[322];
    const double h6_9_16 = h14_3_16 + ABz * h6_3_16;
    const double k6_9_7_2 = h6_9_16 + CDy * h6_9_7;
    const double k6_9_7_5 = k6_9_13_2 + CDx * k6_9_7_2;
    const double h14_3_17 = acc[788] + ABz * acc[323];
    const double h6_9_17 = h14_3_17 + ABz * h6_3_17;
    const double k6_9_7_3 = h6_9_17 + CDz * h6_9_7;
    const double k6_9_7_6 = k6_9_13_3 + CDx * k6_9_7_3;
    const double h14_3_30 = acc[801] + ABz * acc[336];
    const double h6_9_30 = h14_3_30 + ABz * h6_3_30;
    const double k6_9_16_2 = h6_9_30 + CDy * h6_9_16;
    const double k6_9_7_7 = k6_9_16_2 + CDy * k6_9_7_2;
    const double h14_3_31 = acc[802] + ABz * acc[337];
    const double h6_9_31 = h14_3_31 + ABz * h6_3_31;
    const double k6_9_16_3 = h6_9_31 + CDz * h6_9_16;
    const double k6_9_7_8 = k6_9_16_3 + CDy * k6_9_7_3;
    const double h14_3_32 = acc[803] + ABz * acc[338];
    const double h6_9_32 = h14_3_32 + ABz * h6_3_32;
    const double k6_9_17_3 = h6_9_32 + CDz * h6_9_17;
    const double k6_9_7_9 = k6_9_17_3 + CDz * k6_9_7_3;
    const double k6_9_15_1 = h6_9_24 + CDx * h6_9_15;
    const double h14_3_8 = acc[779] + ABz * acc[314];
    const double h6_9_8 = h14_3_8 + ABz * h6_3_8;
    const double k6_9_8_1 = h6_9_15 + CDx * h6_9_8;
    const double k6_9_8_4 = k6_9_15_1 + CDx * k6_9_8_1;
    const double k6_9_8_2 = h6_9_17 + CDy * h6_9_8;
    const double k6_9_8_5 = k6_9_15_2 + CDx * k6_9_8_2;
    const double h14_3_18 = acc[789] + ABz * acc[324];
    const double h6_9_18 = h14_3_18 + ABz * h6_3_18;
    const double k6_9_8_3 = h6_9_18 + CDz * h6_9_8;
    const double k6_9_8_6 = k6_9_15_3 + CDx * k6_9_8_3;
    const double k6_9_17_2 = h6_9_31 + CDy * h6_9_17;
    const double k6_9_8_7 = k6_9_17_2 + CDy * k6_9_8_2;
    const double k6_9_8_8 = k6_9_17_3 + CDy * k6_9_8_3;
    const double h14_3_33 = acc[804] + ABz * acc[339];
    const double h6_9_33 = h14_3_33 + ABz * h6_3_33;
    const double k6_9_18_3 = h6_9_33 + CDz * h6_9_18;
    const double k6_9_8_9 = k6_9_18_3 + CDz * k6_9_8_3;
    const double k6_9_14_1 = h6_9_25 + CDx * h6_9_14;
    const double h14_3_9 = acc[780] + ABz * acc[315];
    const double h6_9_9 = h14_3_9 + ABz * h6_3_9;
    const double k6_9_9_1 = h6_9_14 + CDx * h6_9_9;
    const double k6_9_9_4 = k6_9_14_1 + CDx * k6_9_9_1;
    const double k6_9_14_2 = h6_9_28 + CDy * h6_9_14;
    const double k6_9_9_2 = h6_9_18 + CDy * h6_9_9;
    const double k6_9_9_5 = k6_9_14_2 + CDx * k6_9_9_2;
    const double h14_3_19 = acc[790] + ABz * acc[325];
    const double h6_9_19 = h14_3_19 + ABz * h6_3_19;
    const double k6_9_9_3 = h6_9_19 + CDz * h6_9_9;
    const double k6_9_9_6 = k6_9_14_3 + CDx * k6_9_9_3;
    const double k6_9_18_2 = h6_9_32 + CDy * h6_9_18;
    const double k6_9_9_7 = k6_9_18_2 + CDy * k6_9_9_2;
    const double k6_9_9_8 = k6_9_18_3 + CDy * k6_9_9_3;
    const double h14_3_34 = acc[805] + ABz * acc[340];
    const double h6_9_34 = h14_3_34 + ABz * h6_3_34;
    const double k6_9_19_3 = h6_9_34 + CDz * h6_9_19;
    const double k6_9_9_9 = k6_9_19_3 + CDz * k6_9_9_3;
    const double h13_1_20 = acc[605] + ABx * acc[295];
    const double h7_1_20 = acc[295] + ABx * acc[109];
    const double h7_4_20 = h13_1_20 + ABx * h7_1_20;
    const double h13_1_10 = acc[595] + ABx * acc[285];
    const double h7_1_10 = acc[285] + ABx * acc[99];
    const double h7_4_10 = h13_1_10 + ABx * h7_1_10;
    const double k7_4_10_1 = h7_4_20 + CDx * h7_4_10;
    const double h13_1_4 = acc[589] + ABx * acc[279];
    const double h7_1_4 = acc[279] + ABx * acc[93];
    const double h7_4_4 = h13_1_4 + ABx * h7_1_4;
    const double k7_4_4_1 = h7_4_10 + CDx * h7_4_4;
    const double k7_4_4_4 = k7_4_10_1 + CDx * k7_4_4_1;
    const double h13_1_21 = acc[606] + ABx * acc[296];
    const double h7_1_21 = acc[296] + ABx * acc[110];
    const double h7_4_21 = h13_1_21 + ABx * h7_1_21;
    const double k7_4_10_2 = h7_4_21 + CDy * h7_4_10;
    const double h13_1_11 = acc[596] + ABx * acc[286];
    const double h7_1_11 = acc[286] + ABx * acc[100];
    const double h7_4_11 = h13_1_11 + ABx * h7_1_11;
    const double k7_4_4_2 = h7_4_11 + CDy * h7_4_4;
    const double k7_4_4_5 = k7_4_10_2 + CDx * k7_4_4_2;
    const double h13_1_22 = acc[607] + ABx * acc[297];
    const double h7_1_22 = acc[297] + ABx * acc[111];
    const double h7_4_22 = h13_1_22 + ABx * h7_1_22;
    const double k7_4_10_3 = h7_4_22 + CDz * h7_4_10;
    const double h13_1_12 = acc[597] + ABx * acc[287];
    const double h7_1_12 = acc[287] + ABx * acc[101];
    const double h7_4_12 = h13_1_12 + ABx * h7_1_12;
    const double k7_4_4_3 = h7_4_12 + CDz * h7_4_4;
    const double k7_4_4_6 = k7_4_10_3 + CDx * k7_4_4_3;
    const double h13_1_23 = acc[608] + ABx * acc[298];
    const double h7_1_23 = acc[298] + ABx * acc[112];
    const double h7_4_23 = h13_1_23 + ABx * h7_1_23;
    const double k7_4_11_2 = h7_4_23 + CDy * h7_4_11;
    const double k7_4_4_7 = k7_4_11_2 + CDy * k7_4_4_2;
    const double h13_1_24 = acc[609] + ABx * acc[299];
    const double h7_1_24 = acc[299] + ABx * acc[113];
    const double h7_4_24 = h13_1_24 + ABx * h7_1_24;
    const double k7_4_11_3 = h7_4_24 + CDz * h7_4_11;
    const double k7_4_4_8 = k7_4_11_3 + CDy * k7_4_4_3;
    const double h13_1_25 = acc[610] + ABx * acc[300];
    const double h7_1_25 = acc[300] + ABx * acc[114];
    const double h7_4_25 = h13_1_25 + ABx * h7_1_25;
    const double k7_4_12_3 = h7_4_25 + CDz * h7_4_12;
    const double k7_4_4_9 = k7_4_12_3 + CDz * k7_4_4_3;
    const double k7_4_11_1 = h7_4_21 + CDx * h7_4_11;
    const double h13_1_5 = acc[590] + ABx * acc[280];
    const double h7_1_5 = acc[280] + ABx * acc[94];
    const double h7_4_5 = h13_1_5 + ABx * h7_1_5;
    const double k7_4_5_1 = h7_4_11 + CDx * h7_4_5;
    const double k7_4_5_4 = k7_4_11_1 + CDx * k7_4_5_1;
    const double h13_1_13 = acc[598] + ABx * acc[288];
    const double h7_1_13 = acc[288] + ABx * acc[102];
    const double h7_4_13 = h13_1_13 + ABx * h7_1_13;
    const double k7_4_5_2 = h7_4_13 + CDy * h7_4_5;
    const double k7_4_5_5 = k7_4_11_2 + CDx * k7_4_5_2;
    const double h13_1_15 = acc[600] + ABx * acc[290];
    const double h7_1_15 = acc[290] + ABx * acc[104];
    const double h7_4_15 = h13_1_15 + ABx * h7_1_15;
    const double k7_4_5_3 = h7_4_15 + CDz * h7_4_5;
    const double k7_4_5_6 = k7_4_11_3 + CDx * k7_4_5_3;
    const double h13_1_26 = acc[611] + ABx * acc[301];
    const double h7_1_26 = acc[301] + ABx * acc[115];
    const double h7_4_26 = h13_1_26 + ABx * h7_1_26;
    const double k7_4_13_2 = h7_4_26 + CDy * h7_4_13;
    const double k7_4_5_7 = k7_4_13_2 + CDy * k7_4_5_2;
    const double h13_1_27 = acc[612] + ABx * acc[302];
    const double h7_1_27 = acc[302] + ABx * acc[116];
    const double h7_4_27 = h13_1_27 + ABx * h7_1_27;
    const double k7_4_13_3 = h7_4_27 + CDz * h7_4_13;
    const double k7_4_5_8 = k7_4_13_3 + CDy * k7_4_5_3;
    const double h13_1_28 = acc[613] + ABx * acc[303];
    const double h7_1_28 = acc[303] + ABx * acc[117];
    const double h7_4_28 = h13_1_28 + ABx * h7_1_28;
    const double k7_4_15_3 = h7_4_28 + CDz * h7_4_15;
    const double k7_4_5_9 = k7_4_15_3 + CDz * k7_4_5_3;
    const double k7_4_12_1 = h7_4_22 + CDx * h7_4_12;
    const double h13_1_6 = acc[591] + ABx * acc[281];
    const double h7_1_6 = acc[281] + ABx * acc[95];
    const double h7_4_6 = h13_1_6 + ABx * h7_1_6;
    const double k7_4_6_1 = h7_4_12 + CDx * h7_4_6;
    const double k7_4_6_4 = k7_4_12_1 + CDx * k7_4_6_1;
    const double k7_4_12_2 = h7_4_24 + CDy * h7_4_12;
    const double k7_4_6_2 = h7_4_15 + CDy * h7_4_6;
    const double k7_4_6_5 = k7_4_12_2 + CDx * k7_4_6_2;
    const double h13_1_14 = acc[599] + ABx * acc[289];
    const double h7_1_14 = acc[289] + ABx * acc[103];
    const double h7_4_14 = h13_1_14 + ABx * h7_1_14;
    const double k7_4_6_3 = h7_4_14 + CDz * h7_4_6;
    const double k7_4_6_6 = k7_4_12_3 + CDx * k7_4_6_3;
    const double k7_4_15_2 = h7_4_27 + CDy * h7_4_15;
    const double k7_4_6_7 = k7_4_15_2 + CDy * k7_4_6_2;
    const double k7_4_6_8 = k7_4_15_3 + CDy * k7_4_6_3;
    const double h13_1_29 = acc[614] + ABx * acc[304];
    const double h7_1_29 = acc[304] + ABx * acc[118];
    const double h7_4_29 = h13_1_29 + ABx * h7_1_29;
    const double k7_4_14_3 = h7_4_29 + CDz * h7_4_14;
    const double k7_4_6_9 = k7_4_14_3 + CDz * k7_4_6_3;
    const double k7_4_13_1 = h7_4_23 + CDx * h7_4_13;
    const double h13_1_7 = acc[592] + ABx * acc[282];
    const double h7_1_7 = acc[282] + ABx * acc[96];
    const double h7_4_7 = h13_1_7 + ABx * h7_1_7;
    const double k7_4_7_1 = h7_4_13 + CDx * h7_4_7;
    const double k7_4_7_4 = k7_4_13_1 + CDx * k7_4_7_1;
    const double h13_1_16 = acc[601] + ABx * acc[291];
    const double h7_1_16 = acc[291] + ABx * acc[105];
    const double h7_4_16 = h13_1_16 + ABx * h7_1_16;
    const double k7_4_7_2 = h7_4_16 + CDy * h7_4_7;
    const double k7_4_7_5 = k7_4_13_2 + CDx * k7_4_7_2;
    const double h13_1_17 = acc[602] + ABx * acc[292];
    const double h7_1_17 = acc[292] + ABx * acc[106];
    const double h7_4_17 = h13_1_17 + ABx * h7_1_17;
    const double k7_4_7_3 = h7_4_17 + CDz * h7_4_7;
    const double k7_4_7_6 = k7_4_13_3 + CDx * k7_4_7_3;
    const double h13_1_30 = acc[615] + ABx * acc[305];
    const double h7_1_30 = acc[305] + ABx * acc[119];
    const double h7_4_30 = h13_1_30 + ABx * h7_1_30;
    const double k7_4_16_2 = h7_4_30 + CDy * h7_4_16;
    const double k7_4_7_7 = k7_4_16_2 + CDy * k7_4_7_2;
    const double h13_1_31 = acc[616] + ABx * acc[306];
    const double h7_1_31 = acc[306] + ABx * acc[120];
    const double h7_4_31 = h13_1_31 + ABx * h7_1_31;
    const double k7_4_16_3 = h7_4_31 + CDz * h7_4_16;
    const double k7_4_7_8 = k7_4_16_3 + CDy * k7_4_7_3;
    const double h13_1_32 = acc[617] + ABx * acc[307];
    const double h7_1_32 = acc[307] + ABx * acc[121];
    const double h7_4_32 = h13_1_32 + ABx * h7_1_32;
    const double k7_4_17_3 = h7_4_32 + CDz * h7_4_17;
    const double k7_4_7_9 = k7_4_17_3 + CDz * k7_4_7_3;
    const double k7_4_15_1 = h7_4_24 + CDx * h7_4_15;
    const double h13_1_8 = acc[593] + ABx * acc[283];
    const double h7_1_8 = acc[283] + ABx * acc[97];
    const double h7_4_8 = h13_1_8 + ABx * h7_1_8;
    const double k7_4_8_1 = h7_4_15 + CDx * h7_4_8;
    const double k7_4_8_4 = k7_4_15_1 + CDx * k7_4_8_1;
    const double k7_4_8_2 = h7_4_17 + CDy * h7_4_8;
    const double k7_4_8_5 = k7_4_15_2 + CDx * k7_4_8_2;
    const double h13_1_18 = acc[603] + ABx * acc[293];
    const double h7_1_18 = acc[293] + ABx * acc[107];
    const double h7_4_18 = h13_1_18 + ABx * h7_1_18;
    const double k7_4_8_3 = h7_4_18 + CDz * h7_4_8;
    const double k7_4_8_6 = k7_4_15_3 + CDx * k7_4_8_3;
    const double k7_4_17_2 = h7_4_31 + CDy * h7_4_17;
    const double k7_4_8_7 = k7_4_17_2 + CDy * k7_4_8_2;
    const double k7_4_8_8 = k7_4_17_3 + CDy * k7_4_8_3;
    const double h13_1_33 = acc[618] + ABx * acc[308];
    const double h7_1_33 = acc[308] + ABx * acc[122];
    const double h7_4_33 = h13_1_33 + ABx * h7_1_33;
    const double k7_4_18_3 = h7_4_33 + CDz * h7_4_18;
    const double k7_4_8_9 = k7_4_18_3 + CDz * k7_4_8_3;
    const double k7_4_14_1 = h7_4_25 + CDx * h7_4_14;
    const double h13_1_9 = acc[594] + ABx * acc[284];
    const double h7_1_9 = acc[284] + ABx * acc[98];
    const double h7_4_9 = h13_1_9 + ABx * h7_1_9;
    const double k7_4_9_1 = h7_4_14 + CDx * h7_4_9;
    const double k7_4_9_4 = k7_4_14_1 + CDx * k7_4_9_1;
    const double k7_4_14_2 = h7_4_28 + CDy * h7_4_14;
    const double k7_4_9_2 = h7_4_18 + CDy * h7_4_9;
    const double k7_4_9_5 = k7_4_14_2 + CDx * k7_4_9_2;
    const double h13_1_19 = acc[604] + ABx * acc[294];
    const double h7_1_19 = acc[294] + ABx * acc[108];
    const double h7_4_19 = h13_1_19 + ABx * h7_1_19;
    const double k7_4_9_3 = h7_4_19 + CDz * h7_4_9;
    const double k7_4_9_6 = k7_4_14_3 + CDx * k7_4_9_3;
    const double k7_4_18_2 = h7_4_32 + CDy * h7_4_18;
    const double k7_4_9_7 = k7_4_18_2 + CDy * k7_4_9_2;
    const double k7_4_9_8 = k7_4_18_3 + CDy * k7_4_9_3;
    const double h13_1_34 = acc[619] + ABx * acc[309];
    const double h7_1_34 = acc[309] + ABx * acc[123];
    const double h7_4_34 = h13_1_34 + ABx * h7_1_34;
    const double k7_4_19_3 = h7_4_34 + CDz * h7_4_19;
    const double k7_4_9_9 = k7_4_19_3 + CDz * k7_4_9_3;
    const double h7_2_20 = acc[388] + ABy * acc[109];
    const double h7_5_20 = h13_2_20 + ABx * h7_2_20;
    const double h7_2_10 = acc[378] + ABy * acc[99];
    const double h7_5_10 = h13_2_10 + ABx * h7_2_10;
    const double k7_5_10_1 = h7_5_20 + CDx * h7_5_10;
    const double h7_2_4 = acc[372] + ABy * acc[93];
    const double h7_5_4 = h13_2_4 + ABx * h7_2_4;
    const double k7_5_4_1 = h7_5_10 + CDx * h7_5_4;
    const double k7_5_4_4 = k7_5_10_1 + CDx * k7_5_4_1;
    const double h7_2_21 = acc[389] + ABy * acc[110];
    const double h7_5_21 = h13_2_21 + ABx * h7_2_21;
    const double k7_5_10_2 = h7_5_21 + CDy * h7_5_10;
    const double h7_2_11 = acc[379] + ABy * acc[100];
    const double h7_5_11 = h13_2_11 + ABx * h7_2_11;
    const double k7_5_4_2 = h7_5_11 + CDy * h7_5_4;
    const double k7_5_4_5 = k7_5_10_2 + CDx * k7_5_4_2;
    const double h7_2_22 = acc[390] + ABy * acc[111];
    const double h7_5_22 = h13_2_22 + ABx * h7_2_22;
    const double k7_5_10_3 = h7_5_22 + CDz * h7_5_10;
    const double h7_2_12 = acc[380] + ABy * acc[101];
    const double h7_5_12 = h13_2_12 + ABx * h7_2_12;
    const double k7_5_4_3 = h7_5_12 + CDz * h7_5_4;
    const double k7_5_4_6 = k7_5_10_3 + CDx * k7_5_4_3;
    const double h7_2_23 = acc[391] + ABy * acc[112];
    const double h7_5_23 = h13_2_23 + ABx * h7_2_23;
    const double k7_5_11_2 = h7_5_23 + CDy * h7_5_11;
    const double k7_5_4_7 = k7_5_11_2 + CDy * k7_5_4_2;
    const double h7_2_24 = acc[392] + ABy * acc[113];
    const double h7_5_24 = h13_2_24 + ABx * h7_2_24;
    const double k7_5_11_3 = h7_5_24 + CDz * h7_5_11;
    const double k7_5_4_8 = k7_5_11_3 + CDy * k7_5_4_3;
    const double h7_2_25 = acc[393] + ABy * acc[114];
    const double h7_5_25 = h13_2_25 + ABx * h7_2_25;
    const double k7_5_12_3 = h7_5_25 + CDz * h7_5_12;
    const double k7_5_4_9 = k7_5_12_3 + CDz * k7_5_4_3;
    const double k7_5_11_1 = h7_5_21 + CDx * h7_5_11;
    const double h7_2_5 = acc[373] + ABy * acc[94];
    const double h7_5_5 = h13_2_5 + ABx * h7_2_5;
    const double k7_5_5_1 = h7_5_11 + CDx * h7_5_5;
    const double k7_5_5_4 = k7_5_11_1 + CDx * k7_5_5_1;
    const double h7_2_13 = acc[381] + ABy * acc[102];
    const double h7_5_13 = h13_2_13 + ABx * h7_2_13;
    const double k7_5_5_2 = h7_5_13 + CDy * h7_5_5;
    const double k7_5_5_5 = k7_5_11_2 + CDx * k7_5_5_2;
    const double h7_2_15 = acc[383] + ABy * acc[104];
    const double h7_5_15 = h13_2_15 + ABx * h7_2_15;
    const double k7_5_5_3 = h7_5_15 + CDz * h7_5_5;
    const double k7_5_5_6 = k7_5_11_3 + CDx * k7_5_5_3;
    const double h7_2_26 = acc[394] + ABy * acc[115];
    const double h7_5_26 = h13_2_26 + ABx * h7_2_26;
    const double k7_5_13_2 = h7_5_26 + CDy * h7_5_13;
    const double k7_5_5_7 = k7_5_13_2 + CDy * k7_5_5_2;
    const double h7_2_27 = acc[395] + ABy * acc[116];
    const double h7_5_27 = h13_2_27 + ABx * h7_2_27;
    const double k7_5_13_3 = h7_5_27 + CDz * h7_5_13;
    const double k7_5_5_8 = k7_5_13_3 + CDy * k7_5_5_3;
    const double h7_2_28 = acc[396] + ABy * acc[117];
    const double h7_5_28 = h13_2_28 + ABx * h7_2_28;
    const double k7_5_15_3 = h7_5_28 + CDz * h7_5_15;
    const double k7_5_5_9 = k7_5_15_3 + CDz * k7_5_5_3;
    const double k7_5_12_1 = h7_5_22 + CDx * h7_5_12;
    const double h7_2_6 = acc[374] + ABy * acc[95];
    const double h7_5_6 = h13_2_6 + ABx * h7_2_6;
    const double k7_5_6_1 = h7_5_12 + CDx * h7_5_6;
    const double k7_5_6_4 = k7_5_12_1 + CDx * k7_5_6_1;
    const double k7_5_12_2 = h7_5_24 + CDy * h7_5_12;
    const double k7_5_6_2 = h7_5_15 + CDy * h7_5_6;
    const double k7_5_6_5 = k7_5_12_2 + CDx * k7_5_6_2;
    const double h7_2_14 = acc[382] + ABy * acc[103];
    const double h7_5_14 = h13_2_14 + ABx * h7_2_14;
    const double k7_5_6_3 = h7_5_14 + CDz * h7_5_6;
    const double k7_5_6_6 = k7_5_12_3 + CDx * k7_5_6_3;
    const double k7_5_15_2 = h7_5_27 + CDy * h7_5_15;
    const double k7_5_6_7 = k7_5_15_2 + CDy * k7_5_6_2;
    const double k7_5_6_8 = k7_5_15_3 + CDy * k7_5_6_3;
    const double h7_2_29 = acc[397] + ABy * acc[118];
    const double h7_5_29 = h13_2_29 + ABx * h7_2_29;
    const double k7_5_14_3 = h7_5_29 + CDz * h7_5_14;
    const double k7_5_6_9 = k7_5_14_3 + CDz * k7_5_6_3;
    const double k7_5_13_1 = h7_5_23 + CDx * h7_5_13;
    const double h7_2_7 = acc[375] + ABy * acc[96];
    const double h7_5_7 = h13_2_7 + ABx * h7_2_7;
    const double k7_5_7_1 = h7_5_13 + CDx * h7_5_7;
    const double k7_5_7_4 = k7_5_13_1 + CDx * k7_5_7_1;
    const double h7_2_16 = acc[384] + ABy * acc[105];
    const double h7_5_16 = h13_2_16 + ABx * h7_2_16;
    const double k7_5_7_2 = h7_5_16 + CDy * h7_5_7;
    const double k7_5_7_5 = k7_5_13_2 + CDx * k7_5_7_2;
    const double h7_2_17 = acc[385] + ABy * acc[106];
    const double h7_5_17 = h13_2_17 + ABx * h7_2_17;
    const double k7_5_7_3 = h7_5_17 + CDz * h7_5_7;
    const double k7_5_7_6 = k7_5_13_3 + CDx * k7_5_7_3;
    const double h7_2_30 = acc[398] + ABy * acc[119];
    const double h7_5_30 = h13_2_30 + ABx * h7_2_30;
    const double k7_5_16_2 = h7_5_30 + CDy * h7_5_16;
    const double k7_5_7_7 = k7_5_16_2 + CDy * k7_5_7_2;
    const double h7_2_31 = acc[399] + ABy * acc[120];
    const double h7_5_31 = h13_2_31 + ABx * h7_2_31;
    const double k7_5_16_3 = h7_5_31 + CDz * h7_5_16;
    const double k7_5_7_8 = k7_5_16_3 + CDy * k7_5_7_3;
    const double h7_2_32 = acc[400] + ABy * acc[121];
    const double h7_5_32 = h13_2_32 + ABx * h7_2_32;
    const double k7_5_17_3 = h7_5_32 + CDz * h7_5_17;
    const double k7_5_7_9 = k7_5_17_3 + CDz * k7_5_7_3;
    const double k7_5_15_1 = h7_5_24 + CDx * h7_5_15;
    const double h7_2_8 = acc[376] + ABy * acc[97];
    const double h7_5_8 = h13_2_8 + ABx * h7_2_8;
    const double k7_5_8_1 = h7_5_15 + CDx * h7_5_8;
    const double k7_5_8_4 = k7_5_15_1 + CDx * k7_5_8_1;
    const double k7_5_8_2 = h7_5_17 + CDy * h7_5_8;
    const double k7_5_8_5 = k7_5_15_2 + CDx * k7_5_8_2;
    const double h7_2_18 = acc[386] + ABy * acc[107];
    const double h7_5_18 = h13_2_18 + ABx * h7_2_18;
    const double k7_5_8_3 = h7_5_18 + CDz * h7_5_8;
    const double k7_5_8_6 = k7_5_15_3 + CDx * k7_5_8_3;
    const double k7_5_17_2 = h7_5_31 + CDy * h7_5_17;
    const double k7_5_8_7 = k7_5_17_2 + CDy * k7_5_8_2;
    const double k7_5_8_8 = k7_5_17_3 + CDy * k7_5_8_3;
    const double h7_2_33 = acc[401] + ABy * acc[122];
    const double h7_5_33 = h13_2_33 + ABx * h7_2_33;
    const double k7_5_18_3 = h7_5_33 + CDz * h7_5_18;
    const double k7_5_8_9 = k7_5_18_3 + CDz * k7_5_8_3;
    const double k7_5_14_1 = h7_5_25 + CDx * h7_5_14;
    const double h7_2_9 = acc[377] + ABy * acc[98];
    const double h7_5_9 = h13_2_9 + ABx * h7_2_9;
    const double k7_5_9_1 = h7_5_14 + CDx * h7_5_9;
    const double k7_5_9_4 = k7_5_14_1 + CDx * k7_5_9_1;
    const double k7_5_14_2 = h7_5_28 + CDy * h7_5_14;
    const double k7_5_9_2 = h7_5_18 + CDy * h7_5_9;
    const double k7_5_9_5 = k7_5_14_2 + CDx * k7_5_9_2;
    const double h7_2_19 = acc[387] + ABy * acc[108];
    const double h7_5_19 = h13_2_19 + ABx * h7_2_19;
    const double k7_5_9_3 = h7_5_19 + CDz * h7_5_9;
    const double k7_5_9_6 = k7_5_14_3 + CDx * k7_5_9_3;
    const double k7_5_18_2 = h7_5_32 + CDy * h7_5_18;
    const double k7_5_9_7 = k7_5_18_2 + CDy * k7_5_9_2;
    const double k7_5_9_8 = k7_5_18_3 + CDy * k7_5_9_3;
    const double h7_2_34 = acc[402] + ABy * acc[123];
    const double h7_5_34 = h13_2_34 + ABx * h7_2_34;
    const double k7_5_19_3 = h7_5_34 + CDz * h7_5_19;
    const double k7_5_9_9 = k7_5_19_3 + CDz * k7_5_9_3;
    const double h7_3_20 = acc[419] + ABz * acc[109];
    const double h7_6_20 = h13_3_20 + ABx * h7_3_20;
    const double h7_3_10 = acc[409] + ABz * acc[99];
    const double h7_6_10 = h13_3_10 + ABx * h7_3_10;
    const double k7_6_10_1 = h7_6_20 + CDx * h7_6_10;
    const double h7_3_4 = acc[403] + ABz * acc[93];
    const double h7_6_4 = h13_3_4 + ABx * h7_3_4;
    const double k7_6_4_1 = h7_6_10 + CDx * h7_6_4;
    const double k7_6_4_4 = k7_6_10_1 + CDx * k7_6_4_1;
    const double h7_3_21 = acc[420] + ABz * acc[110];
    const double h7_6_21 = h13_3_21 + ABx * h7_3_21;
    const double k7_6_10_2 = h7_6_21 + CDy * h7_6_10;
    const double h7_3_11 = acc[410] + ABz * acc[100];
    const double h7_6_11 = h13_3_11 + ABx * h7_3_11;
    const double k7_6_4_2 = h7_6_11 + CDy * h7_6_4;
    const double k7_6_4_5 = k7_6_10_2 + CDx * k7_6_4_2;
    const double h7_3_22 = acc[421] + ABz * acc[111];
    const double h7_6_22 = h13_3_22 + ABx * h7_3_22;
    const double k7_6_10_3 = h7_6_22 + CDz * h7_6_10;
    const double h7_3_12 = acc[411] + ABz * acc[101];
    const double h7_6_12 = h13_3_12 + ABx * h7_3_12;
    const double k7_6_4_3 = h7_6_12 + CDz * h7_6_4;
    const double k7_6_4_6 = k7_6_10_3 + CDx * k7_6_4_3;
    const double h7_3_23 = acc[422] + ABz * acc[112];
    const double h7_6_23 = h13_3_23 + ABx * h7_3_23;
    const double k7_6_11_2 = h7_6_23 + CDy * h7_6_11;
    const double k7_6_4_7 = k7_6_11_2 + CDy * k7_6_4_2;
    const double h7_3_24 = acc[423] + ABz * acc[113];
    const double h7_6_24 = h13_3_24 + ABx * h7_3_24;
    const double k7_6_11_3 = h7_6_24 + CDz * h7_6_11;
    const double k7_6_4_8 = k7_6_11_3 + CDy * k7_6_4_3;
    const double h7_3_25 = acc[424] + ABz * acc[114];
    const double h7_6_25 = h13_3_25 + ABx * h7_3_25;
    const double k7_6_12_3 = h7_6_25 + CDz * h7_6_12;
    const double k7_6_4_9 = k7_6_12_3 + CDz * k7_6_4_3;
    const double k7_6_11_1 = h7_6_21 + CDx * h7_6_11;
    const double h7_3_5 = acc[404] + ABz * acc[94];
    const double h7_6_5 = h13_3_5 + ABx * h7_3_5;
    const double k7_6_5_1 = h7_6_11 + CDx * h7_6_5;
    const double k7_6_5_4 = k7_6_11_1 + CDx * k7_6_5_1;
    const double h7_3_13 = acc[412] + ABz * acc[102];
    const double h7_6_13 = h13_3_13 + ABx * h7_3_13;
    const double k7_6_5_2 = h7_6_13 + CDy * h7_6_5;
    const double k7_6_5_5 = k7_6_11_2 + CDx * k7_6_5_2;
    const double h7_3_15 = acc[414] + ABz * acc[104];
    const double h7_6_15 = h13_3_15 + ABx * h7_3_15;
    const double k7_6_5_3 = h7_6_15 + CDz * h7_6_5;
    const double k7_6_5_6 = k7_6_11_3 + CDx * k7_6_5_3;
    const double h7_3_26 = acc[425] + ABz * acc[115];
    const double h7_6_26 = h13_3_26 + ABx * h7_3_26;
    const double k7_6_13_2 = h7_6_26 + CDy * h7_6_13;
    const double k7_6_5_7 = k7_6_13_2 + CDy * k7_6_5_2;
    const double h7_3_27 = acc[426] + ABz * acc[116];
    const double h7_6_27 = h13_3_27 + ABx * h7_3_27;
    const double k7_6_13_3 = h7_6_27 + CDz * h7_6_13;
    const double k7_6_5_8 = k7_6_13_3 + CDy * k7_6_5_3;
    const double h7_3_28 = acc[427] + ABz * acc[117];
    const double h7_6_28 = h13_3_28 + ABx * h7_3_28;
    const double k7_6_15_3 = h7_6_28 + CDz * h7_6_15;
    const double k7_6_5_9 = k7_6_15_3 + CDz * k7_6_5_3;
    const double k7_6_12_1 = h7_6_22 + CDx * h7_6_12;
    const double h7_3_6 = acc[405] + ABz * acc[95];
    const double h7_6_6 = h13_3_6 + ABx * h7_3_6;
    const double k7_6_6_1 = h7_6_12 + CDx * h7_6_6;
    const double k7_6_6_4 = k7_6_12_1 + CDx * k7_6_6_1;
    const double k7_6_12_2 = h7_6_24 + CDy * h7_6_12;
    const double k7_6_6_2 = h7_6_15 + CDy * h7_6_6;
    const double k7_6_6_5 = k7_6_12_2 + CDx * k7_6_6_2;
    const double h7_3_14 = acc[413] + ABz * acc[103];
    const double h7_6_14 = h13_3_14 + ABx * h7_3_14;
    const double k7_6_6_3 = h7_6_14 + CDz * h7_6_6;
    const double k7_6_6_6 = k7_6_12_3 + CDx * k7_6_6_3;
    const double k7_6_15_2 = h7_6_27 + CDy * h7_6_15;
    const double k7_6_6_7 = k7_6_15_2 + CDy * k7_6_6_2;
    const double k7_6_6_8 = k7_6_15_3 + CDy * k7_6_6_3;
    const double h7_3_29 = acc[428] + ABz * acc[118];
    const double h7_6_29 = h13_3_29 + ABx * h7_3_29;
    const double k7_6_14_3 = h7_6_29 + CDz * h7_6_14;
    const double k7_6_6_9 = k7_6_14_3 + CDz * k7_6_6_3;
    const double k7_6_13_1 = h7_6_23 + CDx * h7_6_13;
    const double h7_3_7 = acc[406] + ABz * acc[96];
    const double h7_6_7 = h13_3_7 + ABx * h7_3_7;
    const double k7_6_7_1 = h7_6_13 + CDx * h7_6_7;
    const double k7_6_7_4 = k7_6_13_1 + CDx * k7_6_7_1;
    const double h7_3_16 = acc[415] + ABz * acc[105];
    const double h7_6_16 = h13_3_16 + ABx * h7_3_16;
    const double k7_6_7_2 = h7_6_16 + CDy * h7_6_7;
    const double k7_6_7_5 = k7_6_13_2 + CDx * k7_6_7_2;
    const double h7_3_17 = acc[416] + ABz * acc[106];
    const double h7_6_17 = h13_3_17 + ABx * h7_3_17;
    const double k7_6_7_3 = h7_6_17 + CDz * h7_6_7;
    const double k7_6_7_6 = k7_6_13_3 + CDx * k7_6_7_3;
    const double h7_3_30 = acc[429] + ABz * acc[119];
    const double h7_6_30 = h13_3_30 + ABx * h7_3_30;
    const double k7_6_16_2 = h7_6_30 + CDy * h7_6_16;
    const double k7_6_7_7 = k7_6_16_2 + CDy * k7_6_7_2;
    const double h7_3_31 = acc[430] + ABz * acc[120];
    const double h7_6_31 = h13_3_31 + ABx * h7_3_31;
    const double k7_6_16_3 = h7_6_31 + CDz * h7_6_16;
    const double k7_6_7_8 = k7_6_16_3 + CDy * k7_6_7_3;
    const double h7_3_32 = acc[431] + ABz * acc[121];
    const double h7_6_32 = h13_3_32 + ABx * h7_3_32;
    const double k7_6_17_3 = h7_6_32 + CDz * h7_6_17;
    const double k7_6_7_9 = k7_6_17_3 + CDz * k7_6_7_3;
    const double k7_6_15_1 = h7_6_24 + CDx * h7_6_15;
    const double h7_3_8 = acc[407] + ABz * acc[97];
    const double h7_6_8 = h13_3_8 + ABx * h7_3_8;
    const double k7_6_8_1 = h7_6_15 + CDx * h7_6_8;
    const double k7_6_8_4 = k7_6_15_1 + CDx * k7_6_8_1;
    const double k7_6_8_2 = h7_6_17 + CDy * h7_6_8;
    const double k7_6_8_5 = k7_6_15_2 + CDx * k7_6_8_2;
    const double h7_3_18 = acc[417] + ABz * acc[107];
    const double h7_6_18 = h13_3_18 + ABx * h7_3_18;
    const double k7_6_8_3 = h7_6_18 + CDz * h7_6_8;
    const double k7_6_8_6 = k7_6_15_3 + CDx * k7_6_8_3;
    const double k7_6_17_2 = h7_6_31 + CDy * h7_6_17;
    const double k7_6_8_7 = k7_6_17_2 + CDy * k7_6_8_2;
    const double k7_6_8_8 = k7_6_17_3 + CDy * k7_6_8_3;
    const double h7_3_33 = acc[432] + ABz * acc[122];
    const double h7_6_33 = h13_3_33 + ABx * h7_3_33;
    const double k7_6_18_3 = h7_6_33 + CDz * h7_6_18;
    const double k7_6_8_9 = k7_6_18_3 + CDz * k7_6_8_3;
    const double k7_6_14_1 = h7_6_25 + CDx * h7_6_14;
    const double h7_3_9 = acc[408] + ABz * acc[98];
    const double h7_6_9 = h13_3_9 + ABx * h7_3_9;
    const double k7_6_9_1 = h7_6_14 + CDx * h7_6_9;
    const double k7_6_9_4 = k7_6_14_1 + CDx * k7_6_9_1;
    const double k7_6_14_2 = h7_6_28 + CDy * h7_6_14;
    const double k7_6_9_2 = h7_6_18 + CDy * h7_6_9;
    const double k7_6_9_5 = k7_6_14_2 + CDx * k7_6_9_2;
    const double h7_3_19 = acc[418] + ABz * acc[108];
    const double h7_6_19 = h13_3_19 + ABx * h7_3_19;
    const double k7_6_9_3 = h7_6_19 + CDz * h7_6_9;
    const double k7_6_9_6 = k7_6_14_3 + CDx * k7_6_9_3;
    const double k7_6_18_2 = h7_6_32 + CDy * h7_6_18;
    const double k7_6_9_7 = k7_6_18_2 + CDy * k7_6_9_2;
    const double k7_6_9_8 = k7_6_18_3 + CDy * k7_6_9_3;
    const double h7_3_34 = acc[433] + ABz * acc[123];
    const double h7_6_34 = h13_3_34 + ABx * h7_3_34;
    const double k7_6_19_3 = h7_6_34 + CDz * h7_6_19;
    const double k7_6_9_9 = k7_6_19_3 + CDz * k7_6_9_3;
    const double h16_2_20 = acc[822] + ABy * acc[388];
    const double h7_7_20 = h16_2_20 + ABy * h7_2_20;
    const double h16_2_10 = acc[812] + ABy * acc[378];
    const double h7_7_10 = h16_2_10 + ABy * h7_2_10;
    const double k7_7_10_1 = h7_7_20 + CDx * h7_7_10;
    const double h16_2_4 = acc[806] + ABy * acc[372];
    const double h7_7_4 = h16_2_4 + ABy * h7_2_4;
    const double k7_7_4_1 = h7_7_10 + CDx * h7_7_4;
    const double k7_7_4_4 = k7_7_10_1 + CDx * k7_7_4_1;
    const double h16_2_21 = acc[823] + ABy * acc[389];
    const double h7_7_21 = h16_2_21 + ABy * h7_2_21;
    const double k7_7_10_2 = h7_7_21 + CDy * h7_7_10;
    const double h16_2_11 = acc[813] + ABy * acc[379];
    const double h7_7_11 = h16_2_11 + ABy * h7_2_11;
    const double k7_7_4_2 = h7_7_11 + CDy * h7_7_4;
    const double k7_7_4_5 = k7_7_10_2 + CDx * k7_7_4_2;
    const double h16_2_22 = acc[824] + ABy * acc[390];
    const double h7_7_22 = h16_2_22 + ABy * h7_2_22;
    const double k7_7_10_3 = h7_7_22 + CDz * h7_7_10;
    const double h16_2_12 = acc[814] + ABy * acc[380];
    const double h7_7_12 = h16_2_12 + ABy * h7_2_12;
    const double k7_7_4_3 = h7_7_12 + CDz * h7_7_4;
    const double k7_7_4_6 = k7_7_10_3 + CDx * k7_7_4_3;
    const double h16_2_23 = acc[825] + ABy * acc[391];
    const double h7_7_23 = h16_2_23 + ABy * h7_2_23;
    const double k7_7_11_2 = h7_7_23 + CDy * h7_7_11;
    const double k7_7_4_7 = k7_7_11_2 + CDy * k7_7_4_2;
    const double h16_2_24 = acc[826] + ABy * acc[392];
    const double h7_7_24 = h16_2_24 + ABy * h7_2_24;
    const double k7_7_11_3 = h7_7_24 + CDz * h7_7_11;
    const double k7_7_4_8 = k7_7_11_3 + CDy * k7_7_4_3;
    const double h16_2_25 = acc[827] + ABy * acc[393];
    const double h7_7_25 = h16_2_25 + ABy * h7_2_25;
    const double k7_7_12_3 = h7_7_25 + CDz * h7_7_12;
    const double k7_7_4_9 = k7_7_12_3 + CDz * k7_7_4_3;
    const double k7_7_11_1 = h7_7_21 + CDx * h7_7_11;
    const double h16_2_5 = acc[807] + ABy * acc[373];
    const double h7_7_5 = h16_2_5 + ABy * h7_2_5;
    const double k7_7_5_1 = h7_7_11 + CDx * h7_7_5;
    const double k7_7_5_4 = k7_7_11_1 + CDx * k7_7_5_1;
    const double h16_2_13 = acc[815] + ABy * acc[381];
    const double h7_7_13 = h16_2_13 + ABy * h7_2_13;
    const double k7_7_5_2 = h7_7_13 + CDy * h7_7_5;
    const double k7_7_5_5 = k7_7_11_2 + CDx * k7_7_5_2;
    const double h16_2_15 = acc[817] + ABy * acc[383];
    const double h7_7_15 = h16_2_15 + ABy * h7_2_15;
    const double k7_7_5_3 = h7_7_15 + CDz * h7_7_5;
    const double k7_7_5_6 = k7_7_11_3 + CDx * k7_7_5_3;
    const double h16_2_26 = acc[828] + ABy * acc[394];
    const double h7_7_26 = h16_2_26 + ABy * h7_2_26;
    const double k7_7_13_2 = h7_7_26 + CDy * h7_7_13;
    const double k7_7_5_7 = k7_7_13_2 + CDy * k7_7_5_2;
    const double h16_2_27 = acc[829] + ABy * acc[395];
    const double h7_7_27 = h16_2_27 + ABy * h7_2_27;
    const double k7_7_13_3 = h7_7_27 + CDz * h7_7_13;
    const double k7_7_5_8 = k7_7_13_3 + CDy * k7_7_5_3;
    const double h16_2_28 = acc[830] + ABy * acc[396];
    const double h7_7_28 = h16_2_28 + ABy * h7_2_28;
    const double k7_7_15_3 = h7_7_28 + CDz * h7_7_15;
    const double k7_7_5_9 = k7_7_15_3 + CDz * k7_7_5_3;
    const double k7_7_12_1 = h7_7_22 + CDx * h7_7_12;
    const double h16_2_6 = acc[808] + ABy * acc[374];
    const double h7_7_6 = h16_2_6 + ABy * h7_2_6;
    const double k7_7_6_1 = h7_7_12 + CDx * h7_7_6;
    const double k7_7_6_4 = k7_7_12_1 + CDx * k7_7_6_1;
    const double k7_7_12_2 = h7_7_24 + CDy * h7_7_12;
    const double k7_7_6_2 = h7_7_15 + CDy * h7_7_6;
    const double k7_7_6_5 = k7_7_12_2 + CDx * k7_7_6_2;
    const double h16_2_14 = acc[816] + ABy * acc[382];
    const double h7_7_14 = h16_2_14 + ABy * h7_2_14;
    const double k7_7_6_3 = h7_7_14 + CDz * h7_7_6;
    const double k7_7_6_6 = k7_7_12_3 + CDx * k7_7_6_3;
    const double k7_7_15_2 = h7_7_27 + CDy * h7_7_15;
    const double k7_7_6_7 = k7_7_15_2 + CDy * k7_7_6_2;
    const double k7_7_6_8 = k7_7_15_3 + CDy * k7_7_6_3;
    const double h16_2_29 = acc[831] + ABy * acc[397];
    const double h7_7_29 = h16_2_29 + ABy * h7_2_29;
    const double k7_7_14_3 = h7_7_29 + CDz * h7_7_14;
    const double k7_7_6_9 = k7_7_14_3 + CDz * k7_7_6_3;
    const double k7_7_13_1 = h7_7_23 + CDx * h7_7_13;
    const double h16_2_7 = acc[809] + ABy * acc[375];
    const double h7_7_7 = h16_2_7 + ABy * h7_2_7;
    const double k7_7_7_1 = h7_7_13 + CDx * h7_7_7;
    const double k7_7_7_4 = k7_7_13_1 + CDx * k7_7_7_1;
    const double h16_2_16 = acc[818] + ABy * acc[384];
    const double h7_7_16 = h16_2_16 + ABy * h7_2_16;
    const double k7_7_7_2 = h7_7_16 + CDy * h7_7_7;
    const double k7_7_7_5 = k7_7_13_2 + CDx * k7_7_7_2;
    const double h16_2_17 = acc[819] + ABy * acc[385];
    const double h7_7_17 = h16_2_17 + ABy * h7_2_17;
    const double k7_7_7_3 = h7_7_17 + CDz * h7_7_7;
    const double k7_7_7_6 = k7_7_13_3 + CDx * k7_7_7_3;
    const double h16_2_30 = acc[832] + ABy * acc[398];
    const double h7_7_30 = h16_2_30 + ABy * h7_2_30;
    const double k7_7_16_2 = h7_7_30 + CDy * h7_7_16;
    const double k7_7_7_7 = k7_7_16_2 + CDy * k7_7_7_2;
    const double h16_2_31 = acc[833] + ABy * acc[399];
    const double h7_7_31 = h16_2_31 + ABy * h7_2_31;
    const double k7_7_16_3 = h7_7_31 + CDz * h7_7_16;
    const double k7_7_7_8 = k7_7_16_3 + CDy * k7_7_7_3;
    const double h16_2_32 = acc[834] + ABy * acc[400];
    const double h7_7_32 = h16_2_32 + ABy * h7_2_32;
    const double k7_7_17_3 = h7_7_32 + CDz * h7_7_17;
    const double k7_7_7_9 = k7_7_17_3 + CDz * k7_7_7_3;
    const double k7_7_15_1 = h7_7_24 + CDx * h7_7_15;
    const double h16_2_8 = acc[810] + ABy * acc[376];
    const double h7_7_8 = h16_2_8 + ABy * h7_2_8;
    const double k7_7_8_1 = h7_7_15 + CDx * h7_7_8;
    const double k7_7_8_4 = k7_7_15_1 + CDx * k7_7_8_1;
    const double k7_7_8_2 = h7_7_17 + CDy * h7_7_8;
    const double k7_7_8_5 = k7_7_15_2 + CDx * k7_7_8_2;
    const double h16_2_18 = acc[820] + ABy * acc[386];
    const double h7_7_18 = h16_2_18 + ABy * h7_2_18;
    const double k7_7_8_3 = h7_7_18 + CDz * h7_7_8;
    const double k7_7_8_6 = k7_7_15_3 + CDx * k7_7_8_3;
    const double k7_7_17_2 = h7_7_31 + CDy * h7_7_17;
    const double k7_7_8_7 = k7_7_17_2 + CDy * k7_7_8_2;
    const double k7_7_8_8 = k7_7_17_3 + CDy * k7_7_8_3;
    const double h16_2_33 = acc[835] + ABy * acc[401];
    const double h7_7_33 = h16_2_33 + ABy * h7_2_33;
    const double k7_7_18_3 = h7_7_33 + CDz * h7_7_18;
    const double k7_7_8_9 = k7_7_18_3 + CDz * k7_7_8_3;
    const double k7_7_14_1 = h7_7_25 + CDx * h7_7_14;
    const double h16_2_9 = acc[811] + ABy * acc[377];
    const double h7_7_9 = h16_2_9 + ABy * h7_2_9;
    const double k7_7_9_1 = h7_7_14 + CDx * h7_7_9;
    const double k7_7_9_4 = k7_7_14_1 + CDx * k7_7_9_1;
    const double k7_7_14_2 = h7_7_28 + CDy * h7_7_14;
    const double k7_7_9_2 = h7_7_18 + CDy * h7_7_9;
    const double k7_7_9_5 = k7_7_14_2 + CDx * k7_7_9_2;
    const double h16_2_19 = acc[821] + ABy * acc[387];
    const double h7_7_19 = h16_2_19 + ABy * h7_2_19;
    const double k7_7_9_3 = h7_7_19 + CDz * h7_7_9;
    const double k7_7_9_6 = k7_7_14_3 + CDx * k7_7_9_3;
    const double k7_7_18_2 = h7_7_32 + CDy * h7_7_18;
    const double k7_7_9_7 = k7_7_18_2 + CDy * k7_7_9_2;
    const double k7_7_9_8 = k7_7_18_3 + CDy * k7_7_9_3;
    const double h16_2_34 = acc[836] + ABy * acc[402];
    const double h7_7_34 = h16_2_34 + ABy * h7_2_34;
    const double k7_7_19_3 = h7_7_34 + CDz * h7_7_19;
    const double k7_7_9_9 = k7_7_19_3 + CDz * k7_7_9_3;
    const double h16_3_20 = acc[853] + ABz * acc[388];
    const double h7_8_20 = h16_3_20 + ABy * h7_3_20;
    const double h16_3_10 = acc[843] + ABz * acc[378];
    const double h7_8_10 = h16_3_10 + ABy * h7_3_10;
    const double k7_8_10_1 = h7_8_20 + CDx * h7_8_10;
    const double h16_3_4 = acc[837] + ABz * acc[372];
    const double h7_8_4 = h16_3_4 + ABy * h7_3_4;
    const double k7_8_4_1 = h7_8_10 + CDx * h7_8_4;
    const double k7_8_4_4 = k7_8_10_1 + CDx * k7_8_4_1;
    const double h16_3_21 = acc[854] + ABz * acc[389];
    const double h7_8_21 = h16_3_21 + ABy * h7_3_21;
    const double k7_8_10_2 = h7_8_21 + CDy * h7_8_10;
    const double h16_3_11 = acc[844] + ABz * acc[379];
    const double h7_8_11 = h16_3_11 + ABy * h7_3_11;
    const double k7_8_4_2 = h7_8_11 + CDy * h7_8_4;
    const double k7_8_4_5 = k7_8_10_2 + CDx * k7_8_4_2;
    const double h16_3_22 = acc[855] + ABz * acc[390];
    const double h7_8_22 = h16_3_22 + ABy * h7_3_22;
    const double k7_8_10_3 = h7_8_22 + CDz * h7_8_10;
    const double h16_3_12 = acc[845] + ABz * acc[380];
    const double h7_8_12 = h16_3_12 + ABy * h7_3_12;
    const double k7_8_4_3 = h7_8_12 + CDz * h7_8_4;
    const double k7_8_4_6 = k7_8_10_3 + CDx * k7_8_4_3;
    const double h16_3_23 = acc[856] + ABz * acc[391];
    const double h7_8_23 = h16_3_23 + ABy * h7_3_23;
    const double k7_8_11_2 = h7_8_23 + CDy * h7_8_11;
    const double k7_8_4_7 = k7_8_11_2 + CDy * k7_8_4_2;
    const double h16_3_24 = acc[857] + ABz * acc[392];
    const double h7_8_24 = h16_3_24 + ABy * h7_3_24;
    const double k7_8_11_3 = h7_8_24 + CDz * h7_8_11;
    const double k7_8_4_8 = k7_8_11_3 + CDy * k7_8_4_3;
    const double h16_3_25 = acc[858] + ABz * acc[393];
    const double h7_8_25 = h16_3_25 + ABy * h7_3_25;
    const double k7_8_12_3 = h7_8_25 + CDz * h7_8_12;
    const double k7_8_4_9 = k7_8_12_3 + CDz * k7_8_4_3;
    const double k7_8_11_1 = h7_8_21 + CDx * h7_8_11;
    const double h16_3_5 = acc[838] + ABz * acc[373];
    const double h7_8_5 = h16_3_5 + ABy * h7_3_5;
    const double k7_8_5_1 = h7_8_11 + CDx * h7_8_5;
    const double k7_8_5_4 = k7_8_11_1 + CDx * k7_8_5_1;
    const double h16_3_13 = acc[846] + ABz * acc[381];
    const double h7_8_13 = h16_3_13 + ABy * h7_3_13;
    const double k7_8_5_2 = h7_8_13 + CDy * h7_8_5;
    const double k7_8_5_5 = k7_8_11_2 + CDx * k7_8_5_2;
    const double h16_3_15 = acc[848] + ABz * acc[383];
    const double h7_8_15 = h16_3_15 + ABy * h7_3_15;
    const double k7_8_5_3 = h7_8_15 + CDz * h7_8_5;
    const double k7_8_5_6 = k7_8_11_3 + CDx * k7_8_5_3;
    const double h16_3_26 = acc[859] + ABz * acc[394];
    const double h7_8_26 = h16_3_26 + ABy * h7_3_26;
    const double k7_8_13_2 = h7_8_26 + CDy * h7_8_13;
    const double k7_8_5_7 = k7_8_13_2 + CDy * k7_8_5_2;
    const double h16_3_27 = acc[860] + ABz * acc[395];
    const double h7_8_27 = h16_3_27 + ABy * h7_3_27;
    const double k7_8_13_3 = h7_8_27 + CDz * h7_8_13;
    const double k7_8_5_8 = k7_8_13_3 + CDy * k7_8_5_3;
    const double h16_3_28 = acc[861] + ABz * acc[396];
    const double h7_8_28 = h16_3_28 + ABy * h7_3_28;
    const double k7_8_15_3 = h7_8_28 + CDz * h7_8_15;
    const double k7_8_5_9 = k7_8_15_3 + CDz * k7_8_5_3;
    const double k7_8_12_1 = h7_8_22 + CDx * h7_8_12;
    const double h16_3_6 = acc[839] + ABz * acc[374];
    const double h7_8_6 = h16_3_6 + ABy * h7_3_6;
    const double k7_8_6_1 = h7_8_12 + CDx * h7_8_6;
    const double k7_8_6_4 = k7_8_12_1 + CDx * k7_8_6_1;
    const double k7_8_12_2 = h7_8_24 + CDy * h7_8_12;
    const double k7_8_6_2 = h7_8_15 + CDy * h7_8_6;
    const double k7_8_6_5 = k7_8_12_2 + CDx * k7_8_6_2;
    const double h16_3_14 = acc[847] + ABz * acc[382];
    const double h7_8_14 = h16_3_14 + ABy * h7_3_14;
    const double k7_8_6_3 = h7_8_14 + CDz * h7_8_6;
    const double k7_8_6_6 = k7_8_12_3 + CDx * k7_8_6_3;
    const double k7_8_15_2 = h7_8_27 + CDy * h7_8_15;
    const double k7_8_6_7 = k7_8_15_2 + CDy * k7_8_6_2;
    const double k7_8_6_8 = k7_8_15_3 + CDy * k7_8_6_3;
    const double h16_3_29 = acc[862] + ABz * acc[397];
    const double h7_8_29 = h16_3_29 + ABy * h7_3_29;
    const double k7_8_14_3 = h7_8_29 + CDz * h7_8_14;
    const double k7_8_6_9 = k7_8_14_3 + CDz * k7_8_6_3;
    const double k7_8_13_1 = h7_8_23 + CDx * h7_8_13;
    const double h16_3_7 = acc[840] + ABz * acc[375];
    const double h7_8_7 = h16_3_7 + ABy * h7_3_7;
    const double k7_8_7_1 = h7_8_13 + CDx * h7_8_7;
    const double k7_8_7_4 = k7_8_13_1 + CDx * k7_8_7_1;
    const double h16_3_16 = acc[849] + ABz * acc[384];
    const double h7_8_16 = h16_3_16 + ABy * h7_3_16;
    const double k7_8_7_2 = h7_8_16 + CDy * h7_8_7;
    const double k7_8_7_5 = k7_8_13_2 + CDx * k7_8_7_2;
    const double h16_3_17 = acc[850] + ABz * acc[385];
    const double h7_8_17 = h16_3_17 + ABy * h7_3_17;
    const double k7_8_7_3 = h7_8_17 + CDz * h7_8_7;
    const double k7_8_7_6 = k7_8_13_3 + CDx * k7_8_7_3;
    const double h16_3_30 = acc[863] + ABz * acc[398];
    const double h7_8_30 = h16_3_30 + ABy * h7_3_30;
    const double k7_8_16_2 = h7_8_30 + CDy * h7_8_16;
    const double k7_8_7_7 = k7_8_16_2 + CDy * k7_8_7_2;
    const double h16_3_31 = acc[864] + ABz * acc[399];
    const double h7_8_31 = h16_3_31 + ABy * h7_3_31;
    const double k7_8_16_3 = h7_8_31 + CDz * h7_8_16;
    const double k7_8_7_8 = k7_8_16_3 + CDy * k7_8_7_3;
    const double h16_3_32 = acc[865] + ABz * acc[400];
    const double h7_8_32 = h16_3_32 + ABy * h7_3_32;
    const double k7_8_17_3 = h7_8_32 + CDz * h7_8_17;
    const double k7_8_7_9 = k7_8_17_3 + CDz * k7_8_7_3;
    const double k7_8_15_1 = h7_8_24 + CDx * h7_8_15;
    const double h16_3_8 = acc[841] + ABz * acc[376];
    const double h7_8_8 = h16_3_8 + ABy * h7_3_8;
    const double k7_8_8_1 = h7_8_15 + CDx * h7_8_8;
    const double k7_8_8_4 = k7_8_15_1 + CDx * k7_8_8_1;
    const double k7_8_8_2 = h7_8_17 + CDy * h7_8_8;
    const double k7_8_8_5 = k7_8_15_2 + CDx * k7_8_8_2;
    const double h16_3_18 = acc[851] + ABz * acc[386];
    const double h7_8_18 = h16_3_18 + ABy * h7_3_18;
    const double k7_8_8_3 = h7_8_18 + CDz * h7_8_8;
    const double k7_8_8_6 = k7_8_15_3 + CDx * k7_8_8_3;
    const double k7_8_17_2 = h7_8_31 + CDy * h7_8_17;
    const double k7_8_8_7 = k7_8_17_2 + CDy * k7_8_8_2;
    const double k7_8_8_8 = k7_8_17_3 + CDy * k7_8_8_3;
    const double h16_3_33 = acc[866] + ABz * acc[401];
    const double h7_8_33 = h16_3_33 + ABy * h7_3_33;
    const double k7_8_18_3 = h7_8_33 + CDz * h7_8_18;
    const double k7_8_8_9 = k7_8_18_3 + CDz * k7_8_8_3;
    const double k7_8_14_1 = h7_8_25 + CDx * h7_8_14;
    const double h16_3_9 = acc[842] + ABz * acc[377];
    const double h7_8_9 = h16_3_9 + ABy * h7_3_9;
    const double k7_8_9_1 = h7_8_14 + CDx * h7_8_9;
    const double k7_8_9_4 = k7_8_14_1 + CDx * k7_8_9_1;
    const double k7_8_14_2 = h7_8_28 + CDy * h7_8_14;
    const double k7_8_9_2 = h7_8_18 + CDy * h7_8_9;
    const double k7_8_9_5 = k7_8_14_2 + CDx * k7_8_9_2;
    const double h16_3_19 = acc[852] + ABz * acc[387];
    const double h7_8_19 = h16_3_19 + ABy * h7_3_19;
    const double k7_8_9_3 = h7_8_19 + CDz * h7_8_9;
    const double k7_8_9_6 = k7_8_14_3 + CDx * k7_8_9_3;
    const double k7_8_18_2 = h7_8_32 + CDy * h7_8_18;
    const double k7_8_9_7 = k7_8_18_2 + CDy * k7_8_9_2;
    const double k7_8_9_8 = k7_8_18_3 + CDy * k7_8_9_3;
    const double h16_3_34 = acc[867] + ABz * acc[402];
    const double h7_8_34 = h16_3_34 + ABy * h7_3_34;
    const double k7_8_19_3 = h7_8_34 + CDz * h7_8_19;
    const double k7_8_9_9 = k7_8_19_3 + CDz * k7_8_9_3;
    const double h17_3_20 = acc[884] + ABz * acc[419];
    const double h7_9_20 = h17_3_20 + ABz * h7_3_20;
    const double h17_3_10 = acc[874] + ABz * acc[409];
    const double h7_9_10 = h17_3_10 + ABz * h7_3_10;
    const double k7_9_10_1 = h7_9_20 + CDx * h7_9_10;
    const double h17_3_4 = acc[868] + ABz * acc[403];
    const double h7_9_4 = h17_3_4 + ABz * h7_3_4;
    const double k7_9_4_1 = h7_9_10 + CDx * h7_9_4;
    const double k7_9_4_4 = k7_9_10_1 + CDx * k7_9_4_1;
    const double h17_3_21 = acc[885] + ABz * acc[420];
    const double h7_9_21 = h17_3_21 + ABz * h7_3_21;
    const double k7_9_10_2 = h7_9_21 + CDy * h7_9_10;
    const double h17_3_11 = acc[875] + ABz * acc[410];
    const double h7_9_11 = h17_3_11 + ABz * h7_3_11;
    const double k7_9_4_2 = h7_9_11 + CDy * h7_9_4;
    const double k7_9_4_5 = k7_9_10_2 + CDx * k7_9_4_2;
    const double h17_3_22 = acc[886] + ABz * acc[421];
    const double h7_9_22 = h17_3_22 + ABz * h7_3_22;
    const double k7_9_10_3 = h7_9_22 + CDz * h7_9_10;
    const double h17_3_12 = acc[876] + ABz * acc[411];
    const double h7_9_12 = h17_3_12 + ABz * h7_3_12;
    const double k7_9_4_3 = h7_9_12 + CDz * h7_9_4;
    const double k7_9_4_6 = k7_9_10_3 + CDx * k7_9_4_3;
    const double h17_3_23 = acc[887] + ABz * acc[422];
    const double h7_9_23 = h17_3_23 + ABz * h7_3_23;
    const double k7_9_11_2 = h7_9_23 + CDy * h7_9_11;
    const double k7_9_4_7 = k7_9_11_2 + CDy * k7_9_4_2;
    const double h17_3_24 = acc[888] + ABz * acc[423];
    const double h7_9_24 = h17_3_24 + ABz * h7_3_24;
    const double k7_9_11_3 = h7_9_24 + CDz * h7_9_11;
    const double k7_9_4_8 = k7_9_11_3 + CDy * k7_9_4_3;
    const double h17_3_25 = acc[889] + ABz * acc[424];
    const double h7_9_25 = h17_3_25 + ABz * h7_3_25;
    const double k7_9_12_3 = h7_9_25 + CDz * h7_9_12;
    const double k7_9_4_9 = k7_9_12_3 + CDz * k7_9_4_3;
    const double k7_9_11_1 = h7_9_21 + CDx * h7_9_11;
    const double h17_3_5 = acc[869] + ABz * acc[404];
    const double h7_9_5 = h17_3_5 + ABz * h7_3_5;
    const double k7_9_5_1 = h7_9_11 + CDx * h7_9_5;
    const double k7_9_5_4 = k7_9_11_1 + CDx * k7_9_5_1;
    const double h17_3_13 = acc[877] + ABz * acc[412];
    const double h7_9_13 = h17_3_13 + ABz * h7_3_13;
    const double k7_9_5_2 = h7_9_13 + CDy * h7_9_5;
    const double k7_9_5_5 = k7_9_11_2 + CDx * k7_9_5_2;
    const double h17_3_15 = acc[879] + ABz * acc[414];
    const double h7_9_15 = h17_3_15 + ABz * h7_3_15;
    const double k7_9_5_3 = h7_9_15 + CDz * h7_9_5;
    const double k7_9_5_6 = k7_9_11_3 + CDx * k7_9_5_3;
    const double h17_3_26 = acc[890] + ABz * acc[425];
    const double h7_9_26 = h17_3_26 + ABz * h7_3_26;
    const double k7_9_13_2 = h7_9_26 + CDy * h7_9_13;
    const double k7_9_5_7 = k7_9_13_2 + CDy * k7_9_5_2;
    const double h17_3_27 = acc[891] + ABz * acc[426];
    const double h7_9_27 = h17_3_27 + ABz * h7_3_27;
    const double k7_9_13_3 = h7_9_27 + CDz * h7_9_13;
    const double k7_9_5_8 = k7_9_13_3 + CDy * k7_9_5_3;
    const double h17_3_28 = acc[892] + ABz * acc[427];
    const double h7_9_28 = h17_3_28 + ABz * h7_3_28;
    const double k7_9_15_3 = h7_9_28 + CDz * h7_9_15;
    const double k7_9_5_9 = k7_9_15_3 + CDz * k7_9_5_3;
    const double k7_9_12_1 = h7_9_22 + CDx * h7_9_12;
    const double h17_3_6 = acc[870] + ABz * acc[405];
    const double h7_9_6 = h17_3_6 + ABz * h7_3_6;
    const double k7_9_6_1 = h7_9_12 + CDx * h7_9_6;
    const double k7_9_6_4 = k7_9_12_1 + CDx * k7_9_6_1;
    const double k7_9_12_2 = h7_9_24 + CDy * h7_9_12;
    const double k7_9_6_2 = h7_9_15 + CDy * h7_9_6;
    const double k7_9_6_5 = k7_9_12_2 + CDx * k7_9_6_2;
    const double h17_3_14 = acc[878] + ABz * acc[413];
    const double h7_9_14 = h17_3_14 + ABz * h7_3_14;
    const double k7_9_6_3 = h7_9_14 + CDz * h7_9_6;
    const double k7_9_6_6 = k7_9_12_3 + CDx * k7_9_6_3;
    const double k7_9_15_2 = h7_9_27 + CDy * h7_9_15;
    const double k7_9_6_7 = k7_9_15_2 + CDy * k7_9_6_2;
    const double k7_9_6_8 = k7_9_15_3 + CDy * k7_9_6_3;
    const double h17_3_29 = acc[893] + ABz * acc[428];
    const double h7_9_29 = h17_3_29 + ABz * h7_3_29;
    const double k7_9_14_3 = h7_9_29 + CDz * h7_9_14;
    const double k7_9_6_9 = k7_9_14_3 + CDz * k7_9_6_3;
    const double k7_9_13_1 = h7_9_23 + CDx * h7_9_13;
    const double h17_3_7 = acc[871] + ABz * acc[406];
    const double h7_9_7 = h17_3_7 + ABz * h7_3_7;
    const double k7_9_7_1 = h7_9_13 + CDx * h7_9_7;
    const double k7_9_7_4 = k7_9_13_1 + CDx * k7_9_7_1;
    const double h17_3_16 = acc[880] + ABz * acc[415];
    const double h7_9_16 = h17_3_16 + ABz * h7_3_16;
    const double k7_9_7_2 = h7_9_16 + CDy * h7_9_7;
    const double k7_9_7_5 = k7_9_13_2 + CDx * k7_9_7_2;
    const double h17_3_17 = acc[881] + ABz * acc[416];
    const double h7_9_17 = h17_3_17 + ABz * h7_3_17;
    const double k7_9_7_3 = h7_9_17 + CDz * h7_9_7;
    const double k7_9_7_6 = k7_9_13_3 + CDx * k7_9_7_3;
    const double h17_3_30 = acc[894] + ABz * acc[429];
    const double h7_9_30 = h17_3_30 + ABz * h7_3_30;
    const double k7_9_16_2 = h7_9_30 + CDy * h7_9_16;
    const double k7_9_7_7 = k7_9_16_2 + CDy * k7_9_7_2;
    const double h17_3_31 = acc[895] + ABz * acc[430];
    const double h7_9_31 = h17_3_31 + ABz * h7_3_31;
    const double k7_9_16_3 = h7_9_31 + CDz * h7_9_16;
    const double k7_9_7_8 = k7_9_16_3 + CDy * k7_9_7_3;
    const double h17_3_32 = acc[896] + ABz * acc[431];
    const double h7_9_32 = h17_3_32 + ABz * h7_3_32;
    const double k7_9_17_3 = h7_9_32 + CDz * h7_9_17;
    const double k7_9_7_9 = k7_9_17_3 + CDz * k7_9_7_3;
    const double k7_9_15_1 = h7_9_24 + CDx * h7_9_15;
    const double h17_3_8 = acc[872] + ABz * acc[407];
    const double h7_9_8 = h17_3_8 + ABz * h7_3_8;
    const double k7_9_8_1 = h7_9_15 + CDx * h7_9_8;
    const double k7_9_8_4 = k7_9_15_1 + CDx * k7_9_8_1;
    const double k7_9_8_2 = h7_9_17 + CDy * h7_9_8;
    const double k7_9_8_5 = k7_9_15_2 + CDx * k7_9_8_2;
    const double h17_3_18 = acc[882] + ABz * acc[417];
    const double h7_9_18 = h17_3_18 + ABz * h7_3_18;
    const double k7_9_8_3 = h7_9_18 + CDz * h7_9_8;
    const double k7_9_8_6 = k7_9_15_3 + CDx * k7_9_8_3;
    const double k7_9_17_2 = h7_9_31 + CDy * h7_9_17;
    const double k7_9_8_7 = k7_9_17_2 + CDy * k7_9_8_2;
    const double k7_9_8_8 = k7_9_17_3 + CDy * k7_9_8_3;
    const double h17_3_33 = acc[897] + ABz * acc[432];
    const double h7_9_33 = h17_3_33 + ABz * h7_3_33;
    const double k7_9_18_3 = h7_9_33 + CDz * h7_9_18;
    const double k7_9_8_9 = k7_9_18_3 + CDz * k7_9_8_3;
    const double k7_9_14_1 = h7_9_25 + CDx * h7_9_14;
    const double h17_3_9 = acc[873] + ABz * acc[408];
    const double h7_9_9 = h17_3_9 + ABz * h7_3_9;
    const double k7_9_9_1 = h7_9_14 + CDx * h7_9_9;
    const double k7_9_9_4 = k7_9_14_1 + CDx * k7_9_9_1;
    const double k7_9_14_2 = h7_9_28 + CDy * h7_9_14;
    const double k7_9_9_2 = h7_9_18 + CDy * h7_9_9;
    const double k7_9_9_5 = k7_9_14_2 + CDx * k7_9_9_2;
    const double h17_3_19 = acc[883] + ABz * acc[418];
    const double h7_9_19 = h17_3_19 + ABz * h7_3_19;
    const double k7_9_9_3 = h7_9_19 + CDz * h7_9_9;
    const double k7_9_9_6 = k7_9_14_3 + CDx * k7_9_9_3;
    const double k7_9_18_2 = h7_9_32 + CDy * h7_9_18;
    const double k7_9_9_7 = k7_9_18_2 + CDy * k7_9_9_2;
    const double k7_9_9_8 = k7_9_18_3 + CDy * k7_9_9_3;
    const double h17_3_34 = acc[898] + ABz * acc[433];
    const double h7_9_34 = h17_3_34 + ABz * h7_3_34;
    const double k7_9_19_3 = h7_9_34 + CDz * h7_9_19;
    const double k7_9_9_9 = k7_9_19_3 + CDz * k7_9_9_3;
    const double h15_1_20 = acc[636] + ABx * acc[357];
    const double h8_1_20 = acc[357] + ABx * acc[140];
    const double h8_4_20 = h15_1_20 + ABx * h8_1_20;
    const double h15_1_10 = acc[626] + ABx * acc[347];
    const double h8_1_10 = acc[347] + ABx * acc[130];
    const double h8_4_10 = h15_1_10 + ABx * h8_1_10;
    const double k8_4_10_1 = h8_4_20 + CDx * h8_4_10;
    const double h15_1_4 = acc[620] + ABx * acc[341];
    const double h8_1_4 = acc[341] + ABx * acc[124];
    const double h8_4_4 = h15_1_4 + ABx * h8_1_4;
    const double k8_4_4_1 = h8_4_10 + CDx * h8_4_4;
    const double k8_4_4_4 = k8_4_10_1 + CDx * k8_4_4_1;
    const double h15_1_21 = acc[637] + ABx * acc[358];
    const double h8_1_21 = acc[358] + ABx * acc[141];
    const double h8_4_21 = h15_1_21 + ABx * h8_1_21;
    const double k8_4_10_2 = h8_4_21 + CDy * h8_4_10;
    const double h15_1_11 = acc[627] + ABx * acc[348];
    const double h8_1_11 = acc[348] + ABx * acc[131];
    const double h8_4_11 = h15_1_11 + ABx * h8_1_11;
    const double k8_4_4_2 = h8_4_11 + CDy * h8_4_4;
    const double k8_4_4_5 = k8_4_10_2 + CDx * k8_4_4_2;
    const double h15_1_22 = acc[638] + ABx * acc[359];
    const double h8_1_22 = acc[359] + ABx * acc[142];
    const double h8_4_22 = h15_1_22 + ABx * h8_1_22;
    const double k8_4_10_3 = h8_4_22 + CDz * h8_4_10;
    const double h15_1_12 = acc[628] + ABx * acc[349];
    const double h8_1_12 = acc[349] + ABx * acc[132];
    const double h8_4_12 = h15_1_12 + ABx * h8_1_12;
    const double k8_4_4_3 = h8_4_12 + CDz * h8_4_4;
    const double k8_4_4_6 = k8_4_10_3 + CDx * k8_4_4_3;
    const double h15_1_23 = acc[639] + ABx * acc[360];
    const double h8_1_23 = acc[360] + ABx * acc[143];
    const double h8_4_23 = h15_1_23 + ABx * h8_1_23;
    const double k8_4_11_2 = h8_4_23 + CDy * h8_4_11;
    const double k8_4_4_7 = k8_4_11_2 + CDy * k8_4_4_2;
    const double h15_1_24 = acc[640] + ABx * acc[361];
    const double h8_1_24 = acc[361] + ABx * acc[144];
    const double h8_4_24 = h15_1_24 + ABx * h8_1_24;
    const double k8_4_11_3 = h8_4_24 + CDz * h8_4_11;
    const double k8_4_4_8 = k8_4_11_3 + CDy * k8_4_4_3;
    const double h15_1_25 = acc[641] + ABx * acc[362];
    const double h8_1_25 = acc[362] + ABx * acc[145];
    const double h8_4_25 = h15_1_25 + ABx * h8_1_25;
    const double k8_4_12_3 = h8_4_25 + CDz * h8_4_12;
    const double k8_4_4_9 = k8_4_12_3 + CDz * k8_4_4_3;
    const double k8_4_11_1 = h8_4_21 + CDx * h8_4_11;
    const double h15_1_5 = acc[621] + ABx * acc[342];
    const double h8_1_5 = acc[342] + ABx * acc[125];
    const double h8_4_5 = h15_1_5 + ABx * h8_1_5;
    const double k8_4_5_1 = h8_4_11 + CDx * h8_4_5;
    const double k8_4_5_4 = k8_4_11_1 + CDx * k8_4_5_1;
    const double h15_1_13 = acc[629] + ABx * acc[350];
    const double h8_1_13 = acc[350] + ABx * acc[133];
    const double h8_4_13 = h15_1_13 + ABx * h8_1_13;
    const double k8_4_5_2 = h8_4_13 + CDy * h8_4_5;
    const double k8_4_5_5 = k8_4_11_2 + CDx * k8_4_5_2;
    const double h15_1_15 = acc[631] + ABx * acc[352];
    const double h8_1_15 = acc[352] + ABx * acc[135];
    const double h8_4_15 = h15_1_15 + ABx * h8_1_15;
    const double k8_4_5_3 = h8_4_15 + CDz * h8_4_5;
    const double k8_4_5_6 = k8_4_11_3 + CDx * k8_4_5_3;
    const double h15_1_26 = acc[642] + ABx * acc[363];
    const double h8_1_26 = acc[363] + ABx * acc[146];
    const double h8_4_26 = h15_1_26 + ABx * h8_1_26;
    const double k8_4_13_2 = h8_4_26 + CDy * h8_4_13;
    const double k8_4_5_7 = k8_4_13_2 + CDy * k8_4_5_2;
    const double h15_1_27 = acc[643] + ABx * acc[364];
    const double h8_1_27 = acc[364] + ABx * acc[147];
    const double h8_4_27 = h15_1_27 + ABx * h8_1_27;
    const double k8_4_13_3 = h8_4_27 + CDz * h8_4_13;
    const double k8_4_5_8 = k8_4_13_3 + CDy * k8_4_5_3;
    const double h15_1_28 = acc[644] + ABx * acc[365];
    const double h8_1_28 = acc[365] + ABx * acc[148];
    const double h8_4_28 = h15_1_28 + ABx * h8_1_28;
    const double k8_4_15_3 = h8_4_28 + CDz * h8_4_15;
    const double k8_4_5_9 = k8_4_15_3 + CDz * k8_4_5_3;
    const double k8_4_12_1 = h8_4_22 + CDx * h8_4_12;
    const double h15_1_6 = acc[622] + ABx * acc[343];
    const double h8_1_6 = acc[343] + ABx * acc[126];
    const double h8_4_6 = h15_1_6 + ABx * h8_1_6;
    const double k8_4_6_1 = h8_4_12 + CDx * h8_4_6;
    const double k8_4_6_4 = k8_4_12_1 + CDx * k8_4_6_1;
    const double k8_4_12_2 = h8_4_24 + CDy * h8_4_12;
    const double k8_4_6_2 = h8_4_15 + CDy * h8_4_6;
    const double k8_4_6_5 = k8_4_12_2 + CDx * k8_4_6_2;
    const double h15_1_14 = acc[630] + ABx * acc[351];
    const double h8_1_14 = acc[351] + ABx * acc[134];
    const double h8_4_14 = h15_1_14 + ABx * h8_1_14;
    const double k8_4_6_3 = h8_4_14 + CDz * h8_4_6;
    const double k8_4_6_6 = k8_4_12_3 + CDx * k8_4_6_3;
    const double k8_4_15_2 = h8_4_27 + CDy * h8_4_15;
    const double k8_4_6_7 = k8_4_15_2 + CDy * k8_4_6_2;
    const double k8_4_6_8 = k8_4_15_3 + CDy * k8_4_6_3;
    const double h15_1_29 = acc[645] + ABx * acc[366];
    const double h8_1_29 = acc[366] + ABx * acc[149];
    const double h8_4_29 = h15_1_29 + ABx * h8_1_29;
    const double k8_4_14_3 = h8_4_29 + CDz * h8_4_14;
    const double k8_4_6_9 = k8_4_14_3 + CDz * k8_4_6_3;
    const double k8_4_13_1 = h8_4_23 + CDx * h8_4_13;
    const double h15_1_7 = acc[623] + ABx * acc[344];
    const double h8_1_7 = acc[344] + ABx * acc[127];
    const double h8_4_7 = h15_1_7 + ABx * h8_1_7;
    const double k8_4_7_1 = h8_4_13 + CDx * h8_4_7;
    const double k8_4_7_4 = k8_4_13_1 + CDx * k8_4_7_1;
    const double h15_1_16 = acc[632] + ABx * acc[353];
    const double h8_1_16 = acc[353] + ABx * acc[136];
    const double h8_4_16 = h15_1_16 + ABx * h8_1_16;
    const double k8_4_7_2 = h8_4_16 + CDy * h8_4_7;
    const double k8_4_7_5 = k8_4_13_2 + CDx * k8_4_7_2;
    const double h15_1_17 = acc[633] + ABx * acc[354];
    const double h8_1_17 = acc[354] + ABx * acc[137];
    const double h8_4_17 = h15_1_17 + ABx * h8_1_17;
    const double k8_4_7_3 = h8_4_17 + CDz * h8_4_7;
    const double k8_4_7_6 = k8_4_13_3 + CDx * k8_4_7_3;
    const double h15_1_30 = acc[646] + ABx * acc[367];
    const double h8_1_30 = acc[367] + ABx * acc[150];
    const double h8_4_30 = h15_1_30 + ABx * h8_1_30;
    const double k8_4_16_2 = h8_4_30 + CDy * h8_4_16;
    const double k8_4_7_7 = k8_4_16_2 + CDy * k8_4_7_2;
    const double h15_1_31 = acc[647] + ABx * acc[368];
    const double h8_1_31 = acc[368] + ABx * acc[151];
    const double h8_4_31 = h15_1_31 + ABx * h8_1_31;
    const double k8_4_16_3 = h8_4_31 + CDz * h8_4_16;
    const double k8_4_7_8 = k8_4_16_3 + CDy * k8_4_7_3;
    const double h15_1_32 = acc[648] + ABx * acc[369];
    const double h8_1_32 = acc[369] + ABx * acc[152];
    const double h8_4_32 = h15_1_32 + ABx * h8_1_32;
    const double k8_4_17_3 = h8_4_32 + CDz * h8_4_17;
    const double k8_4_7_9 = k8_4_17_3 + CDz * k8_4_7_3;
    const double k8_4_15_1 = h8_4_24 + CDx * h8_4_15;
    const double h15_1_8 = acc[624] + ABx * acc[345];
    const double h8_1_8 = acc[345] + ABx * acc[128];
    const double h8_4_8 = h15_1_8 + ABx * h8_1_8;
    const double k8_4_8_1 = h8_4_15 + CDx * h8_4_8;
    const double k8_4_8_4 = k8_4_15_1 + CDx * k8_4_8_1;
    const double k8_4_8_2 = h8_4_17 + CDy * h8_4_8;
    const double k8_4_8_5 = k8_4_15_2 + CDx * k8_4_8_2;
    const double h15_1_18 = acc[634] + ABx * acc[355];
    const double h8_1_18 = acc[355] + ABx * acc[138];
    const double h8_4_18 = h15_1_18 + ABx * h8_1_18;
    const double k8_4_8_3 = h8_4_18 + CDz * h8_4_8;
    const double k8_4_8_6 = k8_4_15_3 + CDx * k8_4_8_3;
    const double k8_4_17_2 = h8_4_31 + CDy * h8_4_17;
    const double k8_4_8_7 = k8_4_17_2 + CDy * k8_4_8_2;
    const double k8_4_8_8 = k8_4_17_3 + CDy * k8_4_8_3;
    const double h15_1_33 = acc[649] + ABx * acc[370];
    const double h8_1_33 = acc[370] + ABx * acc[153];
    const double h8_4_33 = h15_1_33 + ABx * h8_1_33;
    const double k8_4_18_3 = h8_4_33 + CDz * h8_4_18;
    const double k8_4_8_9 = k8_4_18_3 + CDz * k8_4_8_3;
    const double k8_4_14_1 = h8_4_25 + CDx * h8_4_14;
    const double h15_1_9 = acc[625] + ABx * acc[346];
    const double h8_1_9 = acc[346] + ABx * acc[129];
    const double h8_4_9 = h15_1_9 + ABx * h8_1_9;
    const double k8_4_9_1 = h8_4_14 + CDx * h8_4_9;
    const double k8_4_9_4 = k8_4_14_1 + CDx * k8_4_9_1;
    const double k8_4_14_2 = h8_4_28 + CDy * h8_4_14;
    const double k8_4_9_2 = h8_4_18 + CDy * h8_4_9;
    const double k8_4_9_5 = k8_4_14_2 + CDx * k8_4_9_2;
    const double h15_1_19 = acc[635] + ABx * acc[356];
    const double h8_1_19 = acc[356] + ABx * acc[139];
    const double h8_4_19 = h15_1_19 + ABx * h8_1_19;
    const double k8_4_9_3 = h8_4_19 + CDz * h8_4_9;
    const double k8_4_9_6 = k8_4_14_3 + CDx * k8_4_9_3;
    const double k8_4_18_2 = h8_4_32 + CDy * h8_4_18;
    const double k8_4_9_7 = k8_4_18_2 + CDy * k8_4_9_2;
    const double k8_4_9_8 = k8_4_18_3 + CDy * k8_4_9_3;
    const double h15_1_34 = acc[650] + ABx * acc[371];
    const double h8_1_34 = acc[371] + ABx * acc[154];
    const double h8_4_34 = h15_1_34 + ABx * h8_1_34;
    const double k8_4_19_3 = h8_4_34 + CDz * h8_4_19;
    const double k8_4_9_9 = k8_4_19_3 + CDz * k8_4_9_3;
    const double h8_2_20 = acc[419] + ABy * acc[140];
    const double h8_5_20 = h15_2_20 + ABx * h8_2_20;
    const double h8_2_10 = acc[409] + ABy * acc[130];
    const double h8_5_10 = h15_2_10 + ABx * h8_2_10;
    const double k8_5_10_1 = h8_5_20 + CDx * h8_5_10;
    const double h8_2_4 = acc[403] + ABy * acc[124];
    const double h8_5_4 = h15_2_4 + ABx * h8_2_4;
    const double k8_5_4_1 = h8_5_10 + CDx * h8_5_4;
    const double k8_5_4_4 = k8_5_10_1 + CDx * k8_5_4_1;
    const double h8_2_21 = acc[420] + ABy * acc[141];
    const double h8_5_21 = h15_2_21 + ABx * h8_2_21;
    const double k8_5_10_2 = h8_5_21 + CDy * h8_5_10;
    const double h8_2_11 = acc[410] + ABy * acc[131];
    const double h8_5_11 = h15_2_11 + ABx * h8_2_11;
    const double k8_5_4_2 = h8_5_11 + CDy * h8_5_4;
    const double k8_5_4_5 = k8_5_10_2 + CDx * k8_5_4_2;
    const double h8_2_22 = acc[421] + ABy * acc[142];
    const double h8_5_22 = h15_2_22 + ABx * h8_2_22;
    const double k8_5_10_3 = h8_5_22 + CDz * h8_5_10;
    const double h8_2_12 = acc[411] + ABy * acc[132];
    const double h8_5_12 = h15_2_12 + ABx * h8_2_12;
    const double k8_5_4_3 = h8_5_12 + CDz * h8_5_4;
    const double k8_5_4_6 = k8_5_10_3 + CDx * k8_5_4_3;
    const double h8_2_23 = acc[422] + ABy * acc[143];
    const double h8_5_23 = h15_2_23 + ABx * h8_2_23;
    const double k8_5_11_2 = h8_5_23 + CDy * h8_5_11;
    const double k8_5_4_7 = k8_5_11_2 + CDy * k8_5_4_2;
    const double h8_2_24 = acc[423] + ABy * acc[144];
    const double h8_5_24 = h15_2_24 + ABx * h8_2_24;
    const double k8_5_11_3 = h8_5_24 + CDz * h8_5_11;
    const double k8_5_4_8 = k8_5_11_3 + CDy * k8_5_4_3;
    const double h8_2_25 = acc[424] + ABy * acc[145];
    const double h8_5_25 = h15_2_25 + ABx * h8_2_25;
    const double k8_5_12_3 = h8_5_25 + CDz * h8_5_12;
    const double k8_5_4_9 = k8_5_12_3 + CDz * k8_5_4_3;
    const double k8_5_11_1 = h8_5_21 + CDx * h8_5_11;
    const double h8_2_5 = acc[404] + ABy * acc[125];
    const double h8_5_5 = h15_2_5 + ABx * h8_2_5;
    const double k8_5_5_1 = h8_5_11 + CDx * h8_5_5;
    const double k8_5_5_4 = k8_5_11_1 + CDx * k8_5_5_1;
    const double h8_2_13 = acc[412] + ABy * acc[133];
    const double h8_5_13 = h15_2_13 + ABx * h8_2_13;
    const double k8_5_5_2 = h8_5_13 + CDy * h8_5_5;
    const double k8_5_5_5 = k8_5_11_2 + CDx * k8_5_5_2;
    const double h8_2_15 = acc[414] + ABy * acc[135];
    const double h8_5_15 = h15_2_15 + ABx * h8_2_15;
    const double k8_5_5_3 = h8_5_15 + CDz * h8_5_5;
    const double k8_5_5_6 = k8_5_11_3 + CDx * k8_5_5_3;
    const double h8_2_26 = acc[425] + ABy * acc[146];
    const double h8_5_26 = h15_2_26 + ABx * h8_2_26;
    const double k8_5_13_2 = h8_5_26 + CDy * h8_5_13;
    const double k8_5_5_7 = k8_5_13_2 + CDy * k8_5_5_2;
    const double h8_2_27 = acc[426] + ABy * acc[147];
    const double h8_5_27 = h15_2_27 + ABx * h8_2_27;
    const double k8_5_13_3 = h8_5_27 + CDz * h8_5_13;
    const double k8_5_5_8 = k8_5_13_3 + CDy * k8_5_5_3;
    const double h8_2_28 = acc[427] + ABy * acc[148];
    const double h8_5_28 = h15_2_28 + ABx * h8_2_28;
    const double k8_5_15_3 = h8_5_28 + CDz * h8_5_15;
    const double k8_5_5_9 = k8_5_15_3 + CDz * k8_5_5_3;
    const double k8_5_12_1 = h8_5_22 + CDx * h8_5_12;
    const double h8_2_6 = acc[405] + ABy * acc[126];
    const double h8_5_6 = h15_2_6 + ABx * h8_2_6;
    const double k8_5_6_1 = h8_5_12 + CDx * h8_5_6;
    const double k8_5_6_4 = k8_5_12_1 + CDx * k8_5_6_1;
    const double k8_5_12_2 = h8_5_24 + CDy * h8_5_12;
    const double k8_5_6_2 = h8_5_15 + CDy * h8_5_6;
    const double k8_5_6_5 = k8_5_12_2 + CDx * k8_5_6_2;
    const double h8_2_14 = acc[413] + ABy * acc[134];
    const double h8_5_14 = h15_2_14 + ABx * h8_2_14;
    const double k8_5_6_3 = h8_5_14 + CDz * h8_5_6;
    const double k8_5_6_6 = k8_5_12_3 + CDx * k8_5_6_3;
    const double k8_5_15_2 = h8_5_27 + CDy * h8_5_15;
    const double k8_5_6_7 = k8_5_15_2 + CDy * k8_5_6_2;
    const double k8_5_6_8 = k8_5_15_3 + CDy * k8_5_6_3;
    const double h8_2_29 = acc[428] + ABy * acc[149];
    const double h8_5_29 = h15_2_29 + ABx * h8_2_29;
    const double k8_5_14_3 = h8_5_29 + CDz * h8_5_14;
    const double k8_5_6_9 = k8_5_14_3 + CDz * k8_5_6_3;
    const double k8_5_13_1 = h8_5_23 + CDx * h8_5_13;
    const double h8_2_7 = acc[406] + ABy * acc[127];
    const double h8_5_7 = h15_2_7 + ABx * h8_2_7;
    const double k8_5_7_1 = h8_5_13 + CDx * h8_5_7;
    const double k8_5_7_4 = k8_5_13_1 + CDx * k8_5_7_1;
    const double h8_2_16 = acc[415] + ABy * acc[136];
    const double h8_5_16 = h15_2_16 + ABx * h8_2_16;
    const double k8_5_7_2 = h8_5_16 + CDy * h8_5_7;
    const double k8_5_7_5 = k8_5_13_2 + CDx * k8_5_7_2;
    const double h8_2_17 = acc[416] + ABy * acc[137];
    const double h8_5_17 = h15_2_17 + ABx * h8_2_17;
    const double k8_5_7_3 = h8_5_17 + CDz * h8_5_7;
    const double k8_5_7_6 = k8_5_13_3 + CDx * k8_5_7_3;
    const double h8_2_30 = acc[429] + ABy * acc[150];
    const double h8_5_30 = h15_2_30 + ABx * h8_2_30;
    const double k8_5_16_2 = h8_5_30 + CDy * h8_5_16;
    const double k8_5_7_7 = k8_5_16_2 + CDy * k8_5_7_2;
    const double h8_2_31 = acc[430] + ABy * acc[151];
    const double h8_5_31 = h15_2_31 + ABx * h8_2_31;
    const double k8_5_16_3 = h8_5_31 + CDz * h8_5_16;
    const double k8_5_7_8 = k8_5_16_3 + CDy * k8_5_7_3;
    const double h8_2_32 = acc[431] + ABy * acc[152];
    const double h8_5_32 = h15_2_32 + ABx * h8_2_32;
    const double k8_5_17_3 = h8_5_32 + CDz * h8_5_17;
    const double k8_5_7_9 = k8_5_17_3 + CDz * k8_5_7_3;
    const double k8_5_15_1 = h8_5_24 + CDx * h8_5_15;
    const double h8_2_8 = acc[407] + ABy * acc[128];
    const double h8_5_8 = h15_2_8 + ABx * h8_2_8;
    const double k8_5_8_1 = h8_5_15 + CDx * h8_5_8;
    const double k8_5_8_4 = k8_5_15_1 + CDx * k8_5_8_1;
    const double k8_5_8_2 = h8_5_17 + CDy * h8_5_8;
    const double k8_5_8_5 = k8_5_15_2 + CDx * k8_5_8_2;
    const double h8_2_18 = acc[417] + ABy * acc[138];
    const double h8_5_18 = h15_2_18 + ABx * h8_2_18;
    const double k8_5_8_3 = h8_5_18 + CDz * h8_5_8;
    const double k8_5_8_6 = k8_5_15_3 + CDx * k8_5_8_3;
    const double k8_5_17_2 = h8_5_31 + CDy * h8_5_17;
    const double k8_5_8_7 = k8_5_17_2 + CDy * k8_5_8_2;
    const double k8_5_8_8 = k8_5_17_3 + CDy * k8_5_8_3;
    const double h8_2_33 = acc[432] + ABy * acc[153];
    const double h8_5_33 = h15_2_33 + ABx * h8_2_33;
    const double k8_5_18_3 = h8_5_33 + CDz * h8_5_18;
    const double k8_5_8_9 = k8_5_18_3 + CDz * k8_5_8_3;
    const double k8_5_14_1 = h8_5_25 + CDx * h8_5_14;
    const double h8_2_9 = acc[408] + ABy * acc[129];
    const double h8_5_9 = h15_2_9 + ABx * h8_2_9;
    const double k8_5_9_1 = h8_5_14 + CDx * h8_5_9;
    const double k8_5_9_4 = k8_5_14_1 + CDx * k8_5_9_1;
    const double k8_5_14_2 = h8_5_28 + CDy * h8_5_14;
    const double k8_5_9_2 = h8_5_18 + CDy * h8_5_9;
    const double k8_5_9_5 = k8_5_14_2 + CDx * k8_5_9_2;
    const double h8_2_19 = acc[418] + ABy * acc[139];
    const double h8_5_19 = h15_2_19 + ABx * h8_2_19;
    const double k8_5_9_3 = h8_5_19 + CDz * h8_5_9;
    const double k8_5_9_6 = k8_5_14_3 + CDx * k8_5_9_3;
    const double k8_5_18_2 = h8_5_32 + CDy * h8_5_18;
    const double k8_5_9_7 = k8_5_18_2 + CDy * k8_5_9_2;
    const double k8_5_9_8 = k8_5_18_3 + CDy * k8_5_9_3;
    const double h8_2_34 = acc[433] + ABy * acc[154];
    const double h8_5_34 = h15_2_34 + ABx * h8_2_34;
    const double k8_5_19_3 = h8_5_34 + CDz * h8_5_19;
    const double k8_5_9_9 = k8_5_19_3 + CDz * k8_5_9_3;
    const double h8_3_20 = acc[450] + ABz * acc[140];
    const double h8_6_20 = h15_3_20 + ABx * h8_3_20;
    const double h8_3_10 = acc[440] + ABz * acc[130];
    const double h8_6_10 = h15_3_10 + ABx * h8_3_10;
    const double k8_6_10_1 = h8_6_20 + CDx * h8_6_10;
    const double h8_3_4 = acc[434] + ABz * acc[124];
    const double h8_6_4 = h15_3_4 + ABx * h8_3_4;
    const double k8_6_4_1 = h8_6_10 + CDx * h8_6_4;
    const double k8_6_4_4 = k8_6_10_1 + CDx * k8_6_4_1;
    const double h8_3_21 = acc[451] + ABz * acc[141];
    const double h8_6_21 = h15_3_21 + ABx * h8_3_21;
    const double k8_6_10_2 = h8_6_21 + CDy * h8_6_10;
    const double h8_3_11 = acc[441] + ABz * acc[131];
    const double h8_6_11 = h15_3_11 + ABx * h8_3_11;
    const double k8_6_4_2 = h8_6_11 + CDy * h8_6_4;
    const double k8_6_4_5 = k8_6_10_2 + CDx * k8_6_4_2;
    const double h8_3_22 = acc[452] + ABz * acc[142];
    const double h8_6_22 = h15_3_22 + ABx * h8_3_22;
    const double k8_6_10_3 = h8_6_22 + CDz * h8_6_10;
    const double h8_3_12 = acc[442] + ABz * acc[132];
    const double h8_6_12 = h15_3_12 + ABx * h8_3_12;
    const double k8_6_4_3 = h8_6_12 + CDz * h8_6_4;
    const double k8_6_4_6 = k8_6_10_3 + CDx * k8_6_4_3;
    const double h8_3_23 = acc[453] + ABz * acc[143];
    const double h8_6_23 = h15_3_23 + ABx * h8_3_23;
    const double k8_6_11_2 = h8_6_23 + CDy * h8_6_11;
    const double k8_6_4_7 = k8_6_11_2 + CDy * k8_6_4_2;
    const double h8_3_24 = acc[454] + ABz * acc[144];
    const double h8_6_24 = h15_3_24 + ABx * h8_3_24;
    const double k8_6_11_3 = h8_6_24 + CDz * h8_6_11;
    const double k8_6_4_8 = k8_6_11_3 + CDy * k8_6_4_3;
    const double h8_3_25 = acc[455] + ABz * acc[145];
    const double h8_6_25 = h15_3_25 + ABx * h8_3_25;
    const double k8_6_12_3 = h8_6_25 + CDz * h8_6_12;
    const double k8_6_4_9 = k8_6_12_3 + CDz * k8_6_4_3;
    const double k8_6_11_1 = h8_6_21 + CDx * h8_6_11;
    const double h8_3_5 = acc[435] + ABz * acc[125];
    const double h8_6_5 = h15_3_5 + ABx * h8_3_5;
    const double k8_6_5_1 = h8_6_11 + CDx * h8_6_5;
    const double k8_6_5_4 = k8_6_11_1 + CDx * k8_6_5_1;
    const double h8_3_13 = acc[443] + ABz * acc[133];
    const double h8_6_13 = h15_3_13 + ABx * h8_3_13;
    const double k8_6_5_2 = h8_6_13 + CDy * h8_6_5;
    const double k8_6_5_5 = k8_6_11_2 + CDx * k8_6_5_2;
    const double h8_3_15 = acc[445] + ABz * acc[135];
    const double h8_6_15 = h15_3_15 + ABx * h8_3_15;
    const double k8_6_5_3 = h8_6_15 + CDz * h8_6_5;
    const double k8_6_5_6 = k8_6_11_3 + CDx * k8_6_5_3;
    const double h8_3_26 = acc[456] + ABz * acc[146];
    const double h8_6_26 = h15_3_26 + ABx * h8_3_26;
    const double k8_6_13_2 = h8_6_26 + CDy * h8_6_13;
    const double k8_6_5_7 = k8_6_13_2 + CDy * k8_6_5_2;
    const double h8_3_27 = acc[457] + ABz * acc[147];
    const double h8_6_27 = h15_3_27 + ABx * h8_3_27;
    const double k8_6_13_3 = h8_6_27 + CDz * h8_6_13;
    const double k8_6_5_8 = k8_6_13_3 + CDy * k8_6_5_3;
    const double h8_3_28 = acc[458] + ABz * acc[148];
    const double h8_6_28 = h15_3_28 + ABx * h8_3_28;
    const double k8_6_15_3 = h8_6_28 + CDz * h8_6_15;
    const double k8_6_5_9 = k8_6_15_3 + CDz * k8_6_5_3;
    const double k8_6_12_1 = h8_6_22 + CDx * h8_6_12;
    const double h8_3_6 = acc[436] + ABz * acc[126];
    const double h8_6_6 = h15_3_6 + ABx * h8_3_6;
    const double k8_6_6_1 = h8_6_12 + CDx * h8_6_6;
    const double k8_6_6_4 = k8_6_12_1 + CDx * k8_6_6_1;
    const double k8_6_12_2 = h8_6_24 + CDy * h8_6_12;
    const double k8_6_6_2 = h8_6_15 + CDy * h8_6_6;
    const double k8_6_6_5 = k8_6_12_2 + CDx * k8_6_6_2;
    const double h8_3_14 = acc[444] + ABz * acc[134];
    const double h8_6_14 = h15_3_14 + ABx * h8_3_14;
    const double k8_6_6_3 = h8_6_14 + CDz * h8_6_6;
    const double k8_6_6_6 = k8_6_12_3 + CDx * k8_6_6_3;
    const double k8_6_15_2 = h8_6_27 + CDy * h8_6_15;
    const double k8_6_6_7 = k8_6_15_2 + CDy * k8_6_6_2;
    const double k8_6_6_8 = k8_6_15_3 + CDy * k8_6_6_3;
    const double h8_3_29 = acc[459] + ABz * acc[149];
    const double h8_6_29 = h15_3_29 + ABx * h8_3_29;
    const double k8_6_14_3 = h8_6_29 + CDz * h8_6_14;
    const double k8_6_6_9 = k8_6_14_3 + CDz * k8_6_6_3;
    const double k8_6_13_1 = h8_6_23 + CDx * h8_6_13;
    const double h8_3_7 = acc[437] + ABz * acc[127];
    const double h8_6_7 = h15_3_7 + ABx * h8_3_7;
    const double k8_6_7_1 = h8_6_13 + CDx * h8_6_7;
    const double k8_6_7_4 = k8_6_13_1 + CDx * k8_6_7_1;
    const double h8_3_16 = acc[446] + ABz * acc[136];
    const double h8_6_16 = h15_3_16 + ABx * h8_3_16;
    const double k8_6_7_2 = h8_6_16 + CDy * h8_6_7;
    const double k8_6_7_5 = k8_6_13_2 + CDx * k8_6_7_2;
    const double h8_3_17 = acc[447] + ABz * acc[137];
    const double h8_6_17 = h15_3_17 + ABx * h8_3_17;
    const double k8_6_7_3 = h8_6_17 + CDz * h8_6_7;
    const double k8_6_7_6 = k8_6_13_3 + CDx * k8_6_7_3;
    const double h8_3_30 = acc[460] + ABz * acc[150];
    const double h8_6_30 = h15_3_30 + ABx * h8_3_30;
    const double k8_6_16_2 = h8_6_30 + CDy * h8_6_16;
    const double k8_6_7_7 = k8_6_16_2 + CDy * k8_6_7_2;
    const double h8_3_31 = acc[461] + ABz * acc[151];
    const double h8_6_31 = h15_3_31 + ABx * h8_3_31;
    const double k8_6_16_3 = h8_6_31 + CDz * h8_6_16;
    const double k8_6_7_8 = k8_6_16_3 + CDy * k8_6_7_3;
    const double h8_3_32 = acc[462] + ABz * acc[152];
    const double h8_6_32 = h15_3_32 + ABx * h8_3_32;
    const double k8_6_17_3 = h8_6_32 + CDz * h8_6_17;
    const double k8_6_7_9 = k8_6_17_3 + CDz * k8_6_7_3;
    const double k8_6_15_1 = h8_6_24 + CDx * h8_6_15;
    const double h8_3_8 = acc[438] + ABz * acc[128];
    const double h8_6_8 = h15_3_8 + ABx * h8_3_8;
    const double k8_6_8_1 = h8_6_15 + CDx * h8_6_8;
    const double k8_6_8_4 = k8_6_15_1 + CDx * k8_6_8_1;
    const double k8_6_8_2 = h8_6_17 + CDy * h8_6_8;
    const double k8_6_8_5 = k8_6_15_2 + CDx * k8_6_8_2;
    const double h8_3_18 = acc[448] + ABz * acc[138];
    const double h8_6_18 = h15_3_18 + ABx * h8_3_18;
    const double k8_6_8_3 = h8_6_18 + CDz * h8_6_8;
    const double k8_6_8_6 = k8_6_15_3 + CDx * k8_6_8_3;
    const double k8_6_17_2 = h8_6_31 + CDy * h8_6_17;
    const double k8_6_8_7 = k8_6_17_2 + CDy * k8_6_8_2;
    const double k8_6_8_8 = k8_6_17_3 + CDy * k8_6_8_3;
    const double h8_3_33 = acc[463] + ABz * acc[153];
    const double h8_6_33 = h15_3_33 + ABx * h8_3_33;
    const double k8_6_18_3 = h8_6_33 + CDz * h8_6_18;
    const double k8_6_8_9 = k8_6_18_3 + CDz * k8_6_8_3;
    const double k8_6_14_1 = h8_6_25 + CDx * h8_6_14;
    const double h8_3_9 = acc[439] + ABz * acc[129];
    const double h8_6_9 = h15_3_9 + ABx * h8_3_9;
    const double k8_6_9_1 = h8_6_14 + CDx * h8_6_9;
    const double k8_6_9_4 = k8_6_14_1 + CDx * k8_6_9_1;
    const double k8_6_14_2 = h8_6_28 + CDy * h8_6_14;
    const double k8_6_9_2 = h8_6_18 + CDy * h8_6_9;
    const double k8_6_9_5 = k8_6_14_2 + CDx * k8_6_9_2;
    const double h8_3_19 = acc[449] + ABz * acc[139];
    const double h8_6_19 = h15_3_19 + ABx * h8_3_19;
    const double k8_6_9_3 = h8_6_19 + CDz * h8_6_9;
    const double k8_6_9_6 = k8_6_14_3 + CDx * k8_6_9_3;
    const double k8_6_18_2 = h8_6_32 + CDy * h8_6_18;
    const double k8_6_9_7 = k8_6_18_2 + CDy * k8_6_9_2;
    const double k8_6_9_8 = k8_6_18_3 + CDy * k8_6_9_3;
    const double h8_3_34 = acc[464] + ABz * acc[154];
    const double h8_6_34 = h15_3_34 + ABx * h8_3_34;
    const double k8_6_19_3 = h8_6_34 + CDz * h8_6_19;
    const double k8_6_9_9 = k8_6_19_3 + CDz * k8_6_9_3;
    const double h17_2_20 = acc[853] + ABy * acc[419];
    const double h8_7_20 = h17_2_20 + ABy * h8_2_20;
    const double h17_2_10 = acc[843] + ABy * acc[409];
    const double h8_7_10 = h17_2_10 + ABy * h8_2_10;
    const double k8_7_10_1 = h8_7_20 + CDx * h8_7_10;
    const double h17_2_4 = acc[837] + ABy * acc[403];
    const double h8_7_4 = h17_2_4 + ABy * h8_2_4;
    const double k8_7_4_1 = h8_7_10 + CDx * h8_7_4;
    const double k8_7_4_4 = k8_7_10_1 + CDx * k8_7_4_1;
    const double h17_2_21 = acc[854] + ABy * acc[420];
    const double h8_7_21 = h17_2_21 + ABy * h8_2_21;
    const double k8_7_10_2 = h8_7_21 + CDy * h8_7_10;
    const double h17_2_11 = acc[844] + ABy * acc[410];
    const double h8_7_11 = h17_2_11 + ABy * h8_2_11;
    const double k8_7_4_2 = h8_7_11 + CDy * h8_7_4;
    const double k8_7_4_5 = k8_7_10_2 + CDx * k8_7_4_2;
    const double h17_2_22 = acc[855] + ABy * acc[421];
    const double h8_7_22 = h17_2_22 + ABy * h8_2_22;
    const double k8_7_10_3 = h8_7_22 + CDz * h8_7_10;
    const double h17_2_12 = acc[845] + ABy * acc[411];
    const double h8_7_12 = h17_2_12 + ABy * h8_2_12;
    const double k8_7_4_3 = h8_7_12 + CDz * h8_7_4;
    const double k8_7_4_6 = k8_7_10_3 + CDx * k8_7_4_3;
    const double h17_2_23 = acc[856] + ABy * acc[422];
    const double h8_7_23 = h17_2_23 + ABy * h8_2_23;
    const double k8_7_11_2 = h8_7_23 + CDy * h8_7_11;
    const double k8_7_4_7 = k8_7_11_2 + CDy * k8_7_4_2;
    const double h17_2_24 = acc[857] + ABy * acc[423];
    const double h8_7_24 = h17_2_24 + ABy * h8_2_24;
    const double k8_7_11_3 = h8_7_24 + CDz * h8_7_11;
    const double k8_7_4_8 = k8_7_11_3 + CDy * k8_7_4_3;
    const double h17_2_25 = acc[858] + ABy * acc[424];
    const double h8_7_25 = h17_2_25 + ABy * h8_2_25;
    const double k8_7_12_3 = h8_7_25 + CDz * h8_7_12;
    const double k8_7_4_9 = k8_7_12_3 + CDz * k8_7_4_3;
    const double k8_7_11_1 = h8_7_21 + CDx * h8_7_11;
    const double h17_2_5 = acc[838] + ABy * acc[404];
    const double h8_7_5 = h17_2_5 + ABy * h8_2_5;
    const double k8_7_5_1 = h8_7_11 + CDx * h8_7_5;
    const double k8_7_5_4 = k8_7_11_1 + CDx * k8_7_5_1;
    const double h17_2_13 = acc[846] + ABy * acc[412];
    const double h8_7_13 = h17_2_13 + ABy * h8_2_13;
    const double k8_7_5_2 = h8_7_13 + CDy * h8_7_5;
    const double k8_7_5_5 = k8_7_11_2 + CDx * k8_7_5_2;
    const double h17_2_15 = acc[848] + ABy * acc[414];
    const double h8_7_15 = h17_2_15 + ABy * h8_2_15;
    const double k8_7_5_3 = h8_7_15 + CDz * h8_7_5;
    const double k8_7_5_6 = k8_7_11_3 + CDx * k8_7_5_3;
    const double h17_2_26 = acc[859] + ABy * acc[425];
    const double h8_7_26 = h17_2_26 + ABy * h8_2_26;
    const double k8_7_13_2 = h8_7_26 + CDy * h8_7_13;
    const double k8_7_5_7 = k8_7_13_2 + CDy * k8_7_5_2;
    const double h17_2_27 = acc[860] + ABy * acc[426];
    const double h8_7_27 = h17_2_27 + ABy * h8_2_27;
    const double k8_7_13_3 = h8_7_27 + CDz * h8_7_13;
    const double k8_7_5_8 = k8_7_13_3 + CDy * k8_7_5_3;
    const double h17_2_28 = acc[861] + ABy * acc[427];
    const double h8_7_28 = h17_2_28 + ABy * h8_2_28;
    const double k8_7_15_3 = h8_7_28 + CDz * h8_7_15;
    const double k8_7_5_9 = k8_7_15_3 + CDz * k8_7_5_3;
    const double k8_7_12_1 = h8_7_22 + CDx * h8_7_12;
    const double h17_2_6 = acc[839] + ABy * acc[405];
    const double h8_7_6 = h17_2_6 + ABy * h8_2_6;
    const double k8_7_6_1 = h8_7_12 + CDx * h8_7_6;
    const double k8_7_6_4 = k8_7_12_1 + CDx * k8_7_6_1;
    const double k8_7_12_2 = h8_7_24 + CDy * h8_7_12;
    const double k8_7_6_2 = h8_7_15 + CDy * h8_7_6;
    const double k8_7_6_5 = k8_7_12_2 + CDx * k8_7_6_2;
    const double h17_2_14 = acc[847] + ABy * acc[413];
    const double h8_7_14 = h17_2_14 + ABy * h8_2_14;
    const double k8_7_6_3 = h8_7_14 + CDz * h8_7_6;
    const double k8_7_6_6 = k8_7_12_3 + CDx * k8_7_6_3;
    const double k8_7_15_2 = h8_7_27 + CDy * h8_7_15;
    const double k8_7_6_7 = k8_7_15_2 + CDy * k8_7_6_2;
    const double k8_7_6_8 = k8_7_15_3 + CDy * k8_7_6_3;
    const double h17_2_29 = acc[862] + ABy * acc[428];
    const double h8_7_29 = h17_2_29 + ABy * h8_2_29;
    const double k8_7_14_3 = h8_7_29 + CDz * h8_7_14;
    const double k8_7_6_9 = k8_7_14_3 + CDz * k8_7_6_3;
    const double k8_7_13_1 = h8_7_23 + CDx * h8_7_13;
    const double h17_2_7 = acc[840] + ABy * acc[406];
    const double h8_7_7 = h17_2_7 + ABy * h8_2_7;
    const double k8_7_7_1 = h8_7_13 + CDx * h8_7_7;
    const double k8_7_7_4 = k8_7_13_1 + CDx * k8_7_7_1;
    const double h17_2_16 = acc[849] + ABy * acc[415];
    const double h8_7_16 = h17_2_16 + ABy * h8_2_16;
    const double k8_7_7_2 = h8_7_16 + CDy * h8_7_7;
    const double k8_7_7_5 = k8_7_13_2 + CDx * k8_7_7_2;
    const double h17_2_17 = acc[850] + ABy * acc[416];
    const double h8_7_17 = h17_2_17 + ABy * h8_2_17;
    const double k8_7_7_3 = h8_7_17 + CDz * h8_7_7;
    const double k8_7_7_6 = k8_7_13_3 + CDx * k8_7_7_3;
    const double h17_2_30 = acc[863] + ABy * acc[429];
    const double h8_7_30 = h17_2_30 + ABy * h8_2_30;
    const double k8_7_16_2 = h8_7_30 + CDy * h8_7_16;
    const double k8_7_7_7 = k8_7_16_2 + CDy * k8_7_7_2;
    const double h17_2_31 = acc[864] + ABy * acc[430];
    const double h8_7_31 = h17_2_31 + ABy * h8_2_31;
    const double k8_7_16_3 = h8_7_31 + CDz * h8_7_16;
    const double k8_7_7_8 = k8_7_16_3 + CDy * k8_7_7_3;
    const double h17_2_32 = acc[865] + ABy * acc[431];
    const double h8_7_32 = h17_2_32 + ABy * h8_2_32;
    const double k8_7_17_3 = h8_7_32 + CDz * h8_7_17;
    const double k8_7_7_9 = k8_7_17_3 + CDz * k8_7_7_3;
    const double k8_7_15_1 = h8_7_24 + CDx * h8_7_15;
    const double h17_2_8 = acc[841] + ABy * acc[407];
    const double h8_7_8 = h17_2_8 + ABy * h8_2_8;
    const double k8_7_8_1 = h8_7_15 + CDx * h8_7_8;
    const double k8_7_8_4 = k8_7_15_1 + CDx * k8_7_8_1;
    const double k8_7_8_2 = h8_7_17 + CDy * h8_7_8;
    const double k8_7_8_5 = k8_7_15_2 + CDx * k8_7_8_2;
    const double h17_2_18 = acc[851] + ABy * acc[417];
    const double h8_7_18 = h17_2_18 + ABy * h8_2_18;
    const double k8_7_8_3 = h8_7_18 + CDz * h8_7_8;
    const double k8_7_8_6 = k8_7_15_3 + CDx * k8_7_8_3;
    const double k8_7_17_2 = h8_7_31 + CDy * h8_7_17;
    const double k8_7_8_7 = k8_7_17_2 + CDy * k8_7_8_2;
    const double k8_7_8_8 = k8_7_17_3 + CDy * k8_7_8_3;
    const double h17_2_33 = acc[866] + ABy * acc[432];
    const double h8_7_33 = h17_2_33 + ABy * h8_2_33;
    const double k8_7_18_3 = h8_7_33 + CDz * h8_7_18;
    const double k8_7_8_9 = k8_7_18_3 + CDz * k8_7_8_3;
    const double k8_7_14_1 = h8_7_25 + CDx * h8_7_14;
    const double h17_2_9 = acc[842] + ABy * acc[408];
    const double h8_7_9 = h17_2_9 + ABy * h8_2_9;
    const double k8_7_9_1 = h8_7_14 + CDx * h8_7_9;
    const double k8_7_9_4 = k8_7_14_1 + CDx * k8_7_9_1;
    const double k8_7_14_2 = h8_7_28 + CDy * h8_7_14;
    const double k8_7_9_2 = h8_7_18 + CDy * h8_7_9;
    const double k8_7_9_5 = k8_7_14_2 + CDx * k8_7_9_2;
    const double h17_2_19 = acc[852] + ABy * acc[418];
    const double h8_7_19 = h17_2_19 + ABy * h8_2_19;
    const double k8_7_9_3 = h8_7_19 + CDz * h8_7_9;
    const double k8_7_9_6 = k8_7_14_3 + CDx * k8_7_9_3;
    const double k8_7_18_2 = h8_7_32 + CDy * h8_7_18;
    const double k8_7_9_7 = k8_7_18_2 + CDy * k8_7_9_2;
    const double k8_7_9_8 = k8_7_18_3 + CDy * k8_7_9_3;
    const double h17_2_34 = acc[867] + ABy * acc[433];
    const double h8_7_34 = h17_2_34 + ABy * h8_2_34;
    const double k8_7_19_3 = h8_7_34 + CDz * h8_7_19;
    const double k8_7_9_9 = k8_7_19_3 + CDz * k8_7_9_3;
    const double h8_8_20 = h17_3_20 + ABy * h8_3_20;
    const double h8_8_10 = h17_3_10 + ABy * h8_3_10;
    const double k8_8_10_1 = h8_8_20 + CDx * h8_8_10;
    const double h8_8_4 = h17_3_4 + ABy * h8_3_4;
    const double k8_8_4_1 = h8_8_10 + CDx * h8_8_4;
    const double k8_8_4_4 = k8_8_10_1 + CDx * k8_8_4_1;
    const double h8_8_21 = h17_3_21 + ABy * h8_3_21;
    const double k8_8_10_2 = h8_8_21 + CDy * h8_8_10;
    const double h8_8_11 = h17_3_11 + ABy * h8_3_11;
    const double k8_8_4_2 = h8_8_11 + CDy * h8_8_4;
    const double k8_8_4_5 = k8_8_10_2 + CDx * k8_8_4_2;
    const double h8_8_22 = h17_3_22 + ABy * h8_3_22;
    const double k8_8_10_3 = h8_8_22 + CDz * h8_8_10;
    const double h8_8_12 = h17_3_12 + ABy * h8_3_12;
    const double k8_8_4_3 = h8_8_12 + CDz * h8_8_4;
    const double k8_8_4_6 = k8_8_10_3 + CDx * k8_8_4_3;
    const double h8_8_23 = h17_3_23 + ABy * h8_3_23;
    const double k8_8_11_2 = h8_8_23 + CDy * h8_8_11;
    const double k8_8_4_7 = k8_8_11_2 + CDy * k8_8_4_2;
    const double h8_8_24 = h17_3_24 + ABy * h8_3_24;
    const double k8_8_11_3 = h8_8_24 + CDz * h8_8_11;
    const double k8_8_4_8 = k8_8_11_3 + CDy * k8_8_4_3;
    const double h8_8_25 = h17_3_25 + ABy * h8_3_25;
    const double k8_8_12_3 = h8_8_25 + CDz * h8_8_12;
    const double k8_8_4_9 = k8_8_12_3 + CDz * k8_8_4_3;
    const double k8_8_11_1 = h8_8_21 + CDx * h8_8_11;
    const double h8_8_5 = h17_3_5 + ABy * h8_3_5;
    const double k8_8_5_1 = h8_8_11 + CDx * h8_8_5;
    const double k8_8_5_4 = k8_8_11_1 + CDx * k8_8_5_1;
    const double h8_8_13 = h17_3_13 + ABy * h8_3_13;
    const double k8_8_5_2 = h8_8_13 + CDy * h8_8_5;
    const double k8_8_5_5 = k8_8_11_2 + CDx * k8_8_5_2;
    const double h8_8_15 = h17_3_15 + ABy * h8_3_15;
    const double k8_8_5_3 = h8_8_15 + CDz * h8_8_5;
    const double k8_8_5_6 = k8_8_11_3 + CDx * k8_8_5_3;
    const double h8_8_26 = h17_3_26 + ABy * h8_3_26;
    const double k8_8_13_2 = h8_8_26 + CDy * h8_8_13;
    const double k8_8_5_7 = k8_8_13_2 + CDy * k8_8_5_2;
    const double h8_8_27 = h17_3_27 + ABy * h8_3_27;
    const double k8_8_13_3 = h8_8_27 + CDz * h8_8_13;
    const double k8_8_5_8 = k8_8_13_3 + CDy * k8_8_5_3;
    const double h8_8_28 = h17_3_28 + ABy * h8_3_28;
    const double k8_8_15_3 = h8_8_28 + CDz * h8_8_15;
    const double k8_8_5_9 = k8_8_15_3 + CDz * k8_8_5_3;
    const double k8_8_12_1 = h8_8_22 + CDx * h8_8_12;
    const double h8_8_6 = h17_3_6 + ABy * h8_3_6;
    const double k8_8_6_1 = h8_8_12 + CDx * h8_8_6;
    const double k8_8_6_4 = k8_8_12_1 + CDx * k8_8_6_1;
    const double k8_8_12_2 = h8_8_24 + CDy * h8_8_12;
    const double k8_8_6_2 = h8_8_15 + CDy * h8_8_6;
    const double k8_8_6_5 = k8_8_12_2 + CDx * k8_8_6_2;
    const double h8_8_14 = h17_3_14 + ABy * h8_3_14;
    const double k8_8_6_3 = h8_8_14 + CDz * h8_8_6;
    const double k8_8_6_6 = k8_8_12_3 + CDx * k8_8_6_3;
    const double k8_8_15_2 = h8_8_27 + CDy * h8_8_15;
    const double k8_8_6_7 = k8_8_15_2 + CDy * k8_8_6_2;
    const double k8_8_6_8 = k8_8_15_3 + CDy * k8_8_6_3;
    const double h8_8_29 = h17_3_29 + ABy * h8_3_29;
    const double k8_8_14_3 = h8_8_29 + CDz * h8_8_14;
    const double k8_8_6_9 = k8_8_14_3 + CDz * k8_8_6_3;
    const double k8_8_13_1 = h8_8_23 + CDx * h8_8_13;
    const double h8_8_7 = h17_3_7 + ABy * h8_3_7;
    const double k8_8_7_1 = h8_8_13 + CDx * h8_8_7;
    const double k8_8_7_4 = k8_8_13_1 + CDx * k8_8_7_1;
    const double h8_8_16 = h17_3_16 + ABy * h8_3_16;
    const double k8_8_7_2 = h8_8_16 + CDy * h8_8_7;
    const double k8_8_7_5 = k8_8_13_2 + CDx * k8_8_7_2;
    const double h8_8_17 = h17_3_17 + ABy * h8_3_17;
    const double k8_8_7_3 = h8_8_17 + CDz * h8_8_7;
    const double k8_8_7_6 = k8_8_13_3 + CDx * k8_8_7_3;
    const double h8_8_30 = h17_3_30 + ABy * h8_3_30;
    const double k8_8_16_2 = h8_8_30 + CDy * h8_8_16;
    const double k8_8_7_7 = k8_8_16_2 + CDy * k8_8_7_2;
    const double h8_8_31 = h17_3_31 + ABy * h8_3_31;
    const double k8_8_16_3 = h8_8_31 + CDz * h8_8_16;
    const double k8_8_7_8 = k8_8_16_3 + CDy * k8_8_7_3;
    const double h8_8_32 = h17_3_32 + ABy * h8_3_32;
    const double k8_8_17_3 = h8_8_32 + CDz * h8_8_17;
    const double k8_8_7_9 = k8_8_17_3 + CDz * k8_8_7_3;
    const double k8_8_15_1 = h8_8_24 + CDx * h8_8_15;
    const double h8_8_8 = h17_3_8 + ABy * h8_3_8;
    const double k8_8_8_1 = h8_8_15 + CDx * h8_8_8;
    const double k8_8_8_4 = k8_8_15_1 + CDx * k8_8_8_1;
    const double k8_8_8_2 = h8_8_17 + CDy * h8_8_8;
    const double k8_8_8_5 = k8_8_15_2 + CDx * k8_8_8_2;
    const double h8_8_18 = h17_3_18 + ABy * h8_3_18;
    const double k8_8_8_3 = h8_8_18 + CDz * h8_8_8;
    const double k8_8_8_6 = k8_8_15_3 + CDx * k8_8_8_3;
    const double k8_8_17_2 = h8_8_31 + CDy * h8_8_17;
    const double k8_8_8_7 = k8_8_17_2 + CDy * k8_8_8_2;
    const double k8_8_8_8 = k8_8_17_3 + CDy * k8_8_8_3;
    const double h8_8_33 = h17_3_33 + ABy * h8_3_33;
    const double k8_8_18_3 = h8_8_33 + CDz * h8_8_18;
    const double k8_8_8_9 = k8_8_18_3 + CDz * k8_8_8_3;
    const double k8_8_14_1 = h8_8_25 + CDx * h8_8_14;
    const double h8_8_9 = h17_3_9 + ABy * h8_3_9;
    const double k8_8_9_1 = h8_8_14 + CDx * h8_8_9;
    const double k8_8_9_4 = k8_8_14_1 + CDx * k8_8_9_1;
    const double k8_8_14_2 = h8_8_28 + CDy * h8_8_14;
    const double k8_8_9_2 = h8_8_18 + CDy * h8_8_9;
    const double k8_8_9_5 = k8_8_14_2 + CDx * k8_8_9_2;
    const double h8_8_19 = h17_3_19 + ABy * h8_3_19;
    const double k8_8_9_3 = h8_8_19 + CDz * h8_8_9;
    const double k8_8_9_6 = k8_8_14_3 + CDx * k8_8_9_3;
    const double k8_8_18_2 = h8_8_32 + CDy * h8_8_18;
    const double k8_8_9_7 = k8_8_18_2 + CDy * k8_8_9_2;
    const double k8_8_9_8 = k8_8_18_3 + CDy * k8_8_9_3;
    const double h8_8_34 = h17_3_34 + ABy * h8_3_34;
    const double k8_8_19_3 = h8_8_34 + CDz * h8_8_19;
    const double k8_8_9_9 = k8_8_19_3 + CDz * k8_8_9_3;
    const double h18_3_20 = acc[915] + ABz * acc[450];
    const double h8_9_20 = h18_3_20 + ABz * h8_3_20;
    const double h18_3_10 = acc[905] + ABz * acc[440];
    const double h8_9_10 = h18_3_10 + ABz * h8_3_10;
    const double k8_9_10_1 = h8_9_20 + CDx * h8_9_10;
    const double h18_3_4 = acc[899] + ABz * acc[434];
    const double h8_9_4 = h18_3_4 + ABz * h8_3_4;
    const double k8_9_4_1 = h8_9_10 + CDx * h8_9_4;
    const double k8_9_4_4 = k8_9_10_1 + CDx * k8_9_4_1;
    const double h18_3_21 = acc[916] + ABz * acc[451];
    const double h8_9_21 = h18_3_21 + ABz * h8_3_21;
    const double k8_9_10_2 = h8_9_21 + CDy * h8_9_10;
    const double h18_3_11 = acc[906] + ABz * acc[441];
    const double h8_9_11 = h18_3_11 + ABz * h8_3_11;
    const double k8_9_4_2 = h8_9_11 + CDy * h8_9_4;
    const double k8_9_4_5 = k8_9_10_2 + CDx * k8_9_4_2;
    const double h18_3_22 = acc[917] + ABz * acc[452];
    const double h8_9_22 = h18_3_22 + ABz * h8_3_22;
    const double k8_9_10_3 = h8_9_22 + CDz * h8_9_10;
    const double h18_3_12 = acc[907] + ABz * acc[442];
    const double h8_9_12 = h18_3_12 + ABz * h8_3_12;
    const double k8_9_4_3 = h8_9_12 + CDz * h8_9_4;
    const double k8_9_4_6 = k8_9_10_3 + CDx * k8_9_4_3;
    const double h18_3_23 = acc[918] + ABz * acc[453];
    const double h8_9_23 = h18_3_23 + ABz * h8_3_23;
    const double k8_9_11_2 = h8_9_23 + CDy * h8_9_11;
    const double k8_9_4_7 = k8_9_11_2 + CDy * k8_9_4_2;
    const double h18_3_24 = acc[919] + ABz * acc[454];
    const double h8_9_24 = h18_3_24 + ABz * h8_3_24;
    const double k8_9_11_3 = h8_9_24 + CDz * h8_9_11;
    const double k8_9_4_8 = k8_9_11_3 + CDy * k8_9_4_3;
    const double h18_3_25 = acc[920] + ABz * acc[455];
    const double h8_9_25 = h18_3_25 + ABz * h8_3_25;
    const double k8_9_12_3 = h8_9_25 + CDz * h8_9_12;
    const double k8_9_4_9 = k8_9_12_3 + CDz * k8_9_4_3;
    const double k8_9_11_1 = h8_9_21 + CDx * h8_9_11;
    const double h18_3_5 = acc[900] + ABz * acc[435];
    const double h8_9_5 = h18_3_5 + ABz * h8_3_5;
    const double k8_9_5_1 = h8_9_11 + CDx * h8_9_5;
    const double k8_9_5_4 = k8_9_11_1 + CDx * k8_9_5_1;
    const double h18_3_13 = acc[908] + ABz * acc[443];
    const double h8_9_13 = h18_3_13 + ABz * h8_3_13;
    const double k8_9_5_2 = h8_9_13 + CDy * h8_9_5;
    const double k8_9_5_5 = k8_9_11_2 + CDx * k8_9_5_2;
    const double h18_3_15 = acc[910] + ABz * acc[445];
    const double h8_9_15 = h18_3_15 + ABz * h8_3_15;
    const double k8_9_5_3 = h8_9_15 + CDz * h8_9_5;
    const double k8_9_5_6 = k8_9_11_3 + CDx * k8_9_5_3;
    const double h18_3_26 = acc[921] + ABz * acc[456];
    const double h8_9_26 = h18_3_26 + ABz * h8_3_26;
    const double k8_9_13_2 = h8_9_26 + CDy * h8_9_13;
    const double k8_9_5_7 = k8_9_13_2 + CDy * k8_9_5_2;
    const double h18_3_27 = acc[922] + ABz * acc[457];
    const double h8_9_27 = h18_3_27 + ABz * h8_3_27;
    const double k8_9_13_3 = h8_9_27 + CDz * h8_9_13;
    const double k8_9_5_8 = k8_9_13_3 + CDy * k8_9_5_3;
    const double h18_3_28 = acc[923] + ABz * acc[458];
    const double h8_9_28 = h18_3_28 + ABz * h8_3_28;
    const double k8_9_15_3 = h8_9_28 + CDz * h8_9_15;
    const double k8_9_5_9 = k8_9_15_3 + CDz * k8_9_5_3;
    const double k8_9_12_1 = h8_9_22 + CDx * h8_9_12;
    const double h18_3_6 = acc[901] + ABz * acc[436];
    const double h8_9_6 = h18_3_6 + ABz * h8_3_6;
    const double k8_9_6_1 = h8_9_12 + CDx * h8_9_6;
    const double k8_9_6_4 = k8_9_12_1 + CDx * k8_9_6_1;
    const double k8_9_12_2 = h8_9_24 + CDy * h8_9_12;
    const double k8_9_6_2 = h8_9_15 + CDy * h8_9_6;
    const double k8_9_6_5 = k8_9_12_2 + CDx * k8_9_6_2;
    const double h18_3_14 = acc[909] + ABz * acc[444];
    const double h8_9_14 = h18_3_14 + ABz * h8_3_14;
    const double k8_9_6_3 = h8_9_14 + CDz * h8_9_6;
    const double k8_9_6_6 = k8_9_12_3 + CDx * k8_9_6_3;
    const double k8_9_15_2 = h8_9_27 + CDy * h8_9_15;
    const double k8_9_6_7 = k8_9_15_2 + CDy * k8_9_6_2;
    const double k8_9_6_8 = k8_9_15_3 + CDy * k8_9_6_3;
    const double h18_3_29 = acc[924] + ABz * acc[459];
    const double h8_9_29 = h18_3_29 + ABz * h8_3_29;
    const double k8_9_14_3 = h8_9_29 + CDz * h8_9_14;
    const double k8_9_6_9 = k8_9_14_3 + CDz * k8_9_6_3;
    const double k8_9_13_1 = h8_9_23 + CDx * h8_9_13;
    const double h18_3_7 = acc[902] + ABz * acc[437];
    const double h8_9_7 = h18_3_7 + ABz * h8_3_7;
    const double k8_9_7_1 = h8_9_13 + CDx * h8_9_7;
    const double k8_9_7_4 = k8_9_13_1 + CDx * k8_9_7_1;
    const double h18_3_16 = acc[911] + ABz * acc[446];
    const double h8_9_16 = h18_3_16 + ABz * h8_3_16;
    const double k8_9_7_2 = h8_9_16 + CDy * h8_9_7;
    const double k8_9_7_5 = k8_9_13_2 + CDx * k8_9_7_2;
    const double h18_3_17 = acc[912] + ABz * acc[447];
    const double h8_9_17 = h18_3_17 + ABz * h8_3_17;
    const double k8_9_7_3 = h8_9_17 + CDz * h8_9_7;
    const double k8_9_7_6 = k8_9_13_3 + CDx * k8_9_7_3;
    const double h18_3_30 = acc[925] + ABz * acc[460];
    const double h8_9_30 = h18_3_30 + ABz * h8_3_30;
    const double k8_9_16_2 = h8_9_30 + CDy * h8_9_16;
    const double k8_9_7_7 = k8_9_16_2 + CDy * k8_9_7_2;
    const double h18_3_31 = acc[926] + ABz * acc[461];
    const double h8_9_31 = h18_3_31 + ABz * h8_3_31;
    const double k8_9_16_3 = h8_9_31 + CDz * h8_9_16;
    const double k8_9_7_8 = k8_9_16_3 + CDy * k8_9_7_3;
    const double h18_3_32 = acc[927] + ABz * acc[462];
    const double h8_9_32 = h18_3_32 + ABz * h8_3_32;
    const double k8_9_17_3 = h8_9_32 + CDz * h8_9_17;
    const double k8_9_7_9 = k8_9_17_3 + CDz * k8_9_7_3;
    const double k8_9_15_1 = h8_9_24 + CDx * h8_9_15;
    const double h18_3_8 = acc[903] + ABz * acc[438];
    const double h8_9_8 = h18_3_8 + ABz * h8_3_8;
    const double k8_9_8_1 = h8_9_15 + CDx * h8_9_8;
    const double k8_9_8_4 = k8_9_15_1 + CDx * k8_9_8_1;
    const double k8_9_8_2 = h8_9_17 + CDy * h8_9_8;
    const double k8_9_8_5 = k8_9_15_2 + CDx * k8_9_8_2;
    const double h18_3_18 = acc[913] + ABz * acc[448];
    const double h8_9_18 = h18_3_18 + ABz * h8_3_18;
    const double k8_9_8_3 = h8_9_18 + CDz * h8_9_8;
    const double k8_9_8_6 = k8_9_15_3 + CDx * k8_9_8_3;
    const double k8_9_17_2 = h8_9_31 + CDy * h8_9_17;
    const double k8_9_8_7 = k8_9_17_2 + CDy * k8_9_8_2;
    const double k8_9_8_8 = k8_9_17_3 + CDy * k8_9_8_3;
    const double h18_3_33 = acc[928] + ABz * acc[463];
    const double h8_9_33 = h18_3_33 + ABz * h8_3_33;
    const double k8_9_18_3 = h8_9_33 + CDz * h8_9_18;
    const double k8_9_8_9 = k8_9_18_3 + CDz * k8_9_8_3;
    const double k8_9_14_1 = h8_9_25 + CDx * h8_9_14;
    const double h18_3_9 = acc[904] + ABz * acc[439];
    const double h8_9_9 = h18_3_9 + ABz * h8_3_9;
    const double k8_9_9_1 = h8_9_14 + CDx * h8_9_9;
    const double k8_9_9_4 = k8_9_14_1 + CDx * k8_9_9_1;
    const double k8_9_14_2 = h8_9_28 + CDy * h8_9_14;
    const double k8_9_9_2 = h8_9_18 + CDy * h8_9_9;
    const double k8_9_9_5 = k8_9_14_2 + CDx * k8_9_9_2;
    const double h18_3_19 = acc[914] + ABz * acc[449];
    const double h8_9_19 = h18_3_19 + ABz * h8_3_19;
    const double k8_9_9_3 = h8_9_19 + CDz * h8_9_9;
    const double k8_9_9_6 = k8_9_14_3 + CDx * k8_9_9_3;
    const double k8_9_18_2 = h8_9_32 + CDy * h8_9_18;
    const double k8_9_9_7 = k8_9_18_2 + CDy * k8_9_9_2;
    const double k8_9_9_8 = k8_9_18_3 + CDy * k8_9_9_3;
    const double h18_3_34 = acc[929] + ABz * acc[464];
    const double h8_9_34 = h18_3_34 + ABz * h8_3_34;
    const double k8_9_19_3 = h8_9_34 + CDz * h8_9_19;
    const double k8_9_9_9 = k8_9_19_3 + CDz * k8_9_9_3;
    const double h14_1_20 = acc[667] + ABx * acc[326];
    const double h9_1_20 = acc[326] + ABx * acc[171];
    const double h9_4_20 = h14_1_20 + ABx * h9_1_20;
    const double h14_1_10 = acc[657] + ABx * acc[316];
    const double h9_1_10 = acc[316] + ABx * acc[161];
    const double h9_4_10 = h14_1_10 + ABx * h9_1_10;
    const double k9_4_10_1 = h9_4_20 + CDx * h9_4_10;
    const double h14_1_4 = acc[651] + ABx * acc[310];
    const double h9_1_4 = acc[310] + ABx * acc[155];
    const double h9_4_4 = h14_1_4 + ABx * h9_1_4;
    const double k9_4_4_1 = h9_4_10 + CDx * h9_4_4;
    const double k9_4_4_4 = k9_4_10_1 + CDx * k9_4_4_1;
    const double h14_1_21 = acc[668] + ABx * acc[327];
    const double h9_1_21 = acc[327] + ABx * acc[172];
    const double h9_4_21 = h14_1_21 + ABx * h9_1_21;
    const double k9_4_10_2 = h9_4_21 + CDy * h9_4_10;
    const double h14_1_11 = acc[658] + ABx * acc[317];
    const double h9_1_11 = acc[317] + ABx * acc[162];
    const double h9_4_11 = h14_1_11 + ABx * h9_1_11;
    const double k9_4_4_2 = h9_4_11 + CDy * h9_4_4;
    const double k9_4_4_5 = k9_4_10_2 + CDx * k9_4_4_2;
    const double h14_1_22 = acc[669] + ABx * acc[328];
    const double h9_1_22 = acc[328] + ABx * acc[173];
    const double h9_4_22 = h14_1_22 + ABx * h9_1_22;
    const double k9_4_10_3 = h9_4_22 + CDz * h9_4_10;
    const double h14_1_12 = acc[659] + ABx * acc[318];
    const double h9_1_12 = acc[318] + ABx * acc[163];
    const double h9_4_12 = h14_1_12 + ABx * h9_1_12;
    const double k9_4_4_3 = h9_4_12 + CDz * h9_4_4;
    const double k9_4_4_6 = k9_4_10_3 + CDx * k9_4_4_3;
    const double h14_1_23 = acc[670] + ABx * acc[329];
    const double h9_1_23 = acc[329] + ABx * acc[174];
    const double h9_4_23 = h14_1_23 + ABx * h9_1_23;
    const double k9_4_11_2 = h9_4_23 + CDy * h9_4_11;
    const double k9_4_4_7 = k9_4_11_2 + CDy * k9_4_4_2;
    const double h14_1_24 = acc[671] + ABx * acc[330];
    const double h9_1_24 = acc[330] + ABx * acc[175];
    const double h9_4_24 = h14_1_24 + ABx * h9_1_24;
    const double k9_4_11_3 = h9_4_24 + CDz * h9_4_11;
    const double k9_4_4_8 = k9_4_11_3 + CDy * k9_4_4_3;
    const double h14_1_25 = acc[672] + ABx * acc[331];
    const double h9_1_25 = acc[331] + ABx * acc[176];
    const double h9_4_25 = h14_1_25 + ABx * h9_1_25;
    const double k9_4_12_3 = h9_4_25 + CDz * h9_4_12;
    const double k9_4_4_9 = k9_4_12_3 + CDz * k9_4_4_3;
    const double k9_4_11_1 = h9_4_21 + CDx * h9_4_11;
    const double h14_1_5 = acc[652] + ABx * acc[311];
    const double h9_1_5 = acc[311] + ABx * acc[156];
    const double h9_4_5 = h14_1_5 + ABx * h9_1_5;
    const double k9_4_5_1 = h9_4_11 + CDx * h9_4_5;
    const double k9_4_5_4 = k9_4_11_1 + CDx * k9_4_5_1;
    const double h14_1_13 = acc[660] + ABx * acc[319];
    const double h9_1_13 = acc[319] + ABx * acc[164];
    const double h9_4_13 = h14_1_13 + ABx * h9_1_13;
    const double k9_4_5_2 = h9_4_13 + CDy * h9_4_5;
    const double k9_4_5_5 = k9_4_11_2 + CDx * k9_4_5_2;
    const double h14_1_15 = acc[662] + ABx * acc[321];
    const double h9_1_15 = acc[321] + ABx * acc[166];
    const double h9_4_15 = h14_1_15 + ABx * h9_1_15;
    const double k9_4_5_3 = h9_4_15 + CDz * h9_4_5;
    const double k9_4_5_6 = k9_4_11_3 + CDx * k9_4_5_3;
    const double h14_1_26 = acc[673] + ABx * acc[332];
    const double h9_1_26 = acc[332] + ABx * acc[177];
    const double h9_4_26 = h14_1_26 + ABx * h9_1_26;
    const double k9_4_13_2 = h9_4_26 + CDy * h9_4_13;
    const double k9_4_5_7 = k9_4_13_2 + CDy * k9_4_5_2;
    const double h14_1_27 = acc[674] + ABx * acc[333];
    const double h9_1_27 = acc[333] + ABx * acc[178];
    const double h9_4_27 = h14_1_27 + ABx * h9_1_27;
    const double k9_4_13_3 = h9_4_27 + CDz * h9_4_13;
    const double k9_4_5_8 = k9_4_13_3 + CDy * k9_4_5_3;
    const double h14_1_28 = acc[675] + ABx * acc[334];
    const double h9_1_28 = acc[334] + ABx * acc[179];
    const double h9_4_28 = h14_1_28 + ABx * h9_1_28;
    const double k9_4_15_3 = h9_4_28 + CDz * h9_4_15;
    const double k9_4_5_9 = k9_4_15_3 + CDz * k9_4_5_3;
    const double k9_4_12_1 = h9_4_22 + CDx * h9_4_12;
    const double h14_1_6 = acc[653] + ABx * acc[312];
    const double h9_1_6 = acc[312] + ABx * acc[157];
    const double h9_4_6 = h14_1_6 + ABx * h9_1_6;
    const double k9_4_6_1 = h9_4_12 + CDx * h9_4_6;
    const double k9_4_6_4 = k9_4_12_1 + CDx * k9_4_6_1;
    const double k9_4_12_2 = h9_4_24 + CDy * h9_4_12;
    const double k9_4_6_2 = h9_4_15 + CDy * h9_4_6;
    const double k9_4_6_5 = k9_4_12_2 + CDx * k9_4_6_2;
    const double h14_1_14 = acc[661] + ABx * acc[320];
    const double h9_1_14 = acc[320] + ABx * acc[165];
    const double h9_4_14 = h14_1_14 + ABx * h9_1_14;
    const double k9_4_6_3 = h9_4_14 + CDz * h9_4_6;
    const double k9_4_6_6 = k9_4_12_3 + CDx * k9_4_6_3;
    const double k9_4_15_2 = h9_4_27 + CDy * h9_4_15;
    const double k9_4_6_7 = k9_4_15_2 + CDy * k9_4_6_2;
    const double k9_4_6_8 = k9_4_15_3 + CDy * k9_4_6_3;
    const double h14_1_29 = acc[676] + ABx * acc[335];
    const double h9_1_29 = acc[335] + ABx * acc[180];
    const double h9_4_29 = h14_1_29 + ABx * h9_1_29;
    const double k9_4_14_3 = h9_4_29 + CDz * h9_4_14;
    const double k9_4_6_9 = k9_4_14_3 + CDz * k9_4_6_3;
    const double k9_4_13_1 = h9_4_23 + CDx * h9_4_13;
    const double h14_1_7 = acc[654] + ABx * acc[313];
    const double h9_1_7 = acc[313] + ABx * acc[158];
    const double h9_4_7 = h14_1_7 + ABx * h9_1_7;
    const double k9_4_7_1 = h9_4_13 + CDx * h9_4_7;
    const double k9_4_7_4 = k9_4_13_1 + CDx * k9_4_7_1;
    const double h14_1_16 = acc[663] + ABx * acc[322];
    const double h9_1_16 = acc[322] + ABx * acc[167];
    const double h9_4_16 = h14_1_16 + ABx * h9_1_16;
    const double k9_4_7_2 = h9_4_16 + CDy * h9_4_7;
    const double k9_4_7_5 = k9_4_13_2 + CDx * k9_4_7_2;
    const double h14_1_17 = acc[664] + ABx * acc[323];
    const double h9_1_17 = acc[323] + ABx * acc[168];
    const double h9_4_17 = h14_1_17 + ABx * h9_1_17;
    const double k9_4_7_3 = h9_4_17 + CDz * h9_4_7;
    const double k9_4_7_6 = k9_4_13_3 + CDx * k9_4_7_3;
    const double h14_1_30 = acc[677] + ABx * acc[336];
    const double h9_1_30 = acc[336] + ABx * acc[181];
    const double h9_4_30 = h14_1_30 + ABx * h9_1_30;
    const double k9_4_16_2 = h9_4_30 + CDy * h9_4_16;
    const double k9_4_7_7 = k9_4_16_2 + CDy * k9_4_7_2;
    const double h14_1_31 = acc[678] + ABx * acc[337];
    const double h9_1_31 = acc[337] + ABx * acc[182];
    const double h9_4_31 = h14_1_31 + ABx * h9_1_31;
    const double k9_4_16_3 = h9_4_31 + CDz * h9_4_16;
    const double k9_4_7_8 = k9_4_16_3 + CDy * k9_4_7_3;
    const double h14_1_32 = acc[679] + ABx * acc[338];
    const double h9_1_32 = acc[338] + ABx * acc[183];
    const double h9_4_32 = h14_1_32 + ABx * h9_1_32;
    const double k9_4_17_3 = h9_4_32 + CDz * h9_4_17;
    const double k9_4_7_9 = k9_4_17_3 + CDz * k9_4_7_3;
    const double k9_4_15_1 = h9_4_24 + CDx * h9_4_15;
    const double h14_1_8 = acc[655] + ABx * acc[314];
    const double h9_1_8 = acc[314] + ABx * acc[159];
    const double h9_4_8 = h14_1_8 + ABx * h9_1_8;
    const double k9_4_8_1 = h9_4_15 + CDx * h9_4_8;
    const double k9_4_8_4 = k9_4_15_1 + CDx * k9_4_8_1;
    const double k9_4_8_2 = h9_4_17 + CDy * h9_4_8;
    const double k9_4_8_5 = k9_4_15_2 + CDx * k9_4_8_2;
    const double h14_1_18 = acc[665] + ABx * acc[324];
    const double h9_1_18 = acc[324] + ABx * acc[169];
    const double h9_4_18 = h14_1_18 + ABx * h9_1_18;
    const double k9_4_8_3 = h9_4_18 + CDz * h9_4_8;
    const double k9_4_8_6 = k9_4_15_3 + CDx * k9_4_8_3;
    const double k9_4_17_2 = h9_4_31 + CDy * h9_4_17;
    const double k9_4_8_7 = k9_4_17_2 + CDy * k9_4_8_2;
    const double k9_4_8_8 = k9_4_17_3 + CDy * k9_4_8_3;
    const double h14_1_33 = acc[680] + ABx * acc[339];
    const double h9_1_33 = acc[339] + ABx * acc[184];
    const double h9_4_33 = h14_1_33 + ABx * h9_1_33;
    const double k9_4_18_3 = h9_4_33 + CDz * h9_4_18;
    const double k9_4_8_9 = k9_4_18_3 + CDz * k9_4_8_3;
    const double k9_4_14_1 = h9_4_25 + CDx * h9_4_14;
    const double h14_1_9 = acc[656] + ABx * acc[315];
    const double h9_1_9 = acc[315] + ABx * acc[160];
    const double h9_4_9 = h14_1_9 + ABx * h9_1_9;
    const double k9_4_9_1 = h9_4_14 + CDx * h9_4_9;
    const double k9_4_9_4 = k9_4_14_1 + CDx * k9_4_9_1;
    const double k9_4_14_2 = h9_4_28 + CDy * h9_4_14;
    const double k9_4_9_2 = h9_4_18 + CDy * h9_4_9;
    const double k9_4_9_5 = k9_4_14_2 + CDx * k9_4_9_2;
    const double h14_1_19 = acc[666] + ABx * acc[325];
    const double h9_1_19 = acc[325] + ABx * acc[170];
    const double h9_4_19 = h14_1_19 + ABx * h9_1_19;
    const double k9_4_9_3 = h9_4_19 + CDz * h9_4_9;
    const double k9_4_9_6 = k9_4_14_3 + CDx * k9_4_9_3;
    const double k9_4_18_2 = h9_4_32 + CDy * h9_4_18;
    const double k9_4_9_7 = k9_4_18_2 + CDy * k9_4_9_2;
    const double k9_4_9_8 = k9_4_18_3 + CDy * k9_4_9_3;
    const double h14_1_34 = acc[681] + ABx * acc[340];
    const double h9_1_34 = acc[340] + ABx * acc[185];
    const double h9_4_34 = h14_1_34 + ABx * h9_1_34;
    const double k9_4_19_3 = h9_4_34 + CDz * h9_4_19;
    const double k9_4_9_9 = k9_4_19_3 + CDz * k9_4_9_3;
    const double h14_2_20 = acc[760] + ABy * acc[326];
    const double h9_2_20 = acc[450] + ABy * acc[171];
    const double h9_5_20 = h14_2_20 + ABx * h9_2_20;
    const double h14_2_10 = acc[750] + ABy * acc[316];
    const double h9_2_10 = acc[440] + ABy * acc[161];
    const double h9_5_10 = h14_2_10 + ABx * h9_2_10;
    const double k9_5_10_1 = h9_5_20 + CDx * h9_5_10;
    const double h14_2_4 = acc[744] + ABy * acc[310];
    const double h9_2_4 = acc[434] + ABy * acc[155];
    const double h9_5_4 = h14_2_4 + ABx * h9_2_4;
    const double k9_5_4_1 = h9_5_10 + CDx * h9_5_4;
    const double k9_5_4_4 = k9_5_10_1 + CDx * k9_5_4_1;
    const double h14_2_21 = acc[761] + ABy * acc[327];
    const double h9_2_21 = acc[451] + ABy * acc[172];
    const double h9_5_21 = h14_2_21 + ABx * h9_2_21;
    const double k9_5_10_2 = h9_5_21 + CDy * h9_5_10;
    const double h14_2_11 = acc[751] + ABy * acc[317];
    const double h9_2_11 = acc[441] + ABy * acc[162];
    const double h9_5_11 = h14_2_11 + ABx * h9_2_11;
    const double k9_5_4_2 = h9_5_11 + CDy * h9_5_4;
    const double k9_5_4_5 = k9_5_10_2 + CDx * k9_5_4_2;
    const double h14_2_22 = acc[762] + ABy * acc[328];
    const double h9_2_22 = acc[452] + ABy * acc[173];
    const double h9_5_22 = h14_2_22 + ABx * h9_2_22;
    const double k9_5_10_3 = h9_5_22 + CDz * h9_5_10;
    const double h14_2_12 = acc[752] + ABy * acc[318];
    const double h9_2_12 = acc[442] + ABy * acc[163];
    const double h9_5_12 = h14_2_12 + ABx * h9_2_12;
    const double k9_5_4_3 = h9_5_12 + CDz * h9_5_4;
    const double k9_5_4_6 = k9_5_10_3 + CDx * k9_5_4_3;
    const double h14_2_23 = acc[763] + ABy * acc[329];
    const double h9_2_23 = acc[453] + ABy * acc[174];
    const double h9_5_23 = h14_2_23 + ABx * h9_2_23;
    const double k9_5_11_2 = h9_5_23 + CDy * h9_5_11;
    const double k9_5_4_7 = k9_5_11_2 + CDy * k9_5_4_2;
    const double h14_2_24 = acc[764] + ABy * acc[330];
    const double h9_2_24 = acc[454] + ABy * acc[175];
    const double h9_5_24 = h14_2_24 + ABx * h9_2_24;
    const double k9_5_11_3 = h9_5_24 + CDz * h9_5_11;
    const double k9_5_4_8 = k9_5_11_3 + CDy * k9_5_4_3;
    const double h14_2_25 = acc[765] + ABy * acc[331];
    const double h9_2_25 = acc[455] + ABy * acc[176];
    const double h9_5_25 = h14_2_25 + ABx * h9_2_25;
    const double k9_5_12_3 = h9_5_25 + CDz * h9_5_12;
    const double k9_5_4_9 = k9_5_12_3 + CDz * k9_5_4_3;
    const double k9_5_11_1 = h9_5_21 + CDx * h9_5_11;
    const double h14_2_5 = acc[745] + ABy * acc[311];
    const double h9_2_5 = acc[435] + ABy * acc[156];
    const double h9_5_5 = h14_2_5 + ABx * h9_2_5;
    const double k9_5_5_1 = h9_5_11 + CDx * h9_5_5;
    const double k9_5_5_4 = k9_5_11_1 + CDx * k9_5_5_1;
    const double h14_2_13 = acc[753] + ABy * acc[319];
    const double h9_2_13 = acc[443] + ABy * acc[164];
    const double h9_5_13 = h14_2_13 + ABx * h9_2_13;
    const double k9_5_5_2 = h9_5_13 + CDy * h9_5_5;
    const double k9_5_5_5 = k9_5_11_2 + CDx * k9_5_5_2;
    const double h14_2_15 = acc[755] + ABy * acc[321];
    const double h9_2_15 = acc[445] + ABy * acc[166];
    const double h9_5_15 = h14_2_15 + ABx * h9_2_15;
    const double k9_5_5_3 = h9_5_15 + CDz * h9_5_5;
    const double k9_5_5_6 = k9_5_11_3 + CDx * k9_5_5_3;
    const double h14_2_26 = acc[766] + ABy * acc[332];
    const double h9_2_26 = acc[456] + ABy * acc[177];
    const double h9_5_26 = h14_2_26 + ABx * h9_2_26;
    const double k9_5_13_2 = h9_5_26 + CDy * h9_5_13;
    const double k9_5_5_7 = k9_5_13_2 + CDy * k9_5_5_2;
    const double h14_2_27 = acc[767] + ABy * acc[333];
    const double h9_2_27 = acc[457] + ABy * acc[178];
    const double h9_5_27 = h14_2_27 + ABx * h9_2_27;
    const double k9_5_13_3 = h9_5_27 + CDz * h9_5_13;
    const double k9_5_5_8 = k9_5_13_3 + CDy * k9_5_5_3;
    const double h14_2_28 = acc[768] + ABy * acc[334];
    const double h9_2_28 = acc[458] + ABy * acc[179];
    const double h9_5_28 = h14_2_28 + ABx * h9_2_28;
    const double k9_5_15_3 = h9_5_28 + CDz * h9_5_15;
    const double k9_5_5_9 = k9_5_15_3 + CDz * k9_5_5_3;
    const double k9_5_12_1 = h9_5_22 + CDx * h9_5_12;
    const double h14_2_6 = acc[746] + ABy * acc[312];
    const double h9_2_6 = acc[436] + ABy * acc[157];
    const double h9_5_6 = h14_2_6 + ABx * h9_2_6;
    const double k9_5_6_1 = h9_5_12 + CDx * h9_5_6;
    const double k9_5_6_4 = k9_5_12_1 + CDx * k9_5_6_1;
    const double k9_5_12_2 = h9_5_24 + CDy * h9_5_12;
    const double k9_5_6_2 = h9_5_15 + CDy * h9_5_6;
    const double k9_5_6_5 = k9_5_12_2 + CDx * k9_5_6_2;
    const double h14_2_14 = acc[754] + ABy * acc[320];
    const double h9_2_14 = acc[444] + ABy * acc[165];
    const double h9_5_14 = h14_2_14 + ABx * h9_2_14;
    const double k9_5_6_3 = h9_5_14 + CDz * h9_5_6;
    const double k9_5_6_6 = k9_5_12_3 + CDx * k9_5_6_3;
    const double k9_5_15_2 = h9_5_27 + CDy * h9_5_15;
    const double k9_5_6_7 = k9_5_15_2 + CDy * k9_5_6_2;
    const double k9_5_6_8 = k9_5_15_3 + CDy * k9_5_6_3;
    const double h14_2_29 = acc[769] + ABy * acc[335];
    const double h9_2_29 = acc[459] + ABy * acc[180];
    const double h9_5_29 = h14_2_29 + ABx * h9_2_29;
    const double k9_5_14_3 = h9_5_29 + CDz * h9_5_14;
    const double k9_5_6_9 = k9_5_14_3 + CDz * k9_5_6_3;
    const double k9_5_13_1 = h9_5_23 + CDx * h9_5_13;
    const double h14_2_7 = acc[747] + ABy * acc[313];
    const double h9_2_7 = acc[437] + ABy * acc[158];
    const double h9_5_7 = h14_2_7 + ABx * h9_2_7;
    const double k9_5_7_1 = h9_5_13 + CDx * h9_5_7;
    const double k9_5_7_4 = k9_5_13_1 + CDx * k9_5_7_1;
    const double h14_2_16 = acc[756] + ABy * acc[322];
    const double h9_2_16 = acc[446] + ABy * acc[167];
    const double h9_5_16 = h14_2_16 + ABx * h9_2_16;
    const double k9_5_7_2 = h9_5_16 + CDy * h9_5_7;
    const double k9_5_7_5 = k9_5_13_2 + CDx * k9_5_7_2;
    const double h14_2_17 = acc[757] + ABy * acc[323];
    const double h9_2_17 = acc[447] + ABy * acc[168];
    const double h9_5_17 = h14_2_17 + ABx * h9_2_17;
    const double k9_5_7_3 = h9_5_17 + CDz * h9_5_7;
    const double k9_5_7_6 = k9_5_13_3 + CDx * k9_5_7_3;
    const double h14_2_30 = acc[770] + ABy * acc[336];
    const double h9_2_30 = acc[460] + ABy * acc[181];
    const double h9_5_30 = h14_2_30 + ABx * h9_2_30;
    const double k9_5_16_2 = h9_5_30 + CDy * h9_5_16;
    const double k9_5_7_7 = k9_5_16_2 + CDy * k9_5_7_2;
    const double h14_2_31 = acc[771] + ABy * acc[337];
    const double h9_2_31 = acc[461] + ABy * acc[182];
    const double h9_5_31 = h14_2_31 + ABx * h9_2_31;
    const double k9_5_16_3 = h9_5_31 + CDz * h9_5_16;
    const double k9_5_7_8 = k9_5_16_3 + CDy * k9_5_7_3;
    const double h14_2_32 = acc[772] + ABy * acc[338];
    const double h9_2_32 = acc[462] + ABy * acc[183];
    const double h9_5_32 = h14_2_32 + ABx * h9_2_32;
    const double k9_5_17_3 = h9_5_32 + CDz * h9_5_17;
    const double k9_5_7_9 = k9_5_17_3 + CDz * k9_5_7_3;
    const double k9_5_15_1 = h9_5_24 + CDx * h9_5_15;
    const double h14_2_8 = acc[748] + ABy * acc[314];
    const double h9_2_8 = acc[438] + ABy * acc[159];
    const double h9_5_8 = h14_2_8 + ABx * h9_2_8;
    const double k9_5_8_1 = h9_5_15 + CDx * h9_5_8;
    const double k9_5_8_4 = k9_5_15_1 + CDx * k9_5_8_1;
    const double k9_5_8_2 = h9_5_17 + CDy * h9_5_8;
    const double k9_5_8_5 = k9_5_15_2 + CDx * k9_5_8_2;
    const double h14_2_18 = acc[758] + ABy * acc[324];
    const double h9_2_18 = acc[448] + ABy * acc[169];
    const double h9_5_18 = h14_2_18 + ABx * h9_2_18;
    const double k9_5_8_3 = h9_5_18 + CDz * h9_5_8;
    const double k9_5_8_6 = k9_5_15_3 + CDx * k9_5_8_3;
    const double k9_5_17_2 = h9_5_31 + CDy * h9_5_17;
    const double k9_5_8_7 = k9_5_17_2 + CDy * k9_5_8_2;
    const double k9_5_8_8 = k9_5_17_3 + CDy * k9_5_8_3;
    const double h14_2_33 = acc[773] + ABy * acc[339];
    const double h9_2_33 = acc[463] + ABy * acc[184];
    const double h9_5_33 = h14_2_33 + ABx * h9_2_33;
    const double k9_5_18_3 = h9_5_33 + CDz * h9_5_18;
    const double k9_5_8_9 = k9_5_18_3 + CDz * k9_5_8_3;
    const double k9_5_14_1 = h9_5_25 + CDx * h9_5_14;
    const double h14_2_9 = acc[749] + ABy * acc[315];
    const double h9_2_9 = acc[439] + ABy * acc[160];
    const double h9_5_9 = h14_2_9 + ABx * h9_2_9;
    const double k9_5_9_1 = h9_5_14 + CDx * h9_5_9;
    const double k9_5_9_4 = k9_5_14_1 + CDx * k9_5_9_1;
    const double k9_5_14_2 = h9_5_28 + CDy * h9_5_14;
    const double k9_5_9_2 = h9_5_18 + CDy * h9_5_9;
    const double k9_5_9_5 = k9_5_14_2 + CDx * k9_5_9_2;
    const double h14_2_19 = acc[759] + ABy * acc[325];
    const double h9_2_19 = acc[449] + ABy * acc[170];
    const double h9_5_19 = h14_2_19 + ABx * h9_2_19;
    const double k9_5_9_3 = h9_5_19 + CDz * h9_5_9;
    const double k9_5_9_6 = k9_5_14_3 + CDx * k9_5_9_3;
    const double k9_5_18_2 = h9_5_32 + CDy * h9_5_18;
    const double k9_5_9_7 = k9_5_18_2 + CDy * k9_5_9_2;
    const double k9_5_9_8 = k9_5_18_3 + CDy * k9_5_9_3;
    const double h14_2_34 = acc[774] + ABy * acc[340];
    const double h9_2_34 = acc[464] + ABy * acc[185];
    const double h9_5_34 = h14_2_34 + ABx * h9_2_34;
    const double k9_5_19_3 = h9_5_34 + CDz * h9_5_19;
    const double k9_5_9_9 = k9_5_19_3 + CDz * k9_5_9_3;
    const double h9_3_20 = acc[481] + ABz * acc[171];
    const double h9_6_20 = h14_3_20 + ABx * h9_3_20;
    const double h9_3_10 = acc[471] + ABz * acc[161];
    const double h9_6_10 = h14_3_10 + ABx * h9_3_10;
    const double k9_6_10_1 = h9_6_20 + CDx * h9_6_10;
    const double h9_3_4 = acc[465] + ABz * acc[155];
    const double h9_6_4 = h14_3_4 + ABx * h9_3_4;
    const double k9_6_4_1 = h9_6_10 + CDx * h9_6_4;
    const double k9_6_4_4 = k9_6_10_1 + CDx * k9_6_4_1;
    const double h9_3_21 = acc[482] + ABz * acc[172];
    const double h9_6_21 = h14_3_21 + ABx * h9_3_21;
    const double k9_6_10_2 = h9_6_21 + CDy * h9_6_10;
    const double h9_3_11 = acc[472] + ABz * acc[162];
    const double h9_6_11 = h14_3_11 + ABx * h9_3_11;
    const double k9_6_4_2 = h9_6_11 + CDy * h9_6_4;
    const double k9_6_4_5 = k9_6_10_2 + CDx * k9_6_4_2;
    const double h9_3_22 = acc[483] + ABz * acc[173];
    const double h9_6_22 = h14_3_22 + ABx * h9_3_22;
    const double k9_6_10_3 = h9_6_22 + CDz * h9_6_10;
    const double h9_3_12 = acc[473] + ABz * acc[163];
    const double h9_6_12 = h14_3_12 + ABx * h9_3_12;
    const double k9_6_4_3 = h9_6_12 + CDz * h9_6_4;
    const double k9_6_4_6 = k9_6_10_3 + CDx * k9_6_4_3;
    const double h9_3_23 = acc[484] + ABz * acc[174];
    const double h9_6_23 = h14_3_23 + ABx * h9_3_23;
    const double k9_6_11_2 = h9_6_23 + CDy * h9_6_11;
    const double k9_6_4_7 = k9_6_11_2 + CDy * k9_6_4_2;
    const double h9_3_24 = acc[485] + ABz * acc[175];
    const double h9_6_24 = h14_3_24 + ABx * h9_3_24;
    const double k9_6_11_3 = h9_6_24 + CDz * h9_6_11;
    const double k9_6_4_8 = k9_6_11_3 + CDy * k9_6_4_3;
    const double h9_3_25 = acc[486] + ABz * acc[176];
    const double h9_6_25 = h14_3_25 + ABx * h9_3_25;
    const double k9_6_12_3 = h9_6_25 + CDz * h9_6_12;
    const double k9_6_4_9 = k9_6_12_3 + CDz * k9_6_4_3;
    const double k9_6_11_1 = h9_6_21 + CDx * h9_6_11;
    const double h9_3_5 = acc[466] + ABz * acc[156];
    const double h9_6_5 = h14_3_5 + ABx * h9_3_5;
    const double k9_6_5_1 = h9_6_11 + CDx * h9_6_5;
    const double k9_6_5_4 = k9_6_11_1 + CDx * k9_6_5_1;
    const double h9_3_13 = acc[474] + ABz * acc[164];
    const double h9_6_13 = h14_3_13 + ABx * h9_3_13;
    const double k9_6_5_2 = h9_6_13 + CDy * h9_6_5;
    const double k9_6_5_5 = k9_6_11_2 + CDx * k9_6_5_2;
    const double h9_3_15 = acc[476] + ABz * acc[166];
    const double h9_6_15 = h14_3_15 + ABx * h9_3_15;
    const double k9_6_5_3 = h9_6_15 + CDz * h9_6_5;
    const double k9_6_5_6 = k9_6_11_3 + CDx * k9_6_5_3;
    const double h9_3_26 = acc[487] + ABz * acc[177];
    const double h9_6_26 = h14_3_26 + ABx * h9_3_26;
    const double k9_6_13_2 = h9_6_26 + CDy * h9_6_13;
    const double k9_6_5_7 = k9_6_13_2 + CDy * k9_6_5_2;
    const double h9_3_27 = acc[488] + ABz * acc[178];
    const double h9_6_27 = h14_3_27 + ABx * h9_3_27;
    const double k9_6_13_3 = h9_6_27 + CDz * h9_6_13;
    const double k9_6_5_8 = k9_6_13_3 + CDy * k9_6_5_3;
    const double h9_3_28 = acc[489] + ABz * acc[179];
    const double h9_6_28 = h14_3_28 + ABx * h9_3_28;
    const double k9_6_15_3 = h9_6_28 + CDz * h9_6_15;
    const double k9_6_5_9 = k9_6_15_3 + CDz * k9_6_5_3;
    const double k9_6_12_1 = h9_6_22 + CDx * h9_6_12;
    const double h9_3_6 = acc[467] + ABz * acc[157];
    const double h9_6_6 = h14_3_6 + ABx * h9_3_6;
    const double k9_6_6_1 = h9_6_12 + CDx * h9_6_6;
    const double k9_6_6_4 = k9_6_12_1 + CDx * k9_6_6_1;
    const double k9_6_12_2 = h9_6_24 + CDy * h9_6_12;
    const double k9_6_6_2 = h9_6_15 + CDy * h9_6_6;
    const double k9_6_6_5 = k9_6_12_2 + CDx * k9_6_6_2;
    const double h9_3_14 = acc[475] + ABz * acc[165];
    const double h9_6_14 = h14_3_14 + ABx * h9_3_14;
    const double k9_6_6_3 = h9_6_14 + CDz * h9_6_6;
    const double k9_6_6_6 = k9_6_12_3 + CDx * k9_6_6_3;
    const double k9_6_15_2 = h9_6_27 + CDy * h9_6_15;
    const double k9_6_6_7 = k9_6_15_2 + CDy * k9_6_6_2;
    const double k9_6_6_8 = k9_6_15_3 + CDy * k9_6_6_3;
    const double h9_3_29 = acc[490] + ABz * acc[180];
    const double h9_6_29 = h14_3_29 + ABx * h9_3_29;
    const double k9_6_14_3 = h9_6_29 + CDz * h9_6_14;
    const double k9_6_6_9 = k9_6_14_3 + CDz * k9_6_6_3;
    const double k9_6_13_1 = h9_6_23 + CDx * h9_6_13;
    const double h9_3_7 = acc[468] + ABz * acc[158];
    const double h9_6_7 = h14_3_7 + ABx * h9_3_7;
    const double k9_6_7_1 = h9_6_13 + CDx * h9_6_7;
    const double k9_6_7_4 = k9_6_13_1 + CDx * k9_6_7_1;
    const double h9_3_16 = acc[477] + ABz * acc[167];
    const double h9_6_16 = h14_3_16 + ABx * h9_3_16;
    const double k9_6_7_2 = h9_6_16 + CDy * h9_6_7;
    const double k9_6_7_5 = k9_6_13_2 + CDx * k9_6_7_2;
    const double h9_3_17 = acc[478] + ABz * acc[168];
    const double h9_6_17 = h14_3_17 + ABx * h9_3_17;
    const double k9_6_7_3 = h9_6_17 + CDz * h9_6_7;
    const double k9_6_7_6 = k9_6_13_3 + CDx * k9_6_7_3;
    const double h9_3_30 = acc[491] + ABz * acc[181];
    const double h9_6_30 = h14_3_30 + ABx * h9_3_30;
    const double k9_6_16_2 = h9_6_30 + CDy * h9_6_16;
    const double k9_6_7_7 = k9_6_16_2 + CDy * k9_6_7_2;
    const double h9_3_31 = acc[492] + ABz * acc[182];
    const double h9_6_31 = h14_3_31 + ABx * h9_3_31;
    const double k9_6_16_3 = h9_6_31 + CDz * h9_6_16;
    const double k9_6_7_8 = k9_6_16_3 + CDy * k9_6_7_3;
    const double h9_3_32 = acc[493] + ABz * acc[183];
    const double h9_6_32 = h14_3_32 + ABx * h9_3_32;
    const double k9_6_17_3 = h9_6_32 + CDz * h9_6_17;
    const double k9_6_7_9 = k9_6_17_3 + CDz * k9_6_7_3;
    const double k9_6_15_1 = h9_6_24 + CDx * h9_6_15;
    const double h9_3_8 = acc[469] + ABz * acc[159];
    const double h9_6_8 = h14_3_8 + ABx * h9_3_8;
    const double k9_6_8_1 = h9_6_15 + CDx * h9_6_8;
    const double k9_6_8_4 = k9_6_15_1 + CDx * k9_6_8_1;
    const double k9_6_8_2 = h9_6_17 + CDy * h9_6_8;
    const double k9_6_8_5 = k9_6_15_2 + CDx * k9_6_8_2;
    const double h9_3_18 = acc[479] + ABz * acc[169];
    const double h9_6_18 = h14_3_18 + ABx * h9_3_18;
    const double k9_6_8_3 = h9_6_18 + CDz * h9_6_8;
    const double k9_6_8_6 = k9_6_15_3 + CDx * k9_6_8_3;
    const double k9_6_17_2 = h9_6_31 + CDy * h9_6_17;
    const double k9_6_8_7 = k9_6_17_2 + CDy * k9_6_8_2;
    const double k9_6_8_8 = k9_6_17_3 + CDy * k9_6_8_3;
    const double h9_3_33 = acc[494] + ABz * acc[184];
    const double h9_6_33 = h14_3_33 + ABx * h9_3_33;
    const double k9_6_18_3 = h9_6_33 + CDz * h9_6_18;
    const double k9_6_8_9 = k9_6_18_3 + CDz * k9_6_8_3;
    const double k9_6_14_1 = h9_6_25 + CDx * h9_6_14;
    const double h9_3_9 = acc[470] + ABz * acc[160];
    const double h9_6_9 = h14_3_9 + ABx * h9_3_9;
    const double k9_6_9_1 = h9_6_14 + CDx * h9_6_9;
    const double k9_6_9_4 = k9_6_14_1 + CDx * k9_6_9_1;
    const double k9_6_14_2 = h9_6_28 + CDy * h9_6_14;
    const double k9_6_9_2 = h9_6_18 + CDy * h9_6_9;
    const double k9_6_9_5 = k9_6_14_2 + CDx * k9_6_9_2;
    const double h9_3_19 = acc[480] + ABz * acc[170];
    const double h9_6_19 = h14_3_19 + ABx * h9_3_19;
    const double k9_6_9_3 = h9_6_19 + CDz * h9_6_9;
    const double k9_6_9_6 = k9_6_14_3 + CDx * k9_6_9_3;
    const double k9_6_18_2 = h9_6_32 + CDy * h9_6_18;
    const double k9_6_9_7 = k9_6_18_2 + CDy * k9_6_9_2;
    const double k9_6_9_8 = k9_6_18_3 + CDy * k9_6_9_3;
    const double h9_3_34 = acc[495] + ABz * acc[185];
    const double h9_6_34 = h14_3_34 + ABx * h9_3_34;
    const double k9_6_19_3 = h9_6_34 + CDz * h9_6_19;
    const double k9_6_9_9 = k9_6_19_3 + CDz * k9_6_9_3;
    const double h18_2_20 = acc[884] + ABy * acc[450];
    const double h9_7_20 = h18_2_20 + ABy * h9_2_20;
    const double h18_2_10 = acc[874] + ABy * acc[440];
    const double h9_7_10 = h18_2_10 + ABy * h9_2_10;
    const double k9_7_10_1 = h9_7_20 + CDx * h9_7_10;
    const double h18_2_4 = acc[868] + ABy * acc[434];
    const double h9_7_4 = h18_2_4 + ABy * h9_2_4;
    const double k9_7_4_1 = h9_7_10 + CDx * h9_7_4;
    const double k9_7_4_4 = k9_7_10_1 + CDx * k9_7_4_1;
    const double h18_2_21 = acc[885] + ABy * acc[451];
    const double h9_7_21 = h18_2_21 + ABy * h9_2_21;
    const double k9_7_10_2 = h9_7_21 + CDy * h9_7_10;
    const double h18_2_11 = acc[875] + ABy * acc[441];
    const double h9_7_11 = h18_2_11 + ABy * h9_2_11;
    const double k9_7_4_2 = h9_7_11 + CDy * h9_7_4;
    const double k9_7_4_5 = k9_7_10_2 + CDx * k9_7_4_2;
    const double h18_2_22 = acc[886] + ABy * acc[452];
    const double h9_7_22 = h18_2_22 + ABy * h9_2_22;
    const double k9_7_10_3 = h9_7_22 + CDz * h9_7_10;
    const double h18_2_12 = acc[876] + ABy * acc[442];
    const double h9_7_12 = h18_2_12 + ABy * h9_2_12;
    const double k9_7_4_3 = h9_7_12 + CDz * h9_7_4;
    const double k9_7_4_6 = k9_7_10_3 + CDx * k9_7_4_3;
    const double h18_2_23 = acc[887] + ABy * acc[453];
    const double h9_7_23 = h18_2_23 + ABy * h9_2_23;
    const double k9_7_11_2 = h9_7_23 + CDy * h9_7_11;
    const double k9_7_4_7 = k9_7_11_2 + CDy * k9_7_4_2;
    const double h18_2_24 = acc[888] + ABy * acc[454];
    const double h9_7_24 = h18_2_24 + ABy * h9_2_24;
    const double k9_7_11_3 = h9_7_24 + CDz * h9_7_11;
    const double k9_7_4_8 = k9_7_11_3 + CDy * k9_7_4_3;
    const double h18_2_25 = acc[889] + ABy * acc[455];
    const double h9_7_25 = h18_2_25 + ABy * h9_2_25;
    const double k9_7_12_3 = h9_7_25 + CDz * h9_7_12;
    const double k9_7_4_9 = k9_7_12_3 + CDz * k9_7_4_3;
    const double k9_7_11_1 = h9_7_21 + CDx * h9_7_11;
    const double h18_2_5 = acc[869] + ABy * acc[435];
    const double h9_7_5 = h18_2_5 + ABy * h9_2_5;
    const double k9_7_5_1 = h9_7_11 + CDx * h9_7_5;
    const double k9_7_5_4 = k9_7_11_1 + CDx * k9_7_5_1;
    const double h18_2_13 = acc[877] + ABy * acc[443];
    const double h9_7_13 = h18_2_13 + ABy * h9_2_13;
    const double k9_7_5_2 = h9_7_13 + CDy * h9_7_5;
    const double k9_7_5_5 = k9_7_11_2 + CDx * k9_7_5_2;
    const double h18_2_15 = acc[879] + ABy * acc[445];
    const double h9_7_15 = h18_2_15 + ABy * h9_2_15;
    const double k9_7_5_3 = h9_7_15 + CDz * h9_7_5;
    const double k9_7_5_6 = k9_7_11_3 + CDx * k9_7_5_3;
    const double h18_2_26 = acc[890] + ABy * acc[456];
    const double h9_7_26 = h18_2_26 + ABy * h9_2_26;
    const double k9_7_13_2 = h9_7_26 + CDy * h9_7_13;
    const double k9_7_5_7 = k9_7_13_2 + CDy * k9_7_5_2;
    const double h18_2_27 = acc[891] + ABy * acc[457];
    const double h9_7_27 = h18_2_27 + ABy * h9_2_27;
    const double k9_7_13_3 = h9_7_27 + CDz * h9_7_13;
    const double k9_7_5_8 = k9_7_13_3 + CDy * k9_7_5_3;
    const double h18_2_28 = acc[892] + ABy * acc[458];
    const double h9_7_28 = h18_2_28 + ABy * h9_2_28;
    const double k9_7_15_3 = h9_7_28 + CDz * h9_7_15;
    const double k9_7_5_9 = k9_7_15_3 + CDz * k9_7_5_3;
    const double k9_7_12_1 = h9_7_22 + CDx * h9_7_12;
    const double h18_2_6 = acc[870] + ABy * acc[436];
    const double h9_7_6 = h18_2_6 + ABy * h9_2_6;
    const double k9_7_6_1 = h9_7_12 + CDx * h9_7_6;
    const double k9_7_6_4 = k9_7_12_1 + CDx * k9_7_6_1;
    const double k9_7_12_2 = h9_7_24 + CDy * h9_7_12;
    const double k9_7_6_2 = h9_7_15 + CDy * h9_7_6;
    const double k9_7_6_5 = k9_7_12_2 + CDx * k9_7_6_2;
    const double h18_2_14 = acc[878] + ABy * acc[444];
    const double h9_7_14 = h18_2_14 + ABy * h9_2_14;
    const double k9_7_6_3 = h9_7_14 + CDz * h9_7_6;
    const double k9_7_6_6 = k9_7_12_3 + CDx * k9_7_6_3;
    const double k9_7_15_2 = h9_7_27 + CDy * h9_7_15;
    const double k9_7_6_7 = k9_7_15_2 + CDy * k9_7_6_2;
    const double k9_7_6_8 = k9_7_15_3 + CDy * k9_7_6_3;
    const double h18_2_29 = acc[893] + ABy * acc[459];
    const double h9_7_29 = h18_2_29 + ABy * h9_2_29;
    const double k9_7_14_3 = h9_7_29 + CDz * h9_7_14;
    const double k9_7_6_9 = k9_7_14_3 + CDz * k9_7_6_3;
    const double k9_7_13_1 = h9_7_23 + CDx * h9_7_13;
    const double h18_2_7 = acc[871] + ABy * acc[437];
    const double h9_7_7 = h18_2_7 + ABy * h9_2_7;
    const double k9_7_7_1 = h9_7_13 + CDx * h9_7_7;
    const double k9_7_7_4 = k9_7_13_1 + CDx * k9_7_7_1;
    const double h18_2_16 = acc[880] + ABy * acc[446];
    const double h9_7_16 = h18_2_16 + ABy * h9_2_16;
    const double k9_7_7_2 = h9_7_16 + CDy * h9_7_7;
    const double k9_7_7_5 = k9_7_13_2 + CDx * k9_7_7_2;
    const double h18_2_17 = acc[881] + ABy * acc[447];
    const double h9_7_17 = h18_2_17 + ABy * h9_2_17;
    const double k9_7_7_3 = h9_7_17 + CDz * h9_7_7;
    const double k9_7_7_6 = k9_7_13_3 + CDx * k9_7_7_3;
    const double h18_2_30 = acc[894] + ABy * acc[460];
    const double h9_7_30 = h18_2_30 + ABy * h9_2_30;
    const double k9_7_16_2 = h9_7_30 + CDy * h9_7_16;
    const double k9_7_7_7 = k9_7_16_2 + CDy * k9_7_7_2;
    const double h18_2_31 = acc[895] + ABy * acc[461];
    const double h9_7_31 = h18_2_31 + ABy * h9_2_31;
    const double k9_7_16_3 = h9_7_31 + CDz * h9_7_16;
    const double k9_7_7_8 = k9_7_16_3 + CDy * k9_7_7_3;
    const double h18_2_32 = acc[896] + ABy * acc[462];
    const double h9_7_32 = h18_2_32 + ABy * h9_2_32;
    const double k9_7_17_3 = h9_7_32 + CDz * h9_7_17;
    const double k9_7_7_9 = k9_7_17_3 + CDz * k9_7_7_3;
    const double k9_7_15_1 = h9_7_24 + CDx * h9_7_15;
    const double h18_2_8 = acc[872] + ABy * acc[438];
    const double h9_7_8 = h18_2_8 + ABy * h9_2_8;
    const double k9_7_8_1 = h9_7_15 + CDx * h9_7_8;
    const double k9_7_8_4 = k9_7_15_1 + CDx * k9_7_8_1;
    const double k9_7_8_2 = h9_7_17 + CDy * h9_7_8;
    const double k9_7_8_5 = k9_7_15_2 + CDx * k9_7_8_2;
    const double h18_2_18 = acc[882] + ABy * acc[448];
    const double h9_7_18 = h18_2_18 + ABy * h9_2_18;
    const double k9_7_8_3 = h9_7_18 + CDz * h9_7_8;
    const double k9_7_8_6 = k9_7_15_3 + CDx * k9_7_8_3;
    const double k9_7_17_2 = h9_7_31 + CDy * h9_7_17;
    const double k9_7_8_7 = k9_7_17_2 + CDy * k9_7_8_2;
    const double k9_7_8_8 = k9_7_17_3 + CDy * k9_7_8_3;
    const double h18_2_33 = acc[897] + ABy * acc[463];
    const double h9_7_33 = h18_2_33 + ABy * h9_2_33;
    const double k9_7_18_3 = h9_7_33 + CDz * h9_7_18;
    const double k9_7_8_9 = k9_7_18_3 + CDz * k9_7_8_3;
    const double k9_7_14_1 = h9_7_25 + CDx * h9_7_14;
    const double h18_2_9 = acc[873] + ABy * acc[439];
    const double h9_7_9 = h18_2_9 + ABy * h9_2_9;
    const double k9_7_9_1 = h9_7_14 + CDx * h9_7_9;
    const double k9_7_9_4 = k9_7_14_1 + CDx * k9_7_9_1;
    const double k9_7_14_2 = h9_7_28 + CDy * h9_7_14;
    const double k9_7_9_2 = h9_7_18 + CDy * h9_7_9;
    const double k9_7_9_5 = k9_7_14_2 + CDx * k9_7_9_2;
    const double h18_2_19 = acc[883] + ABy * acc[449];
    const double h9_7_19 = h18_2_19 + ABy * h9_2_19;
    const double k9_7_9_3 = h9_7_19 + CDz * h9_7_9;
    const double k9_7_9_6 = k9_7_14_3 + CDx * k9_7_9_3;
    const double k9_7_18_2 = h9_7_32 + CDy * h9_7_18;
    const double k9_7_9_7 = k9_7_18_2 + CDy * k9_7_9_2;
    const double k9_7_9_8 = k9_7_18_3 + CDy * k9_7_9_3;
    const double h18_2_34 = acc[898] + ABy * acc[464];
    const double h9_7_34 = h18_2_34 + ABy * h9_2_34;
    const double k9_7_19_3 = h9_7_34 + CDz * h9_7_19;
    const double k9_7_9_9 = k9_7_19_3 + CDz * k9_7_9_3;
    const double h9_8_20 = h18_3_20 + ABy * h9_3_20;
    const double h9_8_10 = h18_3_10 + ABy * h9_3_10;
    const double k9_8_10_1 = h9_8_20 + CDx * h9_8_10;
    const double h9_8_4 = h18_3_4 + ABy * h9_3_4;
    const double k9_8_4_1 = h9_8_10 + CDx * h9_8_4;
    const double k9_8_4_4 = k9_8_10_1 + CDx * k9_8_4_1;
    const double h9_8_21 = h18_3_21 + ABy * h9_3_21;
    const double k9_8_10_2 = h9_8_21 + CDy * h9_8_10;
    const double h9_8_11 = h18_3_11 + ABy * h9_3_11;
    const double k9_8_4_2 = h9_8_11 + CDy * h9_8_4;
    const double k9_8_4_5 = k9_8_10_2 + CDx * k9_8_4_2;
    const double h9_8_22 = h18_3_22 + ABy * h9_3_22;
    const double k9_8_10_3 = h9_8_22 + CDz * h9_8_10;
    const double h9_8_12 = h18_3_12 + ABy * h9_3_12;
    const double k9_8_4_3 = h9_8_12 + CDz * h9_8_4;
    const double k9_8_4_6 = k9_8_10_3 + CDx * k9_8_4_3;
    const double h9_8_23 = h18_3_23 + ABy * h9_3_23;
    const double k9_8_11_2 = h9_8_23 + CDy * h9_8_11;
    const double k9_8_4_7 = k9_8_11_2 + CDy * k9_8_4_2;
    const double h9_8_24 = h18_3_24 + ABy * h9_3_24;
    const double k9_8_11_3 = h9_8_24 + CDz * h9_8_11;
    const double k9_8_4_8 = k9_8_11_3 + CDy * k9_8_4_3;
    const double h9_8_25 = h18_3_25 + ABy * h9_3_25;
    const double k9_8_12_3 = h9_8_25 + CDz * h9_8_12;
    const double k9_8_4_9 = k9_8_12_3 + CDz * k9_8_4_3;
    const double k9_8_11_1 = h9_8_21 + CDx * h9_8_11;
    const double h9_8_5 = h18_3_5 + ABy * h9_3_5;
    const double k9_8_5_1 = h9_8_11 + CDx * h9_8_5;
    const double k9_8_5_4 = k9_8_11_1 + CDx * k9_8_5_1;
    const double h9_8_13 = h18_3_13 + ABy * h9_3_13;
    const double k9_8_5_2 = h9_8_13 + CDy * h9_8_5;
    const double k9_8_5_5 = k9_8_11_2 + CDx * k9_8_5_2;
    const double h9_8_15 = h18_3_15 + ABy * h9_3_15;
    const double k9_8_5_3 = h9_8_15 + CDz * h9_8_5;
    const double k9_8_5_6 = k9_8_11_3 + CDx * k9_8_5_3;
    const double h9_8_26 = h18_3_26 + ABy * h9_3_26;
    const double k9_8_13_2 = h9_8_26 + CDy * h9_8_13;
    const double k9_8_5_7 = k9_8_13_2 + CDy * k9_8_5_2;
    const double h9_8_27 = h18_3_27 + ABy * h9_3_27;
    const double k9_8_13_3 = h9_8_27 + CDz * h9_8_13;
    const double k9_8_5_8 = k9_8_13_3 + CDy * k9_8_5_3;
    const double h9_8_28 = h18_3_28 + ABy * h9_3_28;
    const double k9_8_15_3 = h9_8_28 + CDz * h9_8_15;
    const double k9_8_5_9 = k9_8_15_3 + CDz * k9_8_5_3;
    const double k9_8_12_1 = h9_8_22 + CDx * h9_8_12;
    const double h9_8_6 = h18_3_6 + ABy * h9_3_6;
    const double k9_8_6_1 = h9_8_12 + CDx * h9_8_6;
    const double k9_8_6_4 = k9_8_12_1 + CDx * k9_8_6_1;
    const double k9_8_12_2 = h9_8_24 + CDy * h9_8_12;
    const double k9_8_6_2 = h9_8_15 + CDy * h9_8_6;
    const double k9_8_6_5 = k9_8_12_2 + CDx * k9_8_6_2;
    const double h9_8_14 = h18_3_14 + ABy * h9_3_14;
    const double k9_8_6_3 = h9_8_14 + CDz * h9_8_6;
    const double k9_8_6_6 = k9_8_12_3 + CDx * k9_8_6_3;
    const double k9_8_15_2 = h9_8_27 + CDy * h9_8_15;
    const double k9_8_6_7 = k9_8_15_2 + CDy * k9_8_6_2;
    const double k9_8_6_8 = k9_8_15_3 + CDy * k9_8_6_3;
    const double h9_8_29 = h18_3_29 + ABy * h9_3_29;
    const double k9_8_14_3 = h9_8_29 + CDz * h9_8_14;
    const double k9_8_6_9 = k9_8_14_3 + CDz * k9_8_6_3;
    const double k9_8_13_1 = h9_8_23 + CDx * h9_8_13;
    const double h9_8_7 = h18_3_7 + ABy * h9_3_7;
    const double k9_8_7_1 = h9_8_13 + CDx * h9_8_7;
    const double k9_8_7_4 = k9_8_13_1 + CDx * k9_8_7_1;
    const double h9_8_16 = h18_3_16 + ABy * h9_3_16;
    const double k9_8_7_2 = h9_8_16 + CDy * h9_8_7;
    const double k9_8_7_5 = k9_8_13_2 + CDx * k9_8_7_2;
    const double h9_8_17 = h18_3_17 + ABy * h9_3_17;
    const double k9_8_7_3 = h9_8_17 + CDz * h9_8_7;
    const double k9_8_7_6 = k9_8_13_3 + CDx * k9_8_7_3;
    const double h9_8_30 = h18_3_30 + ABy * h9_3_30;
    const double k9_8_16_2 = h9_8_30 + CDy * h9_8_16;
    const double k9_8_7_7 = k9_8_16_2 + CDy * k9_8_7_2;
    const double h9_8_31 = h18_3_31 + ABy * h9_3_31;
    const double k9_8_16_3 = h9_8_31 + CDz * h9_8_16;
    const double k9_8_7_8 = k9_8_16_3 + CDy * k9_8_7_3;
    const double h9_8_32 = h18_3_32 + ABy * h9_3_32;
    const double k9_8_17_3 = h9_8_32 + CDz * h9_8_17;
    const double k9_8_7_9 = k9_8_17_3 + CDz * k9_8_7_3;
    const double k9_8_15_1 = h9_8_24 + CDx * h9_8_15;
    const double h9_8_8 = h18_3_8 + ABy * h9_3_8;
    const double k9_8_8_1 = h9_8_15 + CDx * h9_8_8;
    const double k9_8_8_4 = k9_8_15_1 + CDx * k9_8_8_1;
    const double k9_8_8_2 = h9_8_17 + CDy * h9_8_8;
    const double k9_8_8_5 = k9_8_15_2 + CDx * k9_8_8_2;
    const double h9_8_18 = h18_3_18 + ABy * h9_3_18;
    const double k9_8_8_3 = h9_8_18 + CDz * h9_8_8;
    const double k9_8_8_6 = k9_8_15_3 + CDx * k9_8_8_3;
    const double k9_8_17_2 = h9_8_31 + CDy * h9_8_17;
    const double k9_8_8_7 = k9_8_17_2 + CDy * k9_8_8_2;
    const double k9_8_8_8 = k9_8_17_3 + CDy * k9_8_8_3;
    const double h9_8_33 = h18_3_33 + ABy * h9_3_33;
    const double k9_8_18_3 = h9_8_33 + CDz * h9_8_18;
    const double k9_8_8_9 = k9_8_18_3 + CDz * k9_8_8_3;
    const double k9_8_14_1 = h9_8_25 + CDx * h9_8_14;
    const double h9_8_9 = h18_3_9 + ABy * h9_3_9;
    const double k9_8_9_1 = h9_8_14 + CDx * h9_8_9;
    const double k9_8_9_4 = k9_8_14_1 + CDx * k9_8_9_1;
    const double k9_8_14_2 = h9_8_28 + CDy * h9_8_14;
    const double k9_8_9_2 = h9_8_18 + CDy * h9_8_9;
    const double k9_8_9_5 = k9_8_14_2 + CDx * k9_8_9_2;
    const double h9_8_19 = h18_3_19 + ABy * h9_3_19;
    const double k9_8_9_3 = h9_8_19 + CDz * h9_8_9;
    const double k9_8_9_6 = k9_8_14_3 + CDx * k9_8_9_3;
    const double k9_8_18_2 = h9_8_32 + CDy * h9_8_18;
    const double k9_8_9_7 = k9_8_18_2 + CDy * k9_8_9_2;
    const double k9_8_9_8 = k9_8_18_3 + CDy * k9_8_9_3;
    const double h9_8_34 = h18_3_34 + ABy * h9_3_34;
    const double k9_8_19_3 = h9_8_34 + CDz * h9_8_19;
    const double k9_8_9_9 = k9_8_19_3 + CDz * k9_8_9_3;
    const double h19_3_20 = acc[946] + ABz * acc[481];
    const double h9_9_20 = h19_3_20 + ABz * h9_3_20;
    const double h19_3_10 = acc[936] + ABz * acc[471];
    const double h9_9_10 = h19_3_10 + ABz * h9_3_10;
    const double k9_9_10_1 = h9_9_20 + CDx * h9_9_10;
    const double h19_3_4 = acc[930] + ABz * acc[465];
    const double h9_9_4 = h19_3_4 + ABz * h9_3_4;
    const double k9_9_4_1 = h9_9_10 + CDx * h9_9_4;
    const double k9_9_4_4 = k9_9_10_1 + CDx * k9_9_4_1;
    const double h19_3_21 = acc[947] + ABz * acc[482];
    const double h9_9_21 = h19_3_21 + ABz * h9_3_21;
    const double k9_9_10_2 = h9_9_21 + CDy * h9_9_10;
    const double h19_3_11 = acc[937] + ABz * acc[472];
    const double h9_9_11 = h19_3_11 + ABz * h9_3_11;
    const double k9_9_4_2 = h9_9_11 + CDy * h9_9_4;
    const double k9_9_4_5 = k9_9_10_2 + CDx * k9_9_4_2;
    const double h19_3_22 = acc[948] + ABz * acc[483];
    const double h9_9_22 = h19_3_22 + ABz * h9_3_22;
    const double k9_9_10_3 = h9_9_22 + CDz * h9_9_10;
    const double h19_3_12 = acc[938] + ABz * acc[473];
    const double h9_9_12 = h19_3_12 + ABz * h9_3_12;
    const double k9_9_4_3 = h9_9_12 + CDz * h9_9_4;
    const double k9_9_4_6 = k9_9_10_3 + CDx * k9_9_4_3;
    const double h19_3_23 = acc[949] + ABz * acc[484];
    const double h9_9_23 = h19_3_23 + ABz * h9_3_23;
    const double k9_9_11_2 = h9_9_23 + CDy * h9_9_11;
    const double k9_9_4_7 = k9_9_11_2 + CDy * k9_9_4_2;
    const double h19_3_24 = acc[950] + ABz * acc[485];
    const double h9_9_24 = h19_3_24 + ABz * h9_3_24;
    const double k9_9_11_3 = h9_9_24 + CDz * h9_9_11;
    const double k9_9_4_8 = k9_9_11_3 + CDy * k9_9_4_3;
    const double h19_3_25 = acc[951] + ABz * acc[486];
    const double h9_9_25 = h19_3_25 + ABz * h9_3_25;
    const double k9_9_12_3 = h9_9_25 + CDz * h9_9_12;
    const double k9_9_4_9 = k9_9_12_3 + CDz * k9_9_4_3;
    const double k9_9_11_1 = h9_9_21 + CDx * h9_9_11;
    const double h19_3_5 = acc[931] + ABz * acc[466];
    const double h9_9_5 = h19_3_5 + ABz * h9_3_5;
    const double k9_9_5_1 = h9_9_11 + CDx * h9_9_5;
    const double k9_9_5_4 = k9_9_11_1 + CDx * k9_9_5_1;
    const double h19_3_13 = acc[939] + ABz * acc[474];
    const double h9_9_13 = h19_3_13 + ABz * h9_3_13;
    const double k9_9_5_2 = h9_9_13 + CDy * h9_9_5;
    const double k9_9_5_5 = k9_9_11_2 + CDx * k9_9_5_2;
    const double h19_3_15 = acc[941] + ABz * acc[476];
    const double h9_9_15 = h19_3_15 + ABz * h9_3_15;
    const double k9_9_5_3 = h9_9_15 + CDz * h9_9_5;
    const double k9_9_5_6 = k9_9_11_3 + CDx * k9_9_5_3;
    const double h19_3_26 = acc[952] + ABz * acc[487];
    const double h9_9_26 = h19_3_26 + ABz * h9_3_26;
    const double k9_9_13_2 = h9_9_26 + CDy * h9_9_13;
    const double k9_9_5_7 = k9_9_13_2 + CDy * k9_9_5_2;
    const double h19_3_27 = acc[953] + ABz * acc[488];
    const double h9_9_27 = h19_3_27 + ABz * h9_3_27;
    const double k9_9_13_3 = h9_9_27 + CDz * h9_9_13;
    const double k9_9_5_8 = k9_9_13_3 + CDy * k9_9_5_3;
    const double h19_3_28 = acc[954] + ABz * acc[489];
    const double h9_9_28 = h19_3_28 + ABz * h9_3_28;
    const double k9_9_15_3 = h9_9_28 + CDz * h9_9_15;
    const double k9_9_5_9 = k9_9_15_3 + CDz * k9_9_5_3;
    const double k9_9_12_1 = h9_9_22 + CDx * h9_9_12;
    const double h19_3_6 = acc[932] + ABz * acc[467];
    const double h9_9_6 = h19_3_6 + ABz * h9_3_6;
    const double k9_9_6_1 = h9_9_12 + CDx * h9_9_6;
    const double k9_9_6_4 = k9_9_12_1 + CDx * k9_9_6_1;
    const double k9_9_12_2 = h9_9_24 + CDy * h9_9_12;
    const double k9_9_6_2 = h9_9_15 + CDy * h9_9_6;
    const double k9_9_6_5 = k9_9_12_2 + CDx * k9_9_6_2;
    const double h19_3_14 = acc[940] + ABz * acc[475];
    const double h9_9_14 = h19_3_14 + ABz * h9_3_14;
    const double k9_9_6_3 = h9_9_14 + CDz * h9_9_6;
    const double k9_9_6_6 = k9_9_12_3 + CDx * k9_9_6_3;
    const double k9_9_15_2 = h9_9_27 + CDy * h9_9_15;
    const double k9_9_6_7 = k9_9_15_2 + CDy * k9_9_6_2;
    const double k9_9_6_8 = k9_9_15_3 + CDy * k9_9_6_3;
    const double h19_3_29 = acc[955] + ABz * acc[490];
    const double h9_9_29 = h19_3_29 + ABz * h9_3_29;
    const double k9_9_14_3 = h9_9_29 + CDz * h9_9_14;
    const double k9_9_6_9 = k9_9_14_3 + CDz * k9_9_6_3;
    const double k9_9_13_1 = h9_9_23 + CDx * h9_9_13;
    const double h19_3_7 = acc[933] + ABz * acc[468];
    const double h9_9_7 = h19_3_7 + ABz * h9_3_7;
    const double k9_9_7_1 = h9_9_13 + CDx * h9_9_7;
    const double k9_9_7_4 = k9_9_13_1 + CDx * k9_9_7_1;
    const double h19_3_16 = acc[942] + ABz * acc[477];
    const double h9_9_16 = h19_3_16 + ABz * h9_3_16;
    const double k9_9_7_2 = h9_9_16 + CDy * h9_9_7;
    const double k9_9_7_5 = k9_9_13_2 + CDx * k9_9_7_2;
    const double h19_3_17 = acc[943] + ABz * acc[478];
    const double h9_9_17 = h19_3_17 + ABz * h9_3_17;
    const double k9_9_7_3 = h9_9_17 + CDz * h9_9_7;
    const double k9_9_7_6 = k9_9_13_3 + CDx * k9_9_7_3;
    const double h19_3_30 = acc[956] + ABz * acc[491];
    const double h9_9_30 = h19_3_30 + ABz * h9_3_30;
    const double k9_9_16_2 = h9_9_30 + CDy * h9_9_16;
    const double k9_9_7_7 = k9_9_16_2 + CDy * k9_9_7_2;
    const double h19_3_31 = acc[957] + ABz * acc[492];
    const double h9_9_31 = h19_3_31 + ABz * h9_3_31;
    const double k9_9_16_3 = h9_9_31 + CDz * h9_9_16;
    const double k9_9_7_8 = k9_9_16_3 + CDy * k9_9_7_3;
    const double h19_3_32 = acc[958] + ABz * acc[493];
    const double h9_9_32 = h19_3_32 + ABz * h9_3_32;
    const double k9_9_17_3 = h9_9_32 + CDz * h9_9_17;
    const double k9_9_7_9 = k9_9_17_3 + CDz * k9_9_7_3;
    const double k9_9_15_1 = h9_9_24 + CDx * h9_9_15;
    const double h19_3_8 = acc[934] + ABz * acc[469];
    const double h9_9_8 = h19_3_8 + ABz * h9_3_8;
    const double k9_9_8_1 = h9_9_15 + CDx * h9_9_8;
    const double k9_9_8_4 = k9_9_15_1 + CDx * k9_9_8_1;
    const double k9_9_8_2 = h9_9_17 + CDy * h9_9_8;
    const double k9_9_8_5 = k9_9_15_2 + CDx * k9_9_8_2;
    const double h19_3_18 = acc[944] + ABz * acc[479];
    const double h9_9_18 = h19_3_18 + ABz * h9_3_18;
    const double k9_9_8_3 = h9_9_18 + CDz * h9_9_8;
    const double k9_9_8_6 = k9_9_15_3 + CDx * k9_9_8_3;
    const double k9_9_17_2 = h9_9_31 + CDy * h9_9_17;
    const double k9_9_8_7 = k9_9_17_2 + CDy * k9_9_8_2;
    const double k9_9_8_8 = k9_9_17_3 + CDy * k9_9_8_3;
    const double h19_3_33 = acc[959] + ABz * acc[494];
    const double h9_9_33 = h19_3_33 + ABz * h9_3_33;
    const double k9_9_18_3 = h9_9_33 + CDz * h9_9_18;
    const double k9_9_8_9 = k9_9_18_3 + CDz * k9_9_8_3;
    const double k9_9_14_1 = h9_9_25 + CDx * h9_9_14;
    const double h19_3_9 = acc[935] + ABz * acc[470];
    const double h9_9_9 = h19_3_9 + ABz * h9_3_9;
    const double k9_9_9_1 = h9_9_14 + CDx * h9_9_9;
    const double k9_9_9_4 = k9_9_14_1 + CDx * k9_9_9_1;
    const double k9_9_14_2 = h9_9_28 + CDy * h9_9_14;
    const double k9_9_9_2 = h9_9_18 + CDy * h9_9_9;
    const double k9_9_9_5 = k9_9_14_2 + CDx * k9_9_9_2;
    const double h19_3_19 = acc[945] + ABz * acc[480];
    const double h9_9_19 = h19_3_19 + ABz * h9_3_19;
    const double k9_9_9_3 = h9_9_19 + CDz * h9_9_9;
    const double k9_9_9_6 = k9_9_14_3 + CDx * k9_9_9_3;
    const double k9_9_18_2 = h9_9_32 + CDy * h9_9_18;
    const double k9_9_9_7 = k9_9_18_2 + CDy * k9_9_9_2;
    const double k9_9_9_8 = k9_9_18_3 + CDy * k9_9_9_3;
    const double h19_3_34 = acc[960] + ABz * acc[495];
    const double h9_9_34 = h19_3_34 + ABz * h9_3_34;
    const double k9_9_19_3 = h9_9_34 + CDz * h9_9_19;
    const double k9_9_9_9 = k9_9_19_3 + CDz * k9_9_9_3;
    res[0] = k4_4_4_4 * 0.11111111111111117;
    res[1] = k4_4_4_5 * 0.19245008972987535;
    res[2] = k4_4_4_6 * 0.19245008972987535;
    res[3] = k4_4_4_7 * 0.11111111111111117;
    res[4] = k4_4_4_8 * 0.19245008972987535;
    res[5] = k4_4_4_9 * 0.11111111111111117;
    res[6] = k4_4_5_4 * 0.19245008972987535;
    res[7] = k4_4_5_5 * 0.3333333333333334;
    res[8] = k4_4_5_6 * 0.3333333333333334;
    res[9] = k4_4_5_7 * 0.19245008972987535;
    res[10] = k4_4_5_8 * 0.3333333333333334;
    res[11] = k4_4_5_9 * 0.19245008972987535;
    res[12] = k4_4_6_4 * 0.19245008972987535;
    res[13] = k4_4_6_5 * 0.3333333333333334;
    res[14] = k4_4_6_6 * 0.3333333333333334;
    res[15] = k4_4_6_7 * 0.19245008972987535;
    res[16] = k4_4_6_8 * 0.3333333333333334;
    res[17] = k4_4_6_9 * 0.19245008972987535;
    res[18] = k4_4_7_4 * 0.11111111111111117;
    res[19] = k4_4_7_5 * 0.19245008972987535;
    res[20] = k4_4_7_6 * 0.19245008972987535;
    res[21] = k4_4_7_7 * 0.11111111111111117;
    res[22] = k4_4_7_8 * 0.19245008972987535;
    res[23] = k4_4_7_9 * 0.11111111111111117;
    res[24] = k4_4_8_4 * 0.19245008972987535;
    res[25] = k4_4_8_5 * 0.3333333333333334;
    res[26] = k4_4_8_6 * 0.3333333333333334;
    res[27] = k4_4_8_7 * 0.19245008972987535;
    res[28] = k4_4_8_8 * 0.3333333333333334;
    res[29] = k4_4_8_9 * 0.19245008972987535;
    res[30] = k4_4_9_4 * 0.11111111111111117;
    res[31] = k4_4_9_5 * 0.19245008972987535;
    res[32] = k4_4_9_6 * 0.19245008972987535;
    res[33] = k4_4_9_7 * 0.11111111111111117;
    res[34] = k4_4_9_8 * 0.19245008972987535;
    res[35] = k4_4_9_9 * 0.11111111111111117;
    res[36] = k4_5_4_4 * 0.19245008972987535;
    res[37] = k4_5_4_5 * 0.3333333333333334;
    res[38] = k4_5_4_6 * 0.3333333333333334;
    res[39] = k4_5_4_7 * 0.19245008972987535;
    res[40] = k4_5_4_8 * 0.3333333333333334;
    res[41] = k4_5_4_9 * 0.19245008972987535;
    res[42] = k4_5_5_4 * 0.3333333333333334;
    res[43] = k4_5_5_5 * 0.5773502691896258;
    res[44] = k4_5_5_6 * 0.5773502691896258;
    res[45] = k4_5_5_7 * 0.3333333333333334;
    res[46] = k4_5_5_8 * 0.5773502691896258;
    res[47] = k4_5_5_9 * 0.3333333333333334;
    res[48] = k4_5_6_4 * 0.3333333333333334;
    res[49] = k4_5_6_5 * 0.5773502691896258;
    res[50] = k4_5_6_6 * 0.5773502691896258;
    res[51] = k4_5_6_7 * 0.3333333333333334;
    res[52] = k4_5_6_8 * 0.5773502691896258;
    res[53] = k4_5_6_9 * 0.3333333333333334;
    res[54] = k4_5_7_4 * 0.19245008972987535;
    res[55] = k4_5_7_5 * 0.3333333333333334;
    res[56] = k4_5_7_6 * 0.3333333333333334;
    res[57] = k4_5_7_7 * 0.19245008972987535;
    res[58] = k4_5_7_8 * 0.3333333333333334;
    res[59] = k4_5_7_9 * 0.19245008972987535;
    res[60] = k4_5_8_4 * 0.3333333333333334;
    res[61] = k4_5_8_5 * 0.5773502691896258;
    res[62] = k4_5_8_6 * 0.5773502691896258;
    res[63] = k4_5_8_7 * 0.3333333333333334;
    res[64] = k4_5_8_8 * 0.5773502691896258;
    res[65] = k4_5_8_9 * 0.3333333333333334;
    res[66] = k4_5_9_4 * 0.19245008972987535;
    res[67] = k4_5_9_5 * 0.3333333333333334;
    res[68] = k4_5_9_6 * 0.3333333333333334;
    res[69] = k4_5_9_7 * 0.19245008972987535;
    res[70] = k4_5_9_8 * 0.3333333333333334;
    res[71] = k4_5_9_9 * 0.19245008972987535;
    res[72] = k4_6_4_4 * 0.19245008972987535;
    res[73] = k4_6_4_5 * 0.3333333333333334;
    res[74] = k4_6_4_6 * 0.3333333333333334;
    res[75] = k4_6_4_7 * 0.19245008972987535;
    res[76] = k4_6_4_8 * 0.3333333333333334;
    res[77] = k4_6_4_9 * 0.19245008972987535;
    res[78] = k4_6_5_4 * 0.3333333333333334;
    res[79] = k4_6_5_5 * 0.5773502691896258;
    res[80] = k4_6_5_6 * 0.5773502691896258;
    res[81] = k4_6_5_7 * 0.3333333333333334;
    res[82] = k4_6_5_8 * 0.5773502691896258;
    res[83] = k4_6_5_9 * 0.3333333333333334;
    res[84] = k4_6_6_4 * 0.3333333333333334;
    res[85] = k4_6_6_5 * 0.5773502691896258;
    res[86] = k4_6_6_6 * 0.5773502691896258;
    res[87] = k4_6_6_7 * 0.3333333333333334;
    res[88] = k4_6_6_8 * 0.5773502691896258;
    res[89] = k4_6_6_9 * 0.3333333333333334;
    res[90] = k4_6_7_4 * 0.19245008972987535;
    res[91] = k4_6_7_5 * 0.3333333333333334;
    res[92] = k4_6_7_6 * 0.3333333333333334;
    res[93] = k4_6_7_7 * 0.19245008972987535;
    res[94] = k4_6_7_8 * 0.3333333333333334;
    res[95] = k4_6_7_9 * 0.19245008972987535;
    res[96] = k4_6_8_4 * 0.3333333333333334;
    res[97] = k4_6_8_5 * 0.5773502691896258;
    res[98] = k4_6_8_6 * 0.5773502691896258;
    res[99] = k4_6_8_7 * 0.3333333333333334;
    res[100] = k4_6_8_8 * 0.5773502691896258;
    res[101] = k4_6_8_9 * 0.3333333333333334;
    res[102] = k4_6_9_4 * 0.19245008972987535;
    res[103] = k4_6_9_5 * 0.3333333333333334;
    res[104] = k4_6_9_6 * 0.3333333333333334;
    res[105] = k4_6_9_7 * 0.19245008972987535;
    res[106] = k4_6_9_8 * 0.3333333333333334;
    res[107] = k4_6_9_9 * 0.19245008972987535;
    res[108] = k4_7_4_4 * 0.11111111111111117;
    res[109] = k4_7_4_5 * 0.19245008972987535;
    res[110] = k4_7_4_6 * 0.19245008972987535;
    res[111] = k4_7_4_7 * 0.11111111111111117;
    res[112] = k4_7_4_8 * 0.19245008972987535;
    res[113] = k4_7_4_9 * 0.11111111111111117;
    res[114] = k4_7_5_4 * 0.19245008972987535;
    res[115] = k4_7_5_5 * 0.3333333333333334;
    res[116] = k4_7_5_6 * 0.3333333333333334;
    res[117] = k4_7_5_7 * 0.19245008972987535;
    res[118] = k4_7_5_8 * 0.3333333333333334;
    res[119] = k4_7_5_9 * 0.19245008972987535;
    res[120] = k4_7_6_4 * 0.19245008972987535;
    res[121] = k4_7_6_5 * 0.3333333333333334;
    res[122] = k4_7_6_6 * 0.3333333333333334;
    res[123] = k4_7_6_7 * 0.19245008972987535;
    res[124] = k4_7_6_8 * 0.3333333333333334;
    res[125] = k4_7_6_9 * 0.19245008972987535;
    res[126] = k4_7_7_4 * 0.11111111111111117;
    res[127] = k4_7_7_5 * 0.19245008972987535;
    res[128] = k4_7_7_6 * 0.19245008972987535;
    res[129] = k4_7_7_7 * 0.11111111111111117;
    res[130] = k4_7_7_8 * 0.19245008972987535;
    res[131] = k4_7_7_9 * 0.11111111111111117;
    res[132] = k4_7_8_4 * 0.19245008972987535;
    res[133] = k4_7_8_5 * 0.3333333333333334;
    res[134] = k4_7_8_6 * 0.3333333333333334;
    res[135] = k4_7_8_7 * 0.19245008972987535;
    res[136] = k4_7_8_8 * 0.3333333333333334;
    res[137] = k4_7_8_9 * 0.19245008972987535;
    res[138] = k4_7_9_4 * 0.11111111111111117;
    res[139] = k4_7_9_5 * 0.19245008972987535;
    res[140] = k4_7_9_6 * 0.19245008972987535;
    res[141] = k4_7_9_7 * 0.11111111111111117;
    res[142] = k4_7_9_8 * 0.19245008972987535;
    res[143] = k4_7_9_9 * 0.11111111111111117;
    res[144] = k4_8_4_4 * 0.19245008972987535;
    res[145] = k4_8_4_5 * 0.3333333333333334;
    res[146] = k4_8_4_6 * 0.3333333333333334;
    res[147] = k4_8_4_7 * 0.19245008972987535;
    res[148] = k4_8_4_8 * 0.3333333333333334;
    res[149] = k4_8_4_9 * 0.19245008972987535;
    res[150] = k4_8_5_4 * 0.3333333333333334;
    res[151] = k4_8_5_5 * 0.5773502691896258;
    res[152] = k4_8_5_6 * 0.5773502691896258;
    res[153] = k4_8_5_7 * 0.3333333333333334;
    res[154] = k4_8_5_8 * 0.5773502691896258;
    res[155] = k4_8_5_9 * 0.3333333333333334;
    res[156] = k4_8_6_4 * 0.3333333333333334;
    res[157] = k4_8_6_5 * 0.5773502691896258;
    res[158] = k4_8_6_6 * 0.5773502691896258;
    res[159] = k4_8_6_7 * 0.3333333333333334;
    res[160] = k4_8_6_8 * 0.5773502691896258;
    res[161] = k4_8_6_9 * 0.3333333333333334;
    res[162] = k4_8_7_4 * 0.19245008972987535;
    res[163] = k4_8_7_5 * 0.3333333333333334;
    res[164] = k4_8_7_6 * 0.3333333333333334;
    res[165] = k4_8_7_7 * 0.19245008972987535;
    res[166] = k4_8_7_8 * 0.3333333333333334;
    res[167] = k4_8_7_9 * 0.19245008972987535;
    res[168] = k4_8_8_4 * 0.3333333333333334;
    res[169] = k4_8_8_5 * 0.5773502691896258;
    res[170] = k4_8_8_6 * 0.5773502691896258;
    res[171] = k4_8_8_7 * 0.3333333333333334;
    res[172] = k4_8_8_8 * 0.5773502691896258;
    res[173] = k4_8_8_9 * 0.3333333333333334;
    res[174] = k4_8_9_4 * 0.19245008972987535;
    res[175] = k4_8_9_5 * 0.3333333333333334;
    res[176] = k4_8_9_6 * 0.3333333333333334;
    res[177] = k4_8_9_7 * 0.19245008972987535;
    res[178] = k4_8_9_8 * 0.3333333333333334;
    res[179] = k4_8_9_9 * 0.19245008972987535;
    res[180] = k4_9_4_4 * 0.11111111111111117;
    res[181] = k4_9_4_5 * 0.19245008972987535;
    res[182] = k4_9_4_6 * 0.19245008972987535;
    res[183] = k4_9_4_7 * 0.11111111111111117;
    res[184] = k4_9_4_8 * 0.19245008972987535;
    res[185] = k4_9_4_9 * 0.11111111111111117;
    res[186] = k4_9_5_4 * 0.19245008972987535;
    res[187] = k4_9_5_5 * 0.3333333333333334;
    res[188] = k4_9_5_6 * 0.3333333333333334;
    res[189] = k4_9_5_7 * 0.19245008972987535;
    res[190] = k4_9_5_8 * 0.3333333333333334;
    res[191] = k4_9_5_9 * 0.19245008972987535;
    res[192] = k4_9_6_4 * 0.19245008972987535;
    res[193] = k4_9_6_5 * 0.3333333333333334;
    res[194] = k4_9_6_6 * 0.3333333333333334;
    res[195] = k4_9_6_7 * 0.19245008972987535;
    res[196] = k4_9_6_8 * 0.3333333333333334;
    res[197] = k4_9_6_9 * 0.19245008972987535;
    res[198] = k4_9_7_4 * 0.11111111111111117;
    res[199] = k4_9_7_5 * 0.19245008972987535;
    res[200] = k4_9_7_6 * 0.19245008972987535;
    res[201] = k4_9_7_7 * 0.11111111111111117;
    res[202] = k4_9_7_8 * 0.19245008972987535;
    res[203] = k4_9_7_9 * 0.11111111111111117;
    res[204] = k4_9_8_4 * 0.19245008972987535;
    res[205] = k4_9_8_5 * 0.3333333333333334;
    res[206] = k4_9_8_6 * 0.3333333333333334;
    res[207] = k4_9_8_7 * 0.19245008972987535;
    res[208] = k4_9_8_8 * 0.3333333333333334;
    res[209] = k4_9_8_9 * 0.19245008972987535;
    res[210] = k4_9_9_4 * 0.11111111111111117;
    res[211] = k4_9_9_5 * 0.19245008972987535;
    res[212] = k4_9_9_6 * 0.19245008972987535;
    res[213] = k4_9_9_7 * 0.11111111111111117;
    res[214] = k4_9_9_8 * 0.19245008972987535;
    res[215] = k4_9_9_9 * 0.11111111111111117;
    res[216] = k5_4_4_4 * 0.19245008972987535;
    res[217] = k5_4_4_5 * 0.3333333333333334;
    res[218] = k5_4_4_6 * 0.3333333333333334;
    res[219] = k5_4_4_7 * 0.19245008972987535;
    res[220] = k5_4_4_8 * 0.3333333333333334;
    res[221] = k5_4_4_9 * 0.19245008972987535;
    res[222] = k5_4_5_4 * 0.3333333333333334;
    res[223] = k5_4_5_5 * 0.5773502691896258;
    res[224] = k5_4_5_6 * 0.5773502691896258;
    res[225] = k5_4_5_7 * 0.3333333333333334;
    res[226] = k5_4_5_8 * 0.5773502691896258;
    res[227] = k5_4_5_9 * 0.3333333333333334;
    res[228] = k5_4_6_4 * 0.3333333333333334;
    res[229] = k5_4_6_5 * 0.5773502691896258;
    res[230] = k5_4_6_6 * 0.5773502691896258;
    res[231] = k5_4_6_7 * 0.3333333333333334;
    res[232] = k5_4_6_8 * 0.5773502691896258;
    res[233] = k5_4_6_9 * 0.3333333333333334;
    res[234] = k5_4_7_4 * 0.19245008972987535;
    res[235] = k5_4_7_5 * 0.3333333333333334;
    res[236] = k5_4_7_6 * 0.3333333333333334;
    res[237] = k5_4_7_7 * 0.19245008972987535;
    res[238] = k5_4_7_8 * 0.3333333333333334;
    res[239] = k5_4_7_9 * 0.19245008972987535;
    res[240] = k5_4_8_4 * 0.3333333333333334;
    res[241] = k5_4_8_5 * 0.5773502691896258;
    res[242] = k5_4_8_6 * 0.5773502691896258;
    res[243] = k5_4_8_7 * 0.3333333333333334;
    res[244] = k5_4_8_8 * 0.5773502691896258;
    res[245] = k5_4_8_9 * 0.3333333333333334;
    res[246] = k5_4_9_4 * 0.19245008972987535;
    res[247] = k5_4_9_5 * 0.3333333333333334;
    res[248] = k5_4_9_6 * 0.3333333333333334;
    res[249] = k5_4_9_7 * 0.19245008972987535;
    res[250] = k5_4_9_8 * 0.3333333333333334;
    res[251] = k5_4_9_9 * 0.19245008972987535;
    res[252] = k5_5_4_4 * 0.3333333333333334;
    res[253] = k5_5_4_5 * 0.5773502691896258;
    res[254] = k5_5_4_6 * 0.5773502691896258;
    res[255] = k5_5_4_7 * 0.3333333333333334;
    res[256] = k5_5_4_8 * 0.5773502691896258;
    res[257] = k5_5_4_9 * 0.3333333333333334;
    res[258] = k5_5_5_4 * 0.5773502691896258;
    res[259] = k5_5_5_5;
    res[260] = k5_5_5_6;
    res[261] = k5_5_5_7 * 0.5773502691896258;
    res[262] = k5_5_5_8;
    res[263] = k5_5_5_9 * 0.5773502691896258;
    res[264] = k5_5_6_4 * 0.5773502691896258;
    res[265] = k5_5_6_5;
    res[266] = k5_5_6_6;
    res[267] = k5_5_6_7 * 0.5773502691896258;
    res[268] = k5_5_6_8;
    res[269] = k5_5_6_9 * 0.5773502691896258;
    res[270] = k5_5_7_4 * 0.3333333333333334;
    res[271] = k5_5_7_5 * 0.5773502691896258;
    res[272] = k5_5_7_6 * 0.5773502691896258;
    res[273] = k5_5_7_7 * 0.3333333333333334;
    res[274] = k5_5_7_8 * 0.5773502691896258;
    res[275] = k5_5_7_9 * 0.3333333333333334;
    res[276] = k5_5_8_4 * 0.5773502691896258;
    res[277] = k5_5_8_5;
    res[278] = k5_5_8_6;
    res[279] = k5_5_8_7 * 0.5773502691896258;
    res[280] = k5_5_8_8;
    res[281] = k5_5_8_9 * 0.5773502691896258;
    res[282] = k5_5_9_4 * 0.3333333333333334;
    res[283] = k5_5_9_5 * 0.5773502691896258;
    res[284] = k5_5_9_6 * 0.5773502691896258;
    res[285] = k5_5_9_7 * 0.3333333333333334;
    res[286] = k5_5_9_8 * 0.5773502691896258;
    res[287] = k5_5_9_9 * 0.3333333333333334;
    res[288] = k5_6_4_4 * 0.3333333333333334;
    res[289] = k5_6_4_5 * 0.5773502691896258;
    res[290] = k5_6_4_6 * 0.5773502691896258;
    res[291] = k5_6_4_7 * 0.3333333333333334;
    res[292] = k5_6_4_8 * 0.5773502691896258;
    res[293] = k5_6_4_9 * 0.3333333333333334;
    res[294] = k5_6_5_4 * 0.5773502691896258;
    res[295] = k5_6_5_5;
    res[296] = k5_6_5_6;
    res[297] = k5_6_5_7 * 0.5773502691896258;
    res[298] = k5_6_5_8;
    res[299] = k5_6_5_9 * 0.5773502691896258;
    res[300] = k5_6_6_4 * 0.5773502691896258;
    res[301] = k5_6_6_5;
    res[302] = k5_6_6_6;
    res[303] = k5_6_6_7 * 0.5773502691896258;
    res[304] = k5_6_6_8;
    res[305] = k5_6_6_9 * 0.5773502691896258;
    res[306] = k5_6_7_4 * 0.3333333333333334;
    res[307] = k5_6_7_5 * 0.5773502691896258;
    res[308] = k5_6_7_6 * 0.5773502691896258;
    res[309] = k5_6_7_7 * 0.3333333333333334;
    res[310] = k5_6_7_8 * 0.5773502691896258;
    res[311] = k5_6_7_9 * 0.3333333333333334;
    res[312] = k5_6_8_4 * 0.5773502691896258;
    res[313] = k5_6_8_5;
    res[314] = k5_6_8_6;
    res[315] = k5_6_8_7 * 0.5773502691896258;
    res[316] = k5_6_8_8;
    res[317] = k5_6_8_9 * 0.5773502691896258;
    res[318] = k5_6_9_4 * 0.3333333333333334;
    res[319] = k5_6_9_5 * 0.5773502691896258;
    res[320] = k5_6_9_6 * 0.5773502691896258;
    res[321] = k5_6_9_7 * 0.3333333333333334;
    res[322] = k5_6_9_8 * 0.5773502691896258;
    res[323] = k5_6_9_9 * 0.3333333333333334;
    res[324] = k5_7_4_4 * 0.19245008972987535;
    res[325] = k5_7_4_5 * 0.3333333333333334;
    res[326] = k5_7_4_6 * 0.3333333333333334;
    res[327] = k5_7_4_7 * 0.19245008972987535;
    res[328] = k5_7_4_8 * 0.3333333333333334;
    res[329] = k5_7_4_9 * 0.19245008972987535;
    res[330] = k5_7_5_4 * 0.3333333333333334;
    res[331] = k5_7_5_5 * 0.5773502691896258;
    res[332] = k5_7_5_6 * 0.5773502691896258;
    res[333] = k5_7_5_7 * 0.3333333333333334;
    res[334] = k5_7_5_8 * 0.5773502691896258;
    res[335] = k5_7_5_9 * 0.3333333333333334;
    res[336] = k5_7_6_4 * 0.3333333333333334;
    res[337] = k5_7_6_5 * 0.5773502691896258;
    res[338] = k5_7_6_6 * 0.5773502691896258;
    res[339] = k5_7_6_7 * 0.3333333333333334;
    res[340] = k5_7_6_8 * 0.5773502691896258;
    res[341] = k5_7_6_9 * 0.3333333333333334;
    res[342] = k5_7_7_4 * 0.19245008972987535;
    res[343] = k5_7_7_5 * 0.3333333333333334;
    res[344] = k5_7_7_6 * 0.3333333333333334;
    res[345] = k5_7_7_7 * 0.19245008972987535;
    res[346] = k5_7_7_8 * 0.3333333333333334;
    res[347] = k5_7_7_9 * 0.19245008972987535;
    res[348] = k5_7_8_4 * 0.3333333333333334;
    res[349] = k5_7_8_5 * 0.5773502691896258;
    res[350] = k5_7_8_6 * 0.5773502691896258;
    res[351] = k5_7_8_7 * 0.3333333333333334;
    res[352] = k5_7_8_8 * 0.5773502691896258;
    res[353] = k5_7_8_9 * 0.3333333333333334;
    res[354] = k5_7_9_4 * 0.19245008972987535;
    res[355] = k5_7_9_5 * 0.3333333333333334;
    res[356] = k5_7_9_6 * 0.3333333333333334;
    res[357] = k5_7_9_7 * 0.19245008972987535;
    res[358] = k5_7_9_8 * 0.3333333333333334;
    res[359] = k5_7_9_9 * 0.19245008972987535;
    res[360] = k5_8_4_4 * 0.3333333333333334;
    res[361] = k5_8_4_5 * 0.5773502691896258;
    res[362] = k5_8_4_6 * 0.5773502691896258;
    res[363] = k5_8_4_7 * 0.3333333333333334;
    res[364] = k5_8_4_8 * 0.5773502691896258;
    res[365] = k5_8_4_9 * 0.3333333333333334;
    res[366] = k5_8_5_4 * 0.5773502691896258;
    res[367] = k5_8_5_5;
    res[368] = k5_8_5_6;
    res[369] = k5_8_5_7 * 0.5773502691896258;
    res[370] = k5_8_5_8;
    res[371] = k5_8_5_9 * 0.5773502691896258;
    res[372] = k5_8_6_4 * 0.5773502691896258;
    res[373] = k5_8_6_5;
    res[374] = k5_8_6_6;
    res[375] = k5_8_6_7 * 0.5773502691896258;
    res[376] = k5_8_6_8;
    res[377] = k5_8_6_9 * 0.5773502691896258;
    res[378] = k5_8_7_4 * 0.3333333333333334;
    res[379] = k5_8_7_5 * 0.5773502691896258;
    res[380] = k5_8_7_6 * 0.5773502691896258;
    res[381] = k5_8_7_7 * 0.3333333333333334;
    res[382] = k5_8_7_8 * 0.5773502691896258;
    res[383] = k5_8_7_9 * 0.3333333333333334;
    res[384] = k5_8_8_4 * 0.5773502691896258;
    res[385] = k5_8_8_5;
    res[386] = k5_8_8_6;
    res[387] = k5_8_8_7 * 0.5773502691896258;
    res[388] = k5_8_8_8;
    res[389] = k5_8_8_9 * 0.5773502691896258;
    res[390] = k5_8_9_4 * 0.3333333333333334;
    res[391] = k5_8_9_5 * 0.5773502691896258;
    res[392] = k5_8_9_6 * 0.5773502691896258;
    res[393] = k5_8_9_7 * 0.3333333333333334;
    res[394] = k5_8_9_8 * 0.5773502691896258;
    res[395] = k5_8_9_9 * 0.3333333333333334;
    res[396] = k5_9_4_4 * 0.19245008972987535;
    res[397] = k5_9_4_5 * 0.3333333333333334;
    res[398] = k5_9_4_6 * 0.3333333333333334;
    res[399] = k5_9_4_7 * 0.19245008972987535;
    res[400] = k5_9_4_8 * 0.3333333333333334;
    res[401] = k5_9_4_9 * 0.19245008972987535;
    res[402] = k5_9_5_4 * 0.3333333333333334;
    res[403] = k5_9_5_5 * 0.5773502691896258;
    res[404] = k5_9_5_6 * 0.5773502691896258;
    res[405] = k5_9_5_7 * 0.3333333333333334;
    res[406] = k5_9_5_8 * 0.5773502691896258;
    res[407] = k5_9_5_9 * 0.3333333333333334;
    res[408] = k5_9_6_4 * 0.3333333333333334;
    res[409] = k5_9_6_5 * 0.5773502691896258;
    res[410] = k5_9_6_6 * 0.5773502691896258;
    res[411] = k5_9_6_7 * 0.3333333333333334;
    res[412] = k5_9_6_8 * 0.5773502691896258;
    res[413] = k5_9_6_9 * 0.3333333333333334;
    res[414] = k5_9_7_4 * 0.19245008972987535;
    res[415] = k5_9_7_5 * 0.3333333333333334;
    res[416] = k5_9_7_6 * 0.3333333333333334;
    res[417] = k5_9_7_7 * 0.19245008972987535;
    res[418] = k5_9_7_8 * 0.3333333333333334;
    res[419] = k5_9_7_9 * 0.19245008972987535;
    res[420] = k5_9_8_4 * 0.3333333333333334;
    res[421] = k5_9_8_5 * 0.5773502691896258;
    res[422] = k5_9_8_6 * 0.5773502691896258;
    res[423] = k5_9_8_7 * 0.3333333333333334;
    res[424] = k5_9_8_8 * 0.5773502691896258;
    res[425] = k5_9_8_9 * 0.3333333333333334;
    res[426] = k5_9_9_4 * 0.19245008972987535;
    res[427] = k5_9_9_5 * 0.3333333333333334;
    res[428] = k5_9_9_6 * 0.3333333333333334;
    res[429] = k5_9_9_7 * 0.19245008972987535;
    res[430] = k5_9_9_8 * 0.3333333333333334;
    res[431] = k5_9_9_9 * 0.19245008972987535;
    res[432] = k6_4_4_4 * 0.19245008972987535;
    res[433] = k6_4_4_5 * 0.3333333333333334;
    res[434] = k6_4_4_6 * 0.3333333333333334;
    res[435] = k6_4_4_7 * 0.19245008972987535;
    res[436] = k6_4_4_8 * 0.3333333333333334;
    res[437] = k6_4_4_9 * 0.19245008972987535;
    res[438] = k6_4_5_4 * 0.3333333333333334;
    res[439] = k6_4_5_5 * 0.5773502691896258;
    res[440] = k6_4_5_6 * 0.5773502691896258;
    res[441] = k6_4_5_7 * 0.3333333333333334;
    res[442] = k6_4_5_8 * 0.5773502691896258;
    res[443] = k6_4_5_9 * 0.3333333333333334;
    res[444] = k6_4_6_4 * 0.3333333333333334;
    res[445] = k6_4_6_5 * 0.5773502691896258;
    res[446] = k6_4_6_6 * 0.5773502691896258;
    res[447] = k6_4_6_7 * 0.3333333333333334;
    res[448] = k6_4_6_8 * 0.5773502691896258;
    res[449] = k6_4_6_9 * 0.3333333333333334;
    res[450] = k6_4_7_4 * 0.19245008972987535;
    res[451] = k6_4_7_5 * 0.3333333333333334;
    res[452] = k6_4_7_6 * 0.3333333333333334;
    res[453] = k6_4_7_7 * 0.19245008972987535;
    res[454] = k6_4_7_8 * 0.3333333333333334;
    res[455] = k6_4_7_9 * 0.19245008972987535;
    res[456] = k6_4_8_4 * 0.3333333333333334;
    res[457] = k6_4_8_5 * 0.5773502691896258;
    res[458] = k6_4_8_6 * 0.5773502691896258;
    res[459] = k6_4_8_7 * 0.3333333333333334;
    res[460] = k6_4_8_8 * 0.5773502691896258;
    res[461] = k6_4_8_9 * 0.3333333333333334;
    res[462] = k6_4_9_4 * 0.19245008972987535;
    res[463] = k6_4_9_5 * 0.3333333333333334;
    res[464] = k6_4_9_6 * 0.3333333333333334;
    res[465] = k6_4_9_7 * 0.19245008972987535;
    res[466] = k6_4_9_8 * 0.3333333333333334;
    res[467] = k6_4_9_9 * 0.19245008972987535;
    res[468] = k6_5_4_4 * 0.3333333333333334;
    res[469] = k6_5_4_5 * 0.5773502691896258;
    res[470] = k6_5_4_6 * 0.5773502691896258;
    res[471] = k6_5_4_7 * 0.3333333333333334;
    res[472] = k6_5_4_8 * 0.5773502691896258;
    res[473] = k6_5_4_9 * 0.3333333333333334;
    res[474] = k6_5_5_4 * 0.5773502691896258;
    res[475] = k6_5_5_5;
    res[476] = k6_5_5_6;
    res[477] = k6_5_5_7 * 0.5773502691896258;
    res[478] = k6_5_5_8;
    res[479] = k6_5_5_9 * 0.5773502691896258;
    res[480] = k6_5_6_4 * 0.5773502691896258;
    res[481] = k6_5_6_5;
    res[482] = k6_5_6_6;
    res[483] = k6_5_6_7 * 0.5773502691896258;
    res[484] = k6_5_6_8;
    res[485] = k6_5_6_9 * 0.5773502691896258;
    res[486] = k6_5_7_4 * 0.3333333333333334;
    res[487] = k6_5_7_5 * 0.5773502691896258;
    res[488] = k6_5_7_6 * 0.5773502691896258;
    res[489] = k6_5_7_7 * 0.3333333333333334;
    res[490] = k6_5_7_8 * 0.5773502691896258;
    res[491] = k6_5_7_9 * 0.3333333333333334;
    res[492] = k6_5_8_4 * 0.5773502691896258;
    res[493] = k6_5_8_5;
    res[494] = k6_5_8_6;
    res[495] = k6_5_8_7 * 0.5773502691896258;
    res[496] = k6_5_8_8;
    res[497] = k6_5_8_9 * 0.5773502691896258;
    res[498] = k6_5_9_4 * 0.3333333333333334;
    res[499] = k6_5_9_5 * 0.5773502691896258;
    res[500] = k6_5_9_6 * 0.5773502691896258;
    res[501] = k6_5_9_7 * 0.3333333333333334;
    res[502] = k6_5_9_8 * 0.5773502691896258;
    res[503] = k6_5_9_9 * 0.3333333333333334;
    res[504] = k6_6_4_4 * 0.3333333333333334;
    res[505] = k6_6_4_5 * 0.5773502691896258;
    res[506] = k6_6_4_6 * 0.5773502691896258;
    res[507] = k6_6_4_7 * 0.3333333333333334;
    res[508] = k6_6_4_8 * 0.5773502691896258;
    res[509] = k6_6_4_9 * 0.3333333333333334;
    res[510] = k6_6_5_4 * 0.5773502691896258;
    res[511] = k6_6_5_5;
    res[512] = k6_6_5_6;
    res[513] = k6_6_5_7 * 0.5773502691896258;
    res[514] = k6_6_5_8;
    res[515] = k6_6_5_9 * 0.5773502691896258;
    res[516] = k6_6_6_4 * 0.5773502691896258;
    res[517] = k6_6_6_5;
    res[518] = k6_6_6_6;
    res[519] = k6_6_6_7 * 0.5773502691896258;
    res[520] = k6_6_6_8;
    res[521] = k6_6_6_9 * 0.5773502691896258;
    res[522] = k6_6_7_4 * 0.3333333333333334;
    res[523] = k6_6_7_5 * 0.5773502691896258;
    res[524] = k6_6_7_6 * 0.5773502691896258;
    res[525] = k6_6_7_7 * 0.3333333333333334;
    res[526] = k6_6_7_8 * 0.5773502691896258;
    res[527] = k6_6_7_9 * 0.3333333333333334;
    res[528] = k6_6_8_4 * 0.5773502691896258;
    res[529] = k6_6_8_5;
    res[530] = k6_6_8_6;
    res[531] = k6_6_8_7 * 0.5773502691896258;
    res[532] = k6_6_8_8;
    res[533] = k6_6_8_9 * 0.5773502691896258;
    res[534] = k6_6_9_4 * 0.3333333333333334;
    res[535] = k6_6_9_5 * 0.5773502691896258;
    res[536] = k6_6_9_6 * 0.5773502691896258;
    res[537] = k6_6_9_7 * 0.3333333333333334;
    res[538] = k6_6_9_8 * 0.5773502691896258;
    res[539] = k6_6_9_9 * 0.3333333333333334;
    res[540] = k6_7_4_4 * 0.19245008972987535;
    res[541] = k6_7_4_5 * 0.3333333333333334;
    res[542] = k6_7_4_6 * 0.3333333333333334;
    res[543] = k6_7_4_7 * 0.19245008972987535;
    res[544] = k6_7_4_8 * 0.3333333333333334;
    res[545] = k6_7_4_9 * 0.19245008972987535;
    res[546] = k6_7_5_4 * 0.3333333333333334;
    res[547] = k6_7_5_5 * 0.5773502691896258;
    res[548] = k6_7_5_6 * 0.5773502691896258;
    res[549] = k6_7_5_7 * 0.3333333333333334;
    res[550] = k6_7_5_8 * 0.5773502691896258;
    res[551] = k6_7_5_9 * 0.3333333333333334;
    res[552] = k6_7_6_4 * 0.3333333333333334;
    res[553] = k6_7_6_5 * 0.5773502691896258;
    res[554] = k6_7_6_6 * 0.5773502691896258;
    res[555] = k6_7_6_7 * 0.3333333333333334;
    res[556] = k6_7_6_8 * 0.5773502691896258;
    res[557] = k6_7_6_9 * 0.3333333333333334;
    res[558] = k6_7_7_4 * 0.19245008972987535;
    res[559] = k6_7_7_5 * 0.3333333333333334;
    res[560] = k6_7_7_6 * 0.3333333333333334;
    res[561] = k6_7_7_7 * 0.19245008972987535;
    res[562] = k6_7_7_8 * 0.3333333333333334;
    res[563] = k6_7_7_9 * 0.19245008972987535;
    res[564] = k6_7_8_4 * 0.3333333333333334;
    res[565] = k6_7_8_5 * 0.5773502691896258;
    res[566] = k6_7_8_6 * 0.5773502691896258;
    res[567] = k6_7_8_7 * 0.3333333333333334;
    res[568] = k6_7_8_8 * 0.5773502691896258;
    res[569] = k6_7_8_9 * 0.3333333333333334;
    res[570] = k6_7_9_4 * 0.19245008972987535;
    res[571] = k6_7_9_5 * 0.3333333333333334;
    res[572] = k6_7_9_6 * 0.3333333333333334;
    res[573] = k6_7_9_7 * 0.19245008972987535;
    res[574] = k6_7_9_8 * 0.3333333333333334;
    res[575] = k6_7_9_9 * 0.19245008972987535;
    res[576] = k6_8_4_4 * 0.3333333333333334;
    res[577] = k6_8_4_5 * 0.5773502691896258;
    res[578] = k6_8_4_6 * 0.5773502691896258;
    res[579] = k6_8_4_7 * 0.3333333333333334;
    res[580] = k6_8_4_8 * 0.5773502691896258;
    res[581] = k6_8_4_9 * 0.3333333333333334;
    res[582] = k6_8_5_4 * 0.5773502691896258;
    res[583] = k6_8_5_5;
    res[584] = k6_8_5_6;
    res[585] = k6_8_5_7 * 0.5773502691896258;
    res[586] = k6_8_5_8;
    res[587] = k6_8_5_9 * 0.5773502691896258;
    res[588] = k6_8_6_4 * 0.5773502691896258;
    res[589] = k6_8_6_5;
    res[590] = k6_8_6_6;
    res[591] = k6_8_6_7 * 0.5773502691896258;
    res[592] = k6_8_6_8;
    res[593] = k6_8_6_9 * 0.5773502691896258;
    res[594] = k6_8_7_4 * 0.3333333333333334;
    res[595] = k6_8_7_5 * 0.5773502691896258;
    res[596] = k6_8_7_6 * 0.5773502691896258;
    res[597] = k6_8_7_7 * 0.3333333333333334;
    res[598] = k6_8_7_8 * 0.5773502691896258;
    res[599] = k6_8_7_9 * 0.3333333333333334;
    res[600] = k6_8_8_4 * 0.5773502691896258;
    res[601] = k6_8_8_5;
    res[602] = k6_8_8_6;
    res[603] = k6_8_8_7 * 0.5773502691896258;
    res[604] = k6_8_8_8;
    res[605] = k6_8_8_9 * 0.5773502691896258;
    res[606] = k6_8_9_4 * 0.3333333333333334;
    res[607] = k6_8_9_5 * 0.5773502691896258;
    res[608] = k6_8_9_6 * 0.5773502691896258;
    res[609] = k6_8_9_7 * 0.3333333333333334;
    res[610] = k6_8_9_8 * 0.5773502691896258;
    res[611] = k6_8_9_9 * 0.3333333333333334;
    res[612] = k6_9_4_4 * 0.19245008972987535;
    res[613] = k6_9_4_5 * 0.3333333333333334;
    res[614] = k6_9_4_6 * 0.3333333333333334;
    res[615] = k6_9_4_7 * 0.19245008972987535;
    res[616] = k6_9_4_8 * 0.3333333333333334;
    res[617] = k6_9_4_9 * 0.19245008972987535;
    res[618] = k6_9_5_4 * 0.3333333333333334;
    res[619] = k6_9_5_5 * 0.5773502691896258;
    res[620] = k6_9_5_6 * 0.5773502691896258;
    res[621] = k6_9_5_7 * 0.3333333333333334;
    res[622] = k6_9_5_8 * 0.5773502691896258;
    res[623] = k6_9_5_9 * 0.3333333333333334;
    res[624] = k6_9_6_4 * 0.3333333333333334;
    res[625] = k6_9_6_5 * 0.5773502691896258;
    res[626] = k6_9_6_6 * 0.5773502691896258;
    res[627] = k6_9_6_7 * 0.3333333333333334;
    res[628] = k6_9_6_8 * 0.5773502691896258;
    res[629] = k6_9_6_9 * 0.3333333333333334;
    res[630] = k6_9_7_4 * 0.19245008972987535;
    res[631] = k6_9_7_5 * 0.3333333333333334;
    res[632] = k6_9_7_6 * 0.3333333333333334;
    res[633] = k6_9_7_7 * 0.19245008972987535;
    res[634] = k6_9_7_8 * 0.3333333333333334;
    res[635] = k6_9_7_9 * 0.19245008972987535;
    res[636] = k6_9_8_4 * 0.3333333333333334;
    res[637] = k6_9_8_5 * 0.5773502691896258;
    res[638] = k6_9_8_6 * 0.5773502691896258;
    res[639] = k6_9_8_7 * 0.3333333333333334;
    res[640] = k6_9_8_8 * 0.5773502691896258;
    res[641] = k6_9_8_9 * 0.3333333333333334;
    res[642] = k6_9_9_4 * 0.19245008972987535;
    res[643] = k6_9_9_5 * 0.3333333333333334;
    res[644] = k6_9_9_6 * 0.3333333333333334;
    res[645] = k6_9_9_7 * 0.19245008972987535;
    res[646] = k6_9_9_8 * 0.3333333333333334;
    res[647] = k6_9_9_9 * 0.19245008972987535;
    res[648] = k7_4_4_4 * 0.11111111111111117;
    res[649] = k7_4_4_5 * 0.19245008972987535;
    res[650] = k7_4_4_6 * 0.19245008972987535;
    res[651] = k7_4_4_7 * 0.11111111111111117;
    res[652] = k7_4_4_8 * 0.19245008972987535;
    res[653] = k7_4_4_9 * 0.11111111111111117;
    res[654] = k7_4_5_4 * 0.19245008972987535;
    res[655] = k7_4_5_5 * 0.3333333333333334;
    res[656] = k7_4_5_6 * 0.3333333333333334;
    res[657] = k7_4_5_7 * 0.19245008972987535;
    res[658] = k7_4_5_8 * 0.3333333333333334;
    res[659] = k7_4_5_9 * 0.19245008972987535;
    res[660] = k7_4_6_4 * 0.19245008972987535;
    res[661] = k7_4_6_5 * 0.3333333333333334;
    res[662] = k7_4_6_6 * 0.3333333333333334;
    res[663] = k7_4_6_7 * 0.19245008972987535;
    res[664] = k7_4_6_8 * 0.3333333333333334;
    res[665] = k7_4_6_9 * 0.19245008972987535;
    res[666] = k7_4_7_4 * 0.11111111111111117;
    res[667] = k7_4_7_5 * 0.19245008972987535;
    res[668] = k7_4_7_6 * 0.19245008972987535;
    res[669] = k7_4_7_7 * 0.11111111111111117;
    res[670] = k7_4_7_8 * 0.19245008972987535;
    res[671] = k7_4_7_9 * 0.11111111111111117;
    res[672] = k7_4_8_4 * 0.19245008972987535;
    res[673] = k7_4_8_5 * 0.3333333333333334;
    res[674] = k7_4_8_6 * 0.3333333333333334;
    res[675] = k7_4_8_7 * 0.19245008972987535;
    res[676] = k7_4_8_8 * 0.3333333333333334;
    res[677] = k7_4_8_9 * 0.19245008972987535;
    res[678] = k7_4_9_4 * 0.11111111111111117;
    res[679] = k7_4_9_5 * 0.19245008972987535;
    res[680] = k7_4_9_6 * 0.19245008972987535;
    res[681] = k7_4_9_7 * 0.11111111111111117;
    res[682] = k7_4_9_8 * 0.19245008972987535;
    res[683] = k7_4_9_9 * 0.11111111111111117;
    res[684] = k7_5_4_4 * 0.19245008972987535;
    res[685] = k7_5_4_5 * 0.3333333333333334;
    res[686] = k7_5_4_6 * 0.3333333333333334;
    res[687] = k7_5_4_7 * 0.19245008972987535;
    res[688] = k7_5_4_8 * 0.3333333333333334;
    res[689] = k7_5_4_9 * 0.19245008972987535;
    res[690] = k7_5_5_4 * 0.3333333333333334;
    res[691] = k7_5_5_5 * 0.5773502691896258;
    res[692] = k7_5_5_6 * 0.5773502691896258;
    res[693] = k7_5_5_7 * 0.3333333333333334;
    res[694] = k7_5_5_8 * 0.5773502691896258;
    res[695] = k7_5_5_9 * 0.3333333333333334;
    res[696] = k7_5_6_4 * 0.3333333333333334;
    res[697] = k7_5_6_5 * 0.5773502691896258;
    res[698] = k7_5_6_6 * 0.5773502691896258;
    res[699] = k7_5_6_7 * 0.3333333333333334;
    res[700] = k7_5_6_8 * 0.5773502691896258;
    res[701] = k7_5_6_9 * 0.3333333333333334;
    res[702] = k7_5_7_4 * 0.19245008972987535;
    res[703] = k7_5_7_5 * 0.3333333333333334;
    res[704] = k7_5_7_6 * 0.3333333333333334;
    res[705] = k7_5_7_7 * 0.19245008972987535;
    res[706] = k7_5_7_8 * 0.3333333333333334;
    res[707] = k7_5_7_9 * 0.19245008972987535;
    res[708] = k7_5_8_4 * 0.3333333333333334;
    res[709] = k7_5_8_5 * 0.5773502691896258;
    res[710] = k7_5_8_6 * 0.5773502691896258;
    res[711] = k7_5_8_7 * 0.3333333333333334;
    res[712] = k7_5_8_8 * 0.5773502691896258;
    res[713] = k7_5_8_9 * 0.3333333333333334;
    res[714] = k7_5_9_4 * 0.19245008972987535;
    res[715] = k7_5_9_5 * 0.3333333333333334;
    res[716] = k7_5_9_6 * 0.3333333333333334;
    res[717] = k7_5_9_7 * 0.19245008972987535;
    res[718] = k7_5_9_8 * 0.3333333333333334;
    res[719] = k7_5_9_9 * 0.19245008972987535;
    res[720] = k7_6_4_4 * 0.19245008972987535;
    res[721] = k7_6_4_5 * 0.3333333333333334;
    res[722] = k7_6_4_6 * 0.3333333333333334;
    res[723] = k7_6_4_7 * 0.19245008972987535;
    res[724] = k7_6_4_8 * 0.3333333333333334;
    res[725] = k7_6_4_9 * 0.19245008972987535;
    res[726] = k7_6_5_4 * 0.3333333333333334;
    res[727] = k7_6_5_5 * 0.5773502691896258;
    res[728] = k7_6_5_6 * 0.5773502691896258;
    res[729] = k7_6_5_7 * 0.3333333333333334;
    res[730] = k7_6_5_8 * 0.5773502691896258;
    res[731] = k7_6_5_9 * 0.3333333333333334;
    res[732] = k7_6_6_4 * 0.3333333333333334;
    res[733] = k7_6_6_5 * 0.5773502691896258;
    res[734] = k7_6_6_6 * 0.5773502691896258;
    res[735] = k7_6_6_7 * 0.3333333333333334;
    res[736] = k7_6_6_8 * 0.5773502691896258;
    res[737] = k7_6_6_9 * 0.3333333333333334;
    res[738] = k7_6_7_4 * 0.19245008972987535;
    res[739] = k7_6_7_5 * 0.3333333333333334;
    res[740] = k7_6_7_6 * 0.3333333333333334;
    res[741] = k7_6_7_7 * 0.19245008972987535;
    res[742] = k7_6_7_8 * 0.3333333333333334;
    res[743] = k7_6_7_9 * 0.19245008972987535;
    res[744] = k7_6_8_4 * 0.3333333333333334;
    res[745] = k7_6_8_5 * 0.5773502691896258;
    res[746] = k7_6_8_6 * 0.5773502691896258;
    res[747] = k7_6_8_7 * 0.3333333333333334;
    res[748] = k7_6_8_8 * 0.5773502691896258;
    res[749] = k7_6_8_9 * 0.3333333333333334;
    res[750] = k7_6_9_4 * 0.19245008972987535;
    res[751] = k7_6_9_5 * 0.3333333333333334;
    res[752] = k7_6_9_6 * 0.3333333333333334;
    res[753] = k7_6_9_7 * 0.19245008972987535;
    res[754] = k7_6_9_8 * 0.3333333333333334;
    res[755] = k7_6_9_9 * 0.19245008972987535;
    res[756] = k7_7_4_4 * 0.11111111111111117;
    res[757] = k7_7_4_5 * 0.19245008972987535;
    res[758] = k7_7_4_6 * 0.19245008972987535;
    res[759] = k7_7_4_7 * 0.11111111111111117;
    res[760] = k7_7_4_8 * 0.19245008972987535;
    res[761] = k7_7_4_9 * 0.11111111111111117;
    res[762] = k7_7_5_4 * 0.19245008972987535;
    res[763] = k7_7_5_5 * 0.3333333333333334;
    res[764] = k7_7_5_6 * 0.3333333333333334;
    res[765] = k7_7_5_7 * 0.19245008972987535;
    res[766] = k7_7_5_8 * 0.3333333333333334;
    res[767] = k7_7_5_9 * 0.19245008972987535;
    res[768] = k7_7_6_4 * 0.19245008972987535;
    res[769] = k7_7_6_5 * 0.3333333333333334;
    res[770] = k7_7_6_6 * 0.3333333333333334;
    res[771] = k7_7_6_7 * 0.19245008972987535;
    res[772] = k7_7_6_8 * 0.3333333333333334;
    res[773] = k7_7_6_9 * 0.19245008972987535;
    res[774] = k7_7_7_4 * 0.11111111111111117;
    res[775] = k7_7_7_5 * 0.19245008972987535;
    res[776] = k7_7_7_6 * 0.19245008972987535;
    res[777] = k7_7_7_7 * 0.11111111111111117;
    res[778] = k7_7_7_8 * 0.19245008972987535;
    res[779] = k7_7_7_9 * 0.11111111111111117;
    res[780] = k7_7_8_4 * 0.19245008972987535;
    res[781] = k7_7_8_5 * 0.3333333333333334;
    res[782] = k7_7_8_6 * 0.3333333333333334;
    res[783] = k7_7_8_7 * 0.19245008972987535;
    res[784] = k7_7_8_8 * 0.3333333333333334;
    res[785] = k7_7_8_9 * 0.19245008972987535;
    res[786] = k7_7_9_4 * 0.11111111111111117;
    res[787] = k7_7_9_5 * 0.19245008972987535;
    res[788] = k7_7_9_6 * 0.19245008972987535;
    res[789] = k7_7_9_7 * 0.11111111111111117;
    res[790] = k7_7_9_8 * 0.19245008972987535;
    res[791] = k7_7_9_9 * 0.11111111111111117;
    res[792] = k7_8_4_4 * 0.19245008972987535;
    res[793] = k7_8_4_5 * 0.3333333333333334;
    res[794] = k7_8_4_6 * 0.3333333333333334;
    res[795] = k7_8_4_7 * 0.19245008972987535;
    res[796] = k7_8_4_8 * 0.3333333333333334;
    res[797] = k7_8_4_9 * 0.19245008972987535;
    res[798] = k7_8_5_4 * 0.3333333333333334;
    res[799] = k7_8_5_5 * 0.5773502691896258;
    res[800] = k7_8_5_6 * 0.5773502691896258;
    res[801] = k7_8_5_7 * 0.3333333333333334;
    res[802] = k7_8_5_8 * 0.5773502691896258;
    res[803] = k7_8_5_9 * 0.3333333333333334;
    res[804] = k7_8_6_4 * 0.3333333333333334;
    res[805] = k7_8_6_5 * 0.5773502691896258;
    res[806] = k7_8_6_6 * 0.5773502691896258;
    res[807] = k7_8_6_7 * 0.3333333333333334;
    res[808] = k7_8_6_8 * 0.5773502691896258;
    res[809] = k7_8_6_9 * 0.3333333333333334;
    res[810] = k7_8_7_4 * 0.19245008972987535;
    res[811] = k7_8_7_5 * 0.3333333333333334;
    res[812] = k7_8_7_6 * 0.3333333333333334;
    res[813] = k7_8_7_7 * 0.19245008972987535;
    res[814] = k7_8_7_8 * 0.3333333333333334;
    res[815] = k7_8_7_9 * 0.19245008972987535;
    res[816] = k7_8_8_4 * 0.3333333333333334;
    res[817] = k7_8_8_5 * 0.5773502691896258;
    res[818] = k7_8_8_6 * 0.5773502691896258;
    res[819] = k7_8_8_7 * 0.3333333333333334;
    res[820] = k7_8_8_8 * 0.5773502691896258;
    res[821] = k7_8_8_9 * 0.3333333333333334;
    res[822] = k7_8_9_4 * 0.19245008972987535;
    res[823] = k7_8_9_5 * 0.3333333333333334;
    res[824] = k7_8_9_6 * 0.3333333333333334;
    res[825] = k7_8_9_7 * 0.19245008972987535;
    res[826] = k7_8_9_8 * 0.3333333333333334;
    res[827] = k7_8_9_9 * 0.19245008972987535;
    res[828] = k7_9_4_4 * 0.11111111111111117;
    res[829] = k7_9_4_5 * 0.19245008972987535;
    res[830] = k7_9_4_6 * 0.19245008972987535;
    res[831] = k7_9_4_7 * 0.11111111111111117;
    res[832] = k7_9_4_8 * 0.19245008972987535;
    res[833] = k7_9_4_9 * 0.11111111111111117;
    res[834] = k7_9_5_4 * 0.19245008972987535;
    res[835] = k7_9_5_5 * 0.3333333333333334;
    res[836] = k7_9_5_6 * 0.3333333333333334;
    res[837] = k7_9_5_7 * 0.19245008972987535;
    res[838] = k7_9_5_8 * 0.3333333333333334;
    res[839] = k7_9_5_9 * 0.19245008972987535;
    res[840] = k7_9_6_4 * 0.19245008972987535;
    res[841] = k7_9_6_5 * 0.3333333333333334;
    res[842] = k7_9_6_6 * 0.3333333333333334;
    res[843] = k7_9_6_7 * 0.19245008972987535;
    res[844] = k7_9_6_8 * 0.3333333333333334;
    res[845] = k7_9_6_9 * 0.19245008972987535;
    res[846] = k7_9_7_4 * 0.11111111111111117;
    res[847] = k7_9_7_5 * 0.19245008972987535;
    res[848] = k7_9_7_6 * 0.19245008972987535;
    res[849] = k7_9_7_7 * 0.11111111111111117;
    res[850] = k7_9_7_8 * 0.19245008972987535;
    res[851] = k7_9_7_9 * 0.11111111111111117;
    res[852] = k7_9_8_4 * 0.19245008972987535;
    res[853] = k7_9_8_5 * 0.3333333333333334;
    res[854] = k7_9_8_6 * 0.3333333333333334;
    res[855] = k7_9_8_7 * 0.19245008972987535;
    res[856] = k7_9_8_8 * 0.3333333333333334;
    res[857] = k7_9_8_9 * 0.19245008972987535;
    res[858] = k7_9_9_4 * 0.11111111111111117;
    res[859] = k7_9_9_5 * 0.19245008972987535;
    res[860] = k7_9_9_6 * 0.19245008972987535;
    res[861] = k7_9_9_7 * 0.11111111111111117;
    res[862] = k7_9_9_8 * 0.19245008972987535;
    res[863] = k7_9_9_9 * 0.11111111111111117;
    res[864] = k8_4_4_4 * 0.19245008972987535;
    res[865] = k8_4_4_5 * 0.3333333333333334;
    res[866] = k8_4_4_6 * 0.3333333333333334;
    res[867] = k8_4_4_7 * 0.19245008972987535;
    res[868] = k8_4_4_8 * 0.3333333333333334;
    res[869] = k8_4_4_9 * 0.19245008972987535;
    res[870] = k8_4_5_4 * 0.3333333333333334;
    res[871] = k8_4_5_5 * 0.5773502691896258;
    res[872] = k8_4_5_6 * 0.5773502691896258;
    res[873] = k8_4_5_7 * 0.3333333333333334;
    res[874] = k8_4_5_8 * 0.5773502691896258;
    res[875] = k8_4_5_9 * 0.3333333333333334;
    res[876] = k8_4_6_4 * 0.3333333333333334;
    res[877] = k8_4_6_5 * 0.5773502691896258;
    res[878] = k8_4_6_6 * 0.5773502691896258;
    res[879] = k8_4_6_7 * 0.3333333333333334;
    res[880] = k8_4_6_8 * 0.5773502691896258;
    res[881] = k8_4_6_9 * 0.3333333333333334;
    res[882] = k8_4_7_4 * 0.19245008972987535;
    res[883] = k8_4_7_5 * 0.3333333333333334;
    res[884] = k8_4_7_6 * 0.3333333333333334;
    res[885] = k8_4_7_7 * 0.19245008972987535;
    res[886] = k8_4_7_8 * 0.3333333333333334;
    res[887] = k8_4_7_9 * 0.19245008972987535;
    res[888] = k8_4_8_4 * 0.3333333333333334;
    res[889] = k8_4_8_5 * 0.5773502691896258;
    res[890] = k8_4_8_6 * 0.5773502691896258;
    res[891] = k8_4_8_7 * 0.3333333333333334;
    res[892] = k8_4_8_8 * 0.5773502691896258;
    res[893] = k8_4_8_9 * 0.3333333333333334;
    res[894] = k8_4_9_4 * 0.19245008972987535;
    res[895] = k8_4_9_5 * 0.3333333333333334;
    res[896] = k8_4_9_6 * 0.3333333333333334;
    res[897] = k8_4_9_7 * 0.19245008972987535;
    res[898] = k8_4_9_8 * 0.3333333333333334;
    res[899] = k8_4_9_9 * 0.19245008972987535;
    res[900] = k8_5_4_4 * 0.3333333333333334;
    res[901] = k8_5_4_5 * 0.5773502691896258;
    res[902] = k8_5_4_6 * 0.5773502691896258;
    res[903] = k8_5_4_7 * 0.3333333333333334;
    res[904] = k8_5_4_8 * 0.5773502691896258;
    res[905] = k8_5_4_9 * 0.3333333333333334;
    res[906] = k8_5_5_4 * 0.5773502691896258;
    res[907] = k8_5_5_5;
    res[908] = k8_5_5_6;
    res[909] = k8_5_5_7 * 0.5773502691896258;
    res[910] = k8_5_5_8;
    res[911] = k8_5_5_9 * 0.5773502691896258;
    res[912] = k8_5_6_4 * 0.5773502691896258;
    res[913] = k8_5_6_5;
    res[914] = k8_5_6_6;
    res[915] = k8_5_6_7 * 0.5773502691896258;
    res[916] = k8_5_6_8;
    res[917] = k8_5_6_9 * 0.5773502691896258;
    res[918] = k8_5_7_4 * 0.3333333333333334;
    res[919] = k8_5_7_5 * 0.5773502691896258;
    res[920] = k8_5_7_6 * 0.5773502691896258;
    res[921] = k8_5_7_7 * 0.3333333333333334;
    res[922] = k8_5_7_8 * 0.5773502691896258;
    res[923] = k8_5_7_9 * 0.3333333333333334;
    res[924] = k8_5_8_4 * 0.5773502691896258;
    res[925] = k8_5_8_5;
    res[926] = k8_5_8_6;
    res[927] = k8_5_8_7 * 0.5773502691896258;
    res[928] = k8_5_8_8;
    res[929] = k8_5_8_9 * 0.5773502691896258;
    res[930] = k8_5_9_4 * 0.3333333333333334;
    res[931] = k8_5_9_5 * 0.5773502691896258;
    res[932] = k8_5_9_6 * 0.5773502691896258;
    res[933] = k8_5_9_7 * 0.3333333333333334;
    res[934] = k8_5_9_8 * 0.5773502691896258;
    res[935] = k8_5_9_9 * 0.3333333333333334;
    res[936] = k8_6_4_4 * 0.3333333333333334;
    res[937] = k8_6_4_5 * 0.5773502691896258;
    res[938] = k8_6_4_6 * 0.5773502691896258;
    res[939] = k8_6_4_7 * 0.3333333333333334;
    res[940] = k8_6_4_8 * 0.5773502691896258;
    res[941] = k8_6_4_9 * 0.3333333333333334;
    res[942] = k8_6_5_4 * 0.5773502691896258;
    res[943] = k8_6_5_5;
    res[944] = k8_6_5_6;
    res[945] = k8_6_5_7 * 0.5773502691896258;
    res[946] = k8_6_5_8;
    res[947] = k8_6_5_9 * 0.5773502691896258;
    res[948] = k8_6_6_4 * 0.5773502691896258;
    res[949] = k8_6_6_5;
    res[950] = k8_6_6_6;
    res[951] = k8_6_6_7 * 0.5773502691896258;
    res[952] = k8_6_6_8;
    res[953] = k8_6_6_9 * 0.5773502691896258;
    res[954] = k8_6_7_4 * 0.3333333333333334;
    res[955] = k8_6_7_5 * 0.5773502691896258;
    res[956] = k8_6_7_6 * 0.5773502691896258;
    res[957] = k8_6_7_7 * 0.3333333333333334;
    res[958] = k8_6_7_8 * 0.5773502691896258;
    res[959] = k8_6_7_9 * 0.3333333333333334;
    res[960] = k8_6_8_4 * 0.5773502691896258;
    res[961] = k8_6_8_5;
    res[962] = k8_6_8_6;
    res[963] = k8_6_8_7 * 0.5773502691896258;
    res[964] = k8_6_8_8;
    res[965] = k8_6_8_9 * 0.5773502691896258;
    res[966] = k8_6_9_4 * 0.3333333333333334;
    res[967] = k8_6_9_5 * 0.5773502691896258;
    res[968] = k8_6_9_6 * 0.5773502691896258;
    res[969] = k8_6_9_7 * 0.3333333333333334;
    res[970] = k8_6_9_8 * 0.5773502691896258;
    res[971] = k8_6_9_9 * 0.3333333333333334;
    res[972] = k8_7_4_4 * 0.19245008972987535;
    res[973] = k8_7_4_5 * 0.3333333333333334;
    res[974] = k8_7_4_6 * 0.3333333333333334;
    res[975] = k8_7_4_7 * 0.19245008972987535;
    res[976] = k8_7_4_8 * 0.3333333333333334;
    res[977] = k8_7_4_9 * 0.19245008972987535;
    res[978] = k8_7_5_4 * 0.3333333333333334;
    res[979] = k8_7_5_5 * 0.5773502691896258;
    res[980] = k8_7_5_6 * 0.5773502691896258;
    res[981] = k8_7_5_7 * 0.3333333333333334;
    res[982] = k8_7_5_8 * 0.5773502691896258;
    res[983] = k8_7_5_9 * 0.3333333333333334;
    res[984] = k8_7_6_4 * 0.3333333333333334;
    res[985] = k8_7_6_5 * 0.5773502691896258;
    res[986] = k8_7_6_6 * 0.5773502691896258;
    res[987] = k8_7_6_7 * 0.3333333333333334;
    res[988] = k8_7_6_8 * 0.5773502691896258;
    res[989] = k8_7_6_9 * 0.3333333333333334;
    res[990] = k8_7_7_4 * 0.19245008972987535;
    res[991] = k8_7_7_5 * 0.3333333333333334;
    res[992] = k8_7_7_6 * 0.3333333333333334;
    res[993] = k8_7_7_7 * 0.19245008972987535;
    res[994] = k8_7_7_8 * 0.3333333333333334;
    res[995] = k8_7_7_9 * 0.19245008972987535;
    res[996] = k8_7_8_4 * 0.3333333333333334;
    res[997] = k8_7_8_5 * 0.5773502691896258;
    res[998] = k8_7_8_6 * 0.5773502691896258;
    res[999] = k8_7_8_7 * 0.3333333333333334;
    res[1000] = k8_7_8_8 * 0.5773502691896258;
    res[1001] = k8_7_8_9 * 0.3333333333333334;
    res[1002] = k8_7_9_4 * 0.19245008972987535;
    res[1003] = k8_7_9_5 * 0.3333333333333334;
    res[1004] = k8_7_9_6 * 0.3333333333333334;
    res[1005] = k8_7_9_7 * 0.19245008972987535;
    res[1006] = k8_7_9_8 * 0.3333333333333334;
    res[1007] = k8_7_9_9 * 0.19245008972987535;
    res[1008] = k8_8_4_4 * 0.3333333333333334;
    res[1009] = k8_8_4_5 * 0.5773502691896258;
    res[1010] = k8_8_4_6 * 0.5773502691896258;
    res[1011] = k8_8_4_7 * 0.3333333333333334;
    res[1012] = k8_8_4_8 * 0.5773502691896258;
    res[1013] = k8_8_4_9 * 0.3333333333333334;
    res[1014] = k8_8_5_4 * 0.5773502691896258;
    res[1015] = k8_8_5_5;
    res[1016] = k8_8_5_6;
    res[1017] = k8_8_5_7 * 0.5773502691896258;
    res[1018] = k8_8_5_8;
    res[1019] = k8_8_5_9 * 0.5773502691896258;
    res[1020] = k8_8_6_4 * 0.5773502691896258;
    res[1021] = k8_8_6_5;
    res[1022] = k8_8_6_6;
    res[1023] = k8_8_6_7 * 0.5773502691896258;
    res[1024] = k8_8_6_8;
    res[1025] = k8_8_6_9 * 0.5773502691896258;
    res[1026] = k8_8_7_4 * 0.3333333333333334;
    res[1027] = k8_8_7_5 * 0.5773502691896258;
    res[1028] = k8_8_7_6 * 0.5773502691896258;
    res[1029] = k8_8_7_7 * 0.3333333333333334;
    res[1030] = k8_8_7_8 * 0.5773502691896258;
    res[1031] = k8_8_7_9 * 0.3333333333333334;
    res[1032] = k8_8_8_4 * 0.5773502691896258;
    res[1033] = k8_8_8_5;
    res[1034] = k8_8_8_6;
    res[1035] = k8_8_8_7 * 0.5773502691896258;
    res[1036] = k8_8_8_8;
    res[1037] = k8_8_8_9 * 0.5773502691896258;
    res[1038] = k8_8_9_4 * 0.3333333333333334;
    res[1039] = k8_8_9_5 * 0.5773502691896258;
    res[1040] = k8_8_9_6 * 0.5773502691896258;
    res[1041] = k8_8_9_7 * 0.3333333333333334;
    res[1042] = k8_8_9_8 * 0.5773502691896258;
    res[1043] = k8_8_9_9 * 0.3333333333333334;
    res[1044] = k8_9_4_4 * 0.19245008972987535;
    res[1045] = k8_9_4_5 * 0.3333333333333334;
    res[1046] = k8_9_4_6 * 0.3333333333333334;
    res[1047] = k8_9_4_7 * 0.19245008972987535;
    res[1048] = k8_9_4_8 * 0.3333333333333334;
    res[1049] = k8_9_4_9 * 0.19245008972987535;
    res[1050] = k8_9_5_4 * 0.3333333333333334;
    res[1051] = k8_9_5_5 * 0.5773502691896258;
    res[1052] = k8_9_5_6 * 0.5773502691896258;
    res[1053] = k8_9_5_7 * 0.3333333333333334;
    res[1054] = k8_9_5_8 * 0.5773502691896258;
    res[1055] = k8_9_5_9 * 0.3333333333333334;
    res[1056] = k8_9_6_4 * 0.3333333333333334;
    res[1057] = k8_9_6_5 * 0.5773502691896258;
    res[1058] = k8_9_6_6 * 0.5773502691896258;
    res[1059] = k8_9_6_7 * 0.3333333333333334;
    res[1060] = k8_9_6_8 * 0.5773502691896258;
    res[1061] = k8_9_6_9 * 0.3333333333333334;
    res[1062] = k8_9_7_4 * 0.19245008972987535;
    res[1063] = k8_9_7_5 * 0.3333333333333334;
    res[1064] = k8_9_7_6 * 0.3333333333333334;
    res[1065] = k8_9_7_7 * 0.19245008972987535;
    res[1066] = k8_9_7_8 * 0.3333333333333334;
    res[1067] = k8_9_7_9 * 0.19245008972987535;
    res[1068] = k8_9_8_4 * 0.3333333333333334;
    res[1069] = k8_9_8_5 * 0.5773502691896258;
    res[1070] = k8_9_8_6 * 0.5773502691896258;
    res[1071] = k8_9_8_7 * 0.3333333333333334;
    res[1072] = k8_9_8_8 * 0.5773502691896258;
    res[1073] = k8_9_8_9 * 0.3333333333333334;
    res[1074] = k8_9_9_4 * 0.19245008972987535;
    res[1075] = k8_9_9_5 * 0.3333333333333334;
    res[1076] = k8_9_9_6 * 0.3333333333333334;
    res[1077] = k8_9_9_7 * 0.19245008972987535;
    res[1078] = k8_9_9_8 * 0.3333333333333334;
    res[1079] = k8_9_9_9 * 0.19245008972987535;
    res[1080] = k9_4_4_4 * 0.11111111111111117;
    res[1081] = k9_4_4_5 * 0.19245008972987535;
    res[1082] = k9_4_4_6 * 0.19245008972987535;
    res[1083] = k9_4_4_7 * 0.11111111111111117;
    res[1084] = k9_4_4_8 * 0.19245008972987535;
    res[1085] = k9_4_4_9 * 0.11111111111111117;
    res[1086] = k9_4_5_4 * 0.19245008972987535;
    res[1087] = k9_4_5_5 * 0.3333333333333334;
    res[1088] = k9_4_5_6 * 0.3333333333333334;
    res[1089] = k9_4_5_7 * 0.19245008972987535;
    res[1090] = k9_4_5_8 * 0.3333333333333334;
    res[1091] = k9_4_5_9 * 0.19245008972987535;
    res[1092] = k9_4_6_4 * 0.19245008972987535;
    res[1093] = k9_4_6_5 * 0.3333333333333334;
    res[1094] = k9_4_6_6 * 0.3333333333333334;
    res[1095] = k9_4_6_7 * 0.19245008972987535;
    res[1096] = k9_4_6_8 * 0.3333333333333334;
    res[1097] = k9_4_6_9 * 0.19245008972987535;
    res[1098] = k9_4_7_4 * 0.11111111111111117;
    res[1099] = k9_4_7_5 * 0.19245008972987535;
    res[1100] = k9_4_7_6 * 0.19245008972987535;
    res[1101] = k9_4_7_7 * 0.11111111111111117;
    res[1102] = k9_4_7_8 * 0.19245008972987535;
    res[1103] = k9_4_7_9 * 0.11111111111111117;
    res[1104] = k9_4_8_4 * 0.19245008972987535;
    res[1105] = k9_4_8_5 * 0.3333333333333334;
    res[1106] = k9_4_8_6 * 0.3333333333333334;
    res[1107] = k9_4_8_7 * 0.19245008972987535;
    res[1108] = k9_4_8_8 * 0.3333333333333334;
    res[1109] = k9_4_8_9 * 0.19245008972987535;
    res[1110] = k9_4_9_4 * 0.11111111111111117;
    res[1111] = k9_4_9_5 * 0.19245008972987535;
    res[1112] = k9_4_9_6 * 0.19245008972987535;
    res[1113] = k9_4_9_7 * 0.11111111111111117;
    res[1114] = k9_4_9_8 * 0.19245008972987535;
    res[1115] = k9_4_9_9 * 0.11111111111111117;
    res[1116] = k9_5_4_4 * 0.19245008972987535;
    res[1117] = k9_5_4_5 * 0.3333333333333334;
    res[1118] = k9_5_4_6 * 0.3333333333333334;
    res[1119] = k9_5_4_7 * 0.19245008972987535;
    res[1120] = k9_5_4_8 * 0.3333333333333334;
    res[1121] = k9_5_4_9 * 0.19245008972987535;
    res[1122] = k9_5_5_4 * 0.3333333333333334;
    res[1123] = k9_5_5_5 * 0.5773502691896258;
    res[1124] = k9_5_5_6 * 0.5773502691896258;
    res[1125] = k9_5_5_7 * 0.3333333333333334;
    res[1126] = k9_5_5_8 * 0.5773502691896258;
    res[1127] = k9_5_5_9 * 0.3333333333333334;
    res[1128] = k9_5_6_4 * 0.3333333333333334;
    res[1129] = k9_5_6_5 * 0.5773502691896258;
    res[1130] = k9_5_6_6 * 0.5773502691896258;
    res[1131] = k9_5_6_7 * 0.3333333333333334;
    res[1132] = k9_5_6_8 * 0.5773502691896258;
    res[1133] = k9_5_6_9 * 0.3333333333333334;
    res[1134] = k9_5_7_4 * 0.19245008972987535;
    res[1135] = k9_5_7_5 * 0.3333333333333334;
    res[1136] = k9_5_7_6 * 0.3333333333333334;
    res[1137] = k9_5_7_7 * 0.19245008972987535;
    res[1138] = k9_5_7_8 * 0.3333333333333334;
    res[1139] = k9_5_7_9 * 0.19245008972987535;
    res[1140] = k9_5_8_4 * 0.3333333333333334;
    res[1141] = k9_5_8_5 * 0.5773502691896258;
    res[1142] = k9_5_8_6 * 0.5773502691896258;
    res[1143] = k9_5_8_7 * 0.3333333333333334;
    res[1144] = k9_5_8_8 * 0.5773502691896258;
    res[1145] = k9_5_8_9 * 0.3333333333333334;
    res[1146] = k9_5_9_4 * 0.19245008972987535;
    res[1147] = k9_5_9_5 * 0.3333333333333334;
    res[1148] = k9_5_9_6 * 0.3333333333333334;
    res[1149] = k9_5_9_7 * 0.19245008972987535;
    res[1150] = k9_5_9_8 * 0.3333333333333334;
    res[1151] = k9_5_9_9 * 0.19245008972987535;
    res[1152] = k9_6_4_4 * 0.19245008972987535;
    res[1153] = k9_6_4_5 * 0.3333333333333334;
    res[1154] = k9_6_4_6 * 0.3333333333333334;
    res[1155] = k9_6_4_7 * 0.19245008972987535;
    res[1156] = k9_6_4_8 * 0.3333333333333334;
    res[1157] = k9_6_4_9 * 0.19245008972987535;
    res[1158] = k9_6_5_4 * 0.3333333333333334;
    res[1159] = k9_6_5_5 * 0.5773502691896258;
    res[1160] = k9_6_5_6 * 0.5773502691896258;
    res[1161] = k9_6_5_7 * 0.3333333333333334;
    res[1162] = k9_6_5_8 * 0.5773502691896258;
    res[1163] = k9_6_5_9 * 0.3333333333333334;
    res[1164] = k9_6_6_4 * 0.3333333333333334;
    res[1165] = k9_6_6_5 * 0.5773502691896258;
    res[1166] = k9_6_6_6 * 0.5773502691896258;
    res[1167] = k9_6_6_7 * 0.3333333333333334;
    res[1168] = k9_6_6_8 * 0.5773502691896258;
    res[1169] = k9_6_6_9 * 0.3333333333333334;
    res[1170] = k9_6_7_4 * 0.19245008972987535;
    res[1171] = k9_6_7_5 * 0.3333333333333334;
    res[1172] = k9_6_7_6 * 0.3333333333333334;
    res[1173] = k9_6_7_7 * 0.19245008972987535;
    res[1174] = k9_6_7_8 * 0.3333333333333334;
    res[1175] = k9_6_7_9 * 0.19245008972987535;
    res[1176] = k9_6_8_4 * 0.3333333333333334;
    res[1177] = k9_6_8_5 * 0.5773502691896258;
    res[1178] = k9_6_8_6 * 0.5773502691896258;
    res[1179] = k9_6_8_7 * 0.3333333333333334;
    res[1180] = k9_6_8_8 * 0.5773502691896258;
    res[1181] = k9_6_8_9 * 0.3333333333333334;
    res[1182] = k9_6_9_4 * 0.19245008972987535;
    res[1183] = k9_6_9_5 * 0.3333333333333334;
    res[1184] = k9_6_9_6 * 0.3333333333333334;
    res[1185] = k9_6_9_7 * 0.19245008972987535;
    res[1186] = k9_6_9_8 * 0.3333333333333334;
    res[1187] = k9_6_9_9 * 0.19245008972987535;
    res[1188] = k9_7_4_4 * 0.11111111111111117;
    res[1189] = k9_7_4_5 * 0.19245008972987535;
    res[1190] = k9_7_4_6 * 0.19245008972987535;
    res[1191] = k9_7_4_7 * 0.11111111111111117;
    res[1192] = k9_7_4_8 * 0.19245008972987535;
    res[1193] = k9_7_4_9 * 0.11111111111111117;
    res[1194] = k9_7_5_4 * 0.19245008972987535;
    res[1195] = k9_7_5_5 * 0.3333333333333334;
    res[1196] = k9_7_5_6 * 0.3333333333333334;
    res[1197] = k9_7_5_7 * 0.19245008972987535;
    res[1198] = k9_7_5_8 * 0.3333333333333334;
    res[1199] = k9_7_5_9 * 0.19245008972987535;
    res[1200] = k9_7_6_4 * 0.19245008972987535;
    res[1201] = k9_7_6_5 * 0.3333333333333334;
    res[1202] = k9_7_6_6 * 0.3333333333333334;
    res[1203] = k9_7_6_7 * 0.19245008972987535;
    res[1204] = k9_7_6_8 * 0.3333333333333334;
    res[1205] = k9_7_6_9 * 0.19245008972987535;
    res[1206] = k9_7_7_4 * 0.11111111111111117;
    res[1207] = k9_7_7_5 * 0.19245008972987535;
    res[1208] = k9_7_7_6 * 0.19245008972987535;
    res[1209] = k9_7_7_7 * 0.11111111111111117;
    res[1210] = k9_7_7_8 * 0.19245008972987535;
    res[1211] = k9_7_7_9 * 0.11111111111111117;
    res[1212] = k9_7_8_4 * 0.19245008972987535;
    res[1213] = k9_7_8_5 * 0.3333333333333334;
    res[1214] = k9_7_8_6 * 0.3333333333333334;
    res[1215] = k9_7_8_7 * 0.19245008972987535;
    res[1216] = k9_7_8_8 * 0.3333333333333334;
    res[1217] = k9_7_8_9 * 0.19245008972987535;
    res[1218] = k9_7_9_4 * 0.11111111111111117;
    res[1219] = k9_7_9_5 * 0.19245008972987535;
    res[1220] = k9_7_9_6 * 0.19245008972987535;
    res[1221] = k9_7_9_7 * 0.11111111111111117;
    res[1222] = k9_7_9_8 * 0.19245008972987535;
    res[1223] = k9_7_9_9 * 0.11111111111111117;
    res[1224] = k9_8_4_4 * 0.19245008972987535;
    res[1225] = k9_8_4_5 * 0.3333333333333334;
    res[1226] = k9_8_4_6 * 0.3333333333333334;
    res[1227] = k9_8_4_7 * 0.19245008972987535;
    res[1228] = k9_8_4_8 * 0.3333333333333334;
    res[1229] = k9_8_4_9 * 0.19245008972987535;
    res[1230] = k9_8_5_4 * 0.3333333333333334;
    res[1231] = k9_8_5_5 * 0.5773502691896258;
    res[1232] = k9_8_5_6 * 0.5773502691896258;
    res[1233] = k9_8_5_7 * 0.3333333333333334;
    res[1234] = k9_8_5_8 * 0.5773502691896258;
    res[1235] = k9_8_5_9 * 0.3333333333333334;
    res[1236] = k9_8_6_4 * 0.3333333333333334;
    res[1237] = k9_8_6_5 * 0.5773502691896258;
    res[1238] = k9_8_6_6 * 0.5773502691896258;
    res[1239] = k9_8_6_7 * 0.3333333333333334;
    res[1240] = k9_8_6_8 * 0.5773502691896258;
    res[1241] = k9_8_6_9 * 0.3333333333333334;
    res[1242] = k9_8_7_4 * 0.19245008972987535;
    res[1243] = k9_8_7_5 * 0.3333333333333334;
    res[1244] = k9_8_7_6 * 0.3333333333333334;
    res[1245] = k9_8_7_7 * 0.19245008972987535;
    res[1246] = k9_8_7_8 * 0.3333333333333334;
    res[1247] = k9_8_7_9 * 0.19245008972987535;
    res[1248] = k9_8_8_4 * 0.3333333333333334;
    res[1249] = k9_8_8_5 * 0.5773502691896258;
    res[1250] = k9_8_8_6 * 0.5773502691896258;
    res[1251] = k9_8_8_7 * 0.3333333333333334;
    res[1252] = k9_8_8_8 * 0.5773502691896258;
    res[1253] = k9_8_8_9 * 0.3333333333333334;
    res[1254] = k9_8_9_4 * 0.19245008972987535;
    res[1255] = k9_8_9_5 * 0.3333333333333334;
    res[1256] = k9_8_9_6 * 0.3333333333333334;
    res[1257] = k9_8_9_7 * 0.19245008972987535;
    res[1258] = k9_8_9_8 * 0.3333333333333334;
    res[1259] = k9_8_9_9 * 0.19245008972987535;
    res[1260] = k9_9_4_4 * 0.11111111111111117;
    res[1261] = k9_9_4_5 * 0.19245008972987535;
    res[1262] = k9_9_4_6 * 0.19245008972987535;
    res[1263] = k9_9_4_7 * 0.11111111111111117;
    res[1264] = k9_9_4_8 * 0.19245008972987535;
    res[1265] = k9_9_4_9 * 0.11111111111111117;
    res[1266] = k9_9_5_4 * 0.19245008972987535;
    res[1267] = k9_9_5_5 * 0.3333333333333334;
    res[1268] = k9_9_5_6 * 0.3333333333333334;
    res[1269] = k9_9_5_7 * 0.19245008972987535;
    res[1270] = k9_9_5_8 * 0.3333333333333334;
    res[1271] = k9_9_5_9 * 0.19245008972987535;
    res[1272] = k9_9_6_4 * 0.19245008972987535;
    res[1273] = k9_9_6_5 * 0.3333333333333334;
    res[1274] = k9_9_6_6 * 0.3333333333333334;
    res[1275] = k9_9_6_7 * 0.19245008972987535;
    res[1276] = k9_9_6_8 * 0.3333333333333334;
    res[1277] = k9_9_6_9 * 0.19245008972987535;
    res[1278] = k9_9_7_4 * 0.11111111111111117;
    res[1279] = k9_9_7_5 * 0.19245008972987535;
    res[1280] = k9_9_7_6 * 0.19245008972987535;
    res[1281] = k9_9_7_7 * 0.11111111111111117;
    res[1282] = k9_9_7_8 * 0.19245008972987535;
    res[1283] = k9_9_7_9 * 0.11111111111111117;
    res[1284] = k9_9_8_4 * 0.19245008972987535;
    res[1285] = k9_9_8_5 * 0.3333333333333334;
    res[1286] = k9_9_8_6 * 0.3333333333333334;
    res[1287] = k9_9_8_7 * 0.19245008972987535;
    res[1288] = k9_9_8_8 * 0.3333333333333334;
    res[1289] = k9_9_8_9 * 0.19245008972987535;
    res[1290] = k9_9_9_4 * 0.11111111111111117;
    res[1291] = k9_9_9_5 * 0.19245008972987535;
    res[1292] = k9_9_9_6 * 0.19245008972987535;
    res[1293] = k9_9_9_7 * 0.11111111111111117;
    res[1294] = k9_9_9_8 * 0.19245008972987535;
    res[1295] = k9_9_9_9 * 0.11111111111111117;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[1296]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_dddd(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[961];
    vrr_dddd<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 961; ++x) acc_out[x] = acc[x];
    }
    hrr_dddd(P, p, q, acc, res);
}

__device__ __forceinline__ void store_dddd(double *__restrict__ out, const int4 ib_, const int4 ik_,
                                            bool same, const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    (void)dab; (void)dcd;
    const long long ij_0_0 = pair_index(ib_.z + 0, ib_.w + 0);
    const long long ij_0_1 = pair_index(ib_.z + 0, ib_.w + 1);
    const long long ij_0_2 = pair_index(ib_.z + 0, ib_.w + 2);
    const long long ij_0_3 = pair_index(ib_.z + 0, ib_.w + 3);
    const long long ij_0_4 = pair_index(ib_.z + 0, ib_.w + 4);
    const long long ij_0_5 = pair_index(ib_.z + 0, ib_.w + 5);
    const long long ij_1_0 = pair_index(ib_.z + 1, ib_.w + 0);
    const long long ij_1_1 = pair_index(ib_.z + 1, ib_.w + 1);
    const long long ij_1_2 = pair_index(ib_.z + 1, ib_.w + 2);
    const long long ij_1_3 = pair_index(ib_.z + 1, ib_.w + 3);
    const long long ij_1_4 = pair_index(ib_.z + 1, ib_.w + 4);
    const long long ij_1_5 = pair_index(ib_.z + 1, ib_.w + 5);
    const long long ij_2_0 = pair_index(ib_.z + 2, ib_.w + 0);
    const long long ij_2_1 = pair_index(ib_.z + 2, ib_.w + 1);
    const long long ij_2_2 = pair_index(ib_.z + 2, ib_.w + 2);
    const long long ij_2_3 = pair_index(ib_.z + 2, ib_.w + 3);
    const long long ij_2_4 = pair_index(ib_.z + 2, ib_.w + 4);
    const long long ij_2_5 = pair_index(ib_.z + 2, ib_.w + 5);
    const long long ij_3_0 = pair_index(ib_.z + 3, ib_.w + 0);
    const long long ij_3_1 = pair_index(ib_.z + 3, ib_.w + 1);
    const long long ij_3_2 = pair_index(ib_.z + 3, ib_.w + 2);
    const long long ij_3_3 = pair_index(ib_.z + 3, ib_.w + 3);
    const long long ij_3_4 = pair_index(ib_.z + 3, ib_.w + 4);
    const long long ij_3_5 = pair_index(ib_.z + 3, ib_.w + 5);
    const long long ij_4_0 = pair_index(ib_.z + 4, ib_.w + 0);
    const long long ij_4_1 = pair_index(ib_.z + 4, ib_.w + 1);
    const long long ij_4_2 = pair_index(ib_.z + 4, ib_.w + 2);
    const long long ij_4_3 = pair_index(ib_.z + 4, ib_.w + 3);
    const long long ij_4_4 = pair_index(ib_.z + 4, ib_.w + 4);
    const long long ij_4_5 = pair_index(ib_.z + 4, ib_.w + 5);
    const long long ij_5_0 = pair_index(ib_.z + 5, ib_.w + 0);
    const long long ij_5_1 = pair_index(ib_.z + 5, ib_.w + 1);
    const long long ij_5_2 = pair_index(ib_.z + 5, ib_.w + 2);
    const long long ij_5_3 = pair_index(ib_.z + 5, ib_.w + 3);
    const long long ij_5_4 = pair_index(ib_.z + 5, ib_.w + 4);
    const long long ij_5_5 = pair_index(ib_.z + 5, ib_.w + 5);
    const long long kl_0_0 = pair_index(ik_.z + 0, ik_.w + 0);
    const long long kl_0_1 = pair_index(ik_.z + 0, ik_.w + 1);
    const long long kl_0_2 = pair_index(ik_.z + 0, ik_.w + 2);
    const long long kl_0_3 = pair_index(ik_.z + 0, ik_.w + 3);
    const long long kl_0_4 = pair_index(ik_.z + 0, ik_.w + 4);
    const long long kl_0_5 = pair_index(ik_.z + 0, ik_.w + 5);
    const long long kl_1_0 = pair_index(ik_.z + 1, ik_.w + 0);
    const long long kl_1_1 = pair_index(ik_.z + 1, ik_.w + 1);
    const long long kl_1_2 = pair_index(ik_.z + 1, ik_.w + 2);
    const long long kl_1_3 = pair_index(ik_.z + 1, ik_.w + 3);
    const long long kl_1_4 = pair_index(ik_.z + 1, ik_.w + 4);
    const long long kl_1_5 = pair_index(ik_.z + 1, ik_.w + 5);
    const long long kl_2_0 = pair_index(ik_.z + 2, ik_.w + 0);
    const long long kl_2_1 = pair_index(ik_.z + 2, ik_.w + 1);
    const long long kl_2_2 = pair_index(ik_.z + 2, ik_.w + 2);
    const long long kl_2_3 = pair_index(ik_.z + 2, ik_.w + 3);
    const long long kl_2_4 = pair_index(ik_.z + 2, ik_.w + 4);
    const long long kl_2_5 = pair_index(ik_.z + 2, ik_.w + 5);
    const long long kl_3_0 = pair_index(ik_.z + 3, ik_.w + 0);
    const long long kl_3_1 = pair_index(ik_.z + 3, ik_.w + 1);
    const long long kl_3_2 = pair_index(ik_.z + 3, ik_.w + 2);
    const long long kl_3_3 = pair_index(ik_.z + 3, ik_.w + 3);
    const long long kl_3_4 = pair_index(ik_.z + 3, ik_.w + 4);
    const long long kl_3_5 = pair_index(ik_.z + 3, ik_.w + 5);
    const long long kl_4_0 = pair_index(ik_.z + 4, ik_.w + 0);
    const long long kl_4_1 = pair_index(ik_.z + 4, ik_.w + 1);
    const long long kl_4_2 = pair_index(ik_.z + 4, ik_.w + 2);
    const long long kl_4_3 = pair_index(ik_.z + 4, ik_.w + 3);
    const long long kl_4_4 = pair_index(ik_.z + 4, ik_.w + 4);
    const long long kl_4_5 = pair_index(ik_.z + 4, ik_.w + 5);
    const long long kl_5_0 = pair_index(ik_.z + 5, ik_.w + 0);
    const long long kl_5_1 = pair_index(ik_.z + 5, ik_.w + 1);
    const long long kl_5_2 = pair_index(ik_.z + 5, ik_.w + 2);
    const long long kl_5_3 = pair_index(ik_.z + 5, ik_.w + 3);
    const long long kl_5_4 = pair_index(ik_.z + 5, ik_.w + 4);
    const long long kl_5_5 = pair_index(ik_.z + 5, ik_.w + 5);
    { const long long ij = ij_0_0, kl = kl_0_0;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_0_1;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_0_2;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_0, kl = kl_0_3;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_0, kl = kl_0_4;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_0, kl = kl_0_5;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_0, kl = kl_1_1;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_0, kl = kl_1_2;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_0_0, kl = kl_1_3;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_0_0, kl = kl_1_4;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_0_0, kl = kl_1_5;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_0_0, kl = kl_2_1;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_0_0, kl = kl_2_2;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_0_0, kl = kl_2_3;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_0_0, kl = kl_2_4;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_0_0, kl = kl_2_5;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_0_0, kl = kl_3_0;
      if ((!dab || 0 >= 0) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_0_0, kl = kl_3_1;
      if ((!dab || 0 >= 0) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_0_0, kl = kl_3_2;
      if ((!dab || 0 >= 0) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_0_0, kl = kl_3_3;
      if ((!dab || 0 >= 0) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_0_0, kl = kl_3_4;
      if ((!dab || 0 >= 0) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_0_0, kl = kl_3_5;
      if ((!dab || 0 >= 0) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_0_0, kl = kl_4_0;
      if ((!dab || 0 >= 0) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_0_0, kl = kl_4_1;
      if ((!dab || 0 >= 0) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_0_0, kl = kl_4_2;
      if ((!dab || 0 >= 0) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_0_0, kl = kl_4_3;
      if ((!dab || 0 >= 0) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_0_0, kl = kl_4_4;
      if ((!dab || 0 >= 0) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_0_0, kl = kl_4_5;
      if ((!dab || 0 >= 0) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_0_0, kl = kl_5_0;
      if ((!dab || 0 >= 0) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_0_0, kl = kl_5_1;
      if ((!dab || 0 >= 0) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_0_0, kl = kl_5_2;
      if ((!dab || 0 >= 0) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_0_0, kl = kl_5_3;
      if ((!dab || 0 >= 0) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_0_0, kl = kl_5_4;
      if ((!dab || 0 >= 0) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_0_0, kl = kl_5_5;
      if ((!dab || 0 >= 0) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_0_1, kl = kl_0_1;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_0_1, kl = kl_0_2;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_0_1, kl = kl_0_3;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_0_1, kl = kl_0_4;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_0_1, kl = kl_0_5;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_0_1, kl = kl_1_0;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_0_1, kl = kl_1_1;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_0_1, kl = kl_1_2;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_0_1, kl = kl_1_3;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_0_1, kl = kl_1_4;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_0_1, kl = kl_1_5;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_0_1, kl = kl_2_0;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_0_1, kl = kl_2_1;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_0_1, kl = kl_2_2;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_0_1, kl = kl_2_3;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_0_1, kl = kl_2_4;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_0_1, kl = kl_2_5;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_0_1, kl = kl_3_0;
      if ((!dab || 0 >= 1) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_0_1, kl = kl_3_1;
      if ((!dab || 0 >= 1) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_0_1, kl = kl_3_2;
      if ((!dab || 0 >= 1) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_0_1, kl = kl_3_3;
      if ((!dab || 0 >= 1) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_0_1, kl = kl_3_4;
      if ((!dab || 0 >= 1) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_0_1, kl = kl_3_5;
      if ((!dab || 0 >= 1) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_0_1, kl = kl_4_0;
      if ((!dab || 0 >= 1) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_0_1, kl = kl_4_1;
      if ((!dab || 0 >= 1) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_0_1, kl = kl_4_2;
      if ((!dab || 0 >= 1) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_0_1, kl = kl_4_3;
      if ((!dab || 0 >= 1) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_0_1, kl = kl_4_4;
      if ((!dab || 0 >= 1) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_0_1, kl = kl_4_5;
      if ((!dab || 0 >= 1) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_0_1, kl = kl_5_0;
      if ((!dab || 0 >= 1) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_0_1, kl = kl_5_1;
      if ((!dab || 0 >= 1) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_0_1, kl = kl_5_2;
      if ((!dab || 0 >= 1) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_0_1, kl = kl_5_3;
      if ((!dab || 0 >= 1) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_0_1, kl = kl_5_4;
      if ((!dab || 0 >= 1) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_0_1, kl = kl_5_5;
      if ((!dab || 0 >= 1) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_0_2, kl = kl_0_1;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_0_2, kl = kl_0_2;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_0_2, kl = kl_0_3;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_0_2, kl = kl_0_4;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_0_2, kl = kl_0_5;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_0_2, kl = kl_1_0;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_0_2, kl = kl_1_1;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_0_2, kl = kl_1_2;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_0_2, kl = kl_1_3;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_0_2, kl = kl_1_4;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_0_2, kl = kl_1_5;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_0_2, kl = kl_2_0;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_0_2, kl = kl_2_1;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_0_2, kl = kl_2_2;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_0_2, kl = kl_2_3;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_0_2, kl = kl_2_4;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_0_2, kl = kl_2_5;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_0_2, kl = kl_3_0;
      if ((!dab || 0 >= 2) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_0_2, kl = kl_3_1;
      if ((!dab || 0 >= 2) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_0_2, kl = kl_3_2;
      if ((!dab || 0 >= 2) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_0_2, kl = kl_3_3;
      if ((!dab || 0 >= 2) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_0_2, kl = kl_3_4;
      if ((!dab || 0 >= 2) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_0_2, kl = kl_3_5;
      if ((!dab || 0 >= 2) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_0_2, kl = kl_4_0;
      if ((!dab || 0 >= 2) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_0_2, kl = kl_4_1;
      if ((!dab || 0 >= 2) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_0_2, kl = kl_4_2;
      if ((!dab || 0 >= 2) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_0_2, kl = kl_4_3;
      if ((!dab || 0 >= 2) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
    { const long long ij = ij_0_2, kl = kl_4_4;
      if ((!dab || 0 >= 2) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[100]; }
    { const long long ij = ij_0_2, kl = kl_4_5;
      if ((!dab || 0 >= 2) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[101]; }
    { const long long ij = ij_0_2, kl = kl_5_0;
      if ((!dab || 0 >= 2) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[102]; }
    { const long long ij = ij_0_2, kl = kl_5_1;
      if ((!dab || 0 >= 2) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[103]; }
    { const long long ij = ij_0_2, kl = kl_5_2;
      if ((!dab || 0 >= 2) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[104]; }
    { const long long ij = ij_0_2, kl = kl_5_3;
      if ((!dab || 0 >= 2) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[105]; }
    { const long long ij = ij_0_2, kl = kl_5_4;
      if ((!dab || 0 >= 2) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[106]; }
    { const long long ij = ij_0_2, kl = kl_5_5;
      if ((!dab || 0 >= 2) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[107]; }
    { const long long ij = ij_0_3, kl = kl_0_0;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[108]; }
    { const long long ij = ij_0_3, kl = kl_0_1;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[109]; }
    { const long long ij = ij_0_3, kl = kl_0_2;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[110]; }
    { const long long ij = ij_0_3, kl = kl_0_3;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[111]; }
    { const long long ij = ij_0_3, kl = kl_0_4;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[112]; }
    { const long long ij = ij_0_3, kl = kl_0_5;
      if ((!dab || 0 >= 3) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[113]; }
    { const long long ij = ij_0_3, kl = kl_1_0;
      if ((!dab || 0 >= 3) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[114]; }
    { const long long ij = ij_0_3, kl = kl_1_1;
      if ((!dab || 0 >= 3) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[115]; }
    { const long long ij = ij_0_3, kl = kl_1_2;
      if ((!dab || 0 >= 3) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[116]; }
    { const long long ij = ij_0_3, kl = kl_1_3;
      if ((!dab || 0 >= 3) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[117]; }
    { const long long ij = ij_0_3, kl = kl_1_4;
      if ((!dab || 0 >= 3) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[118]; }
    { const long long ij = ij_0_3, kl = kl_1_5;
      if ((!dab || 0 >= 3) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[119]; }
    { const long long ij = ij_0_3, kl = kl_2_0;
      if ((!dab || 0 >= 3) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[120]; }
    { const long long ij = ij_0_3, kl = kl_2_1;
      if ((!dab || 0 >= 3) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[121]; }
    { const long long ij = ij_0_3, kl = kl_2_2;
      if ((!dab || 0 >= 3) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[122]; }
    { const long long ij = ij_0_3, kl = kl_2_3;
      if ((!dab || 0 >= 3) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[123]; }
    { const long long ij = ij_0_3, kl = kl_2_4;
      if ((!dab || 0 >= 3) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[124]; }
    { const long long ij = ij_0_3, kl = kl_2_5;
      if ((!dab || 0 >= 3) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[125]; }
    { const long long ij = ij_0_3, kl = kl_3_0;
      if ((!dab || 0 >= 3) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[126]; }
    { const long long ij = ij_0_3, kl = kl_3_1;
      if ((!dab || 0 >= 3) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[127]; }
    { const long long ij = ij_0_3, kl = kl_3_2;
      if ((!dab || 0 >= 3) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[128]; }
    { const long long ij = ij_0_3, kl = kl_3_3;
      if ((!dab || 0 >= 3) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[129]; }
    { const long long ij = ij_0_3, kl = kl_3_4;
      if ((!dab || 0 >= 3) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[130]; }
    { const long long ij = ij_0_3, kl = kl_3_5;
      if ((!dab || 0 >= 3) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[131]; }
    { const long long ij = ij_0_3, kl = kl_4_0;
      if ((!dab || 0 >= 3) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[132]; }
    { const long long ij = ij_0_3, kl = kl_4_1;
      if ((!dab || 0 >= 3) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[133]; }
    { const long long ij = ij_0_3, kl = kl_4_2;
      if ((!dab || 0 >= 3) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[134]; }
    { const long long ij = ij_0_3, kl = kl_4_3;
      if ((!dab || 0 >= 3) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[135]; }
    { const long long ij = ij_0_3, kl = kl_4_4;
      if ((!dab || 0 >= 3) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[136]; }
    { const long long ij = ij_0_3, kl = kl_4_5;
      if ((!dab || 0 >= 3) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[137]; }
    { const long long ij = ij_0_3, kl = kl_5_0;
      if ((!dab || 0 >= 3) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[138]; }
    { const long long ij = ij_0_3, kl = kl_5_1;
      if ((!dab || 0 >= 3) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[139]; }
    { const long long ij = ij_0_3, kl = kl_5_2;
      if ((!dab || 0 >= 3) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[140]; }
    { const long long ij = ij_0_3, kl = kl_5_3;
      if ((!dab || 0 >= 3) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[141]; }
    { const long long ij = ij_0_3, kl = kl_5_4;
      if ((!dab || 0 >= 3) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[142]; }
    { const long long ij = ij_0_3, kl = kl_5_5;
      if ((!dab || 0 >= 3) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[143]; }
    { const long long ij = ij_0_4, kl = kl_0_0;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[144]; }
    { const long long ij = ij_0_4, kl = kl_0_1;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[145]; }
    { const long long ij = ij_0_4, kl = kl_0_2;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[146]; }
    { const long long ij = ij_0_4, kl = kl_0_3;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[147]; }
    { const long long ij = ij_0_4, kl = kl_0_4;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[148]; }
    { const long long ij = ij_0_4, kl = kl_0_5;
      if ((!dab || 0 >= 4) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[149]; }
    { const long long ij = ij_0_4, kl = kl_1_0;
      if ((!dab || 0 >= 4) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[150]; }
    { const long long ij = ij_0_4, kl = kl_1_1;
      if ((!dab || 0 >= 4) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[151]; }
    { const long long ij = ij_0_4, kl = kl_1_2;
      if ((!dab || 0 >= 4) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[152]; }
    { const long long ij = ij_0_4, kl = kl_1_3;
      if ((!dab || 0 >= 4) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[153]; }
    { const long long ij = ij_0_4, kl = kl_1_4;
      if ((!dab || 0 >= 4) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[154]; }
    { const long long ij = ij_0_4, kl = kl_1_5;
      if ((!dab || 0 >= 4) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[155]; }
    { const long long ij = ij_0_4, kl = kl_2_0;
      if ((!dab || 0 >= 4) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[156]; }
    { const long long ij = ij_0_4, kl = kl_2_1;
      if ((!dab || 0 >= 4) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[157]; }
    { const long long ij = ij_0_4, kl = kl_2_2;
      if ((!dab || 0 >= 4) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[158]; }
    { const long long ij = ij_0_4, kl = kl_2_3;
      if ((!dab || 0 >= 4) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[159]; }
    { const long long ij = ij_0_4, kl = kl_2_4;
      if ((!dab || 0 >= 4) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[160]; }
    { const long long ij = ij_0_4, kl = kl_2_5;
      if ((!dab || 0 >= 4) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[161]; }
    { const long long ij = ij_0_4, kl = kl_3_0;
      if ((!dab || 0 >= 4) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[162]; }
    { const long long ij = ij_0_4, kl = kl_3_1;
      if ((!dab || 0 >= 4) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[163]; }
    { const long long ij = ij_0_4, kl = kl_3_2;
      if ((!dab || 0 >= 4) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[164]; }
    { const long long ij = ij_0_4, kl = kl_3_3;
      if ((!dab || 0 >= 4) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[165]; }
    { const long long ij = ij_0_4, kl = kl_3_4;
      if ((!dab || 0 >= 4) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[166]; }
    { const long long ij = ij_0_4, kl = kl_3_5;
      if ((!dab || 0 >= 4) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[167]; }
    { const long long ij = ij_0_4, kl = kl_4_0;
      if ((!dab || 0 >= 4) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[168]; }
    { const long long ij = ij_0_4, kl = kl_4_1;
      if ((!dab || 0 >= 4) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[169]; }
    { const long long ij = ij_0_4, kl = kl_4_2;
      if ((!dab || 0 >= 4) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[170]; }
    { const long long ij = ij_0_4, kl = kl_4_3;
      if ((!dab || 0 >= 4) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[171]; }
    { const long long ij = ij_0_4, kl = kl_4_4;
      if ((!dab || 0 >= 4) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[172]; }
    { const long long ij = ij_0_4, kl = kl_4_5;
      if ((!dab || 0 >= 4) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[173]; }
    { const long long ij = ij_0_4, kl = kl_5_0;
      if ((!dab || 0 >= 4) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[174]; }
    { const long long ij = ij_0_4, kl = kl_5_1;
      if ((!dab || 0 >= 4) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[175]; }
    { const long long ij = ij_0_4, kl = kl_5_2;
      if ((!dab || 0 >= 4) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[176]; }
    { const long long ij = ij_0_4, kl = kl_5_3;
      if ((!dab || 0 >= 4) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[177]; }
    { const long long ij = ij_0_4, kl = kl_5_4;
      if ((!dab || 0 >= 4) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[178]; }
    { const long long ij = ij_0_4, kl = kl_5_5;
      if ((!dab || 0 >= 4) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[179]; }
    { const long long ij = ij_0_5, kl = kl_0_0;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[180]; }
    { const long long ij = ij_0_5, kl = kl_0_1;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[181]; }
    { const long long ij = ij_0_5, kl = kl_0_2;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[182]; }
    { const long long ij = ij_0_5, kl = kl_0_3;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[183]; }
    { const long long ij = ij_0_5, kl = kl_0_4;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[184]; }
    { const long long ij = ij_0_5, kl = kl_0_5;
      if ((!dab || 0 >= 5) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[185]; }
    { const long long ij = ij_0_5, kl = kl_1_0;
      if ((!dab || 0 >= 5) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[186]; }
    { const long long ij = ij_0_5, kl = kl_1_1;
      if ((!dab || 0 >= 5) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[187]; }
    { const long long ij = ij_0_5, kl = kl_1_2;
      if ((!dab || 0 >= 5) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[188]; }
    { const long long ij = ij_0_5, kl = kl_1_3;
      if ((!dab || 0 >= 5) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[189]; }
    { const long long ij = ij_0_5, kl = kl_1_4;
      if ((!dab || 0 >= 5) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[190]; }
    { const long long ij = ij_0_5, kl = kl_1_5;
      if ((!dab || 0 >= 5) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[191]; }
    { const long long ij = ij_0_5, kl = kl_2_0;
      if ((!dab || 0 >= 5) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[192]; }
    { const long long ij = ij_0_5, kl = kl_2_1;
      if ((!dab || 0 >= 5) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[193]; }
    { const long long ij = ij_0_5, kl = kl_2_2;
      if ((!dab || 0 >= 5) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[194]; }
    { const long long ij = ij_0_5, kl = kl_2_3;
      if ((!dab || 0 >= 5) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[195]; }
    { const long long ij = ij_0_5, kl = kl_2_4;
      if ((!dab || 0 >= 5) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[196]; }
    { const long long ij = ij_0_5, kl = kl_2_5;
      if ((!dab || 0 >= 5) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[197]; }
    { const long long ij = ij_0_5, kl = kl_3_0;
      if ((!dab || 0 >= 5) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[198]; }
    { const long long ij = ij_0_5, kl = kl_3_1;
      if ((!dab || 0 >= 5) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[199]; }
    { const long long ij = ij_0_5, kl = kl_3_2;
      if ((!dab || 0 >= 5) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[200]; }
    { const long long ij = ij_0_5, kl = kl_3_3;
      if ((!dab || 0 >= 5) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[201]; }
    { const long long ij = ij_0_5, kl = kl_3_4;
      if ((!dab || 0 >= 5) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[202]; }
    { const long long ij = ij_0_5, kl = kl_3_5;
      if ((!dab || 0 >= 5) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[203]; }
    { const long long ij = ij_0_5, kl = kl_4_0;
      if ((!dab || 0 >= 5) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[204]; }
    { const long long ij = ij_0_5, kl = kl_4_1;
      if ((!dab || 0 >= 5) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[205]; }
    { const long long ij = ij_0_5, kl = kl_4_2;
      if ((!dab || 0 >= 5) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[206]; }
    { const long long ij = ij_0_5, kl = kl_4_3;
      if ((!dab || 0 >= 5) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[207]; }
    { const long long ij = ij_0_5, kl = kl_4_4;
      if ((!dab || 0 >= 5) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[208]; }
    { const long long ij = ij_0_5, kl = kl_4_5;
      if ((!dab || 0 >= 5) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[209]; }
    { const long long ij = ij_0_5, kl = kl_5_0;
      if ((!dab || 0 >= 5) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[210]; }
    { const long long ij = ij_0_5, kl = kl_5_1;
      if ((!dab || 0 >= 5) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[211]; }
    { const long long ij = ij_0_5, kl = kl_5_2;
      if ((!dab || 0 >= 5) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[212]; }
    { const long long ij = ij_0_5, kl = kl_5_3;
      if ((!dab || 0 >= 5) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[213]; }
    { const long long ij = ij_0_5, kl = kl_5_4;
      if ((!dab || 0 >= 5) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[214]; }
    { const long long ij = ij_0_5, kl = kl_5_5;
      if ((!dab || 0 >= 5) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[215]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[216]; }
    { const long long ij = ij_1_0, kl = kl_0_1;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[217]; }
    { const long long ij = ij_1_0, kl = kl_0_2;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[218]; }
    { const long long ij = ij_1_0, kl = kl_0_3;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[219]; }
    { const long long ij = ij_1_0, kl = kl_0_4;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[220]; }
    { const long long ij = ij_1_0, kl = kl_0_5;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[221]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[222]; }
    { const long long ij = ij_1_0, kl = kl_1_1;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[223]; }
    { const long long ij = ij_1_0, kl = kl_1_2;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[224]; }
    { const long long ij = ij_1_0, kl = kl_1_3;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[225]; }
    { const long long ij = ij_1_0, kl = kl_1_4;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[226]; }
    { const long long ij = ij_1_0, kl = kl_1_5;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[227]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[228]; }
    { const long long ij = ij_1_0, kl = kl_2_1;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[229]; }
    { const long long ij = ij_1_0, kl = kl_2_2;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[230]; }
    { const long long ij = ij_1_0, kl = kl_2_3;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[231]; }
    { const long long ij = ij_1_0, kl = kl_2_4;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[232]; }
    { const long long ij = ij_1_0, kl = kl_2_5;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[233]; }
    { const long long ij = ij_1_0, kl = kl_3_0;
      if ((!dab || 1 >= 0) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[234]; }
    { const long long ij = ij_1_0, kl = kl_3_1;
      if ((!dab || 1 >= 0) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[235]; }
    { const long long ij = ij_1_0, kl = kl_3_2;
      if ((!dab || 1 >= 0) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[236]; }
    { const long long ij = ij_1_0, kl = kl_3_3;
      if ((!dab || 1 >= 0) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[237]; }
    { const long long ij = ij_1_0, kl = kl_3_4;
      if ((!dab || 1 >= 0) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[238]; }
    { const long long ij = ij_1_0, kl = kl_3_5;
      if ((!dab || 1 >= 0) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[239]; }
    { const long long ij = ij_1_0, kl = kl_4_0;
      if ((!dab || 1 >= 0) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[240]; }
    { const long long ij = ij_1_0, kl = kl_4_1;
      if ((!dab || 1 >= 0) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[241]; }
    { const long long ij = ij_1_0, kl = kl_4_2;
      if ((!dab || 1 >= 0) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[242]; }
    { const long long ij = ij_1_0, kl = kl_4_3;
      if ((!dab || 1 >= 0) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[243]; }
    { const long long ij = ij_1_0, kl = kl_4_4;
      if ((!dab || 1 >= 0) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[244]; }
    { const long long ij = ij_1_0, kl = kl_4_5;
      if ((!dab || 1 >= 0) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[245]; }
    { const long long ij = ij_1_0, kl = kl_5_0;
      if ((!dab || 1 >= 0) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[246]; }
    { const long long ij = ij_1_0, kl = kl_5_1;
      if ((!dab || 1 >= 0) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[247]; }
    { const long long ij = ij_1_0, kl = kl_5_2;
      if ((!dab || 1 >= 0) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[248]; }
    { const long long ij = ij_1_0, kl = kl_5_3;
      if ((!dab || 1 >= 0) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[249]; }
    { const long long ij = ij_1_0, kl = kl_5_4;
      if ((!dab || 1 >= 0) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[250]; }
    { const long long ij = ij_1_0, kl = kl_5_5;
      if ((!dab || 1 >= 0) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[251]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[252]; }
    { const long long ij = ij_1_1, kl = kl_0_1;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[253]; }
    { const long long ij = ij_1_1, kl = kl_0_2;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[254]; }
    { const long long ij = ij_1_1, kl = kl_0_3;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[255]; }
    { const long long ij = ij_1_1, kl = kl_0_4;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[256]; }
    { const long long ij = ij_1_1, kl = kl_0_5;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[257]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[258]; }
    { const long long ij = ij_1_1, kl = kl_1_1;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[259]; }
    { const long long ij = ij_1_1, kl = kl_1_2;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[260]; }
    { const long long ij = ij_1_1, kl = kl_1_3;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[261]; }
    { const long long ij = ij_1_1, kl = kl_1_4;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[262]; }
    { const long long ij = ij_1_1, kl = kl_1_5;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[263]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[264]; }
    { const long long ij = ij_1_1, kl = kl_2_1;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[265]; }
    { const long long ij = ij_1_1, kl = kl_2_2;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[266]; }
    { const long long ij = ij_1_1, kl = kl_2_3;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[267]; }
    { const long long ij = ij_1_1, kl = kl_2_4;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[268]; }
    { const long long ij = ij_1_1, kl = kl_2_5;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[269]; }
    { const long long ij = ij_1_1, kl = kl_3_0;
      if ((!dab || 1 >= 1) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[270]; }
    { const long long ij = ij_1_1, kl = kl_3_1;
      if ((!dab || 1 >= 1) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[271]; }
    { const long long ij = ij_1_1, kl = kl_3_2;
      if ((!dab || 1 >= 1) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[272]; }
    { const long long ij = ij_1_1, kl = kl_3_3;
      if ((!dab || 1 >= 1) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[273]; }
    { const long long ij = ij_1_1, kl = kl_3_4;
      if ((!dab || 1 >= 1) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[274]; }
    { const long long ij = ij_1_1, kl = kl_3_5;
      if ((!dab || 1 >= 1) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[275]; }
    { const long long ij = ij_1_1, kl = kl_4_0;
      if ((!dab || 1 >= 1) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[276]; }
    { const long long ij = ij_1_1, kl = kl_4_1;
      if ((!dab || 1 >= 1) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[277]; }
    { const long long ij = ij_1_1, kl = kl_4_2;
      if ((!dab || 1 >= 1) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[278]; }
    { const long long ij = ij_1_1, kl = kl_4_3;
      if ((!dab || 1 >= 1) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[279]; }
    { const long long ij = ij_1_1, kl = kl_4_4;
      if ((!dab || 1 >= 1) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[280]; }
    { const long long ij = ij_1_1, kl = kl_4_5;
      if ((!dab || 1 >= 1) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[281]; }
    { const long long ij = ij_1_1, kl = kl_5_0;
      if ((!dab || 1 >= 1) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[282]; }
    { const long long ij = ij_1_1, kl = kl_5_1;
      if ((!dab || 1 >= 1) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[283]; }
    { const long long ij = ij_1_1, kl = kl_5_2;
      if ((!dab || 1 >= 1) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[284]; }
    { const long long ij = ij_1_1, kl = kl_5_3;
      if ((!dab || 1 >= 1) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[285]; }
    { const long long ij = ij_1_1, kl = kl_5_4;
      if ((!dab || 1 >= 1) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[286]; }
    { const long long ij = ij_1_1, kl = kl_5_5;
      if ((!dab || 1 >= 1) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[287]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[288]; }
    { const long long ij = ij_1_2, kl = kl_0_1;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[289]; }
    { const long long ij = ij_1_2, kl = kl_0_2;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[290]; }
    { const long long ij = ij_1_2, kl = kl_0_3;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[291]; }
    { const long long ij = ij_1_2, kl = kl_0_4;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[292]; }
    { const long long ij = ij_1_2, kl = kl_0_5;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[293]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[294]; }
    { const long long ij = ij_1_2, kl = kl_1_1;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[295]; }
    { const long long ij = ij_1_2, kl = kl_1_2;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[296]; }
    { const long long ij = ij_1_2, kl = kl_1_3;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[297]; }
    { const long long ij = ij_1_2, kl = kl_1_4;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[298]; }
    { const long long ij = ij_1_2, kl = kl_1_5;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[299]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[300]; }
    { const long long ij = ij_1_2, kl = kl_2_1;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[301]; }
    { const long long ij = ij_1_2, kl = kl_2_2;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[302]; }
    { const long long ij = ij_1_2, kl = kl_2_3;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[303]; }
    { const long long ij = ij_1_2, kl = kl_2_4;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[304]; }
    { const long long ij = ij_1_2, kl = kl_2_5;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[305]; }
    { const long long ij = ij_1_2, kl = kl_3_0;
      if ((!dab || 1 >= 2) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[306]; }
    { const long long ij = ij_1_2, kl = kl_3_1;
      if ((!dab || 1 >= 2) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[307]; }
    { const long long ij = ij_1_2, kl = kl_3_2;
      if ((!dab || 1 >= 2) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[308]; }
    { const long long ij = ij_1_2, kl = kl_3_3;
      if ((!dab || 1 >= 2) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[309]; }
    { const long long ij = ij_1_2, kl = kl_3_4;
      if ((!dab || 1 >= 2) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[310]; }
    { const long long ij = ij_1_2, kl = kl_3_5;
      if ((!dab || 1 >= 2) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[311]; }
    { const long long ij = ij_1_2, kl = kl_4_0;
      if ((!dab || 1 >= 2) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[312]; }
    { const long long ij = ij_1_2, kl = kl_4_1;
      if ((!dab || 1 >= 2) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[313]; }
    { const long long ij = ij_1_2, kl = kl_4_2;
      if ((!dab || 1 >= 2) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[314]; }
    { const long long ij = ij_1_2, kl = kl_4_3;
      if ((!dab || 1 >= 2) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[315]; }
    { const long long ij = ij_1_2, kl = kl_4_4;
      if ((!dab || 1 >= 2) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[316]; }
    { const long long ij = ij_1_2, kl = kl_4_5;
      if ((!dab || 1 >= 2) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[317]; }
    { const long long ij = ij_1_2, kl = kl_5_0;
      if ((!dab || 1 >= 2) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[318]; }
    { const long long ij = ij_1_2, kl = kl_5_1;
      if ((!dab || 1 >= 2) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[319]; }
    { const long long ij = ij_1_2, kl = kl_5_2;
      if ((!dab || 1 >= 2) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[320]; }
    { const long long ij = ij_1_2, kl = kl_5_3;
      if ((!dab || 1 >= 2) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[321]; }
    { const long long ij = ij_1_2, kl = kl_5_4;
      if ((!dab || 1 >= 2) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[322]; }
    { const long long ij = ij_1_2, kl = kl_5_5;
      if ((!dab || 1 >= 2) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[323]; }
    { const long long ij = ij_1_3, kl = kl_0_0;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[324]; }
    { const long long ij = ij_1_3, kl = kl_0_1;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[325]; }
    { const long long ij = ij_1_3, kl = kl_0_2;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[326]; }
    { const long long ij = ij_1_3, kl = kl_0_3;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[327]; }
    { const long long ij = ij_1_3, kl = kl_0_4;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[328]; }
    { const long long ij = ij_1_3, kl = kl_0_5;
      if ((!dab || 1 >= 3) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[329]; }
    { const long long ij = ij_1_3, kl = kl_1_0;
      if ((!dab || 1 >= 3) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[330]; }
    { const long long ij = ij_1_3, kl = kl_1_1;
      if ((!dab || 1 >= 3) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[331]; }
    { const long long ij = ij_1_3, kl = kl_1_2;
      if ((!dab || 1 >= 3) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[332]; }
    { const long long ij = ij_1_3, kl = kl_1_3;
      if ((!dab || 1 >= 3) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[333]; }
    { const long long ij = ij_1_3, kl = kl_1_4;
      if ((!dab || 1 >= 3) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[334]; }
    { const long long ij = ij_1_3, kl = kl_1_5;
      if ((!dab || 1 >= 3) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[335]; }
    { const long long ij = ij_1_3, kl = kl_2_0;
      if ((!dab || 1 >= 3) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[336]; }
    { const long long ij = ij_1_3, kl = kl_2_1;
      if ((!dab || 1 >= 3) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[337]; }
    { const long long ij = ij_1_3, kl = kl_2_2;
      if ((!dab || 1 >= 3) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[338]; }
    { const long long ij = ij_1_3, kl = kl_2_3;
      if ((!dab || 1 >= 3) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[339]; }
    { const long long ij = ij_1_3, kl = kl_2_4;
      if ((!dab || 1 >= 3) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[340]; }
    { const long long ij = ij_1_3, kl = kl_2_5;
      if ((!dab || 1 >= 3) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[341]; }
    { const long long ij = ij_1_3, kl = kl_3_0;
      if ((!dab || 1 >= 3) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[342]; }
    { const long long ij = ij_1_3, kl = kl_3_1;
      if ((!dab || 1 >= 3) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[343]; }
    { const long long ij = ij_1_3, kl = kl_3_2;
      if ((!dab || 1 >= 3) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[344]; }
    { const long long ij = ij_1_3, kl = kl_3_3;
      if ((!dab || 1 >= 3) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[345]; }
    { const long long ij = ij_1_3, kl = kl_3_4;
      if ((!dab || 1 >= 3) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[346]; }
    { const long long ij = ij_1_3, kl = kl_3_5;
      if ((!dab || 1 >= 3) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[347]; }
    { const long long ij = ij_1_3, kl = kl_4_0;
      if ((!dab || 1 >= 3) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[348]; }
    { const long long ij = ij_1_3, kl = kl_4_1;
      if ((!dab || 1 >= 3) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[349]; }
    { const long long ij = ij_1_3, kl = kl_4_2;
      if ((!dab || 1 >= 3) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[350]; }
    { const long long ij = ij_1_3, kl = kl_4_3;
      if ((!dab || 1 >= 3) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[351]; }
    { const long long ij = ij_1_3, kl = kl_4_4;
      if ((!dab || 1 >= 3) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[352]; }
    { const long long ij = ij_1_3, kl = kl_4_5;
      if ((!dab || 1 >= 3) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[353]; }
    { const long long ij = ij_1_3, kl = kl_5_0;
      if ((!dab || 1 >= 3) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[354]; }
    { const long long ij = ij_1_3, kl = kl_5_1;
      if ((!dab || 1 >= 3) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[355]; }
    { const long long ij = ij_1_3, kl = kl_5_2;
      if ((!dab || 1 >= 3) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[356]; }
    { const long long ij = ij_1_3, kl = kl_5_3;
      if ((!dab || 1 >= 3) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[357]; }
    { const long long ij = ij_1_3, kl = kl_5_4;
      if ((!dab || 1 >= 3) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[358]; }
    { const long long ij = ij_1_3, kl = kl_5_5;
      if ((!dab || 1 >= 3) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[359]; }
    { const long long ij = ij_1_4, kl = kl_0_0;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[360]; }
    { const long long ij = ij_1_4, kl = kl_0_1;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[361]; }
    { const long long ij = ij_1_4, kl = kl_0_2;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[362]; }
    { const long long ij = ij_1_4, kl = kl_0_3;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[363]; }
    { const long long ij = ij_1_4, kl = kl_0_4;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[364]; }
    { const long long ij = ij_1_4, kl = kl_0_5;
      if ((!dab || 1 >= 4) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[365]; }
    { const long long ij = ij_1_4, kl = kl_1_0;
      if ((!dab || 1 >= 4) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[366]; }
    { const long long ij = ij_1_4, kl = kl_1_1;
      if ((!dab || 1 >= 4) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[367]; }
    { const long long ij = ij_1_4, kl = kl_1_2;
      if ((!dab || 1 >= 4) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[368]; }
    { const long long ij = ij_1_4, kl = kl_1_3;
      if ((!dab || 1 >= 4) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[369]; }
    { const long long ij = ij_1_4, kl = kl_1_4;
      if ((!dab || 1 >= 4) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[370]; }
    { const long long ij = ij_1_4, kl = kl_1_5;
      if ((!dab || 1 >= 4) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[371]; }
    { const long long ij = ij_1_4, kl = kl_2_0;
      if ((!dab || 1 >= 4) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[372]; }
    { const long long ij = ij_1_4, kl = kl_2_1;
      if ((!dab || 1 >= 4) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[373]; }
    { const long long ij = ij_1_4, kl = kl_2_2;
      if ((!dab || 1 >= 4) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[374]; }
    { const long long ij = ij_1_4, kl = kl_2_3;
      if ((!dab || 1 >= 4) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[375]; }
    { const long long ij = ij_1_4, kl = kl_2_4;
      if ((!dab || 1 >= 4) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[376]; }
    { const long long ij = ij_1_4, kl = kl_2_5;
      if ((!dab || 1 >= 4) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[377]; }
    { const long long ij = ij_1_4, kl = kl_3_0;
      if ((!dab || 1 >= 4) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[378]; }
    { const long long ij = ij_1_4, kl = kl_3_1;
      if ((!dab || 1 >= 4) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[379]; }
    { const long long ij = ij_1_4, kl = kl_3_2;
      if ((!dab || 1 >= 4) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[380]; }
    { const long long ij = ij_1_4, kl = kl_3_3;
      if ((!dab || 1 >= 4) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[381]; }
    { const long long ij = ij_1_4, kl = kl_3_4;
      if ((!dab || 1 >= 4) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[382]; }
    { const long long ij = ij_1_4, kl = kl_3_5;
      if ((!dab || 1 >= 4) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[383]; }
    { const long long ij = ij_1_4, kl = kl_4_0;
      if ((!dab || 1 >= 4) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[384]; }
    { const long long ij = ij_1_4, kl = kl_4_1;
      if ((!dab || 1 >= 4) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[385]; }
    { const long long ij = ij_1_4, kl = kl_4_2;
      if ((!dab || 1 >= 4) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[386]; }
    { const long long ij = ij_1_4, kl = kl_4_3;
      if ((!dab || 1 >= 4) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[387]; }
    { const long long ij = ij_1_4, kl = kl_4_4;
      if ((!dab || 1 >= 4) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[388]; }
    { const long long ij = ij_1_4, kl = kl_4_5;
      if ((!dab || 1 >= 4) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[389]; }
    { const long long ij = ij_1_4, kl = kl_5_0;
      if ((!dab || 1 >= 4) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[390]; }
    { const long long ij = ij_1_4, kl = kl_5_1;
      if ((!dab || 1 >= 4) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[391]; }
    { const long long ij = ij_1_4, kl = kl_5_2;
      if ((!dab || 1 >= 4) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[392]; }
    { const long long ij = ij_1_4, kl = kl_5_3;
      if ((!dab || 1 >= 4) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[393]; }
    { const long long ij = ij_1_4, kl = kl_5_4;
      if ((!dab || 1 >= 4) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[394]; }
    { const long long ij = ij_1_4, kl = kl_5_5;
      if ((!dab || 1 >= 4) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[395]; }
    { const long long ij = ij_1_5, kl = kl_0_0;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[396]; }
    { const long long ij = ij_1_5, kl = kl_0_1;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[397]; }
    { const long long ij = ij_1_5, kl = kl_0_2;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[398]; }
    { const long long ij = ij_1_5, kl = kl_0_3;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[399]; }
    { const long long ij = ij_1_5, kl = kl_0_4;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[400]; }
    { const long long ij = ij_1_5, kl = kl_0_5;
      if ((!dab || 1 >= 5) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[401]; }
    { const long long ij = ij_1_5, kl = kl_1_0;
      if ((!dab || 1 >= 5) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[402]; }
    { const long long ij = ij_1_5, kl = kl_1_1;
      if ((!dab || 1 >= 5) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[403]; }
    { const long long ij = ij_1_5, kl = kl_1_2;
      if ((!dab || 1 >= 5) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[404]; }
    { const long long ij = ij_1_5, kl = kl_1_3;
      if ((!dab || 1 >= 5) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[405]; }
    { const long long ij = ij_1_5, kl = kl_1_4;
      if ((!dab || 1 >= 5) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[406]; }
    { const long long ij = ij_1_5, kl = kl_1_5;
      if ((!dab || 1 >= 5) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[407]; }
    { const long long ij = ij_1_5, kl = kl_2_0;
      if ((!dab || 1 >= 5) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[408]; }
    { const long long ij = ij_1_5, kl = kl_2_1;
      if ((!dab || 1 >= 5) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[409]; }
    { const long long ij = ij_1_5, kl = kl_2_2;
      if ((!dab || 1 >= 5) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[410]; }
    { const long long ij = ij_1_5, kl = kl_2_3;
      if ((!dab || 1 >= 5) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[411]; }
    { const long long ij = ij_1_5, kl = kl_2_4;
      if ((!dab || 1 >= 5) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[412]; }
    { const long long ij = ij_1_5, kl = kl_2_5;
      if ((!dab || 1 >= 5) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[413]; }
    { const long long ij = ij_1_5, kl = kl_3_0;
      if ((!dab || 1 >= 5) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[414]; }
    { const long long ij = ij_1_5, kl = kl_3_1;
      if ((!dab || 1 >= 5) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[415]; }
    { const long long ij = ij_1_5, kl = kl_3_2;
      if ((!dab || 1 >= 5) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[416]; }
    { const long long ij = ij_1_5, kl = kl_3_3;
      if ((!dab || 1 >= 5) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[417]; }
    { const long long ij = ij_1_5, kl = kl_3_4;
      if ((!dab || 1 >= 5) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[418]; }
    { const long long ij = ij_1_5, kl = kl_3_5;
      if ((!dab || 1 >= 5) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[419]; }
    { const long long ij = ij_1_5, kl = kl_4_0;
      if ((!dab || 1 >= 5) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[420]; }
    { const long long ij = ij_1_5, kl = kl_4_1;
      if ((!dab || 1 >= 5) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[421]; }
    { const long long ij = ij_1_5, kl = kl_4_2;
      if ((!dab || 1 >= 5) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[422]; }
    { const long long ij = ij_1_5, kl = kl_4_3;
      if ((!dab || 1 >= 5) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[423]; }
    { const long long ij = ij_1_5, kl = kl_4_4;
      if ((!dab || 1 >= 5) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[424]; }
    { const long long ij = ij_1_5, kl = kl_4_5;
      if ((!dab || 1 >= 5) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[425]; }
    { const long long ij = ij_1_5, kl = kl_5_0;
      if ((!dab || 1 >= 5) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[426]; }
    { const long long ij = ij_1_5, kl = kl_5_1;
      if ((!dab || 1 >= 5) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[427]; }
    { const long long ij = ij_1_5, kl = kl_5_2;
      if ((!dab || 1 >= 5) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[428]; }
    { const long long ij = ij_1_5, kl = kl_5_3;
      if ((!dab || 1 >= 5) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[429]; }
    { const long long ij = ij_1_5, kl = kl_5_4;
      if ((!dab || 1 >= 5) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[430]; }
    { const long long ij = ij_1_5, kl = kl_5_5;
      if ((!dab || 1 >= 5) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[431]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[432]; }
    { const long long ij = ij_2_0, kl = kl_0_1;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[433]; }
    { const long long ij = ij_2_0, kl = kl_0_2;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[434]; }
    { const long long ij = ij_2_0, kl = kl_0_3;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[435]; }
    { const long long ij = ij_2_0, kl = kl_0_4;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[436]; }
    { const long long ij = ij_2_0, kl = kl_0_5;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[437]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[438]; }
    { const long long ij = ij_2_0, kl = kl_1_1;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[439]; }
    { const long long ij = ij_2_0, kl = kl_1_2;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[440]; }
    { const long long ij = ij_2_0, kl = kl_1_3;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[441]; }
    { const long long ij = ij_2_0, kl = kl_1_4;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[442]; }
    { const long long ij = ij_2_0, kl = kl_1_5;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[443]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[444]; }
    { const long long ij = ij_2_0, kl = kl_2_1;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[445]; }
    { const long long ij = ij_2_0, kl = kl_2_2;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[446]; }
    { const long long ij = ij_2_0, kl = kl_2_3;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[447]; }
    { const long long ij = ij_2_0, kl = kl_2_4;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[448]; }
    { const long long ij = ij_2_0, kl = kl_2_5;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[449]; }
    { const long long ij = ij_2_0, kl = kl_3_0;
      if ((!dab || 2 >= 0) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[450]; }
    { const long long ij = ij_2_0, kl = kl_3_1;
      if ((!dab || 2 >= 0) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[451]; }
    { const long long ij = ij_2_0, kl = kl_3_2;
      if ((!dab || 2 >= 0) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[452]; }
    { const long long ij = ij_2_0, kl = kl_3_3;
      if ((!dab || 2 >= 0) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[453]; }
    { const long long ij = ij_2_0, kl = kl_3_4;
      if ((!dab || 2 >= 0) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[454]; }
    { const long long ij = ij_2_0, kl = kl_3_5;
      if ((!dab || 2 >= 0) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[455]; }
    { const long long ij = ij_2_0, kl = kl_4_0;
      if ((!dab || 2 >= 0) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[456]; }
    { const long long ij = ij_2_0, kl = kl_4_1;
      if ((!dab || 2 >= 0) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[457]; }
    { const long long ij = ij_2_0, kl = kl_4_2;
      if ((!dab || 2 >= 0) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[458]; }
    { const long long ij = ij_2_0, kl = kl_4_3;
      if ((!dab || 2 >= 0) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[459]; }
    { const long long ij = ij_2_0, kl = kl_4_4;
      if ((!dab || 2 >= 0) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[460]; }
    { const long long ij = ij_2_0, kl = kl_4_5;
      if ((!dab || 2 >= 0) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[461]; }
    { const long long ij = ij_2_0, kl = kl_5_0;
      if ((!dab || 2 >= 0) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[462]; }
    { const long long ij = ij_2_0, kl = kl_5_1;
      if ((!dab || 2 >= 0) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[463]; }
    { const long long ij = ij_2_0, kl = kl_5_2;
      if ((!dab || 2 >= 0) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[464]; }
    { const long long ij = ij_2_0, kl = kl_5_3;
      if ((!dab || 2 >= 0) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[465]; }
    { const long long ij = ij_2_0, kl = kl_5_4;
      if ((!dab || 2 >= 0) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[466]; }
    { const long long ij = ij_2_0, kl = kl_5_5;
      if ((!dab || 2 >= 0) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[467]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[468]; }
    { const long long ij = ij_2_1, kl = kl_0_1;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[469]; }
    { const long long ij = ij_2_1, kl = kl_0_2;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[470]; }
    { const long long ij = ij_2_1, kl = kl_0_3;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[471]; }
    { const long long ij = ij_2_1, kl = kl_0_4;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[472]; }
    { const long long ij = ij_2_1, kl = kl_0_5;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[473]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[474]; }
    { const long long ij = ij_2_1, kl = kl_1_1;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[475]; }
    { const long long ij = ij_2_1, kl = kl_1_2;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[476]; }
    { const long long ij = ij_2_1, kl = kl_1_3;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[477]; }
    { const long long ij = ij_2_1, kl = kl_1_4;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[478]; }
    { const long long ij = ij_2_1, kl = kl_1_5;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[479]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[480]; }
    { const long long ij = ij_2_1, kl = kl_2_1;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[481]; }
    { const long long ij = ij_2_1, kl = kl_2_2;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[482]; }
    { const long long ij = ij_2_1, kl = kl_2_3;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[483]; }
    { const long long ij = ij_2_1, kl = kl_2_4;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[484]; }
    { const long long ij = ij_2_1, kl = kl_2_5;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[485]; }
    { const long long ij = ij_2_1, kl = kl_3_0;
      if ((!dab || 2 >= 1) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[486]; }
    { const long long ij = ij_2_1, kl = kl_3_1;
      if ((!dab || 2 >= 1) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[487]; }
    { const long long ij = ij_2_1, kl = kl_3_2;
      if ((!dab || 2 >= 1) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[488]; }
    { const long long ij = ij_2_1, kl = kl_3_3;
      if ((!dab || 2 >= 1) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[489]; }
    { const long long ij = ij_2_1, kl = kl_3_4;
      if ((!dab || 2 >= 1) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[490]; }
    { const long long ij = ij_2_1, kl = kl_3_5;
      if ((!dab || 2 >= 1) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[491]; }
    { const long long ij = ij_2_1, kl = kl_4_0;
      if ((!dab || 2 >= 1) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[492]; }
    { const long long ij = ij_2_1, kl = kl_4_1;
      if ((!dab || 2 >= 1) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[493]; }
    { const long long ij = ij_2_1, kl = kl_4_2;
      if ((!dab || 2 >= 1) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[494]; }
    { const long long ij = ij_2_1, kl = kl_4_3;
      if ((!dab || 2 >= 1) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[495]; }
    { const long long ij = ij_2_1, kl = kl_4_4;
      if ((!dab || 2 >= 1) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[496]; }
    { const long long ij = ij_2_1, kl = kl_4_5;
      if ((!dab || 2 >= 1) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[497]; }
    { const long long ij = ij_2_1, kl = kl_5_0;
      if ((!dab || 2 >= 1) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[498]; }
    { const long long ij = ij_2_1, kl = kl_5_1;
      if ((!dab || 2 >= 1) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[499]; }
    { const long long ij = ij_2_1, kl = kl_5_2;
      if ((!dab || 2 >= 1) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[500]; }
    { const long long ij = ij_2_1, kl = kl_5_3;
      if ((!dab || 2 >= 1) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[501]; }
    { const long long ij = ij_2_1, kl = kl_5_4;
      if ((!dab || 2 >= 1) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[502]; }
    { const long long ij = ij_2_1, kl = kl_5_5;
      if ((!dab || 2 >= 1) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[503]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[504]; }
    { const long long ij = ij_2_2, kl = kl_0_1;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[505]; }
    { const long long ij = ij_2_2, kl = kl_0_2;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[506]; }
    { const long long ij = ij_2_2, kl = kl_0_3;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[507]; }
    { const long long ij = ij_2_2, kl = kl_0_4;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[508]; }
    { const long long ij = ij_2_2, kl = kl_0_5;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[509]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[510]; }
    { const long long ij = ij_2_2, kl = kl_1_1;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[511]; }
    { const long long ij = ij_2_2, kl = kl_1_2;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[512]; }
    { const long long ij = ij_2_2, kl = kl_1_3;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[513]; }
    { const long long ij = ij_2_2, kl = kl_1_4;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[514]; }
    { const long long ij = ij_2_2, kl = kl_1_5;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[515]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[516]; }
    { const long long ij = ij_2_2, kl = kl_2_1;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[517]; }
    { const long long ij = ij_2_2, kl = kl_2_2;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[518]; }
    { const long long ij = ij_2_2, kl = kl_2_3;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[519]; }
    { const long long ij = ij_2_2, kl = kl_2_4;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[520]; }
    { const long long ij = ij_2_2, kl = kl_2_5;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[521]; }
    { const long long ij = ij_2_2, kl = kl_3_0;
      if ((!dab || 2 >= 2) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[522]; }
    { const long long ij = ij_2_2, kl = kl_3_1;
      if ((!dab || 2 >= 2) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[523]; }
    { const long long ij = ij_2_2, kl = kl_3_2;
      if ((!dab || 2 >= 2) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[524]; }
    { const long long ij = ij_2_2, kl = kl_3_3;
      if ((!dab || 2 >= 2) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[525]; }
    { const long long ij = ij_2_2, kl = kl_3_4;
      if ((!dab || 2 >= 2) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[526]; }
    { const long long ij = ij_2_2, kl = kl_3_5;
      if ((!dab || 2 >= 2) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[527]; }
    { const long long ij = ij_2_2, kl = kl_4_0;
      if ((!dab || 2 >= 2) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[528]; }
    { const long long ij = ij_2_2, kl = kl_4_1;
      if ((!dab || 2 >= 2) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[529]; }
    { const long long ij = ij_2_2, kl = kl_4_2;
      if ((!dab || 2 >= 2) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[530]; }
    { const long long ij = ij_2_2, kl = kl_4_3;
      if ((!dab || 2 >= 2) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[531]; }
    { const long long ij = ij_2_2, kl = kl_4_4;
      if ((!dab || 2 >= 2) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[532]; }
    { const long long ij = ij_2_2, kl = kl_4_5;
      if ((!dab || 2 >= 2) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[533]; }
    { const long long ij = ij_2_2, kl = kl_5_0;
      if ((!dab || 2 >= 2) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[534]; }
    { const long long ij = ij_2_2, kl = kl_5_1;
      if ((!dab || 2 >= 2) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[535]; }
    { const long long ij = ij_2_2, kl = kl_5_2;
      if ((!dab || 2 >= 2) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[536]; }
    { const long long ij = ij_2_2, kl = kl_5_3;
      if ((!dab || 2 >= 2) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[537]; }
    { const long long ij = ij_2_2, kl = kl_5_4;
      if ((!dab || 2 >= 2) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[538]; }
    { const long long ij = ij_2_2, kl = kl_5_5;
      if ((!dab || 2 >= 2) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[539]; }
    { const long long ij = ij_2_3, kl = kl_0_0;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[540]; }
    { const long long ij = ij_2_3, kl = kl_0_1;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[541]; }
    { const long long ij = ij_2_3, kl = kl_0_2;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[542]; }
    { const long long ij = ij_2_3, kl = kl_0_3;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[543]; }
    { const long long ij = ij_2_3, kl = kl_0_4;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[544]; }
    { const long long ij = ij_2_3, kl = kl_0_5;
      if ((!dab || 2 >= 3) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[545]; }
    { const long long ij = ij_2_3, kl = kl_1_0;
      if ((!dab || 2 >= 3) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[546]; }
    { const long long ij = ij_2_3, kl = kl_1_1;
      if ((!dab || 2 >= 3) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[547]; }
    { const long long ij = ij_2_3, kl = kl_1_2;
      if ((!dab || 2 >= 3) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[548]; }
    { const long long ij = ij_2_3, kl = kl_1_3;
      if ((!dab || 2 >= 3) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[549]; }
    { const long long ij = ij_2_3, kl = kl_1_4;
      if ((!dab || 2 >= 3) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[550]; }
    { const long long ij = ij_2_3, kl = kl_1_5;
      if ((!dab || 2 >= 3) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[551]; }
    { const long long ij = ij_2_3, kl = kl_2_0;
      if ((!dab || 2 >= 3) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[552]; }
    { const long long ij = ij_2_3, kl = kl_2_1;
      if ((!dab || 2 >= 3) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[553]; }
    { const long long ij = ij_2_3, kl = kl_2_2;
      if ((!dab || 2 >= 3) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[554]; }
    { const long long ij = ij_2_3, kl = kl_2_3;
      if ((!dab || 2 >= 3) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[555]; }
    { const long long ij = ij_2_3, kl = kl_2_4;
      if ((!dab || 2 >= 3) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[556]; }
    { const long long ij = ij_2_3, kl = kl_2_5;
      if ((!dab || 2 >= 3) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[557]; }
    { const long long ij = ij_2_3, kl = kl_3_0;
      if ((!dab || 2 >= 3) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[558]; }
    { const long long ij = ij_2_3, kl = kl_3_1;
      if ((!dab || 2 >= 3) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[559]; }
    { const long long ij = ij_2_3, kl = kl_3_2;
      if ((!dab || 2 >= 3) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[560]; }
    { const long long ij = ij_2_3, kl = kl_3_3;
      if ((!dab || 2 >= 3) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[561]; }
    { const long long ij = ij_2_3, kl = kl_3_4;
      if ((!dab || 2 >= 3) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[562]; }
    { const long long ij = ij_2_3, kl = kl_3_5;
      if ((!dab || 2 >= 3) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[563]; }
    { const long long ij = ij_2_3, kl = kl_4_0;
      if ((!dab || 2 >= 3) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[564]; }
    { const long long ij = ij_2_3, kl = kl_4_1;
      if ((!dab || 2 >= 3) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[565]; }
    { const long long ij = ij_2_3, kl = kl_4_2;
      if ((!dab || 2 >= 3) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[566]; }
    { const long long ij = ij_2_3, kl = kl_4_3;
      if ((!dab || 2 >= 3) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[567]; }
    { const long long ij = ij_2_3, kl = kl_4_4;
      if ((!dab || 2 >= 3) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[568]; }
    { const long long ij = ij_2_3, kl = kl_4_5;
      if ((!dab || 2 >= 3) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[569]; }
    { const long long ij = ij_2_3, kl = kl_5_0;
      if ((!dab || 2 >= 3) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[570]; }
    { const long long ij = ij_2_3, kl = kl_5_1;
      if ((!dab || 2 >= 3) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[571]; }
    { const long long ij = ij_2_3, kl = kl_5_2;
      if ((!dab || 2 >= 3) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[572]; }
    { const long long ij = ij_2_3, kl = kl_5_3;
      if ((!dab || 2 >= 3) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[573]; }
    { const long long ij = ij_2_3, kl = kl_5_4;
      if ((!dab || 2 >= 3) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[574]; }
    { const long long ij = ij_2_3, kl = kl_5_5;
      if ((!dab || 2 >= 3) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[575]; }
    { const long long ij = ij_2_4, kl = kl_0_0;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[576]; }
    { const long long ij = ij_2_4, kl = kl_0_1;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[577]; }
    { const long long ij = ij_2_4, kl = kl_0_2;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[578]; }
    { const long long ij = ij_2_4, kl = kl_0_3;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[579]; }
    { const long long ij = ij_2_4, kl = kl_0_4;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[580]; }
    { const long long ij = ij_2_4, kl = kl_0_5;
      if ((!dab || 2 >= 4) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[581]; }
    { const long long ij = ij_2_4, kl = kl_1_0;
      if ((!dab || 2 >= 4) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[582]; }
    { const long long ij = ij_2_4, kl = kl_1_1;
      if ((!dab || 2 >= 4) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[583]; }
    { const long long ij = ij_2_4, kl = kl_1_2;
      if ((!dab || 2 >= 4) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[584]; }
    { const long long ij = ij_2_4, kl = kl_1_3;
      if ((!dab || 2 >= 4) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[585]; }
    { const long long ij = ij_2_4, kl = kl_1_4;
      if ((!dab || 2 >= 4) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[586]; }
    { const long long ij = ij_2_4, kl = kl_1_5;
      if ((!dab || 2 >= 4) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[587]; }
    { const long long ij = ij_2_4, kl = kl_2_0;
      if ((!dab || 2 >= 4) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[588]; }
    { const long long ij = ij_2_4, kl = kl_2_1;
      if ((!dab || 2 >= 4) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[589]; }
    { const long long ij = ij_2_4, kl = kl_2_2;
      if ((!dab || 2 >= 4) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[590]; }
    { const long long ij = ij_2_4, kl = kl_2_3;
      if ((!dab || 2 >= 4) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[591]; }
    { const long long ij = ij_2_4, kl = kl_2_4;
      if ((!dab || 2 >= 4) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[592]; }
    { const long long ij = ij_2_4, kl = kl_2_5;
      if ((!dab || 2 >= 4) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[593]; }
    { const long long ij = ij_2_4, kl = kl_3_0;
      if ((!dab || 2 >= 4) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[594]; }
    { const long long ij = ij_2_4, kl = kl_3_1;
      if ((!dab || 2 >= 4) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[595]; }
    { const long long ij = ij_2_4, kl = kl_3_2;
      if ((!dab || 2 >= 4) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[596]; }
    { const long long ij = ij_2_4, kl = kl_3_3;
      if ((!dab || 2 >= 4) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[597]; }
    { const long long ij = ij_2_4, kl = kl_3_4;
      if ((!dab || 2 >= 4) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[598]; }
    { const long long ij = ij_2_4, kl = kl_3_5;
      if ((!dab || 2 >= 4) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[599]; }
    { const long long ij = ij_2_4, kl = kl_4_0;
      if ((!dab || 2 >= 4) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[600]; }
    { const long long ij = ij_2_4, kl = kl_4_1;
      if ((!dab || 2 >= 4) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[601]; }
    { const long long ij = ij_2_4, kl = kl_4_2;
      if ((!dab || 2 >= 4) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[602]; }
    { const long long ij = ij_2_4, kl = kl_4_3;
      if ((!dab || 2 >= 4) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[603]; }
    { const long long ij = ij_2_4, kl = kl_4_4;
      if ((!dab || 2 >= 4) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[604]; }
    { const long long ij = ij_2_4, kl = kl_4_5;
      if ((!dab || 2 >= 4) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[605]; }
    { const long long ij = ij_2_4, kl = kl_5_0;
      if ((!dab || 2 >= 4) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[606]; }
    { const long long ij = ij_2_4, kl = kl_5_1;
      if ((!dab || 2 >= 4) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[607]; }
    { const long long ij = ij_2_4, kl = kl_5_2;
      if ((!dab || 2 >= 4) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[608]; }
    { const long long ij = ij_2_4, kl = kl_5_3;
      if ((!dab || 2 >= 4) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[609]; }
    { const long long ij = ij_2_4, kl = kl_5_4;
      if ((!dab || 2 >= 4) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[610]; }
    { const long long ij = ij_2_4, kl = kl_5_5;
      if ((!dab || 2 >= 4) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[611]; }
    { const long long ij = ij_2_5, kl = kl_0_0;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[612]; }
    { const long long ij = ij_2_5, kl = kl_0_1;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[613]; }
    { const long long ij = ij_2_5, kl = kl_0_2;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[614]; }
    { const long long ij = ij_2_5, kl = kl_0_3;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[615]; }
    { const long long ij = ij_2_5, kl = kl_0_4;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[616]; }
    { const long long ij = ij_2_5, kl = kl_0_5;
      if ((!dab || 2 >= 5) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[617]; }
    { const long long ij = ij_2_5, kl = kl_1_0;
      if ((!dab || 2 >= 5) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[618]; }
    { const long long ij = ij_2_5, kl = kl_1_1;
      if ((!dab || 2 >= 5) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[619]; }
    { const long long ij = ij_2_5, kl = kl_1_2;
      if ((!dab || 2 >= 5) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[620]; }
    { const long long ij = ij_2_5, kl = kl_1_3;
      if ((!dab || 2 >= 5) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[621]; }
    { const long long ij = ij_2_5, kl = kl_1_4;
      if ((!dab || 2 >= 5) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[622]; }
    { const long long ij = ij_2_5, kl = kl_1_5;
      if ((!dab || 2 >= 5) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[623]; }
    { const long long ij = ij_2_5, kl = kl_2_0;
      if ((!dab || 2 >= 5) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[624]; }
    { const long long ij = ij_2_5, kl = kl_2_1;
      if ((!dab || 2 >= 5) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[625]; }
    { const long long ij = ij_2_5, kl = kl_2_2;
      if ((!dab || 2 >= 5) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[626]; }
    { const long long ij = ij_2_5, kl = kl_2_3;
      if ((!dab || 2 >= 5) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[627]; }
    { const long long ij = ij_2_5, kl = kl_2_4;
      if ((!dab || 2 >= 5) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[628]; }
    { const long long ij = ij_2_5, kl = kl_2_5;
      if ((!dab || 2 >= 5) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[629]; }
    { const long long ij = ij_2_5, kl = kl_3_0;
      if ((!dab || 2 >= 5) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[630]; }
    { const long long ij = ij_2_5, kl = kl_3_1;
      if ((!dab || 2 >= 5) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[631]; }
    { const long long ij = ij_2_5, kl = kl_3_2;
      if ((!dab || 2 >= 5) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[632]; }
    { const long long ij = ij_2_5, kl = kl_3_3;
      if ((!dab || 2 >= 5) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[633]; }
    { const long long ij = ij_2_5, kl = kl_3_4;
      if ((!dab || 2 >= 5) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[634]; }
    { const long long ij = ij_2_5, kl = kl_3_5;
      if ((!dab || 2 >= 5) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[635]; }
    { const long long ij = ij_2_5, kl = kl_4_0;
      if ((!dab || 2 >= 5) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[636]; }
    { const long long ij = ij_2_5, kl = kl_4_1;
      if ((!dab || 2 >= 5) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[637]; }
    { const long long ij = ij_2_5, kl = kl_4_2;
      if ((!dab || 2 >= 5) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[638]; }
    { const long long ij = ij_2_5, kl = kl_4_3;
      if ((!dab || 2 >= 5) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[639]; }
    { const long long ij = ij_2_5, kl = kl_4_4;
      if ((!dab || 2 >= 5) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[640]; }
    { const long long ij = ij_2_5, kl = kl_4_5;
      if ((!dab || 2 >= 5) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[641]; }
    { const long long ij = ij_2_5, kl = kl_5_0;
      if ((!dab || 2 >= 5) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[642]; }
    { const long long ij = ij_2_5, kl = kl_5_1;
      if ((!dab || 2 >= 5) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[643]; }
    { const long long ij = ij_2_5, kl = kl_5_2;
      if ((!dab || 2 >= 5) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[644]; }
    { const long long ij = ij_2_5, kl = kl_5_3;
      if ((!dab || 2 >= 5) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[645]; }
    { const long long ij = ij_2_5, kl = kl_5_4;
      if ((!dab || 2 >= 5) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[646]; }
    { const long long ij = ij_2_5, kl = kl_5_5;
      if ((!dab || 2 >= 5) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[647]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[648]; }
    { const long long ij = ij_3_0, kl = kl_0_1;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[649]; }
    { const long long ij = ij_3_0, kl = kl_0_2;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[650]; }
    { const long long ij = ij_3_0, kl = kl_0_3;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[651]; }
    { const long long ij = ij_3_0, kl = kl_0_4;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[652]; }
    { const long long ij = ij_3_0, kl = kl_0_5;
      if ((!dab || 3 >= 0) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[653]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if ((!dab || 3 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[654]; }
    { const long long ij = ij_3_0, kl = kl_1_1;
      if ((!dab || 3 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[655]; }
    { const long long ij = ij_3_0, kl = kl_1_2;
      if ((!dab || 3 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[656]; }
    { const long long ij = ij_3_0, kl = kl_1_3;
      if ((!dab || 3 >= 0) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[657]; }
    { const long long ij = ij_3_0, kl = kl_1_4;
      if ((!dab || 3 >= 0) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[658]; }
    { const long long ij = ij_3_0, kl = kl_1_5;
      if ((!dab || 3 >= 0) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[659]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if ((!dab || 3 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[660]; }
    { const long long ij = ij_3_0, kl = kl_2_1;
      if ((!dab || 3 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[661]; }
    { const long long ij = ij_3_0, kl = kl_2_2;
      if ((!dab || 3 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[662]; }
    { const long long ij = ij_3_0, kl = kl_2_3;
      if ((!dab || 3 >= 0) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[663]; }
    { const long long ij = ij_3_0, kl = kl_2_4;
      if ((!dab || 3 >= 0) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[664]; }
    { const long long ij = ij_3_0, kl = kl_2_5;
      if ((!dab || 3 >= 0) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[665]; }
    { const long long ij = ij_3_0, kl = kl_3_0;
      if ((!dab || 3 >= 0) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[666]; }
    { const long long ij = ij_3_0, kl = kl_3_1;
      if ((!dab || 3 >= 0) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[667]; }
    { const long long ij = ij_3_0, kl = kl_3_2;
      if ((!dab || 3 >= 0) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[668]; }
    { const long long ij = ij_3_0, kl = kl_3_3;
      if ((!dab || 3 >= 0) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[669]; }
    { const long long ij = ij_3_0, kl = kl_3_4;
      if ((!dab || 3 >= 0) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[670]; }
    { const long long ij = ij_3_0, kl = kl_3_5;
      if ((!dab || 3 >= 0) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[671]; }
    { const long long ij = ij_3_0, kl = kl_4_0;
      if ((!dab || 3 >= 0) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[672]; }
    { const long long ij = ij_3_0, kl = kl_4_1;
      if ((!dab || 3 >= 0) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[673]; }
    { const long long ij = ij_3_0, kl = kl_4_2;
      if ((!dab || 3 >= 0) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[674]; }
    { const long long ij = ij_3_0, kl = kl_4_3;
      if ((!dab || 3 >= 0) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[675]; }
    { const long long ij = ij_3_0, kl = kl_4_4;
      if ((!dab || 3 >= 0) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[676]; }
    { const long long ij = ij_3_0, kl = kl_4_5;
      if ((!dab || 3 >= 0) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[677]; }
    { const long long ij = ij_3_0, kl = kl_5_0;
      if ((!dab || 3 >= 0) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[678]; }
    { const long long ij = ij_3_0, kl = kl_5_1;
      if ((!dab || 3 >= 0) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[679]; }
    { const long long ij = ij_3_0, kl = kl_5_2;
      if ((!dab || 3 >= 0) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[680]; }
    { const long long ij = ij_3_0, kl = kl_5_3;
      if ((!dab || 3 >= 0) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[681]; }
    { const long long ij = ij_3_0, kl = kl_5_4;
      if ((!dab || 3 >= 0) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[682]; }
    { const long long ij = ij_3_0, kl = kl_5_5;
      if ((!dab || 3 >= 0) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[683]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[684]; }
    { const long long ij = ij_3_1, kl = kl_0_1;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[685]; }
    { const long long ij = ij_3_1, kl = kl_0_2;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[686]; }
    { const long long ij = ij_3_1, kl = kl_0_3;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[687]; }
    { const long long ij = ij_3_1, kl = kl_0_4;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[688]; }
    { const long long ij = ij_3_1, kl = kl_0_5;
      if ((!dab || 3 >= 1) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[689]; }
    { const long long ij = ij_3_1, kl = kl_1_0;
      if ((!dab || 3 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[690]; }
    { const long long ij = ij_3_1, kl = kl_1_1;
      if ((!dab || 3 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[691]; }
    { const long long ij = ij_3_1, kl = kl_1_2;
      if ((!dab || 3 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[692]; }
    { const long long ij = ij_3_1, kl = kl_1_3;
      if ((!dab || 3 >= 1) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[693]; }
    { const long long ij = ij_3_1, kl = kl_1_4;
      if ((!dab || 3 >= 1) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[694]; }
    { const long long ij = ij_3_1, kl = kl_1_5;
      if ((!dab || 3 >= 1) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[695]; }
    { const long long ij = ij_3_1, kl = kl_2_0;
      if ((!dab || 3 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[696]; }
    { const long long ij = ij_3_1, kl = kl_2_1;
      if ((!dab || 3 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[697]; }
    { const long long ij = ij_3_1, kl = kl_2_2;
      if ((!dab || 3 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[698]; }
    { const long long ij = ij_3_1, kl = kl_2_3;
      if ((!dab || 3 >= 1) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[699]; }
    { const long long ij = ij_3_1, kl = kl_2_4;
      if ((!dab || 3 >= 1) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[700]; }
    { const long long ij = ij_3_1, kl = kl_2_5;
      if ((!dab || 3 >= 1) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[701]; }
    { const long long ij = ij_3_1, kl = kl_3_0;
      if ((!dab || 3 >= 1) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[702]; }
    { const long long ij = ij_3_1, kl = kl_3_1;
      if ((!dab || 3 >= 1) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[703]; }
    { const long long ij = ij_3_1, kl = kl_3_2;
      if ((!dab || 3 >= 1) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[704]; }
    { const long long ij = ij_3_1, kl = kl_3_3;
      if ((!dab || 3 >= 1) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[705]; }
    { const long long ij = ij_3_1, kl = kl_3_4;
      if ((!dab || 3 >= 1) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[706]; }
    { const long long ij = ij_3_1, kl = kl_3_5;
      if ((!dab || 3 >= 1) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[707]; }
    { const long long ij = ij_3_1, kl = kl_4_0;
      if ((!dab || 3 >= 1) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[708]; }
    { const long long ij = ij_3_1, kl = kl_4_1;
      if ((!dab || 3 >= 1) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[709]; }
    { const long long ij = ij_3_1, kl = kl_4_2;
      if ((!dab || 3 >= 1) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[710]; }
    { const long long ij = ij_3_1, kl = kl_4_3;
      if ((!dab || 3 >= 1) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[711]; }
    { const long long ij = ij_3_1, kl = kl_4_4;
      if ((!dab || 3 >= 1) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[712]; }
    { const long long ij = ij_3_1, kl = kl_4_5;
      if ((!dab || 3 >= 1) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[713]; }
    { const long long ij = ij_3_1, kl = kl_5_0;
      if ((!dab || 3 >= 1) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[714]; }
    { const long long ij = ij_3_1, kl = kl_5_1;
      if ((!dab || 3 >= 1) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[715]; }
    { const long long ij = ij_3_1, kl = kl_5_2;
      if ((!dab || 3 >= 1) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[716]; }
    { const long long ij = ij_3_1, kl = kl_5_3;
      if ((!dab || 3 >= 1) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[717]; }
    { const long long ij = ij_3_1, kl = kl_5_4;
      if ((!dab || 3 >= 1) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[718]; }
    { const long long ij = ij_3_1, kl = kl_5_5;
      if ((!dab || 3 >= 1) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[719]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[720]; }
    { const long long ij = ij_3_2, kl = kl_0_1;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[721]; }
    { const long long ij = ij_3_2, kl = kl_0_2;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[722]; }
    { const long long ij = ij_3_2, kl = kl_0_3;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[723]; }
    { const long long ij = ij_3_2, kl = kl_0_4;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[724]; }
    { const long long ij = ij_3_2, kl = kl_0_5;
      if ((!dab || 3 >= 2) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[725]; }
    { const long long ij = ij_3_2, kl = kl_1_0;
      if ((!dab || 3 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[726]; }
    { const long long ij = ij_3_2, kl = kl_1_1;
      if ((!dab || 3 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[727]; }
    { const long long ij = ij_3_2, kl = kl_1_2;
      if ((!dab || 3 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[728]; }
    { const long long ij = ij_3_2, kl = kl_1_3;
      if ((!dab || 3 >= 2) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[729]; }
    { const long long ij = ij_3_2, kl = kl_1_4;
      if ((!dab || 3 >= 2) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[730]; }
    { const long long ij = ij_3_2, kl = kl_1_5;
      if ((!dab || 3 >= 2) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[731]; }
    { const long long ij = ij_3_2, kl = kl_2_0;
      if ((!dab || 3 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[732]; }
    { const long long ij = ij_3_2, kl = kl_2_1;
      if ((!dab || 3 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[733]; }
    { const long long ij = ij_3_2, kl = kl_2_2;
      if ((!dab || 3 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[734]; }
    { const long long ij = ij_3_2, kl = kl_2_3;
      if ((!dab || 3 >= 2) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[735]; }
    { const long long ij = ij_3_2, kl = kl_2_4;
      if ((!dab || 3 >= 2) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[736]; }
    { const long long ij = ij_3_2, kl = kl_2_5;
      if ((!dab || 3 >= 2) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[737]; }
    { const long long ij = ij_3_2, kl = kl_3_0;
      if ((!dab || 3 >= 2) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[738]; }
    { const long long ij = ij_3_2, kl = kl_3_1;
      if ((!dab || 3 >= 2) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[739]; }
    { const long long ij = ij_3_2, kl = kl_3_2;
      if ((!dab || 3 >= 2) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[740]; }
    { const long long ij = ij_3_2, kl = kl_3_3;
      if ((!dab || 3 >= 2) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[741]; }
    { const long long ij = ij_3_2, kl = kl_3_4;
      if ((!dab || 3 >= 2) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[742]; }
    { const long long ij = ij_3_2, kl = kl_3_5;
      if ((!dab || 3 >= 2) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[743]; }
    { const long long ij = ij_3_2, kl = kl_4_0;
      if ((!dab || 3 >= 2) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[744]; }
    { const long long ij = ij_3_2, kl = kl_4_1;
      if ((!dab || 3 >= 2) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[745]; }
    { const long long ij = ij_3_2, kl = kl_4_2;
      if ((!dab || 3 >= 2) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[746]; }
    { const long long ij = ij_3_2, kl = kl_4_3;
      if ((!dab || 3 >= 2) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[747]; }
    { const long long ij = ij_3_2, kl = kl_4_4;
      if ((!dab || 3 >= 2) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[748]; }
    { const long long ij = ij_3_2, kl = kl_4_5;
      if ((!dab || 3 >= 2) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[749]; }
    { const long long ij = ij_3_2, kl = kl_5_0;
      if ((!dab || 3 >= 2) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[750]; }
    { const long long ij = ij_3_2, kl = kl_5_1;
      if ((!dab || 3 >= 2) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[751]; }
    { const long long ij = ij_3_2, kl = kl_5_2;
      if ((!dab || 3 >= 2) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[752]; }
    { const long long ij = ij_3_2, kl = kl_5_3;
      if ((!dab || 3 >= 2) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[753]; }
    { const long long ij = ij_3_2, kl = kl_5_4;
      if ((!dab || 3 >= 2) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[754]; }
    { const long long ij = ij_3_2, kl = kl_5_5;
      if ((!dab || 3 >= 2) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[755]; }
    { const long long ij = ij_3_3, kl = kl_0_0;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[756]; }
    { const long long ij = ij_3_3, kl = kl_0_1;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[757]; }
    { const long long ij = ij_3_3, kl = kl_0_2;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[758]; }
    { const long long ij = ij_3_3, kl = kl_0_3;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[759]; }
    { const long long ij = ij_3_3, kl = kl_0_4;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[760]; }
    { const long long ij = ij_3_3, kl = kl_0_5;
      if ((!dab || 3 >= 3) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[761]; }
    { const long long ij = ij_3_3, kl = kl_1_0;
      if ((!dab || 3 >= 3) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[762]; }
    { const long long ij = ij_3_3, kl = kl_1_1;
      if ((!dab || 3 >= 3) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[763]; }
    { const long long ij = ij_3_3, kl = kl_1_2;
      if ((!dab || 3 >= 3) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[764]; }
    { const long long ij = ij_3_3, kl = kl_1_3;
      if ((!dab || 3 >= 3) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[765]; }
    { const long long ij = ij_3_3, kl = kl_1_4;
      if ((!dab || 3 >= 3) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[766]; }
    { const long long ij = ij_3_3, kl = kl_1_5;
      if ((!dab || 3 >= 3) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[767]; }
    { const long long ij = ij_3_3, kl = kl_2_0;
      if ((!dab || 3 >= 3) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[768]; }
    { const long long ij = ij_3_3, kl = kl_2_1;
      if ((!dab || 3 >= 3) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[769]; }
    { const long long ij = ij_3_3, kl = kl_2_2;
      if ((!dab || 3 >= 3) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[770]; }
    { const long long ij = ij_3_3, kl = kl_2_3;
      if ((!dab || 3 >= 3) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[771]; }
    { const long long ij = ij_3_3, kl = kl_2_4;
      if ((!dab || 3 >= 3) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[772]; }
    { const long long ij = ij_3_3, kl = kl_2_5;
      if ((!dab || 3 >= 3) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[773]; }
    { const long long ij = ij_3_3, kl = kl_3_0;
      if ((!dab || 3 >= 3) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[774]; }
    { const long long ij = ij_3_3, kl = kl_3_1;
      if ((!dab || 3 >= 3) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[775]; }
    { const long long ij = ij_3_3, kl = kl_3_2;
      if ((!dab || 3 >= 3) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[776]; }
    { const long long ij = ij_3_3, kl = kl_3_3;
      if ((!dab || 3 >= 3) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[777]; }
    { const long long ij = ij_3_3, kl = kl_3_4;
      if ((!dab || 3 >= 3) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[778]; }
    { const long long ij = ij_3_3, kl = kl_3_5;
      if ((!dab || 3 >= 3) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[779]; }
    { const long long ij = ij_3_3, kl = kl_4_0;
      if ((!dab || 3 >= 3) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[780]; }
    { const long long ij = ij_3_3, kl = kl_4_1;
      if ((!dab || 3 >= 3) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[781]; }
    { const long long ij = ij_3_3, kl = kl_4_2;
      if ((!dab || 3 >= 3) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[782]; }
    { const long long ij = ij_3_3, kl = kl_4_3;
      if ((!dab || 3 >= 3) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[783]; }
    { const long long ij = ij_3_3, kl = kl_4_4;
      if ((!dab || 3 >= 3) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[784]; }
    { const long long ij = ij_3_3, kl = kl_4_5;
      if ((!dab || 3 >= 3) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[785]; }
    { const long long ij = ij_3_3, kl = kl_5_0;
      if ((!dab || 3 >= 3) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[786]; }
    { const long long ij = ij_3_3, kl = kl_5_1;
      if ((!dab || 3 >= 3) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[787]; }
    { const long long ij = ij_3_3, kl = kl_5_2;
      if ((!dab || 3 >= 3) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[788]; }
    { const long long ij = ij_3_3, kl = kl_5_3;
      if ((!dab || 3 >= 3) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[789]; }
    { const long long ij = ij_3_3, kl = kl_5_4;
      if ((!dab || 3 >= 3) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[790]; }
    { const long long ij = ij_3_3, kl = kl_5_5;
      if ((!dab || 3 >= 3) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[791]; }
    { const long long ij = ij_3_4, kl = kl_0_0;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[792]; }
    { const long long ij = ij_3_4, kl = kl_0_1;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[793]; }
    { const long long ij = ij_3_4, kl = kl_0_2;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[794]; }
    { const long long ij = ij_3_4, kl = kl_0_3;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[795]; }
    { const long long ij = ij_3_4, kl = kl_0_4;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[796]; }
    { const long long ij = ij_3_4, kl = kl_0_5;
      if ((!dab || 3 >= 4) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[797]; }
    { const long long ij = ij_3_4, kl = kl_1_0;
      if ((!dab || 3 >= 4) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[798]; }
    { const long long ij = ij_3_4, kl = kl_1_1;
      if ((!dab || 3 >= 4) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[799]; }
    { const long long ij = ij_3_4, kl = kl_1_2;
      if ((!dab || 3 >= 4) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[800]; }
    { const long long ij = ij_3_4, kl = kl_1_3;
      if ((!dab || 3 >= 4) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[801]; }
    { const long long ij = ij_3_4, kl = kl_1_4;
      if ((!dab || 3 >= 4) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[802]; }
    { const long long ij = ij_3_4, kl = kl_1_5;
      if ((!dab || 3 >= 4) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[803]; }
    { const long long ij = ij_3_4, kl = kl_2_0;
      if ((!dab || 3 >= 4) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[804]; }
    { const long long ij = ij_3_4, kl = kl_2_1;
      if ((!dab || 3 >= 4) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[805]; }
    { const long long ij = ij_3_4, kl = kl_2_2;
      if ((!dab || 3 >= 4) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[806]; }
    { const long long ij = ij_3_4, kl = kl_2_3;
      if ((!dab || 3 >= 4) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[807]; }
    { const long long ij = ij_3_4, kl = kl_2_4;
      if ((!dab || 3 >= 4) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[808]; }
    { const long long ij = ij_3_4, kl = kl_2_5;
      if ((!dab || 3 >= 4) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[809]; }
    { const long long ij = ij_3_4, kl = kl_3_0;
      if ((!dab || 3 >= 4) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[810]; }
    { const long long ij = ij_3_4, kl = kl_3_1;
      if ((!dab || 3 >= 4) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[811]; }
    { const long long ij = ij_3_4, kl = kl_3_2;
      if ((!dab || 3 >= 4) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[812]; }
    { const long long ij = ij_3_4, kl = kl_3_3;
      if ((!dab || 3 >= 4) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[813]; }
    { const long long ij = ij_3_4, kl = kl_3_4;
      if ((!dab || 3 >= 4) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[814]; }
    { const long long ij = ij_3_4, kl = kl_3_5;
      if ((!dab || 3 >= 4) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[815]; }
    { const long long ij = ij_3_4, kl = kl_4_0;
      if ((!dab || 3 >= 4) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[816]; }
    { const long long ij = ij_3_4, kl = kl_4_1;
      if ((!dab || 3 >= 4) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[817]; }
    { const long long ij = ij_3_4, kl = kl_4_2;
      if ((!dab || 3 >= 4) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[818]; }
    { const long long ij = ij_3_4, kl = kl_4_3;
      if ((!dab || 3 >= 4) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[819]; }
    { const long long ij = ij_3_4, kl = kl_4_4;
      if ((!dab || 3 >= 4) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[820]; }
    { const long long ij = ij_3_4, kl = kl_4_5;
      if ((!dab || 3 >= 4) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[821]; }
    { const long long ij = ij_3_4, kl = kl_5_0;
      if ((!dab || 3 >= 4) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[822]; }
    { const long long ij = ij_3_4, kl = kl_5_1;
      if ((!dab || 3 >= 4) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[823]; }
    { const long long ij = ij_3_4, kl = kl_5_2;
      if ((!dab || 3 >= 4) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[824]; }
    { const long long ij = ij_3_4, kl = kl_5_3;
      if ((!dab || 3 >= 4) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[825]; }
    { const long long ij = ij_3_4, kl = kl_5_4;
      if ((!dab || 3 >= 4) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[826]; }
    { const long long ij = ij_3_4, kl = kl_5_5;
      if ((!dab || 3 >= 4) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[827]; }
    { const long long ij = ij_3_5, kl = kl_0_0;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[828]; }
    { const long long ij = ij_3_5, kl = kl_0_1;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[829]; }
    { const long long ij = ij_3_5, kl = kl_0_2;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[830]; }
    { const long long ij = ij_3_5, kl = kl_0_3;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[831]; }
    { const long long ij = ij_3_5, kl = kl_0_4;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[832]; }
    { const long long ij = ij_3_5, kl = kl_0_5;
      if ((!dab || 3 >= 5) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[833]; }
    { const long long ij = ij_3_5, kl = kl_1_0;
      if ((!dab || 3 >= 5) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[834]; }
    { const long long ij = ij_3_5, kl = kl_1_1;
      if ((!dab || 3 >= 5) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[835]; }
    { const long long ij = ij_3_5, kl = kl_1_2;
      if ((!dab || 3 >= 5) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[836]; }
    { const long long ij = ij_3_5, kl = kl_1_3;
      if ((!dab || 3 >= 5) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[837]; }
    { const long long ij = ij_3_5, kl = kl_1_4;
      if ((!dab || 3 >= 5) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[838]; }
    { const long long ij = ij_3_5, kl = kl_1_5;
      if ((!dab || 3 >= 5) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[839]; }
    { const long long ij = ij_3_5, kl = kl_2_0;
      if ((!dab || 3 >= 5) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[840]; }
    { const long long ij = ij_3_5, kl = kl_2_1;
      if ((!dab || 3 >= 5) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[841]; }
    { const long long ij = ij_3_5, kl = kl_2_2;
      if ((!dab || 3 >= 5) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[842]; }
    { const long long ij = ij_3_5, kl = kl_2_3;
      if ((!dab || 3 >= 5) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[843]; }
    { const long long ij = ij_3_5, kl = kl_2_4;
      if ((!dab || 3 >= 5) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[844]; }
    { const long long ij = ij_3_5, kl = kl_2_5;
      if ((!dab || 3 >= 5) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[845]; }
    { const long long ij = ij_3_5, kl = kl_3_0;
      if ((!dab || 3 >= 5) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[846]; }
    { const long long ij = ij_3_5, kl = kl_3_1;
      if ((!dab || 3 >= 5) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[847]; }
    { const long long ij = ij_3_5, kl = kl_3_2;
      if ((!dab || 3 >= 5) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[848]; }
    { const long long ij = ij_3_5, kl = kl_3_3;
      if ((!dab || 3 >= 5) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[849]; }
    { const long long ij = ij_3_5, kl = kl_3_4;
      if ((!dab || 3 >= 5) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[850]; }
    { const long long ij = ij_3_5, kl = kl_3_5;
      if ((!dab || 3 >= 5) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[851]; }
    { const long long ij = ij_3_5, kl = kl_4_0;
      if ((!dab || 3 >= 5) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[852]; }
    { const long long ij = ij_3_5, kl = kl_4_1;
      if ((!dab || 3 >= 5) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[853]; }
    { const long long ij = ij_3_5, kl = kl_4_2;
      if ((!dab || 3 >= 5) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[854]; }
    { const long long ij = ij_3_5, kl = kl_4_3;
      if ((!dab || 3 >= 5) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[855]; }
    { const long long ij = ij_3_5, kl = kl_4_4;
      if ((!dab || 3 >= 5) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[856]; }
    { const long long ij = ij_3_5, kl = kl_4_5;
      if ((!dab || 3 >= 5) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[857]; }
    { const long long ij = ij_3_5, kl = kl_5_0;
      if ((!dab || 3 >= 5) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[858]; }
    { const long long ij = ij_3_5, kl = kl_5_1;
      if ((!dab || 3 >= 5) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[859]; }
    { const long long ij = ij_3_5, kl = kl_5_2;
      if ((!dab || 3 >= 5) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[860]; }
    { const long long ij = ij_3_5, kl = kl_5_3;
      if ((!dab || 3 >= 5) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[861]; }
    { const long long ij = ij_3_5, kl = kl_5_4;
      if ((!dab || 3 >= 5) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[862]; }
    { const long long ij = ij_3_5, kl = kl_5_5;
      if ((!dab || 3 >= 5) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[863]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[864]; }
    { const long long ij = ij_4_0, kl = kl_0_1;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[865]; }
    { const long long ij = ij_4_0, kl = kl_0_2;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[866]; }
    { const long long ij = ij_4_0, kl = kl_0_3;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[867]; }
    { const long long ij = ij_4_0, kl = kl_0_4;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[868]; }
    { const long long ij = ij_4_0, kl = kl_0_5;
      if ((!dab || 4 >= 0) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[869]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if ((!dab || 4 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[870]; }
    { const long long ij = ij_4_0, kl = kl_1_1;
      if ((!dab || 4 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[871]; }
    { const long long ij = ij_4_0, kl = kl_1_2;
      if ((!dab || 4 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[872]; }
    { const long long ij = ij_4_0, kl = kl_1_3;
      if ((!dab || 4 >= 0) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[873]; }
    { const long long ij = ij_4_0, kl = kl_1_4;
      if ((!dab || 4 >= 0) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[874]; }
    { const long long ij = ij_4_0, kl = kl_1_5;
      if ((!dab || 4 >= 0) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[875]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if ((!dab || 4 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[876]; }
    { const long long ij = ij_4_0, kl = kl_2_1;
      if ((!dab || 4 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[877]; }
    { const long long ij = ij_4_0, kl = kl_2_2;
      if ((!dab || 4 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[878]; }
    { const long long ij = ij_4_0, kl = kl_2_3;
      if ((!dab || 4 >= 0) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[879]; }
    { const long long ij = ij_4_0, kl = kl_2_4;
      if ((!dab || 4 >= 0) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[880]; }
    { const long long ij = ij_4_0, kl = kl_2_5;
      if ((!dab || 4 >= 0) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[881]; }
    { const long long ij = ij_4_0, kl = kl_3_0;
      if ((!dab || 4 >= 0) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[882]; }
    { const long long ij = ij_4_0, kl = kl_3_1;
      if ((!dab || 4 >= 0) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[883]; }
    { const long long ij = ij_4_0, kl = kl_3_2;
      if ((!dab || 4 >= 0) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[884]; }
    { const long long ij = ij_4_0, kl = kl_3_3;
      if ((!dab || 4 >= 0) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[885]; }
    { const long long ij = ij_4_0, kl = kl_3_4;
      if ((!dab || 4 >= 0) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[886]; }
    { const long long ij = ij_4_0, kl = kl_3_5;
      if ((!dab || 4 >= 0) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[887]; }
    { const long long ij = ij_4_0, kl = kl_4_0;
      if ((!dab || 4 >= 0) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[888]; }
    { const long long ij = ij_4_0, kl = kl_4_1;
      if ((!dab || 4 >= 0) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[889]; }
    { const long long ij = ij_4_0, kl = kl_4_2;
      if ((!dab || 4 >= 0) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[890]; }
    { const long long ij = ij_4_0, kl = kl_4_3;
      if ((!dab || 4 >= 0) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[891]; }
    { const long long ij = ij_4_0, kl = kl_4_4;
      if ((!dab || 4 >= 0) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[892]; }
    { const long long ij = ij_4_0, kl = kl_4_5;
      if ((!dab || 4 >= 0) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[893]; }
    { const long long ij = ij_4_0, kl = kl_5_0;
      if ((!dab || 4 >= 0) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[894]; }
    { const long long ij = ij_4_0, kl = kl_5_1;
      if ((!dab || 4 >= 0) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[895]; }
    { const long long ij = ij_4_0, kl = kl_5_2;
      if ((!dab || 4 >= 0) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[896]; }
    { const long long ij = ij_4_0, kl = kl_5_3;
      if ((!dab || 4 >= 0) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[897]; }
    { const long long ij = ij_4_0, kl = kl_5_4;
      if ((!dab || 4 >= 0) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[898]; }
    { const long long ij = ij_4_0, kl = kl_5_5;
      if ((!dab || 4 >= 0) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[899]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[900]; }
    { const long long ij = ij_4_1, kl = kl_0_1;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[901]; }
    { const long long ij = ij_4_1, kl = kl_0_2;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[902]; }
    { const long long ij = ij_4_1, kl = kl_0_3;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[903]; }
    { const long long ij = ij_4_1, kl = kl_0_4;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[904]; }
    { const long long ij = ij_4_1, kl = kl_0_5;
      if ((!dab || 4 >= 1) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[905]; }
    { const long long ij = ij_4_1, kl = kl_1_0;
      if ((!dab || 4 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[906]; }
    { const long long ij = ij_4_1, kl = kl_1_1;
      if ((!dab || 4 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[907]; }
    { const long long ij = ij_4_1, kl = kl_1_2;
      if ((!dab || 4 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[908]; }
    { const long long ij = ij_4_1, kl = kl_1_3;
      if ((!dab || 4 >= 1) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[909]; }
    { const long long ij = ij_4_1, kl = kl_1_4;
      if ((!dab || 4 >= 1) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[910]; }
    { const long long ij = ij_4_1, kl = kl_1_5;
      if ((!dab || 4 >= 1) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[911]; }
    { const long long ij = ij_4_1, kl = kl_2_0;
      if ((!dab || 4 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[912]; }
    { const long long ij = ij_4_1, kl = kl_2_1;
      if ((!dab || 4 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[913]; }
    { const long long ij = ij_4_1, kl = kl_2_2;
      if ((!dab || 4 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[914]; }
    { const long long ij = ij_4_1, kl = kl_2_3;
      if ((!dab || 4 >= 1) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[915]; }
    { const long long ij = ij_4_1, kl = kl_2_4;
      if ((!dab || 4 >= 1) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[916]; }
    { const long long ij = ij_4_1, kl = kl_2_5;
      if ((!dab || 4 >= 1) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[917]; }
    { const long long ij = ij_4_1, kl = kl_3_0;
      if ((!dab || 4 >= 1) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[918]; }
    { const long long ij = ij_4_1, kl = kl_3_1;
      if ((!dab || 4 >= 1) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[919]; }
    { const long long ij = ij_4_1, kl = kl_3_2;
      if ((!dab || 4 >= 1) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[920]; }
    { const long long ij = ij_4_1, kl = kl_3_3;
      if ((!dab || 4 >= 1) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[921]; }
    { const long long ij = ij_4_1, kl = kl_3_4;
      if ((!dab || 4 >= 1) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[922]; }
    { const long long ij = ij_4_1, kl = kl_3_5;
      if ((!dab || 4 >= 1) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[923]; }
    { const long long ij = ij_4_1, kl = kl_4_0;
      if ((!dab || 4 >= 1) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[924]; }
    { const long long ij = ij_4_1, kl = kl_4_1;
      if ((!dab || 4 >= 1) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[925]; }
    { const long long ij = ij_4_1, kl = kl_4_2;
      if ((!dab || 4 >= 1) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[926]; }
    { const long long ij = ij_4_1, kl = kl_4_3;
      if ((!dab || 4 >= 1) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[927]; }
    { const long long ij = ij_4_1, kl = kl_4_4;
      if ((!dab || 4 >= 1) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[928]; }
    { const long long ij = ij_4_1, kl = kl_4_5;
      if ((!dab || 4 >= 1) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[929]; }
    { const long long ij = ij_4_1, kl = kl_5_0;
      if ((!dab || 4 >= 1) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[930]; }
    { const long long ij = ij_4_1, kl = kl_5_1;
      if ((!dab || 4 >= 1) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[931]; }
    { const long long ij = ij_4_1, kl = kl_5_2;
      if ((!dab || 4 >= 1) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[932]; }
    { const long long ij = ij_4_1, kl = kl_5_3;
      if ((!dab || 4 >= 1) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[933]; }
    { const long long ij = ij_4_1, kl = kl_5_4;
      if ((!dab || 4 >= 1) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[934]; }
    { const long long ij = ij_4_1, kl = kl_5_5;
      if ((!dab || 4 >= 1) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[935]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[936]; }
    { const long long ij = ij_4_2, kl = kl_0_1;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[937]; }
    { const long long ij = ij_4_2, kl = kl_0_2;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[938]; }
    { const long long ij = ij_4_2, kl = kl_0_3;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[939]; }
    { const long long ij = ij_4_2, kl = kl_0_4;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[940]; }
    { const long long ij = ij_4_2, kl = kl_0_5;
      if ((!dab || 4 >= 2) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[941]; }
    { const long long ij = ij_4_2, kl = kl_1_0;
      if ((!dab || 4 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[942]; }
    { const long long ij = ij_4_2, kl = kl_1_1;
      if ((!dab || 4 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[943]; }
    { const long long ij = ij_4_2, kl = kl_1_2;
      if ((!dab || 4 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[944]; }
    { const long long ij = ij_4_2, kl = kl_1_3;
      if ((!dab || 4 >= 2) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[945]; }
    { const long long ij = ij_4_2, kl = kl_1_4;
      if ((!dab || 4 >= 2) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[946]; }
    { const long long ij = ij_4_2, kl = kl_1_5;
      if ((!dab || 4 >= 2) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[947]; }
    { const long long ij = ij_4_2, kl = kl_2_0;
      if ((!dab || 4 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[948]; }
    { const long long ij = ij_4_2, kl = kl_2_1;
      if ((!dab || 4 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[949]; }
    { const long long ij = ij_4_2, kl = kl_2_2;
      if ((!dab || 4 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[950]; }
    { const long long ij = ij_4_2, kl = kl_2_3;
      if ((!dab || 4 >= 2) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[951]; }
    { const long long ij = ij_4_2, kl = kl_2_4;
      if ((!dab || 4 >= 2) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[952]; }
    { const long long ij = ij_4_2, kl = kl_2_5;
      if ((!dab || 4 >= 2) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[953]; }
    { const long long ij = ij_4_2, kl = kl_3_0;
      if ((!dab || 4 >= 2) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[954]; }
    { const long long ij = ij_4_2, kl = kl_3_1;
      if ((!dab || 4 >= 2) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[955]; }
    { const long long ij = ij_4_2, kl = kl_3_2;
      if ((!dab || 4 >= 2) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[956]; }
    { const long long ij = ij_4_2, kl = kl_3_3;
      if ((!dab || 4 >= 2) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[957]; }
    { const long long ij = ij_4_2, kl = kl_3_4;
      if ((!dab || 4 >= 2) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[958]; }
    { const long long ij = ij_4_2, kl = kl_3_5;
      if ((!dab || 4 >= 2) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[959]; }
    { const long long ij = ij_4_2, kl = kl_4_0;
      if ((!dab || 4 >= 2) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[960]; }
    { const long long ij = ij_4_2, kl = kl_4_1;
      if ((!dab || 4 >= 2) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[961]; }
    { const long long ij = ij_4_2, kl = kl_4_2;
      if ((!dab || 4 >= 2) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[962]; }
    { const long long ij = ij_4_2, kl = kl_4_3;
      if ((!dab || 4 >= 2) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[963]; }
    { const long long ij = ij_4_2, kl = kl_4_4;
      if ((!dab || 4 >= 2) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[964]; }
    { const long long ij = ij_4_2, kl = kl_4_5;
      if ((!dab || 4 >= 2) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[965]; }
    { const long long ij = ij_4_2, kl = kl_5_0;
      if ((!dab || 4 >= 2) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[966]; }
    { const long long ij = ij_4_2, kl = kl_5_1;
      if ((!dab || 4 >= 2) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[967]; }
    { const long long ij = ij_4_2, kl = kl_5_2;
      if ((!dab || 4 >= 2) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[968]; }
    { const long long ij = ij_4_2, kl = kl_5_3;
      if ((!dab || 4 >= 2) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[969]; }
    { const long long ij = ij_4_2, kl = kl_5_4;
      if ((!dab || 4 >= 2) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[970]; }
    { const long long ij = ij_4_2, kl = kl_5_5;
      if ((!dab || 4 >= 2) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[971]; }
    { const long long ij = ij_4_3, kl = kl_0_0;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[972]; }
    { const long long ij = ij_4_3, kl = kl_0_1;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[973]; }
    { const long long ij = ij_4_3, kl = kl_0_2;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[974]; }
    { const long long ij = ij_4_3, kl = kl_0_3;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[975]; }
    { const long long ij = ij_4_3, kl = kl_0_4;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[976]; }
    { const long long ij = ij_4_3, kl = kl_0_5;
      if ((!dab || 4 >= 3) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[977]; }
    { const long long ij = ij_4_3, kl = kl_1_0;
      if ((!dab || 4 >= 3) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[978]; }
    { const long long ij = ij_4_3, kl = kl_1_1;
      if ((!dab || 4 >= 3) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[979]; }
    { const long long ij = ij_4_3, kl = kl_1_2;
      if ((!dab || 4 >= 3) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[980]; }
    { const long long ij = ij_4_3, kl = kl_1_3;
      if ((!dab || 4 >= 3) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[981]; }
    { const long long ij = ij_4_3, kl = kl_1_4;
      if ((!dab || 4 >= 3) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[982]; }
    { const long long ij = ij_4_3, kl = kl_1_5;
      if ((!dab || 4 >= 3) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[983]; }
    { const long long ij = ij_4_3, kl = kl_2_0;
      if ((!dab || 4 >= 3) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[984]; }
    { const long long ij = ij_4_3, kl = kl_2_1;
      if ((!dab || 4 >= 3) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[985]; }
    { const long long ij = ij_4_3, kl = kl_2_2;
      if ((!dab || 4 >= 3) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[986]; }
    { const long long ij = ij_4_3, kl = kl_2_3;
      if ((!dab || 4 >= 3) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[987]; }
    { const long long ij = ij_4_3, kl = kl_2_4;
      if ((!dab || 4 >= 3) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[988]; }
    { const long long ij = ij_4_3, kl = kl_2_5;
      if ((!dab || 4 >= 3) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[989]; }
    { const long long ij = ij_4_3, kl = kl_3_0;
      if ((!dab || 4 >= 3) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[990]; }
    { const long long ij = ij_4_3, kl = kl_3_1;
      if ((!dab || 4 >= 3) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[991]; }
    { const long long ij = ij_4_3, kl = kl_3_2;
      if ((!dab || 4 >= 3) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[992]; }
    { const long long ij = ij_4_3, kl = kl_3_3;
      if ((!dab || 4 >= 3) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[993]; }
    { const long long ij = ij_4_3, kl = kl_3_4;
      if ((!dab || 4 >= 3) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[994]; }
    { const long long ij = ij_4_3, kl = kl_3_5;
      if ((!dab || 4 >= 3) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[995]; }
    { const long long ij = ij_4_3, kl = kl_4_0;
      if ((!dab || 4 >= 3) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[996]; }
    { const long long ij = ij_4_3, kl = kl_4_1;
      if ((!dab || 4 >= 3) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[997]; }
    { const long long ij = ij_4_3, kl = kl_4_2;
      if ((!dab || 4 >= 3) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[998]; }
    { const long long ij = ij_4_3, kl = kl_4_3;
      if ((!dab || 4 >= 3) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[999]; }
    { const long long ij = ij_4_3, kl = kl_4_4;
      if ((!dab || 4 >= 3) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1000]; }
    { const long long ij = ij_4_3, kl = kl_4_5;
      if ((!dab || 4 >= 3) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1001]; }
    { const long long ij = ij_4_3, kl = kl_5_0;
      if ((!dab || 4 >= 3) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1002]; }
    { const long long ij = ij_4_3, kl = kl_5_1;
      if ((!dab || 4 >= 3) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1003]; }
    { const long long ij = ij_4_3, kl = kl_5_2;
      if ((!dab || 4 >= 3) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1004]; }
    { const long long ij = ij_4_3, kl = kl_5_3;
      if ((!dab || 4 >= 3) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1005]; }
    { const long long ij = ij_4_3, kl = kl_5_4;
      if ((!dab || 4 >= 3) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1006]; }
    { const long long ij = ij_4_3, kl = kl_5_5;
      if ((!dab || 4 >= 3) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1007]; }
    { const long long ij = ij_4_4, kl = kl_0_0;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1008]; }
    { const long long ij = ij_4_4, kl = kl_0_1;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1009]; }
    { const long long ij = ij_4_4, kl = kl_0_2;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1010]; }
    { const long long ij = ij_4_4, kl = kl_0_3;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1011]; }
    { const long long ij = ij_4_4, kl = kl_0_4;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1012]; }
    { const long long ij = ij_4_4, kl = kl_0_5;
      if ((!dab || 4 >= 4) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1013]; }
    { const long long ij = ij_4_4, kl = kl_1_0;
      if ((!dab || 4 >= 4) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1014]; }
    { const long long ij = ij_4_4, kl = kl_1_1;
      if ((!dab || 4 >= 4) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1015]; }
    { const long long ij = ij_4_4, kl = kl_1_2;
      if ((!dab || 4 >= 4) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1016]; }
    { const long long ij = ij_4_4, kl = kl_1_3;
      if ((!dab || 4 >= 4) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1017]; }
    { const long long ij = ij_4_4, kl = kl_1_4;
      if ((!dab || 4 >= 4) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1018]; }
    { const long long ij = ij_4_4, kl = kl_1_5;
      if ((!dab || 4 >= 4) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1019]; }
    { const long long ij = ij_4_4, kl = kl_2_0;
      if ((!dab || 4 >= 4) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1020]; }
    { const long long ij = ij_4_4, kl = kl_2_1;
      if ((!dab || 4 >= 4) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1021]; }
    { const long long ij = ij_4_4, kl = kl_2_2;
      if ((!dab || 4 >= 4) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1022]; }
    { const long long ij = ij_4_4, kl = kl_2_3;
      if ((!dab || 4 >= 4) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1023]; }
    { const long long ij = ij_4_4, kl = kl_2_4;
      if ((!dab || 4 >= 4) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1024]; }
    { const long long ij = ij_4_4, kl = kl_2_5;
      if ((!dab || 4 >= 4) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1025]; }
    { const long long ij = ij_4_4, kl = kl_3_0;
      if ((!dab || 4 >= 4) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1026]; }
    { const long long ij = ij_4_4, kl = kl_3_1;
      if ((!dab || 4 >= 4) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1027]; }
    { const long long ij = ij_4_4, kl = kl_3_2;
      if ((!dab || 4 >= 4) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1028]; }
    { const long long ij = ij_4_4, kl = kl_3_3;
      if ((!dab || 4 >= 4) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1029]; }
    { const long long ij = ij_4_4, kl = kl_3_4;
      if ((!dab || 4 >= 4) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1030]; }
    { const long long ij = ij_4_4, kl = kl_3_5;
      if ((!dab || 4 >= 4) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1031]; }
    { const long long ij = ij_4_4, kl = kl_4_0;
      if ((!dab || 4 >= 4) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1032]; }
    { const long long ij = ij_4_4, kl = kl_4_1;
      if ((!dab || 4 >= 4) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1033]; }
    { const long long ij = ij_4_4, kl = kl_4_2;
      if ((!dab || 4 >= 4) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1034]; }
    { const long long ij = ij_4_4, kl = kl_4_3;
      if ((!dab || 4 >= 4) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1035]; }
    { const long long ij = ij_4_4, kl = kl_4_4;
      if ((!dab || 4 >= 4) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1036]; }
    { const long long ij = ij_4_4, kl = kl_4_5;
      if ((!dab || 4 >= 4) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1037]; }
    { const long long ij = ij_4_4, kl = kl_5_0;
      if ((!dab || 4 >= 4) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1038]; }
    { const long long ij = ij_4_4, kl = kl_5_1;
      if ((!dab || 4 >= 4) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1039]; }
    { const long long ij = ij_4_4, kl = kl_5_2;
      if ((!dab || 4 >= 4) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1040]; }
    { const long long ij = ij_4_4, kl = kl_5_3;
      if ((!dab || 4 >= 4) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1041]; }
    { const long long ij = ij_4_4, kl = kl_5_4;
      if ((!dab || 4 >= 4) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1042]; }
    { const long long ij = ij_4_4, kl = kl_5_5;
      if ((!dab || 4 >= 4) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1043]; }
    { const long long ij = ij_4_5, kl = kl_0_0;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1044]; }
    { const long long ij = ij_4_5, kl = kl_0_1;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1045]; }
    { const long long ij = ij_4_5, kl = kl_0_2;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1046]; }
    { const long long ij = ij_4_5, kl = kl_0_3;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1047]; }
    { const long long ij = ij_4_5, kl = kl_0_4;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1048]; }
    { const long long ij = ij_4_5, kl = kl_0_5;
      if ((!dab || 4 >= 5) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1049]; }
    { const long long ij = ij_4_5, kl = kl_1_0;
      if ((!dab || 4 >= 5) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1050]; }
    { const long long ij = ij_4_5, kl = kl_1_1;
      if ((!dab || 4 >= 5) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1051]; }
    { const long long ij = ij_4_5, kl = kl_1_2;
      if ((!dab || 4 >= 5) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1052]; }
    { const long long ij = ij_4_5, kl = kl_1_3;
      if ((!dab || 4 >= 5) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1053]; }
    { const long long ij = ij_4_5, kl = kl_1_4;
      if ((!dab || 4 >= 5) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1054]; }
    { const long long ij = ij_4_5, kl = kl_1_5;
      if ((!dab || 4 >= 5) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1055]; }
    { const long long ij = ij_4_5, kl = kl_2_0;
      if ((!dab || 4 >= 5) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1056]; }
    { const long long ij = ij_4_5, kl = kl_2_1;
      if ((!dab || 4 >= 5) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1057]; }
    { const long long ij = ij_4_5, kl = kl_2_2;
      if ((!dab || 4 >= 5) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1058]; }
    { const long long ij = ij_4_5, kl = kl_2_3;
      if ((!dab || 4 >= 5) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1059]; }
    { const long long ij = ij_4_5, kl = kl_2_4;
      if ((!dab || 4 >= 5) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1060]; }
    { const long long ij = ij_4_5, kl = kl_2_5;
      if ((!dab || 4 >= 5) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1061]; }
    { const long long ij = ij_4_5, kl = kl_3_0;
      if ((!dab || 4 >= 5) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1062]; }
    { const long long ij = ij_4_5, kl = kl_3_1;
      if ((!dab || 4 >= 5) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1063]; }
    { const long long ij = ij_4_5, kl = kl_3_2;
      if ((!dab || 4 >= 5) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1064]; }
    { const long long ij = ij_4_5, kl = kl_3_3;
      if ((!dab || 4 >= 5) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1065]; }
    { const long long ij = ij_4_5, kl = kl_3_4;
      if ((!dab || 4 >= 5) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1066]; }
    { const long long ij = ij_4_5, kl = kl_3_5;
      if ((!dab || 4 >= 5) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1067]; }
    { const long long ij = ij_4_5, kl = kl_4_0;
      if ((!dab || 4 >= 5) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1068]; }
    { const long long ij = ij_4_5, kl = kl_4_1;
      if ((!dab || 4 >= 5) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1069]; }
    { const long long ij = ij_4_5, kl = kl_4_2;
      if ((!dab || 4 >= 5) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1070]; }
    { const long long ij = ij_4_5, kl = kl_4_3;
      if ((!dab || 4 >= 5) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1071]; }
    { const long long ij = ij_4_5, kl = kl_4_4;
      if ((!dab || 4 >= 5) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1072]; }
    { const long long ij = ij_4_5, kl = kl_4_5;
      if ((!dab || 4 >= 5) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1073]; }
    { const long long ij = ij_4_5, kl = kl_5_0;
      if ((!dab || 4 >= 5) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1074]; }
    { const long long ij = ij_4_5, kl = kl_5_1;
      if ((!dab || 4 >= 5) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1075]; }
    { const long long ij = ij_4_5, kl = kl_5_2;
      if ((!dab || 4 >= 5) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1076]; }
    { const long long ij = ij_4_5, kl = kl_5_3;
      if ((!dab || 4 >= 5) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1077]; }
    { const long long ij = ij_4_5, kl = kl_5_4;
      if ((!dab || 4 >= 5) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1078]; }
    { const long long ij = ij_4_5, kl = kl_5_5;
      if ((!dab || 4 >= 5) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1079]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1080]; }
    { const long long ij = ij_5_0, kl = kl_0_1;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1081]; }
    { const long long ij = ij_5_0, kl = kl_0_2;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1082]; }
    { const long long ij = ij_5_0, kl = kl_0_3;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1083]; }
    { const long long ij = ij_5_0, kl = kl_0_4;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1084]; }
    { const long long ij = ij_5_0, kl = kl_0_5;
      if ((!dab || 5 >= 0) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1085]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if ((!dab || 5 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1086]; }
    { const long long ij = ij_5_0, kl = kl_1_1;
      if ((!dab || 5 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1087]; }
    { const long long ij = ij_5_0, kl = kl_1_2;
      if ((!dab || 5 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1088]; }
    { const long long ij = ij_5_0, kl = kl_1_3;
      if ((!dab || 5 >= 0) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1089]; }
    { const long long ij = ij_5_0, kl = kl_1_4;
      if ((!dab || 5 >= 0) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1090]; }
    { const long long ij = ij_5_0, kl = kl_1_5;
      if ((!dab || 5 >= 0) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1091]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if ((!dab || 5 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1092]; }
    { const long long ij = ij_5_0, kl = kl_2_1;
      if ((!dab || 5 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1093]; }
    { const long long ij = ij_5_0, kl = kl_2_2;
      if ((!dab || 5 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1094]; }
    { const long long ij = ij_5_0, kl = kl_2_3;
      if ((!dab || 5 >= 0) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1095]; }
    { const long long ij = ij_5_0, kl = kl_2_4;
      if ((!dab || 5 >= 0) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1096]; }
    { const long long ij = ij_5_0, kl = kl_2_5;
      if ((!dab || 5 >= 0) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1097]; }
    { const long long ij = ij_5_0, kl = kl_3_0;
      if ((!dab || 5 >= 0) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1098]; }
    { const long long ij = ij_5_0, kl = kl_3_1;
      if ((!dab || 5 >= 0) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1099]; }
    { const long long ij = ij_5_0, kl = kl_3_2;
      if ((!dab || 5 >= 0) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1100]; }
    { const long long ij = ij_5_0, kl = kl_3_3;
      if ((!dab || 5 >= 0) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1101]; }
    { const long long ij = ij_5_0, kl = kl_3_4;
      if ((!dab || 5 >= 0) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1102]; }
    { const long long ij = ij_5_0, kl = kl_3_5;
      if ((!dab || 5 >= 0) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1103]; }
    { const long long ij = ij_5_0, kl = kl_4_0;
      if ((!dab || 5 >= 0) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1104]; }
    { const long long ij = ij_5_0, kl = kl_4_1;
      if ((!dab || 5 >= 0) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1105]; }
    { const long long ij = ij_5_0, kl = kl_4_2;
      if ((!dab || 5 >= 0) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1106]; }
    { const long long ij = ij_5_0, kl = kl_4_3;
      if ((!dab || 5 >= 0) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1107]; }
    { const long long ij = ij_5_0, kl = kl_4_4;
      if ((!dab || 5 >= 0) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1108]; }
    { const long long ij = ij_5_0, kl = kl_4_5;
      if ((!dab || 5 >= 0) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1109]; }
    { const long long ij = ij_5_0, kl = kl_5_0;
      if ((!dab || 5 >= 0) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1110]; }
    { const long long ij = ij_5_0, kl = kl_5_1;
      if ((!dab || 5 >= 0) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1111]; }
    { const long long ij = ij_5_0, kl = kl_5_2;
      if ((!dab || 5 >= 0) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1112]; }
    { const long long ij = ij_5_0, kl = kl_5_3;
      if ((!dab || 5 >= 0) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1113]; }
    { const long long ij = ij_5_0, kl = kl_5_4;
      if ((!dab || 5 >= 0) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1114]; }
    { const long long ij = ij_5_0, kl = kl_5_5;
      if ((!dab || 5 >= 0) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1115]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1116]; }
    { const long long ij = ij_5_1, kl = kl_0_1;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1117]; }
    { const long long ij = ij_5_1, kl = kl_0_2;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1118]; }
    { const long long ij = ij_5_1, kl = kl_0_3;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1119]; }
    { const long long ij = ij_5_1, kl = kl_0_4;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1120]; }
    { const long long ij = ij_5_1, kl = kl_0_5;
      if ((!dab || 5 >= 1) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1121]; }
    { const long long ij = ij_5_1, kl = kl_1_0;
      if ((!dab || 5 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1122]; }
    { const long long ij = ij_5_1, kl = kl_1_1;
      if ((!dab || 5 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1123]; }
    { const long long ij = ij_5_1, kl = kl_1_2;
      if ((!dab || 5 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1124]; }
    { const long long ij = ij_5_1, kl = kl_1_3;
      if ((!dab || 5 >= 1) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1125]; }
    { const long long ij = ij_5_1, kl = kl_1_4;
      if ((!dab || 5 >= 1) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1126]; }
    { const long long ij = ij_5_1, kl = kl_1_5;
      if ((!dab || 5 >= 1) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1127]; }
    { const long long ij = ij_5_1, kl = kl_2_0;
      if ((!dab || 5 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1128]; }
    { const long long ij = ij_5_1, kl = kl_2_1;
      if ((!dab || 5 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1129]; }
    { const long long ij = ij_5_1, kl = kl_2_2;
      if ((!dab || 5 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1130]; }
    { const long long ij = ij_5_1, kl = kl_2_3;
      if ((!dab || 5 >= 1) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1131]; }
    { const long long ij = ij_5_1, kl = kl_2_4;
      if ((!dab || 5 >= 1) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1132]; }
    { const long long ij = ij_5_1, kl = kl_2_5;
      if ((!dab || 5 >= 1) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1133]; }
    { const long long ij = ij_5_1, kl = kl_3_0;
      if ((!dab || 5 >= 1) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1134]; }
    { const long long ij = ij_5_1, kl = kl_3_1;
      if ((!dab || 5 >= 1) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1135]; }
    { const long long ij = ij_5_1, kl = kl_3_2;
      if ((!dab || 5 >= 1) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1136]; }
    { const long long ij = ij_5_1, kl = kl_3_3;
      if ((!dab || 5 >= 1) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1137]; }
    { const long long ij = ij_5_1, kl = kl_3_4;
      if ((!dab || 5 >= 1) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1138]; }
    { const long long ij = ij_5_1, kl = kl_3_5;
      if ((!dab || 5 >= 1) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1139]; }
    { const long long ij = ij_5_1, kl = kl_4_0;
      if ((!dab || 5 >= 1) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1140]; }
    { const long long ij = ij_5_1, kl = kl_4_1;
      if ((!dab || 5 >= 1) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1141]; }
    { const long long ij = ij_5_1, kl = kl_4_2;
      if ((!dab || 5 >= 1) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1142]; }
    { const long long ij = ij_5_1, kl = kl_4_3;
      if ((!dab || 5 >= 1) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1143]; }
    { const long long ij = ij_5_1, kl = kl_4_4;
      if ((!dab || 5 >= 1) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1144]; }
    { const long long ij = ij_5_1, kl = kl_4_5;
      if ((!dab || 5 >= 1) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1145]; }
    { const long long ij = ij_5_1, kl = kl_5_0;
      if ((!dab || 5 >= 1) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1146]; }
    { const long long ij = ij_5_1, kl = kl_5_1;
      if ((!dab || 5 >= 1) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1147]; }
    { const long long ij = ij_5_1, kl = kl_5_2;
      if ((!dab || 5 >= 1) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1148]; }
    { const long long ij = ij_5_1, kl = kl_5_3;
      if ((!dab || 5 >= 1) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1149]; }
    { const long long ij = ij_5_1, kl = kl_5_4;
      if ((!dab || 5 >= 1) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1150]; }
    { const long long ij = ij_5_1, kl = kl_5_5;
      if ((!dab || 5 >= 1) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1151]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1152]; }
    { const long long ij = ij_5_2, kl = kl_0_1;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1153]; }
    { const long long ij = ij_5_2, kl = kl_0_2;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1154]; }
    { const long long ij = ij_5_2, kl = kl_0_3;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1155]; }
    { const long long ij = ij_5_2, kl = kl_0_4;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1156]; }
    { const long long ij = ij_5_2, kl = kl_0_5;
      if ((!dab || 5 >= 2) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1157]; }
    { const long long ij = ij_5_2, kl = kl_1_0;
      if ((!dab || 5 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1158]; }
    { const long long ij = ij_5_2, kl = kl_1_1;
      if ((!dab || 5 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1159]; }
    { const long long ij = ij_5_2, kl = kl_1_2;
      if ((!dab || 5 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1160]; }
    { const long long ij = ij_5_2, kl = kl_1_3;
      if ((!dab || 5 >= 2) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1161]; }
    { const long long ij = ij_5_2, kl = kl_1_4;
      if ((!dab || 5 >= 2) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1162]; }
    { const long long ij = ij_5_2, kl = kl_1_5;
      if ((!dab || 5 >= 2) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1163]; }
    { const long long ij = ij_5_2, kl = kl_2_0;
      if ((!dab || 5 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1164]; }
    { const long long ij = ij_5_2, kl = kl_2_1;
      if ((!dab || 5 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1165]; }
    { const long long ij = ij_5_2, kl = kl_2_2;
      if ((!dab || 5 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1166]; }
    { const long long ij = ij_5_2, kl = kl_2_3;
      if ((!dab || 5 >= 2) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1167]; }
    { const long long ij = ij_5_2, kl = kl_2_4;
      if ((!dab || 5 >= 2) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1168]; }
    { const long long ij = ij_5_2, kl = kl_2_5;
      if ((!dab || 5 >= 2) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1169]; }
    { const long long ij = ij_5_2, kl = kl_3_0;
      if ((!dab || 5 >= 2) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1170]; }
    { const long long ij = ij_5_2, kl = kl_3_1;
      if ((!dab || 5 >= 2) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1171]; }
    { const long long ij = ij_5_2, kl = kl_3_2;
      if ((!dab || 5 >= 2) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1172]; }
    { const long long ij = ij_5_2, kl = kl_3_3;
      if ((!dab || 5 >= 2) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1173]; }
    { const long long ij = ij_5_2, kl = kl_3_4;
      if ((!dab || 5 >= 2) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1174]; }
    { const long long ij = ij_5_2, kl = kl_3_5;
      if ((!dab || 5 >= 2) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1175]; }
    { const long long ij = ij_5_2, kl = kl_4_0;
      if ((!dab || 5 >= 2) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1176]; }
    { const long long ij = ij_5_2, kl = kl_4_1;
      if ((!dab || 5 >= 2) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1177]; }
    { const long long ij = ij_5_2, kl = kl_4_2;
      if ((!dab || 5 >= 2) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1178]; }
    { const long long ij = ij_5_2, kl = kl_4_3;
      if ((!dab || 5 >= 2) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1179]; }
    { const long long ij = ij_5_2, kl = kl_4_4;
      if ((!dab || 5 >= 2) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1180]; }
    { const long long ij = ij_5_2, kl = kl_4_5;
      if ((!dab || 5 >= 2) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1181]; }
    { const long long ij = ij_5_2, kl = kl_5_0;
      if ((!dab || 5 >= 2) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1182]; }
    { const long long ij = ij_5_2, kl = kl_5_1;
      if ((!dab || 5 >= 2) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1183]; }
    { const long long ij = ij_5_2, kl = kl_5_2;
      if ((!dab || 5 >= 2) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1184]; }
    { const long long ij = ij_5_2, kl = kl_5_3;
      if ((!dab || 5 >= 2) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1185]; }
    { const long long ij = ij_5_2, kl = kl_5_4;
      if ((!dab || 5 >= 2) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1186]; }
    { const long long ij = ij_5_2, kl = kl_5_5;
      if ((!dab || 5 >= 2) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1187]; }
    { const long long ij = ij_5_3, kl = kl_0_0;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1188]; }
    { const long long ij = ij_5_3, kl = kl_0_1;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1189]; }
    { const long long ij = ij_5_3, kl = kl_0_2;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1190]; }
    { const long long ij = ij_5_3, kl = kl_0_3;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1191]; }
    { const long long ij = ij_5_3, kl = kl_0_4;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1192]; }
    { const long long ij = ij_5_3, kl = kl_0_5;
      if ((!dab || 5 >= 3) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1193]; }
    { const long long ij = ij_5_3, kl = kl_1_0;
      if ((!dab || 5 >= 3) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1194]; }
    { const long long ij = ij_5_3, kl = kl_1_1;
      if ((!dab || 5 >= 3) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1195]; }
    { const long long ij = ij_5_3, kl = kl_1_2;
      if ((!dab || 5 >= 3) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1196]; }
    { const long long ij = ij_5_3, kl = kl_1_3;
      if ((!dab || 5 >= 3) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1197]; }
    { const long long ij = ij_5_3, kl = kl_1_4;
      if ((!dab || 5 >= 3) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1198]; }
    { const long long ij = ij_5_3, kl = kl_1_5;
      if ((!dab || 5 >= 3) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1199]; }
    { const long long ij = ij_5_3, kl = kl_2_0;
      if ((!dab || 5 >= 3) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1200]; }
    { const long long ij = ij_5_3, kl = kl_2_1;
      if ((!dab || 5 >= 3) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1201]; }
    { const long long ij = ij_5_3, kl = kl_2_2;
      if ((!dab || 5 >= 3) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1202]; }
    { const long long ij = ij_5_3, kl = kl_2_3;
      if ((!dab || 5 >= 3) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1203]; }
    { const long long ij = ij_5_3, kl = kl_2_4;
      if ((!dab || 5 >= 3) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1204]; }
    { const long long ij = ij_5_3, kl = kl_2_5;
      if ((!dab || 5 >= 3) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1205]; }
    { const long long ij = ij_5_3, kl = kl_3_0;
      if ((!dab || 5 >= 3) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1206]; }
    { const long long ij = ij_5_3, kl = kl_3_1;
      if ((!dab || 5 >= 3) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1207]; }
    { const long long ij = ij_5_3, kl = kl_3_2;
      if ((!dab || 5 >= 3) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1208]; }
    { const long long ij = ij_5_3, kl = kl_3_3;
      if ((!dab || 5 >= 3) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1209]; }
    { const long long ij = ij_5_3, kl = kl_3_4;
      if ((!dab || 5 >= 3) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1210]; }
    { const long long ij = ij_5_3, kl = kl_3_5;
      if ((!dab || 5 >= 3) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1211]; }
    { const long long ij = ij_5_3, kl = kl_4_0;
      if ((!dab || 5 >= 3) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1212]; }
    { const long long ij = ij_5_3, kl = kl_4_1;
      if ((!dab || 5 >= 3) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1213]; }
    { const long long ij = ij_5_3, kl = kl_4_2;
      if ((!dab || 5 >= 3) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1214]; }
    { const long long ij = ij_5_3, kl = kl_4_3;
      if ((!dab || 5 >= 3) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1215]; }
    { const long long ij = ij_5_3, kl = kl_4_4;
      if ((!dab || 5 >= 3) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1216]; }
    { const long long ij = ij_5_3, kl = kl_4_5;
      if ((!dab || 5 >= 3) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1217]; }
    { const long long ij = ij_5_3, kl = kl_5_0;
      if ((!dab || 5 >= 3) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1218]; }
    { const long long ij = ij_5_3, kl = kl_5_1;
      if ((!dab || 5 >= 3) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1219]; }
    { const long long ij = ij_5_3, kl = kl_5_2;
      if ((!dab || 5 >= 3) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1220]; }
    { const long long ij = ij_5_3, kl = kl_5_3;
      if ((!dab || 5 >= 3) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1221]; }
    { const long long ij = ij_5_3, kl = kl_5_4;
      if ((!dab || 5 >= 3) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1222]; }
    { const long long ij = ij_5_3, kl = kl_5_5;
      if ((!dab || 5 >= 3) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1223]; }
    { const long long ij = ij_5_4, kl = kl_0_0;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1224]; }
    { const long long ij = ij_5_4, kl = kl_0_1;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1225]; }
    { const long long ij = ij_5_4, kl = kl_0_2;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1226]; }
    { const long long ij = ij_5_4, kl = kl_0_3;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1227]; }
    { const long long ij = ij_5_4, kl = kl_0_4;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1228]; }
    { const long long ij = ij_5_4, kl = kl_0_5;
      if ((!dab || 5 >= 4) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1229]; }
    { const long long ij = ij_5_4, kl = kl_1_0;
      if ((!dab || 5 >= 4) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1230]; }
    { const long long ij = ij_5_4, kl = kl_1_1;
      if ((!dab || 5 >= 4) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1231]; }
    { const long long ij = ij_5_4, kl = kl_1_2;
      if ((!dab || 5 >= 4) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1232]; }
    { const long long ij = ij_5_4, kl = kl_1_3;
      if ((!dab || 5 >= 4) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1233]; }
    { const long long ij = ij_5_4, kl = kl_1_4;
      if ((!dab || 5 >= 4) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1234]; }
    { const long long ij = ij_5_4, kl = kl_1_5;
      if ((!dab || 5 >= 4) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1235]; }
    { const long long ij = ij_5_4, kl = kl_2_0;
      if ((!dab || 5 >= 4) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1236]; }
    { const long long ij = ij_5_4, kl = kl_2_1;
      if ((!dab || 5 >= 4) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1237]; }
    { const long long ij = ij_5_4, kl = kl_2_2;
      if ((!dab || 5 >= 4) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1238]; }
    { const long long ij = ij_5_4, kl = kl_2_3;
      if ((!dab || 5 >= 4) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1239]; }
    { const long long ij = ij_5_4, kl = kl_2_4;
      if ((!dab || 5 >= 4) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1240]; }
    { const long long ij = ij_5_4, kl = kl_2_5;
      if ((!dab || 5 >= 4) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1241]; }
    { const long long ij = ij_5_4, kl = kl_3_0;
      if ((!dab || 5 >= 4) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1242]; }
    { const long long ij = ij_5_4, kl = kl_3_1;
      if ((!dab || 5 >= 4) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1243]; }
    { const long long ij = ij_5_4, kl = kl_3_2;
      if ((!dab || 5 >= 4) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1244]; }
    { const long long ij = ij_5_4, kl = kl_3_3;
      if ((!dab || 5 >= 4) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1245]; }
    { const long long ij = ij_5_4, kl = kl_3_4;
      if ((!dab || 5 >= 4) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1246]; }
    { const long long ij = ij_5_4, kl = kl_3_5;
      if ((!dab || 5 >= 4) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1247]; }
    { const long long ij = ij_5_4, kl = kl_4_0;
      if ((!dab || 5 >= 4) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1248]; }
    { const long long ij = ij_5_4, kl = kl_4_1;
      if ((!dab || 5 >= 4) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1249]; }
    { const long long ij = ij_5_4, kl = kl_4_2;
      if ((!dab || 5 >= 4) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1250]; }
    { const long long ij = ij_5_4, kl = kl_4_3;
      if ((!dab || 5 >= 4) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1251]; }
    { const long long ij = ij_5_4, kl = kl_4_4;
      if ((!dab || 5 >= 4) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1252]; }
    { const long long ij = ij_5_4, kl = kl_4_5;
      if ((!dab || 5 >= 4) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1253]; }
    { const long long ij = ij_5_4, kl = kl_5_0;
      if ((!dab || 5 >= 4) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1254]; }
    { const long long ij = ij_5_4, kl = kl_5_1;
      if ((!dab || 5 >= 4) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1255]; }
    { const long long ij = ij_5_4, kl = kl_5_2;
      if ((!dab || 5 >= 4) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1256]; }
    { const long long ij = ij_5_4, kl = kl_5_3;
      if ((!dab || 5 >= 4) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1257]; }
    { const long long ij = ij_5_4, kl = kl_5_4;
      if ((!dab || 5 >= 4) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1258]; }
    { const long long ij = ij_5_4, kl = kl_5_5;
      if ((!dab || 5 >= 4) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1259]; }
    { const long long ij = ij_5_5, kl = kl_0_0;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1260]; }
    { const long long ij = ij_5_5, kl = kl_0_1;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1261]; }
    { const long long ij = ij_5_5, kl = kl_0_2;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1262]; }
    { const long long ij = ij_5_5, kl = kl_0_3;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1263]; }
    { const long long ij = ij_5_5, kl = kl_0_4;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1264]; }
    { const long long ij = ij_5_5, kl = kl_0_5;
      if ((!dab || 5 >= 5) && (!dcd || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1265]; }
    { const long long ij = ij_5_5, kl = kl_1_0;
      if ((!dab || 5 >= 5) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1266]; }
    { const long long ij = ij_5_5, kl = kl_1_1;
      if ((!dab || 5 >= 5) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1267]; }
    { const long long ij = ij_5_5, kl = kl_1_2;
      if ((!dab || 5 >= 5) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1268]; }
    { const long long ij = ij_5_5, kl = kl_1_3;
      if ((!dab || 5 >= 5) && (!dcd || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1269]; }
    { const long long ij = ij_5_5, kl = kl_1_4;
      if ((!dab || 5 >= 5) && (!dcd || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1270]; }
    { const long long ij = ij_5_5, kl = kl_1_5;
      if ((!dab || 5 >= 5) && (!dcd || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1271]; }
    { const long long ij = ij_5_5, kl = kl_2_0;
      if ((!dab || 5 >= 5) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1272]; }
    { const long long ij = ij_5_5, kl = kl_2_1;
      if ((!dab || 5 >= 5) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1273]; }
    { const long long ij = ij_5_5, kl = kl_2_2;
      if ((!dab || 5 >= 5) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1274]; }
    { const long long ij = ij_5_5, kl = kl_2_3;
      if ((!dab || 5 >= 5) && (!dcd || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1275]; }
    { const long long ij = ij_5_5, kl = kl_2_4;
      if ((!dab || 5 >= 5) && (!dcd || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1276]; }
    { const long long ij = ij_5_5, kl = kl_2_5;
      if ((!dab || 5 >= 5) && (!dcd || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1277]; }
    { const long long ij = ij_5_5, kl = kl_3_0;
      if ((!dab || 5 >= 5) && (!dcd || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1278]; }
    { const long long ij = ij_5_5, kl = kl_3_1;
      if ((!dab || 5 >= 5) && (!dcd || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1279]; }
    { const long long ij = ij_5_5, kl = kl_3_2;
      if ((!dab || 5 >= 5) && (!dcd || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1280]; }
    { const long long ij = ij_5_5, kl = kl_3_3;
      if ((!dab || 5 >= 5) && (!dcd || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1281]; }
    { const long long ij = ij_5_5, kl = kl_3_4;
      if ((!dab || 5 >= 5) && (!dcd || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1282]; }
    { const long long ij = ij_5_5, kl = kl_3_5;
      if ((!dab || 5 >= 5) && (!dcd || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1283]; }
    { const long long ij = ij_5_5, kl = kl_4_0;
      if ((!dab || 5 >= 5) && (!dcd || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1284]; }
    { const long long ij = ij_5_5, kl = kl_4_1;
      if ((!dab || 5 >= 5) && (!dcd || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1285]; }
    { const long long ij = ij_5_5, kl = kl_4_2;
      if ((!dab || 5 >= 5) && (!dcd || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1286]; }
    { const long long ij = ij_5_5, kl = kl_4_3;
      if ((!dab || 5 >= 5) && (!dcd || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1287]; }
    { const long long ij = ij_5_5, kl = kl_4_4;
      if ((!dab || 5 >= 5) && (!dcd || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1288]; }
    { const long long ij = ij_5_5, kl = kl_4_5;
      if ((!dab || 5 >= 5) && (!dcd || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1289]; }
    { const long long ij = ij_5_5, kl = kl_5_0;
      if ((!dab || 5 >= 5) && (!dcd || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1290]; }
    { const long long ij = ij_5_5, kl = kl_5_1;
      if ((!dab || 5 >= 5) && (!dcd || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1291]; }
    { const long long ij = ij_5_5, kl = kl_5_2;
      if ((!dab || 5 >= 5) && (!dcd || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1292]; }
    { const long long ij = ij_5_5, kl = kl_5_3;
      if ((!dab || 5 >= 5) && (!dcd || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1293]; }
    { const long long ij = ij_5_5, kl = kl_5_4;
      if ((!dab || 5 >= 5) && (!dcd || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1294]; }
    { const long long ij = ij_5_5, kl = kl_5_5;
      if ((!dab || 5 >= 5) && (!dcd || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1295]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_dddd(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 1296; ++x) {
        const int ia = x / 216, ibb = (x / 36) % 6, ic = (x / 6) % 6, id = x % 6;
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
__global__ void __launch_bounds__(128) eri_queue_dddd(const EriQueue Q) {
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
        double acc[961];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 961; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_dddd<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_dddd<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 961; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: each leader stores its quartet's whole block at its slot
            if (lead) {
                double res[1296];
                hrr_dddd(Q.pairs, p, q, acc, res);
                double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                    (__ldg(&Q.chunk_slot[c]) + base + kq) * (long long)1296;
#pragma unroll
                for (int x = 0; x < 1296; ++x) dst[x] = res[x];
            }
        } else if (lead) {
            double res[1296];
            hrr_dddd(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_dddd(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_dddd(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_dddd(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    constexpr size_t smem = 0;
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_dddd<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_dddd<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_dddd<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_dddd<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_dddd(int mixed) {

    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dddd<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dddd<0, 0>, 128, 0);
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
__global__ void __launch_bounds__(128) schwarz_kernel_dddd(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[1296];
    if (full) {
        quartet_dddd<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[37]));
    m = fmax(m, fabs(res[74]));
    m = fmax(m, fabs(res[111]));
    m = fmax(m, fabs(res[148]));
    m = fmax(m, fabs(res[185]));
    m = fmax(m, fabs(res[222]));
    m = fmax(m, fabs(res[259]));
    m = fmax(m, fabs(res[296]));
    m = fmax(m, fabs(res[333]));
    m = fmax(m, fabs(res[370]));
    m = fmax(m, fabs(res[407]));
    m = fmax(m, fabs(res[444]));
    m = fmax(m, fabs(res[481]));
    m = fmax(m, fabs(res[518]));
    m = fmax(m, fabs(res[555]));
    m = fmax(m, fabs(res[592]));
    m = fmax(m, fabs(res[629]));
    m = fmax(m, fabs(res[666]));
    m = fmax(m, fabs(res[703]));
    m = fmax(m, fabs(res[740]));
    m = fmax(m, fabs(res[777]));
    m = fmax(m, fabs(res[814]));
    m = fmax(m, fabs(res[851]));
    m = fmax(m, fabs(res[888]));
    m = fmax(m, fabs(res[925]));
    m = fmax(m, fabs(res[962]));
    m = fmax(m, fabs(res[999]));
    m = fmax(m, fabs(res[1036]));
    m = fmax(m, fabs(res[1073]));
    m = fmax(m, fabs(res[1110]));
    m = fmax(m, fabs(res[1147]));
    m = fmax(m, fabs(res[1184]));
    m = fmax(m, fabs(res[1221]));
    m = fmax(m, fabs(res[1258]));
    m = fmax(m, fabs(res[1295]));
        qout[p] = sqrt(m);
        return;
    }
    double acc[961];
    for (int k = 0; k < in.y; ++k) {
        quartet_dddd<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[37]));
    m = fmax(m, fabs(res[74]));
    m = fmax(m, fabs(res[111]));
    m = fmax(m, fabs(res[148]));
    m = fmax(m, fabs(res[185]));
    m = fmax(m, fabs(res[222]));
    m = fmax(m, fabs(res[259]));
    m = fmax(m, fabs(res[296]));
    m = fmax(m, fabs(res[333]));
    m = fmax(m, fabs(res[370]));
    m = fmax(m, fabs(res[407]));
    m = fmax(m, fabs(res[444]));
    m = fmax(m, fabs(res[481]));
    m = fmax(m, fabs(res[518]));
    m = fmax(m, fabs(res[555]));
    m = fmax(m, fabs(res[592]));
    m = fmax(m, fabs(res[629]));
    m = fmax(m, fabs(res[666]));
    m = fmax(m, fabs(res[703]));
    m = fmax(m, fabs(res[740]));
    m = fmax(m, fabs(res[777]));
    m = fmax(m, fabs(res[814]));
    m = fmax(m, fabs(res[851]));
    m = fmax(m, fabs(res[888]));
    m = fmax(m, fabs(res[925]));
    m = fmax(m, fabs(res[962]));
    m = fmax(m, fabs(res[999]));
    m = fmax(m, fabs(res[1036]));
    m = fmax(m, fabs(res[1073]));
    m = fmax(m, fabs(res[1110]));
    m = fmax(m, fabs(res[1147]));
    m = fmax(m, fabs(res[1184]));
    m = fmax(m, fabs(res[1221]));
    m = fmax(m, fabs(res[1258]));
    m = fmax(m, fabs(res[1295]));
        w = fmax(w, fabs(acc[0]));
        w = fmax(w, fabs(acc[32]));
        w = fmax(w, fabs(acc[64]));
        w = fmax(w, fabs(acc[96]));
        w = fmax(w, fabs(acc[128]));
        w = fmax(w, fabs(acc[160]));
        w = fmax(w, fabs(acc[192]));
        w = fmax(w, fabs(acc[224]));
        w = fmax(w, fabs(acc[256]));
        w = fmax(w, fabs(acc[288]));
        w = fmax(w, fabs(acc[320]));
        w = fmax(w, fabs(acc[352]));
        w = fmax(w, fabs(acc[384]));
        w = fmax(w, fabs(acc[416]));
        w = fmax(w, fabs(acc[448]));
        w = fmax(w, fabs(acc[480]));
        w = fmax(w, fabs(acc[512]));
        w = fmax(w, fabs(acc[544]));
        w = fmax(w, fabs(acc[576]));
        w = fmax(w, fabs(acc[608]));
        w = fmax(w, fabs(acc[640]));
        w = fmax(w, fabs(acc[672]));
        w = fmax(w, fabs(acc[704]));
        w = fmax(w, fabs(acc[736]));
        w = fmax(w, fabs(acc[768]));
        w = fmax(w, fabs(acc[800]));
        w = fmax(w, fabs(acc[832]));
        w = fmax(w, fabs(acc[864]));
        w = fmax(w, fabs(acc[896]));
        w = fmax(w, fabs(acc[928]));
        w = fmax(w, fabs(acc[960]));
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }
}

void launch_schwarz_dddd(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    schwarz_kernel_dddd<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}

}  // namespace molints

// Generated by gen_eri.py -- class (fd|ps).  Do not edit.
// VRR entries: 320, contracted block: 138, HRR lines: 387, outputs: 180.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[138], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_fdps(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 138; ++x) acc[x] = 0.0;
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
            const VT v35_1_0 = QCx * v35_0_0 + WQx * v35_0_1 + (VT)5.0 * oo2ze * v20_0_1;
            const VT v36_1_0 = QCx * v36_0_0 + WQx * v36_0_1 + (VT)4.0 * oo2ze * v21_0_1;
            const VT v37_1_0 = QCx * v37_0_0 + WQx * v37_0_1 + (VT)4.0 * oo2ze * v22_0_1;
            const VT v38_1_0 = QCx * v38_0_0 + WQx * v38_0_1 + (VT)3.0 * oo2ze * v23_0_1;
            const VT v39_1_0 = QCx * v39_0_0 + WQx * v39_0_1 + (VT)3.0 * oo2ze * v24_0_1;
            const VT v40_1_0 = QCx * v40_0_0 + WQx * v40_0_1 + (VT)3.0 * oo2ze * v25_0_1;
            const VT v41_1_0 = QCx * v41_0_0 + WQx * v41_0_1 + (VT)2.0 * oo2ze * v26_0_1;
            const VT v42_1_0 = QCx * v42_0_0 + WQx * v42_0_1 + (VT)2.0 * oo2ze * v27_0_1;
            const VT v43_1_0 = QCx * v43_0_0 + WQx * v43_0_1 + (VT)2.0 * oo2ze * v28_0_1;
            const VT v44_1_0 = QCx * v44_0_0 + WQx * v44_0_1 + (VT)2.0 * oo2ze * v29_0_1;
            const VT v45_1_0 = QCx * v45_0_0 + WQx * v45_0_1 + (VT)1.0 * oo2ze * v30_0_1;
            const VT v46_1_0 = QCx * v46_0_0 + WQx * v46_0_1 + (VT)1.0 * oo2ze * v31_0_1;
            const VT v47_1_0 = QCx * v47_0_0 + WQx * v47_0_1 + (VT)1.0 * oo2ze * v32_0_1;
            const VT v48_1_0 = QCx * v48_0_0 + WQx * v48_0_1 + (VT)1.0 * oo2ze * v33_0_1;
            const VT v49_1_0 = QCx * v49_0_0 + WQx * v49_0_1 + (VT)1.0 * oo2ze * v34_0_1;
            const VT v50_1_0 = QCx * v50_0_0 + WQx * v50_0_1;
            const VT v51_1_0 = QCx * v51_0_0 + WQx * v51_0_1;
            const VT v52_1_0 = QCx * v52_0_0 + WQx * v52_0_1;
            const VT v53_1_0 = QCx * v53_0_0 + WQx * v53_0_1;
            const VT v54_1_0 = QCx * v54_0_0 + WQx * v54_0_1;
            const VT v55_1_0 = QCx * v55_0_0 + WQx * v55_0_1;
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
            const VT v35_2_0 = QCy * v35_0_0 + WQy * v35_0_1;
            const VT v36_2_0 = QCy * v36_0_0 + WQy * v36_0_1 + (VT)1.0 * oo2ze * v20_0_1;
            const VT v37_2_0 = QCy * v37_0_0 + WQy * v37_0_1;
            const VT v38_2_0 = QCy * v38_0_0 + WQy * v38_0_1 + (VT)2.0 * oo2ze * v21_0_1;
            const VT v39_2_0 = QCy * v39_0_0 + WQy * v39_0_1 + (VT)1.0 * oo2ze * v22_0_1;
            const VT v40_2_0 = QCy * v40_0_0 + WQy * v40_0_1;
            const VT v41_2_0 = QCy * v41_0_0 + WQy * v41_0_1 + (VT)3.0 * oo2ze * v23_0_1;
            const VT v42_2_0 = QCy * v42_0_0 + WQy * v42_0_1 + (VT)2.0 * oo2ze * v24_0_1;
            const VT v43_2_0 = QCy * v43_0_0 + WQy * v43_0_1 + (VT)1.0 * oo2ze * v25_0_1;
            const VT v44_2_0 = QCy * v44_0_0 + WQy * v44_0_1;
            const VT v45_2_0 = QCy * v45_0_0 + WQy * v45_0_1 + (VT)4.0 * oo2ze * v26_0_1;
            const VT v46_2_0 = QCy * v46_0_0 + WQy * v46_0_1 + (VT)3.0 * oo2ze * v27_0_1;
            const VT v47_2_0 = QCy * v47_0_0 + WQy * v47_0_1 + (VT)2.0 * oo2ze * v28_0_1;
            const VT v48_2_0 = QCy * v48_0_0 + WQy * v48_0_1 + (VT)1.0 * oo2ze * v29_0_1;
            const VT v49_2_0 = QCy * v49_0_0 + WQy * v49_0_1;
            const VT v50_2_0 = QCy * v50_0_0 + WQy * v50_0_1 + (VT)5.0 * oo2ze * v30_0_1;
            const VT v51_2_0 = QCy * v51_0_0 + WQy * v51_0_1 + (VT)4.0 * oo2ze * v31_0_1;
            const VT v52_2_0 = QCy * v52_0_0 + WQy * v52_0_1 + (VT)3.0 * oo2ze * v32_0_1;
            const VT v53_2_0 = QCy * v53_0_0 + WQy * v53_0_1 + (VT)2.0 * oo2ze * v33_0_1;
            const VT v54_2_0 = QCy * v54_0_0 + WQy * v54_0_1 + (VT)1.0 * oo2ze * v34_0_1;
            const VT v55_2_0 = QCy * v55_0_0 + WQy * v55_0_1;
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
            const VT v35_3_0 = QCz * v35_0_0 + WQz * v35_0_1;
            const VT v36_3_0 = QCz * v36_0_0 + WQz * v36_0_1;
            const VT v37_3_0 = QCz * v37_0_0 + WQz * v37_0_1 + (VT)1.0 * oo2ze * v20_0_1;
            const VT v38_3_0 = QCz * v38_0_0 + WQz * v38_0_1;
            const VT v39_3_0 = QCz * v39_0_0 + WQz * v39_0_1 + (VT)1.0 * oo2ze * v21_0_1;
            const VT v40_3_0 = QCz * v40_0_0 + WQz * v40_0_1 + (VT)2.0 * oo2ze * v22_0_1;
            const VT v41_3_0 = QCz * v41_0_0 + WQz * v41_0_1;
            const VT v42_3_0 = QCz * v42_0_0 + WQz * v42_0_1 + (VT)1.0 * oo2ze * v23_0_1;
            const VT v43_3_0 = QCz * v43_0_0 + WQz * v43_0_1 + (VT)2.0 * oo2ze * v24_0_1;
            const VT v44_3_0 = QCz * v44_0_0 + WQz * v44_0_1 + (VT)3.0 * oo2ze * v25_0_1;
            const VT v45_3_0 = QCz * v45_0_0 + WQz * v45_0_1;
            const VT v46_3_0 = QCz * v46_0_0 + WQz * v46_0_1 + (VT)1.0 * oo2ze * v26_0_1;
            const VT v47_3_0 = QCz * v47_0_0 + WQz * v47_0_1 + (VT)2.0 * oo2ze * v27_0_1;
            const VT v48_3_0 = QCz * v48_0_0 + WQz * v48_0_1 + (VT)3.0 * oo2ze * v28_0_1;
            const VT v49_3_0 = QCz * v49_0_0 + WQz * v49_0_1 + (VT)4.0 * oo2ze * v29_0_1;
            const VT v50_3_0 = QCz * v50_0_0 + WQz * v50_0_1;
            const VT v51_3_0 = QCz * v51_0_0 + WQz * v51_0_1 + (VT)1.0 * oo2ze * v30_0_1;
            const VT v52_3_0 = QCz * v52_0_0 + WQz * v52_0_1 + (VT)2.0 * oo2ze * v31_0_1;
            const VT v53_3_0 = QCz * v53_0_0 + WQz * v53_0_1 + (VT)3.0 * oo2ze * v32_0_1;
            const VT v54_3_0 = QCz * v54_0_0 + WQz * v54_0_1 + (VT)4.0 * oo2ze * v33_0_1;
            const VT v55_3_0 = QCz * v55_0_0 + WQz * v55_0_1 + (VT)5.0 * oo2ze * v34_0_1;
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
            acc[75] += (double)v35_1_0;
            acc[76] += (double)v35_2_0;
            acc[77] += (double)v35_3_0;
            acc[78] += (double)v36_1_0;
            acc[79] += (double)v36_2_0;
            acc[80] += (double)v36_3_0;
            acc[81] += (double)v37_1_0;
            acc[82] += (double)v37_2_0;
            acc[83] += (double)v37_3_0;
            acc[84] += (double)v38_1_0;
            acc[85] += (double)v38_2_0;
            acc[86] += (double)v38_3_0;
            acc[87] += (double)v39_1_0;
            acc[88] += (double)v39_2_0;
            acc[89] += (double)v39_3_0;
            acc[90] += (double)v40_1_0;
            acc[91] += (double)v40_2_0;
            acc[92] += (double)v40_3_0;
            acc[93] += (double)v41_1_0;
            acc[94] += (double)v41_2_0;
            acc[95] += (double)v41_3_0;
            acc[96] += (double)v42_1_0;
            acc[97] += (double)v42_2_0;
            acc[98] += (double)v42_3_0;
            acc[99] += (double)v43_1_0;
            acc[100] += (double)v43_2_0;
            acc[101] += (double)v43_3_0;
            acc[102] += (double)v44_1_0;
            acc[103] += (double)v44_2_0;
            acc[104] += (double)v44_3_0;
            acc[105] += (double)v45_1_0;
            acc[106] += (double)v45_2_0;
            acc[107] += (double)v45_3_0;
            acc[108] += (double)v46_1_0;
            acc[109] += (double)v46_2_0;
            acc[110] += (double)v46_3_0;
            acc[111] += (double)v47_1_0;
            acc[112] += (double)v47_2_0;
            acc[113] += (double)v47_3_0;
            acc[114] += (double)v48_1_0;
            acc[115] += (double)v48_2_0;
            acc[116] += (double)v48_3_0;
            acc[117] += (double)v49_1_0;
            acc[118] += (double)v49_2_0;
            acc[119] += (double)v49_3_0;
            acc[120] += (double)v50_1_0;
            acc[121] += (double)v50_2_0;
            acc[122] += (double)v50_3_0;
            acc[123] += (double)v51_1_0;
            acc[124] += (double)v51_2_0;
            acc[125] += (double)v51_3_0;
            acc[126] += (double)v52_1_0;
            acc[127] += (double)v52_2_0;
            acc[128] += (double)v52_3_0;
            acc[129] += (double)v53_1_0;
            acc[130] += (double)v53_2_0;
            acc[131] += (double)v53_3_0;
            acc[132] += (double)v54_1_0;
            acc[133] += (double)v54_2_0;
            acc[134] += (double)v54_3_0;
            acc[135] += (double)v55_1_0;
            acc[136] += (double)v55_2_0;
            acc[137] += (double)v55_3_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[180] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_fdps(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h20_1_1 = acc[75] + ABx * acc[30];
    const double h10_1_1 = acc[30] + ABx * acc[0];
    const double h10_4_1 = h20_1_1 + ABx * h10_1_1;
    const double h20_1_2 = acc[76] + ABx * acc[31];
    const double h10_1_2 = acc[31] + ABx * acc[1];
    const double h10_4_2 = h20_1_2 + ABx * h10_1_2;
    const double h20_1_3 = acc[77] + ABx * acc[32];
    const double h10_1_3 = acc[32] + ABx * acc[2];
    const double h10_4_3 = h20_1_3 + ABx * h10_1_3;
    const double h20_2_1 = acc[78] + ABy * acc[30];
    const double h10_2_1 = acc[33] + ABy * acc[0];
    const double h10_5_1 = h20_2_1 + ABx * h10_2_1;
    const double h20_2_2 = acc[79] + ABy * acc[31];
    const double h10_2_2 = acc[34] + ABy * acc[1];
    const double h10_5_2 = h20_2_2 + ABx * h10_2_2;
    const double h20_2_3 = acc[80] + ABy * acc[32];
    const double h10_2_3 = acc[35] + ABy * acc[2];
    const double h10_5_3 = h20_2_3 + ABx * h10_2_3;
    const double h20_3_1 = acc[81] + ABz * acc[30];
    const double h10_3_1 = acc[36] + ABz * acc[0];
    const double h10_6_1 = h20_3_1 + ABx * h10_3_1;
    const double h20_3_2 = acc[82] + ABz * acc[31];
    const double h10_3_2 = acc[37] + ABz * acc[1];
    const double h10_6_2 = h20_3_2 + ABx * h10_3_2;
    const double h20_3_3 = acc[83] + ABz * acc[32];
    const double h10_3_3 = acc[38] + ABz * acc[2];
    const double h10_6_3 = h20_3_3 + ABx * h10_3_3;
    const double h21_2_1 = acc[84] + ABy * acc[33];
    const double h10_7_1 = h21_2_1 + ABy * h10_2_1;
    const double h21_2_2 = acc[85] + ABy * acc[34];
    const double h10_7_2 = h21_2_2 + ABy * h10_2_2;
    const double h21_2_3 = acc[86] + ABy * acc[35];
    const double h10_7_3 = h21_2_3 + ABy * h10_2_3;
    const double h21_3_1 = acc[87] + ABz * acc[33];
    const double h10_8_1 = h21_3_1 + ABy * h10_3_1;
    const double h21_3_2 = acc[88] + ABz * acc[34];
    const double h10_8_2 = h21_3_2 + ABy * h10_3_2;
    const double h21_3_3 = acc[89] + ABz * acc[35];
    const double h10_8_3 = h21_3_3 + ABy * h10_3_3;
    const double h22_3_1 = acc[90] + ABz * acc[36];
    const double h10_9_1 = h22_3_1 + ABz * h10_3_1;
    const double h22_3_2 = acc[91] + ABz * acc[37];
    const double h10_9_2 = h22_3_2 + ABz * h10_3_2;
    const double h22_3_3 = acc[92] + ABz * acc[38];
    const double h10_9_3 = h22_3_3 + ABz * h10_3_3;
    const double h21_1_1 = acc[78] + ABx * acc[33];
    const double h11_1_1 = acc[33] + ABx * acc[3];
    const double h11_4_1 = h21_1_1 + ABx * h11_1_1;
    const double h21_1_2 = acc[79] + ABx * acc[34];
    const double h11_1_2 = acc[34] + ABx * acc[4];
    const double h11_4_2 = h21_1_2 + ABx * h11_1_2;
    const double h21_1_3 = acc[80] + ABx * acc[35];
    const double h11_1_3 = acc[35] + ABx * acc[5];
    const double h11_4_3 = h21_1_3 + ABx * h11_1_3;
    const double h11_2_1 = acc[39] + ABy * acc[3];
    const double h11_5_1 = h21_2_1 + ABx * h11_2_1;
    const double h11_2_2 = acc[40] + ABy * acc[4];
    const double h11_5_2 = h21_2_2 + ABx * h11_2_2;
    const double h11_2_3 = acc[41] + ABy * acc[5];
    const double h11_5_3 = h21_2_3 + ABx * h11_2_3;
    const double h11_3_1 = acc[42] + ABz * acc[3];
    const double h11_6_1 = h21_3_1 + ABx * h11_3_1;
    const double h11_3_2 = acc[43] + ABz * acc[4];
    const double h11_6_2 = h21_3_2 + ABx * h11_3_2;
    const double h11_3_3 = acc[44] + ABz * acc[5];
    const double h11_6_3 = h21_3_3 + ABx * h11_3_3;
    const double h23_2_1 = acc[93] + ABy * acc[39];
    const double h11_7_1 = h23_2_1 + ABy * h11_2_1;
    const double h23_2_2 = acc[94] + ABy * acc[40];
    const double h11_7_2 = h23_2_2 + ABy * h11_2_2;
    const double h23_2_3 = acc[95] + ABy * acc[41];
    const double h11_7_3 = h23_2_3 + ABy * h11_2_3;
    const double h23_3_1 = acc[96] + ABz * acc[39];
    const double h11_8_1 = h23_3_1 + ABy * h11_3_1;
    const double h23_3_2 = acc[97] + ABz * acc[40];
    const double h11_8_2 = h23_3_2 + ABy * h11_3_2;
    const double h23_3_3 = acc[98] + ABz * acc[41];
    const double h11_8_3 = h23_3_3 + ABy * h11_3_3;
    const double h24_3_1 = acc[99] + ABz * acc[42];
    const double h11_9_1 = h24_3_1 + ABz * h11_3_1;
    const double h24_3_2 = acc[100] + ABz * acc[43];
    const double h11_9_2 = h24_3_2 + ABz * h11_3_2;
    const double h24_3_3 = acc[101] + ABz * acc[44];
    const double h11_9_3 = h24_3_3 + ABz * h11_3_3;
    const double h22_1_1 = acc[81] + ABx * acc[36];
    const double h12_1_1 = acc[36] + ABx * acc[6];
    const double h12_4_1 = h22_1_1 + ABx * h12_1_1;
    const double h22_1_2 = acc[82] + ABx * acc[37];
    const double h12_1_2 = acc[37] + ABx * acc[7];
    const double h12_4_2 = h22_1_2 + ABx * h12_1_2;
    const double h22_1_3 = acc[83] + ABx * acc[38];
    const double h12_1_3 = acc[38] + ABx * acc[8];
    const double h12_4_3 = h22_1_3 + ABx * h12_1_3;
    const double h22_2_1 = acc[87] + ABy * acc[36];
    const double h12_2_1 = acc[42] + ABy * acc[6];
    const double h12_5_1 = h22_2_1 + ABx * h12_2_1;
    const double h22_2_2 = acc[88] + ABy * acc[37];
    const double h12_2_2 = acc[43] + ABy * acc[7];
    const double h12_5_2 = h22_2_2 + ABx * h12_2_2;
    const double h22_2_3 = acc[89] + ABy * acc[38];
    const double h12_2_3 = acc[44] + ABy * acc[8];
    const double h12_5_3 = h22_2_3 + ABx * h12_2_3;
    const double h12_3_1 = acc[45] + ABz * acc[6];
    const double h12_6_1 = h22_3_1 + ABx * h12_3_1;
    const double h12_3_2 = acc[46] + ABz * acc[7];
    const double h12_6_2 = h22_3_2 + ABx * h12_3_2;
    const double h12_3_3 = acc[47] + ABz * acc[8];
    const double h12_6_3 = h22_3_3 + ABx * h12_3_3;
    const double h24_2_1 = acc[96] + ABy * acc[42];
    const double h12_7_1 = h24_2_1 + ABy * h12_2_1;
    const double h24_2_2 = acc[97] + ABy * acc[43];
    const double h12_7_2 = h24_2_2 + ABy * h12_2_2;
    const double h24_2_3 = acc[98] + ABy * acc[44];
    const double h12_7_3 = h24_2_3 + ABy * h12_2_3;
    const double h12_8_1 = h24_3_1 + ABy * h12_3_1;
    const double h12_8_2 = h24_3_2 + ABy * h12_3_2;
    const double h12_8_3 = h24_3_3 + ABy * h12_3_3;
    const double h25_3_1 = acc[102] + ABz * acc[45];
    const double h12_9_1 = h25_3_1 + ABz * h12_3_1;
    const double h25_3_2 = acc[103] + ABz * acc[46];
    const double h12_9_2 = h25_3_2 + ABz * h12_3_2;
    const double h25_3_3 = acc[104] + ABz * acc[47];
    const double h12_9_3 = h25_3_3 + ABz * h12_3_3;
    const double h23_1_1 = acc[84] + ABx * acc[39];
    const double h13_1_1 = acc[39] + ABx * acc[9];
    const double h13_4_1 = h23_1_1 + ABx * h13_1_1;
    const double h23_1_2 = acc[85] + ABx * acc[40];
    const double h13_1_2 = acc[40] + ABx * acc[10];
    const double h13_4_2 = h23_1_2 + ABx * h13_1_2;
    const double h23_1_3 = acc[86] + ABx * acc[41];
    const double h13_1_3 = acc[41] + ABx * acc[11];
    const double h13_4_3 = h23_1_3 + ABx * h13_1_3;
    const double h13_2_1 = acc[48] + ABy * acc[9];
    const double h13_5_1 = h23_2_1 + ABx * h13_2_1;
    const double h13_2_2 = acc[49] + ABy * acc[10];
    const double h13_5_2 = h23_2_2 + ABx * h13_2_2;
    const double h13_2_3 = acc[50] + ABy * acc[11];
    const double h13_5_3 = h23_2_3 + ABx * h13_2_3;
    const double h13_3_1 = acc[51] + ABz * acc[9];
    const double h13_6_1 = h23_3_1 + ABx * h13_3_1;
    const double h13_3_2 = acc[52] + ABz * acc[10];
    const double h13_6_2 = h23_3_2 + ABx * h13_3_2;
    const double h13_3_3 = acc[53] + ABz * acc[11];
    const double h13_6_3 = h23_3_3 + ABx * h13_3_3;
    const double h26_2_1 = acc[105] + ABy * acc[48];
    const double h13_7_1 = h26_2_1 + ABy * h13_2_1;
    const double h26_2_2 = acc[106] + ABy * acc[49];
    const double h13_7_2 = h26_2_2 + ABy * h13_2_2;
    const double h26_2_3 = acc[107] + ABy * acc[50];
    const double h13_7_3 = h26_2_3 + ABy * h13_2_3;
    const double h26_3_1 = acc[108] + ABz * acc[48];
    const double h13_8_1 = h26_3_1 + ABy * h13_3_1;
    const double h26_3_2 = acc[109] + ABz * acc[49];
    const double h13_8_2 = h26_3_2 + ABy * h13_3_2;
    const double h26_3_3 = acc[110] + ABz * acc[50];
    const double h13_8_3 = h26_3_3 + ABy * h13_3_3;
    const double h27_3_1 = acc[111] + ABz * acc[51];
    const double h13_9_1 = h27_3_1 + ABz * h13_3_1;
    const double h27_3_2 = acc[112] + ABz * acc[52];
    const double h13_9_2 = h27_3_2 + ABz * h13_3_2;
    const double h27_3_3 = acc[113] + ABz * acc[53];
    const double h13_9_3 = h27_3_3 + ABz * h13_3_3;
    const double h25_1_1 = acc[90] + ABx * acc[45];
    const double h14_1_1 = acc[45] + ABx * acc[12];
    const double h14_4_1 = h25_1_1 + ABx * h14_1_1;
    const double h25_1_2 = acc[91] + ABx * acc[46];
    const double h14_1_2 = acc[46] + ABx * acc[13];
    const double h14_4_2 = h25_1_2 + ABx * h14_1_2;
    const double h25_1_3 = acc[92] + ABx * acc[47];
    const double h14_1_3 = acc[47] + ABx * acc[14];
    const double h14_4_3 = h25_1_3 + ABx * h14_1_3;
    const double h25_2_1 = acc[99] + ABy * acc[45];
    const double h14_2_1 = acc[54] + ABy * acc[12];
    const double h14_5_1 = h25_2_1 + ABx * h14_2_1;
    const double h25_2_2 = acc[100] + ABy * acc[46];
    const double h14_2_2 = acc[55] + ABy * acc[13];
    const double h14_5_2 = h25_2_2 + ABx * h14_2_2;
    const double h25_2_3 = acc[101] + ABy * acc[47];
    const double h14_2_3 = acc[56] + ABy * acc[14];
    const double h14_5_3 = h25_2_3 + ABx * h14_2_3;
    const double h14_3_1 = acc[57] + ABz * acc[12];
    const double h14_6_1 = h25_3_1 + ABx * h14_3_1;
    const double h14_3_2 = acc[58] + ABz * acc[13];
    const double h14_6_2 = h25_3_2 + ABx * h14_3_2;
    const double h14_3_3 = acc[59] + ABz * acc[14];
    const double h14_6_3 = h25_3_3 + ABx * h14_3_3;
    const double h28_2_1 = acc[111] + ABy * acc[54];
    const double h14_7_1 = h28_2_1 + ABy * h14_2_1;
    const double h28_2_2 = acc[112] + ABy * acc[55];
    const double h14_7_2 = h28_2_2 + ABy * h14_2_2;
    const double h28_2_3 = acc[113] + ABy * acc[56];
    const double h14_7_3 = h28_2_3 + ABy * h14_2_3;
    const double h28_3_1 = acc[114] + ABz * acc[54];
    const double h14_8_1 = h28_3_1 + ABy * h14_3_1;
    const double h28_3_2 = acc[115] + ABz * acc[55];
    const double h14_8_2 = h28_3_2 + ABy * h14_3_2;
    const double h28_3_3 = acc[116] + ABz * acc[56];
    const double h14_8_3 = h28_3_3 + ABy * h14_3_3;
    const double h29_3_1 = acc[117] + ABz * acc[57];
    const double h14_9_1 = h29_3_1 + ABz * h14_3_1;
    const double h29_3_2 = acc[118] + ABz * acc[58];
    const double h14_9_2 = h29_3_2 + ABz * h14_3_2;
    const double h29_3_3 = acc[119] + ABz * acc[59];
    const double h14_9_3 = h29_3_3 + ABz * h14_3_3;
    const double h24_1_1 = acc[87] + ABx * acc[42];
    const double h15_1_1 = acc[42] + ABx * acc[15];
    const double h15_4_1 = h24_1_1 + ABx * h15_1_1;
    const double h24_1_2 = acc[88] + ABx * acc[43];
    const double h15_1_2 = acc[43] + ABx * acc[16];
    const double h15_4_2 = h24_1_2 + ABx * h15_1_2;
    const double h24_1_3 = acc[89] + ABx * acc[44];
    const double h15_1_3 = acc[44] + ABx * acc[17];
    const double h15_4_3 = h24_1_3 + ABx * h15_1_3;
    const double h15_2_1 = acc[51] + ABy * acc[15];
    const double h15_5_1 = h24_2_1 + ABx * h15_2_1;
    const double h15_2_2 = acc[52] + ABy * acc[16];
    const double h15_5_2 = h24_2_2 + ABx * h15_2_2;
    const double h15_2_3 = acc[53] + ABy * acc[17];
    const double h15_5_3 = h24_2_3 + ABx * h15_2_3;
    const double h15_3_1 = acc[54] + ABz * acc[15];
    const double h15_6_1 = h24_3_1 + ABx * h15_3_1;
    const double h15_3_2 = acc[55] + ABz * acc[16];
    const double h15_6_2 = h24_3_2 + ABx * h15_3_2;
    const double h15_3_3 = acc[56] + ABz * acc[17];
    const double h15_6_3 = h24_3_3 + ABx * h15_3_3;
    const double h27_2_1 = acc[108] + ABy * acc[51];
    const double h15_7_1 = h27_2_1 + ABy * h15_2_1;
    const double h27_2_2 = acc[109] + ABy * acc[52];
    const double h15_7_2 = h27_2_2 + ABy * h15_2_2;
    const double h27_2_3 = acc[110] + ABy * acc[53];
    const double h15_7_3 = h27_2_3 + ABy * h15_2_3;
    const double h15_8_1 = h27_3_1 + ABy * h15_3_1;
    const double h15_8_2 = h27_3_2 + ABy * h15_3_2;
    const double h15_8_3 = h27_3_3 + ABy * h15_3_3;
    const double h15_9_1 = h28_3_1 + ABz * h15_3_1;
    const double h15_9_2 = h28_3_2 + ABz * h15_3_2;
    const double h15_9_3 = h28_3_3 + ABz * h15_3_3;
    const double h26_1_1 = acc[93] + ABx * acc[48];
    const double h16_1_1 = acc[48] + ABx * acc[18];
    const double h16_4_1 = h26_1_1 + ABx * h16_1_1;
    const double h26_1_2 = acc[94] + ABx * acc[49];
    const double h16_1_2 = acc[49] + ABx * acc[19];
    const double h16_4_2 = h26_1_2 + ABx * h16_1_2;
    const double h26_1_3 = acc[95] + ABx * acc[50];
    const double h16_1_3 = acc[50] + ABx * acc[20];
    const double h16_4_3 = h26_1_3 + ABx * h16_1_3;
    const double h16_2_1 = acc[60] + ABy * acc[18];
    const double h16_5_1 = h26_2_1 + ABx * h16_2_1;
    const double h16_2_2 = acc[61] + ABy * acc[19];
    const double h16_5_2 = h26_2_2 + ABx * h16_2_2;
    const double h16_2_3 = acc[62] + ABy * acc[20];
    const double h16_5_3 = h26_2_3 + ABx * h16_2_3;
    const double h16_3_1 = acc[63] + ABz * acc[18];
    const double h16_6_1 = h26_3_1 + ABx * h16_3_1;
    const double h16_3_2 = acc[64] + ABz * acc[19];
    const double h16_6_2 = h26_3_2 + ABx * h16_3_2;
    const double h16_3_3 = acc[65] + ABz * acc[20];
    const double h16_6_3 = h26_3_3 + ABx * h16_3_3;
    const double h30_2_1 = acc[120] + ABy * acc[60];
    const double h16_7_1 = h30_2_1 + ABy * h16_2_1;
    const double h30_2_2 = acc[121] + ABy * acc[61];
    const double h16_7_2 = h30_2_2 + ABy * h16_2_2;
    const double h30_2_3 = acc[122] + ABy * acc[62];
    const double h16_7_3 = h30_2_3 + ABy * h16_2_3;
    const double h30_3_1 = acc[123] + ABz * acc[60];
    const double h16_8_1 = h30_3_1 + ABy * h16_3_1;
    const double h30_3_2 = acc[124] + ABz * acc[61];
    const double h16_8_2 = h30_3_2 + ABy * h16_3_2;
    const double h30_3_3 = acc[125] + ABz * acc[62];
    const double h16_8_3 = h30_3_3 + ABy * h16_3_3;
    const double h31_3_1 = acc[126] + ABz * acc[63];
    const double h16_9_1 = h31_3_1 + ABz * h16_3_1;
    const double h31_3_2 = acc[127] + ABz * acc[64];
    const double h16_9_2 = h31_3_2 + ABz * h16_3_2;
    const double h31_3_3 = acc[128] + ABz * acc[65];
    const double h16_9_3 = h31_3_3 + ABz * h16_3_3;
    const double h27_1_1 = acc[96] + ABx * acc[51];
    const double h17_1_1 = acc[51] + ABx * acc[21];
    const double h17_4_1 = h27_1_1 + ABx * h17_1_1;
    const double h27_1_2 = acc[97] + ABx * acc[52];
    const double h17_1_2 = acc[52] + ABx * acc[22];
    const double h17_4_2 = h27_1_2 + ABx * h17_1_2;
    const double h27_1_3 = acc[98] + ABx * acc[53];
    const double h17_1_3 = acc[53] + ABx * acc[23];
    const double h17_4_3 = h27_1_3 + ABx * h17_1_3;
    const double h17_2_1 = acc[63] + ABy * acc[21];
    const double h17_5_1 = h27_2_1 + ABx * h17_2_1;
    const double h17_2_2 = acc[64] + ABy * acc[22];
    const double h17_5_2 = h27_2_2 + ABx * h17_2_2;
    const double h17_2_3 = acc[65] + ABy * acc[23];
    const double h17_5_3 = h27_2_3 + ABx * h17_2_3;
    const double h17_3_1 = acc[66] + ABz * acc[21];
    const double h17_6_1 = h27_3_1 + ABx * h17_3_1;
    const double h17_3_2 = acc[67] + ABz * acc[22];
    const double h17_6_2 = h27_3_2 + ABx * h17_3_2;
    const double h17_3_3 = acc[68] + ABz * acc[23];
    const double h17_6_3 = h27_3_3 + ABx * h17_3_3;
    const double h31_2_1 = acc[123] + ABy * acc[63];
    const double h17_7_1 = h31_2_1 + ABy * h17_2_1;
    const double h31_2_2 = acc[124] + ABy * acc[64];
    const double h17_7_2 = h31_2_2 + ABy * h17_2_2;
    const double h31_2_3 = acc[125] + ABy * acc[65];
    const double h17_7_3 = h31_2_3 + ABy * h17_2_3;
    const double h17_8_1 = h31_3_1 + ABy * h17_3_1;
    const double h17_8_2 = h31_3_2 + ABy * h17_3_2;
    const double h17_8_3 = h31_3_3 + ABy * h17_3_3;
    const double h32_3_1 = acc[129] + ABz * acc[66];
    const double h17_9_1 = h32_3_1 + ABz * h17_3_1;
    const double h32_3_2 = acc[130] + ABz * acc[67];
    const double h17_9_2 = h32_3_2 + ABz * h17_3_2;
    const double h32_3_3 = acc[131] + ABz * acc[68];
    const double h17_9_3 = h32_3_3 + ABz * h17_3_3;
    const double h28_1_1 = acc[99] + ABx * acc[54];
    const double h18_1_1 = acc[54] + ABx * acc[24];
    const double h18_4_1 = h28_1_1 + ABx * h18_1_1;
    const double h28_1_2 = acc[100] + ABx * acc[55];
    const double h18_1_2 = acc[55] + ABx * acc[25];
    const double h18_4_2 = h28_1_2 + ABx * h18_1_2;
    const double h28_1_3 = acc[101] + ABx * acc[56];
    const double h18_1_3 = acc[56] + ABx * acc[26];
    const double h18_4_3 = h28_1_3 + ABx * h18_1_3;
    const double h18_2_1 = acc[66] + ABy * acc[24];
    const double h18_5_1 = h28_2_1 + ABx * h18_2_1;
    const double h18_2_2 = acc[67] + ABy * acc[25];
    const double h18_5_2 = h28_2_2 + ABx * h18_2_2;
    const double h18_2_3 = acc[68] + ABy * acc[26];
    const double h18_5_3 = h28_2_3 + ABx * h18_2_3;
    const double h18_3_1 = acc[69] + ABz * acc[24];
    const double h18_6_1 = h28_3_1 + ABx * h18_3_1;
    const double h18_3_2 = acc[70] + ABz * acc[25];
    const double h18_6_2 = h28_3_2 + ABx * h18_3_2;
    const double h18_3_3 = acc[71] + ABz * acc[26];
    const double h18_6_3 = h28_3_3 + ABx * h18_3_3;
    const double h32_2_1 = acc[126] + ABy * acc[66];
    const double h18_7_1 = h32_2_1 + ABy * h18_2_1;
    const double h32_2_2 = acc[127] + ABy * acc[67];
    const double h18_7_2 = h32_2_2 + ABy * h18_2_2;
    const double h32_2_3 = acc[128] + ABy * acc[68];
    const double h18_7_3 = h32_2_3 + ABy * h18_2_3;
    const double h18_8_1 = h32_3_1 + ABy * h18_3_1;
    const double h18_8_2 = h32_3_2 + ABy * h18_3_2;
    const double h18_8_3 = h32_3_3 + ABy * h18_3_3;
    const double h33_3_1 = acc[132] + ABz * acc[69];
    const double h18_9_1 = h33_3_1 + ABz * h18_3_1;
    const double h33_3_2 = acc[133] + ABz * acc[70];
    const double h18_9_2 = h33_3_2 + ABz * h18_3_2;
    const double h33_3_3 = acc[134] + ABz * acc[71];
    const double h18_9_3 = h33_3_3 + ABz * h18_3_3;
    const double h29_1_1 = acc[102] + ABx * acc[57];
    const double h19_1_1 = acc[57] + ABx * acc[27];
    const double h19_4_1 = h29_1_1 + ABx * h19_1_1;
    const double h29_1_2 = acc[103] + ABx * acc[58];
    const double h19_1_2 = acc[58] + ABx * acc[28];
    const double h19_4_2 = h29_1_2 + ABx * h19_1_2;
    const double h29_1_3 = acc[104] + ABx * acc[59];
    const double h19_1_3 = acc[59] + ABx * acc[29];
    const double h19_4_3 = h29_1_3 + ABx * h19_1_3;
    const double h29_2_1 = acc[114] + ABy * acc[57];
    const double h19_2_1 = acc[69] + ABy * acc[27];
    const double h19_5_1 = h29_2_1 + ABx * h19_2_1;
    const double h29_2_2 = acc[115] + ABy * acc[58];
    const double h19_2_2 = acc[70] + ABy * acc[28];
    const double h19_5_2 = h29_2_2 + ABx * h19_2_2;
    const double h29_2_3 = acc[116] + ABy * acc[59];
    const double h19_2_3 = acc[71] + ABy * acc[29];
    const double h19_5_3 = h29_2_3 + ABx * h19_2_3;
    const double h19_3_1 = acc[72] + ABz * acc[27];
    const double h19_6_1 = h29_3_1 + ABx * h19_3_1;
    const double h19_3_2 = acc[73] + ABz * acc[28];
    const double h19_6_2 = h29_3_2 + ABx * h19_3_2;
    const double h19_3_3 = acc[74] + ABz * acc[29];
    const double h19_6_3 = h29_3_3 + ABx * h19_3_3;
    const double h33_2_1 = acc[129] + ABy * acc[69];
    const double h19_7_1 = h33_2_1 + ABy * h19_2_1;
    const double h33_2_2 = acc[130] + ABy * acc[70];
    const double h19_7_2 = h33_2_2 + ABy * h19_2_2;
    const double h33_2_3 = acc[131] + ABy * acc[71];
    const double h19_7_3 = h33_2_3 + ABy * h19_2_3;
    const double h19_8_1 = h33_3_1 + ABy * h19_3_1;
    const double h19_8_2 = h33_3_2 + ABy * h19_3_2;
    const double h19_8_3 = h33_3_3 + ABy * h19_3_3;
    const double h34_3_1 = acc[135] + ABz * acc[72];
    const double h19_9_1 = h34_3_1 + ABz * h19_3_1;
    const double h34_3_2 = acc[136] + ABz * acc[73];
    const double h19_9_2 = h34_3_2 + ABz * h19_3_2;
    const double h34_3_3 = acc[137] + ABz * acc[74];
    const double h19_9_3 = h34_3_3 + ABz * h19_3_3;
    res[0] = h10_4_1 * 0.14907119849998599;
    res[1] = h10_4_2 * 0.14907119849998599;
    res[2] = h10_4_3 * 0.14907119849998599;
    res[3] = h10_5_1 * 0.2581988897471611;
    res[4] = h10_5_2 * 0.2581988897471611;
    res[5] = h10_5_3 * 0.2581988897471611;
    res[6] = h10_6_1 * 0.2581988897471611;
    res[7] = h10_6_2 * 0.2581988897471611;
    res[8] = h10_6_3 * 0.2581988897471611;
    res[9] = h10_7_1 * 0.14907119849998599;
    res[10] = h10_7_2 * 0.14907119849998599;
    res[11] = h10_7_3 * 0.14907119849998599;
    res[12] = h10_8_1 * 0.2581988897471611;
    res[13] = h10_8_2 * 0.2581988897471611;
    res[14] = h10_8_3 * 0.2581988897471611;
    res[15] = h10_9_1 * 0.14907119849998599;
    res[16] = h10_9_2 * 0.14907119849998599;
    res[17] = h10_9_3 * 0.14907119849998599;
    res[18] = h11_4_1 * 0.3333333333333334;
    res[19] = h11_4_2 * 0.3333333333333334;
    res[20] = h11_4_3 * 0.3333333333333334;
    res[21] = h11_5_1 * 0.5773502691896258;
    res[22] = h11_5_2 * 0.5773502691896258;
    res[23] = h11_5_3 * 0.5773502691896258;
    res[24] = h11_6_1 * 0.5773502691896258;
    res[25] = h11_6_2 * 0.5773502691896258;
    res[26] = h11_6_3 * 0.5773502691896258;
    res[27] = h11_7_1 * 0.3333333333333334;
    res[28] = h11_7_2 * 0.3333333333333334;
    res[29] = h11_7_3 * 0.3333333333333334;
    res[30] = h11_8_1 * 0.5773502691896258;
    res[31] = h11_8_2 * 0.5773502691896258;
    res[32] = h11_8_3 * 0.5773502691896258;
    res[33] = h11_9_1 * 0.3333333333333334;
    res[34] = h11_9_2 * 0.3333333333333334;
    res[35] = h11_9_3 * 0.3333333333333334;
    res[36] = h12_4_1 * 0.3333333333333334;
    res[37] = h12_4_2 * 0.3333333333333334;
    res[38] = h12_4_3 * 0.3333333333333334;
    res[39] = h12_5_1 * 0.5773502691896258;
    res[40] = h12_5_2 * 0.5773502691896258;
    res[41] = h12_5_3 * 0.5773502691896258;
    res[42] = h12_6_1 * 0.5773502691896258;
    res[43] = h12_6_2 * 0.5773502691896258;
    res[44] = h12_6_3 * 0.5773502691896258;
    res[45] = h12_7_1 * 0.3333333333333334;
    res[46] = h12_7_2 * 0.3333333333333334;
    res[47] = h12_7_3 * 0.3333333333333334;
    res[48] = h12_8_1 * 0.5773502691896258;
    res[49] = h12_8_2 * 0.5773502691896258;
    res[50] = h12_8_3 * 0.5773502691896258;
    res[51] = h12_9_1 * 0.3333333333333334;
    res[52] = h12_9_2 * 0.3333333333333334;
    res[53] = h12_9_3 * 0.3333333333333334;
    res[54] = h13_4_1 * 0.3333333333333334;
    res[55] = h13_4_2 * 0.3333333333333334;
    res[56] = h13_4_3 * 0.3333333333333334;
    res[57] = h13_5_1 * 0.5773502691896258;
    res[58] = h13_5_2 * 0.5773502691896258;
    res[59] = h13_5_3 * 0.5773502691896258;
    res[60] = h13_6_1 * 0.5773502691896258;
    res[61] = h13_6_2 * 0.5773502691896258;
    res[62] = h13_6_3 * 0.5773502691896258;
    res[63] = h13_7_1 * 0.3333333333333334;
    res[64] = h13_7_2 * 0.3333333333333334;
    res[65] = h13_7_3 * 0.3333333333333334;
    res[66] = h13_8_1 * 0.5773502691896258;
    res[67] = h13_8_2 * 0.5773502691896258;
    res[68] = h13_8_3 * 0.5773502691896258;
    res[69] = h13_9_1 * 0.3333333333333334;
    res[70] = h13_9_2 * 0.3333333333333334;
    res[71] = h13_9_3 * 0.3333333333333334;
    res[72] = h14_4_1 * 0.3333333333333334;
    res[73] = h14_4_2 * 0.3333333333333334;
    res[74] = h14_4_3 * 0.3333333333333334;
    res[75] = h14_5_1 * 0.5773502691896258;
    res[76] = h14_5_2 * 0.5773502691896258;
    res[77] = h14_5_3 * 0.5773502691896258;
    res[78] = h14_6_1 * 0.5773502691896258;
    res[79] = h14_6_2 * 0.5773502691896258;
    res[80] = h14_6_3 * 0.5773502691896258;
    res[81] = h14_7_1 * 0.3333333333333334;
    res[82] = h14_7_2 * 0.3333333333333334;
    res[83] = h14_7_3 * 0.3333333333333334;
    res[84] = h14_8_1 * 0.5773502691896258;
    res[85] = h14_8_2 * 0.5773502691896258;
    res[86] = h14_8_3 * 0.5773502691896258;
    res[87] = h14_9_1 * 0.3333333333333334;
    res[88] = h14_9_2 * 0.3333333333333334;
    res[89] = h14_9_3 * 0.3333333333333334;
    res[90] = h15_4_1 * 0.5773502691896258;
    res[91] = h15_4_2 * 0.5773502691896258;
    res[92] = h15_4_3 * 0.5773502691896258;
    res[93] = h15_5_1;
    res[94] = h15_5_2;
    res[95] = h15_5_3;
    res[96] = h15_6_1;
    res[97] = h15_6_2;
    res[98] = h15_6_3;
    res[99] = h15_7_1 * 0.5773502691896258;
    res[100] = h15_7_2 * 0.5773502691896258;
    res[101] = h15_7_3 * 0.5773502691896258;
    res[102] = h15_8_1;
    res[103] = h15_8_2;
    res[104] = h15_8_3;
    res[105] = h15_9_1 * 0.5773502691896258;
    res[106] = h15_9_2 * 0.5773502691896258;
    res[107] = h15_9_3 * 0.5773502691896258;
    res[108] = h16_4_1 * 0.14907119849998599;
    res[109] = h16_4_2 * 0.14907119849998599;
    res[110] = h16_4_3 * 0.14907119849998599;
    res[111] = h16_5_1 * 0.2581988897471611;
    res[112] = h16_5_2 * 0.2581988897471611;
    res[113] = h16_5_3 * 0.2581988897471611;
    res[114] = h16_6_1 * 0.2581988897471611;
    res[115] = h16_6_2 * 0.2581988897471611;
    res[116] = h16_6_3 * 0.2581988897471611;
    res[117] = h16_7_1 * 0.14907119849998599;
    res[118] = h16_7_2 * 0.14907119849998599;
    res[119] = h16_7_3 * 0.14907119849998599;
    res[120] = h16_8_1 * 0.2581988897471611;
    res[121] = h16_8_2 * 0.2581988897471611;
    res[122] = h16_8_3 * 0.2581988897471611;
    res[123] = h16_9_1 * 0.14907119849998599;
    res[124] = h16_9_2 * 0.14907119849998599;
    res[125] = h16_9_3 * 0.14907119849998599;
    res[126] = h17_4_1 * 0.3333333333333334;
    res[127] = h17_4_2 * 0.3333333333333334;
    res[128] = h17_4_3 * 0.3333333333333334;
    res[129] = h17_5_1 * 0.5773502691896258;
    res[130] = h17_5_2 * 0.5773502691896258;
    res[131] = h17_5_3 * 0.5773502691896258;
    res[132] = h17_6_1 * 0.5773502691896258;
    res[133] = h17_6_2 * 0.5773502691896258;
    res[134] = h17_6_3 * 0.5773502691896258;
    res[135] = h17_7_1 * 0.3333333333333334;
    res[136] = h17_7_2 * 0.3333333333333334;
    res[137] = h17_7_3 * 0.3333333333333334;
    res[138] = h17_8_1 * 0.5773502691896258;
    res[139] = h17_8_2 * 0.5773502691896258;
    res[140] = h17_8_3 * 0.5773502691896258;
    res[141] = h17_9_1 * 0.3333333333333334;
    res[142] = h17_9_2 * 0.3333333333333334;
    res[143] = h17_9_3 * 0.3333333333333334;
    res[144] = h18_4_1 * 0.3333333333333334;
    res[145] = h18_4_2 * 0.3333333333333334;
    res[146] = h18_4_3 * 0.3333333333333334;
    res[147] = h18_5_1 * 0.5773502691896258;
    res[148] = h18_5_2 * 0.5773502691896258;
    res[149] = h18_5_3 * 0.5773502691896258;
    res[150] = h18_6_1 * 0.5773502691896258;
    res[151] = h18_6_2 * 0.5773502691896258;
    res[152] = h18_6_3 * 0.5773502691896258;
    res[153] = h18_7_1 * 0.3333333333333334;
    res[154] = h18_7_2 * 0.3333333333333334;
    res[155] = h18_7_3 * 0.3333333333333334;
    res[156] = h18_8_1 * 0.5773502691896258;
    res[157] = h18_8_2 * 0.5773502691896258;
    res[158] = h18_8_3 * 0.5773502691896258;
    res[159] = h18_9_1 * 0.3333333333333334;
    res[160] = h18_9_2 * 0.3333333333333334;
    res[161] = h18_9_3 * 0.3333333333333334;
    res[162] = h19_4_1 * 0.14907119849998599;
    res[163] = h19_4_2 * 0.14907119849998599;
    res[164] = h19_4_3 * 0.14907119849998599;
    res[165] = h19_5_1 * 0.2581988897471611;
    res[166] = h19_5_2 * 0.2581988897471611;
    res[167] = h19_5_3 * 0.2581988897471611;
    res[168] = h19_6_1 * 0.2581988897471611;
    res[169] = h19_6_2 * 0.2581988897471611;
    res[170] = h19_6_3 * 0.2581988897471611;
    res[171] = h19_7_1 * 0.14907119849998599;
    res[172] = h19_7_2 * 0.14907119849998599;
    res[173] = h19_7_3 * 0.14907119849998599;
    res[174] = h19_8_1 * 0.2581988897471611;
    res[175] = h19_8_2 * 0.2581988897471611;
    res[176] = h19_8_3 * 0.2581988897471611;
    res[177] = h19_9_1 * 0.14907119849998599;
    res[178] = h19_9_2 * 0.14907119849998599;
    res[179] = h19_9_3 * 0.14907119849998599;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[180]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_fdps(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[138];
    vrr_fdps<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 138; ++x) acc_out[x] = acc[x];
    }
    hrr_fdps(P, p, q, acc, res);
}

__device__ __forceinline__ void store_fdps(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
    const long long ij_6_0 = pair_index(ib_.z + 6, ib_.w + 0);
    const long long ij_6_1 = pair_index(ib_.z + 6, ib_.w + 1);
    const long long ij_6_2 = pair_index(ib_.z + 6, ib_.w + 2);
    const long long ij_6_3 = pair_index(ib_.z + 6, ib_.w + 3);
    const long long ij_6_4 = pair_index(ib_.z + 6, ib_.w + 4);
    const long long ij_6_5 = pair_index(ib_.z + 6, ib_.w + 5);
    const long long ij_7_0 = pair_index(ib_.z + 7, ib_.w + 0);
    const long long ij_7_1 = pair_index(ib_.z + 7, ib_.w + 1);
    const long long ij_7_2 = pair_index(ib_.z + 7, ib_.w + 2);
    const long long ij_7_3 = pair_index(ib_.z + 7, ib_.w + 3);
    const long long ij_7_4 = pair_index(ib_.z + 7, ib_.w + 4);
    const long long ij_7_5 = pair_index(ib_.z + 7, ib_.w + 5);
    const long long ij_8_0 = pair_index(ib_.z + 8, ib_.w + 0);
    const long long ij_8_1 = pair_index(ib_.z + 8, ib_.w + 1);
    const long long ij_8_2 = pair_index(ib_.z + 8, ib_.w + 2);
    const long long ij_8_3 = pair_index(ib_.z + 8, ib_.w + 3);
    const long long ij_8_4 = pair_index(ib_.z + 8, ib_.w + 4);
    const long long ij_8_5 = pair_index(ib_.z + 8, ib_.w + 5);
    const long long ij_9_0 = pair_index(ib_.z + 9, ib_.w + 0);
    const long long ij_9_1 = pair_index(ib_.z + 9, ib_.w + 1);
    const long long ij_9_2 = pair_index(ib_.z + 9, ib_.w + 2);
    const long long ij_9_3 = pair_index(ib_.z + 9, ib_.w + 3);
    const long long ij_9_4 = pair_index(ib_.z + 9, ib_.w + 4);
    const long long ij_9_5 = pair_index(ib_.z + 9, ib_.w + 5);
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
    { const long long ij = ij_0_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_0_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_0_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_0_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_0_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_0_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_0_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_0_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_0_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_1_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_1_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_1_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_1_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_1_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_1_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_1_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_1_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_1_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_2_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_2_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_2_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_2_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_2_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_2_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_2_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_2_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_2_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_3_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_3_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_3_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_3_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_3_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_3_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_3_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_3_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_3_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_3_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_3_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_3_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_3_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_4_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_4_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_4_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_4_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_4_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_4_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_4_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_4_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_4_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_4_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_4_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_4_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_4_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_5_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_5_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_5_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_5_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_5_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
    { const long long ij = ij_5_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[100]; }
    { const long long ij = ij_5_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[101]; }
    { const long long ij = ij_5_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[102]; }
    { const long long ij = ij_5_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[103]; }
    { const long long ij = ij_5_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[104]; }
    { const long long ij = ij_5_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[105]; }
    { const long long ij = ij_5_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[106]; }
    { const long long ij = ij_5_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[107]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[108]; }
    { const long long ij = ij_6_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[109]; }
    { const long long ij = ij_6_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[110]; }
    { const long long ij = ij_6_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[111]; }
    { const long long ij = ij_6_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[112]; }
    { const long long ij = ij_6_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[113]; }
    { const long long ij = ij_6_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[114]; }
    { const long long ij = ij_6_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[115]; }
    { const long long ij = ij_6_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[116]; }
    { const long long ij = ij_6_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[117]; }
    { const long long ij = ij_6_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[118]; }
    { const long long ij = ij_6_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[119]; }
    { const long long ij = ij_6_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[120]; }
    { const long long ij = ij_6_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[121]; }
    { const long long ij = ij_6_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[122]; }
    { const long long ij = ij_6_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[123]; }
    { const long long ij = ij_6_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[124]; }
    { const long long ij = ij_6_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[125]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[126]; }
    { const long long ij = ij_7_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[127]; }
    { const long long ij = ij_7_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[128]; }
    { const long long ij = ij_7_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[129]; }
    { const long long ij = ij_7_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[130]; }
    { const long long ij = ij_7_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[131]; }
    { const long long ij = ij_7_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[132]; }
    { const long long ij = ij_7_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[133]; }
    { const long long ij = ij_7_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[134]; }
    { const long long ij = ij_7_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[135]; }
    { const long long ij = ij_7_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[136]; }
    { const long long ij = ij_7_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[137]; }
    { const long long ij = ij_7_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[138]; }
    { const long long ij = ij_7_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[139]; }
    { const long long ij = ij_7_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[140]; }
    { const long long ij = ij_7_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[141]; }
    { const long long ij = ij_7_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[142]; }
    { const long long ij = ij_7_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[143]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[144]; }
    { const long long ij = ij_8_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[145]; }
    { const long long ij = ij_8_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[146]; }
    { const long long ij = ij_8_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[147]; }
    { const long long ij = ij_8_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[148]; }
    { const long long ij = ij_8_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[149]; }
    { const long long ij = ij_8_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[150]; }
    { const long long ij = ij_8_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[151]; }
    { const long long ij = ij_8_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[152]; }
    { const long long ij = ij_8_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[153]; }
    { const long long ij = ij_8_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[154]; }
    { const long long ij = ij_8_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[155]; }
    { const long long ij = ij_8_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[156]; }
    { const long long ij = ij_8_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[157]; }
    { const long long ij = ij_8_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[158]; }
    { const long long ij = ij_8_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[159]; }
    { const long long ij = ij_8_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[160]; }
    { const long long ij = ij_8_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[161]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[162]; }
    { const long long ij = ij_9_0, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[163]; }
    { const long long ij = ij_9_0, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[164]; }
    { const long long ij = ij_9_1, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[165]; }
    { const long long ij = ij_9_1, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[166]; }
    { const long long ij = ij_9_1, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[167]; }
    { const long long ij = ij_9_2, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[168]; }
    { const long long ij = ij_9_2, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[169]; }
    { const long long ij = ij_9_2, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[170]; }
    { const long long ij = ij_9_3, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[171]; }
    { const long long ij = ij_9_3, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[172]; }
    { const long long ij = ij_9_3, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[173]; }
    { const long long ij = ij_9_4, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[174]; }
    { const long long ij = ij_9_4, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[175]; }
    { const long long ij = ij_9_4, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[176]; }
    { const long long ij = ij_9_5, kl = kl_0_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[177]; }
    { const long long ij = ij_9_5, kl = kl_1_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[178]; }
    { const long long ij = ij_9_5, kl = kl_2_0;
      if (true && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[179]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_fdps(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 180; ++x) {
        const int ia = x / 18, ibb = (x / 3) % 6, ic = (x / 1) % 3, id = x % 1;
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
__global__ void __launch_bounds__(128) eri_queue_fdps(const EriQueue Q) {
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
        double acc[138];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 138; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_fdps<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_fdps<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 138; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: each leader stores its quartet's whole block at its slot
            if (lead) {
                double res[180];
                hrr_fdps(Q.pairs, p, q, acc, res);
                double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                    (__ldg(&Q.chunk_slot[c]) + base + kq) * (long long)180;
#pragma unroll
                for (int x = 0; x < 180; ++x) dst[x] = res[x];
            }
        } else if (lead) {
            double res[180];
            hrr_fdps(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_fdps(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_fdps(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_fdps(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    constexpr size_t smem = 0;
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_fdps<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_fdps<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_fdps<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_fdps<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_fdps(int mixed) {

    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fdps<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fdps<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

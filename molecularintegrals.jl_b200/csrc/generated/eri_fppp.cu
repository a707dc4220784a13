// Generated by gen_eri.py -- class (fp|pp).  Do not edit.
// VRR entries: 458, contracted block: 225, HRR lines: 540, outputs: 270.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[225], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_fppp(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 225; ++x) acc[x] = 0.0;
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
            const VT v20_1_0 = QCx * v20_0_0 + WQx * v20_0_1 + (VT)4.0 * oo2ze * v10_0_1;
            const VT v20_1_1 = QCx * v20_0_1 + WQx * v20_0_2 + (VT)4.0 * oo2ze * v10_0_2;
            const VT v21_1_0 = QCx * v21_0_0 + WQx * v21_0_1 + (VT)3.0 * oo2ze * v11_0_1;
            const VT v21_1_1 = QCx * v21_0_1 + WQx * v21_0_2 + (VT)3.0 * oo2ze * v11_0_2;
            const VT v22_1_0 = QCx * v22_0_0 + WQx * v22_0_1 + (VT)3.0 * oo2ze * v12_0_1;
            const VT v22_1_1 = QCx * v22_0_1 + WQx * v22_0_2 + (VT)3.0 * oo2ze * v12_0_2;
            const VT v23_1_0 = QCx * v23_0_0 + WQx * v23_0_1 + (VT)2.0 * oo2ze * v13_0_1;
            const VT v23_1_1 = QCx * v23_0_1 + WQx * v23_0_2 + (VT)2.0 * oo2ze * v13_0_2;
            const VT v24_1_0 = QCx * v24_0_0 + WQx * v24_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v24_1_1 = QCx * v24_0_1 + WQx * v24_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v25_1_0 = QCx * v25_0_0 + WQx * v25_0_1 + (VT)2.0 * oo2ze * v14_0_1;
            const VT v25_1_1 = QCx * v25_0_1 + WQx * v25_0_2 + (VT)2.0 * oo2ze * v14_0_2;
            const VT v26_1_0 = QCx * v26_0_0 + WQx * v26_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v26_1_1 = QCx * v26_0_1 + WQx * v26_0_2 + (VT)1.0 * oo2ze * v16_0_2;
            const VT v27_1_0 = QCx * v27_0_0 + WQx * v27_0_1 + (VT)1.0 * oo2ze * v17_0_1;
            const VT v27_1_1 = QCx * v27_0_1 + WQx * v27_0_2 + (VT)1.0 * oo2ze * v17_0_2;
            const VT v28_1_0 = QCx * v28_0_0 + WQx * v28_0_1 + (VT)1.0 * oo2ze * v18_0_1;
            const VT v28_1_1 = QCx * v28_0_1 + WQx * v28_0_2 + (VT)1.0 * oo2ze * v18_0_2;
            const VT v29_1_0 = QCx * v29_0_0 + WQx * v29_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v29_1_1 = QCx * v29_0_1 + WQx * v29_0_2 + (VT)1.0 * oo2ze * v19_0_2;
            const VT v30_1_0 = QCx * v30_0_0 + WQx * v30_0_1;
            const VT v30_1_1 = QCx * v30_0_1 + WQx * v30_0_2;
            const VT v31_1_0 = QCx * v31_0_0 + WQx * v31_0_1;
            const VT v31_1_1 = QCx * v31_0_1 + WQx * v31_0_2;
            const VT v32_1_0 = QCx * v32_0_0 + WQx * v32_0_1;
            const VT v32_1_1 = QCx * v32_0_1 + WQx * v32_0_2;
            const VT v33_1_0 = QCx * v33_0_0 + WQx * v33_0_1;
            const VT v33_1_1 = QCx * v33_0_1 + WQx * v33_0_2;
            const VT v34_1_0 = QCx * v34_0_0 + WQx * v34_0_1;
            const VT v34_1_1 = QCx * v34_0_1 + WQx * v34_0_2;
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
            const VT v20_2_0 = QCy * v20_0_0 + WQy * v20_0_1;
            const VT v20_2_1 = QCy * v20_0_1 + WQy * v20_0_2;
            const VT v21_2_0 = QCy * v21_0_0 + WQy * v21_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v21_2_1 = QCy * v21_0_1 + WQy * v21_0_2 + (VT)1.0 * oo2ze * v10_0_2;
            const VT v22_2_0 = QCy * v22_0_0 + WQy * v22_0_1;
            const VT v22_2_1 = QCy * v22_0_1 + WQy * v22_0_2;
            const VT v23_2_0 = QCy * v23_0_0 + WQy * v23_0_1 + (VT)2.0 * oo2ze * v11_0_1;
            const VT v23_2_1 = QCy * v23_0_1 + WQy * v23_0_2 + (VT)2.0 * oo2ze * v11_0_2;
            const VT v24_2_0 = QCy * v24_0_0 + WQy * v24_0_1 + (VT)1.0 * oo2ze * v12_0_1;
            const VT v24_2_1 = QCy * v24_0_1 + WQy * v24_0_2 + (VT)1.0 * oo2ze * v12_0_2;
            const VT v25_2_0 = QCy * v25_0_0 + WQy * v25_0_1;
            const VT v25_2_1 = QCy * v25_0_1 + WQy * v25_0_2;
            const VT v26_2_0 = QCy * v26_0_0 + WQy * v26_0_1 + (VT)3.0 * oo2ze * v13_0_1;
            const VT v26_2_1 = QCy * v26_0_1 + WQy * v26_0_2 + (VT)3.0 * oo2ze * v13_0_2;
            const VT v27_2_0 = QCy * v27_0_0 + WQy * v27_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v27_2_1 = QCy * v27_0_1 + WQy * v27_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v28_2_0 = QCy * v28_0_0 + WQy * v28_0_1 + (VT)1.0 * oo2ze * v14_0_1;
            const VT v28_2_1 = QCy * v28_0_1 + WQy * v28_0_2 + (VT)1.0 * oo2ze * v14_0_2;
            const VT v29_2_0 = QCy * v29_0_0 + WQy * v29_0_1;
            const VT v29_2_1 = QCy * v29_0_1 + WQy * v29_0_2;
            const VT v30_2_0 = QCy * v30_0_0 + WQy * v30_0_1 + (VT)4.0 * oo2ze * v16_0_1;
            const VT v30_2_1 = QCy * v30_0_1 + WQy * v30_0_2 + (VT)4.0 * oo2ze * v16_0_2;
            const VT v31_2_0 = QCy * v31_0_0 + WQy * v31_0_1 + (VT)3.0 * oo2ze * v17_0_1;
            const VT v31_2_1 = QCy * v31_0_1 + WQy * v31_0_2 + (VT)3.0 * oo2ze * v17_0_2;
            const VT v32_2_0 = QCy * v32_0_0 + WQy * v32_0_1 + (VT)2.0 * oo2ze * v18_0_1;
            const VT v32_2_1 = QCy * v32_0_1 + WQy * v32_0_2 + (VT)2.0 * oo2ze * v18_0_2;
            const VT v33_2_0 = QCy * v33_0_0 + WQy * v33_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v33_2_1 = QCy * v33_0_1 + WQy * v33_0_2 + (VT)1.0 * oo2ze * v19_0_2;
            const VT v34_2_0 = QCy * v34_0_0 + WQy * v34_0_1;
            const VT v34_2_1 = QCy * v34_0_1 + WQy * v34_0_2;
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
            const VT v20_3_0 = QCz * v20_0_0 + WQz * v20_0_1;
            const VT v20_3_1 = QCz * v20_0_1 + WQz * v20_0_2;
            const VT v21_3_0 = QCz * v21_0_0 + WQz * v21_0_1;
            const VT v21_3_1 = QCz * v21_0_1 + WQz * v21_0_2;
            const VT v22_3_0 = QCz * v22_0_0 + WQz * v22_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v22_3_1 = QCz * v22_0_1 + WQz * v22_0_2 + (VT)1.0 * oo2ze * v10_0_2;
            const VT v23_3_0 = QCz * v23_0_0 + WQz * v23_0_1;
            const VT v23_3_1 = QCz * v23_0_1 + WQz * v23_0_2;
            const VT v24_3_0 = QCz * v24_0_0 + WQz * v24_0_1 + (VT)1.0 * oo2ze * v11_0_1;
            const VT v24_3_1 = QCz * v24_0_1 + WQz * v24_0_2 + (VT)1.0 * oo2ze * v11_0_2;
            const VT v25_3_0 = QCz * v25_0_0 + WQz * v25_0_1 + (VT)2.0 * oo2ze * v12_0_1;
            const VT v25_3_1 = QCz * v25_0_1 + WQz * v25_0_2 + (VT)2.0 * oo2ze * v12_0_2;
            const VT v26_3_0 = QCz * v26_0_0 + WQz * v26_0_1;
            const VT v26_3_1 = QCz * v26_0_1 + WQz * v26_0_2;
            const VT v27_3_0 = QCz * v27_0_0 + WQz * v27_0_1 + (VT)1.0 * oo2ze * v13_0_1;
            const VT v27_3_1 = QCz * v27_0_1 + WQz * v27_0_2 + (VT)1.0 * oo2ze * v13_0_2;
            const VT v28_3_0 = QCz * v28_0_0 + WQz * v28_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v28_3_1 = QCz * v28_0_1 + WQz * v28_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v29_3_0 = QCz * v29_0_0 + WQz * v29_0_1 + (VT)3.0 * oo2ze * v14_0_1;
            const VT v29_3_1 = QCz * v29_0_1 + WQz * v29_0_2 + (VT)3.0 * oo2ze * v14_0_2;
            const VT v30_3_0 = QCz * v30_0_0 + WQz * v30_0_1;
            const VT v30_3_1 = QCz * v30_0_1 + WQz * v30_0_2;
            const VT v31_3_0 = QCz * v31_0_0 + WQz * v31_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v31_3_1 = QCz * v31_0_1 + WQz * v31_0_2 + (VT)1.0 * oo2ze * v16_0_2;
            const VT v32_3_0 = QCz * v32_0_0 + WQz * v32_0_1 + (VT)2.0 * oo2ze * v17_0_1;
            const VT v32_3_1 = QCz * v32_0_1 + WQz * v32_0_2 + (VT)2.0 * oo2ze * v17_0_2;
            const VT v33_3_0 = QCz * v33_0_0 + WQz * v33_0_1 + (VT)3.0 * oo2ze * v18_0_1;
            const VT v33_3_1 = QCz * v33_0_1 + WQz * v33_0_2 + (VT)3.0 * oo2ze * v18_0_2;
            const VT v34_3_0 = QCz * v34_0_0 + WQz * v34_0_1 + (VT)4.0 * oo2ze * v19_0_1;
            const VT v34_3_1 = QCz * v34_0_1 + WQz * v34_0_2 + (VT)4.0 * oo2ze * v19_0_2;
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
            const VT v20_4_0 = QCx * v20_1_0 + WQx * v20_1_1 + (VT)4.0 * oo2ze * v10_1_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v21_4_0 = QCx * v21_1_0 + WQx * v21_1_1 + (VT)3.0 * oo2ze * v11_1_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v22_4_0 = QCx * v22_1_0 + WQx * v22_1_1 + (VT)3.0 * oo2ze * v12_1_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v23_4_0 = QCx * v23_1_0 + WQx * v23_1_1 + (VT)2.0 * oo2ze * v13_1_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v24_4_0 = QCx * v24_1_0 + WQx * v24_1_1 + (VT)2.0 * oo2ze * v15_1_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v25_4_0 = QCx * v25_1_0 + WQx * v25_1_1 + (VT)2.0 * oo2ze * v14_1_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v26_4_0 = QCx * v26_1_0 + WQx * v26_1_1 + (VT)1.0 * oo2ze * v16_1_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v27_4_0 = QCx * v27_1_0 + WQx * v27_1_1 + (VT)1.0 * oo2ze * v17_1_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v28_4_0 = QCx * v28_1_0 + WQx * v28_1_1 + (VT)1.0 * oo2ze * v18_1_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v29_4_0 = QCx * v29_1_0 + WQx * v29_1_1 + (VT)1.0 * oo2ze * v19_1_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v30_4_0 = QCx * v30_1_0 + WQx * v30_1_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v31_4_0 = QCx * v31_1_0 + WQx * v31_1_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v32_4_0 = QCx * v32_1_0 + WQx * v32_1_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v33_4_0 = QCx * v33_1_0 + WQx * v33_1_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v34_4_0 = QCx * v34_1_0 + WQx * v34_1_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
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
            const VT v20_5_0 = QCx * v20_2_0 + WQx * v20_2_1 + (VT)4.0 * oo2ze * v10_2_1;
            const VT v21_5_0 = QCx * v21_2_0 + WQx * v21_2_1 + (VT)3.0 * oo2ze * v11_2_1;
            const VT v22_5_0 = QCx * v22_2_0 + WQx * v22_2_1 + (VT)3.0 * oo2ze * v12_2_1;
            const VT v23_5_0 = QCx * v23_2_0 + WQx * v23_2_1 + (VT)2.0 * oo2ze * v13_2_1;
            const VT v24_5_0 = QCx * v24_2_0 + WQx * v24_2_1 + (VT)2.0 * oo2ze * v15_2_1;
            const VT v25_5_0 = QCx * v25_2_0 + WQx * v25_2_1 + (VT)2.0 * oo2ze * v14_2_1;
            const VT v26_5_0 = QCx * v26_2_0 + WQx * v26_2_1 + (VT)1.0 * oo2ze * v16_2_1;
            const VT v27_5_0 = QCx * v27_2_0 + WQx * v27_2_1 + (VT)1.0 * oo2ze * v17_2_1;
            const VT v28_5_0 = QCx * v28_2_0 + WQx * v28_2_1 + (VT)1.0 * oo2ze * v18_2_1;
            const VT v29_5_0 = QCx * v29_2_0 + WQx * v29_2_1 + (VT)1.0 * oo2ze * v19_2_1;
            const VT v30_5_0 = QCx * v30_2_0 + WQx * v30_2_1;
            const VT v31_5_0 = QCx * v31_2_0 + WQx * v31_2_1;
            const VT v32_5_0 = QCx * v32_2_0 + WQx * v32_2_1;
            const VT v33_5_0 = QCx * v33_2_0 + WQx * v33_2_1;
            const VT v34_5_0 = QCx * v34_2_0 + WQx * v34_2_1;
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
            const VT v20_6_0 = QCx * v20_3_0 + WQx * v20_3_1 + (VT)4.0 * oo2ze * v10_3_1;
            const VT v21_6_0 = QCx * v21_3_0 + WQx * v21_3_1 + (VT)3.0 * oo2ze * v11_3_1;
            const VT v22_6_0 = QCx * v22_3_0 + WQx * v22_3_1 + (VT)3.0 * oo2ze * v12_3_1;
            const VT v23_6_0 = QCx * v23_3_0 + WQx * v23_3_1 + (VT)2.0 * oo2ze * v13_3_1;
            const VT v24_6_0 = QCx * v24_3_0 + WQx * v24_3_1 + (VT)2.0 * oo2ze * v15_3_1;
            const VT v25_6_0 = QCx * v25_3_0 + WQx * v25_3_1 + (VT)2.0 * oo2ze * v14_3_1;
            const VT v26_6_0 = QCx * v26_3_0 + WQx * v26_3_1 + (VT)1.0 * oo2ze * v16_3_1;
            const VT v27_6_0 = QCx * v27_3_0 + WQx * v27_3_1 + (VT)1.0 * oo2ze * v17_3_1;
            const VT v28_6_0 = QCx * v28_3_0 + WQx * v28_3_1 + (VT)1.0 * oo2ze * v18_3_1;
            const VT v29_6_0 = QCx * v29_3_0 + WQx * v29_3_1 + (VT)1.0 * oo2ze * v19_3_1;
            const VT v30_6_0 = QCx * v30_3_0 + WQx * v30_3_1;
            const VT v31_6_0 = QCx * v31_3_0 + WQx * v31_3_1;
            const VT v32_6_0 = QCx * v32_3_0 + WQx * v32_3_1;
            const VT v33_6_0 = QCx * v33_3_0 + WQx * v33_3_1;
            const VT v34_6_0 = QCx * v34_3_0 + WQx * v34_3_1;
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
            const VT v20_7_0 = QCy * v20_2_0 + WQy * v20_2_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v21_7_0 = QCy * v21_2_0 + WQy * v21_2_1 + (VT)1.0 * oo2ze * v10_2_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v22_7_0 = QCy * v22_2_0 + WQy * v22_2_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v23_7_0 = QCy * v23_2_0 + WQy * v23_2_1 + (VT)2.0 * oo2ze * v11_2_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v24_7_0 = QCy * v24_2_0 + WQy * v24_2_1 + (VT)1.0 * oo2ze * v12_2_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v25_7_0 = QCy * v25_2_0 + WQy * v25_2_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v26_7_0 = QCy * v26_2_0 + WQy * v26_2_1 + (VT)3.0 * oo2ze * v13_2_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v27_7_0 = QCy * v27_2_0 + WQy * v27_2_1 + (VT)2.0 * oo2ze * v15_2_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v28_7_0 = QCy * v28_2_0 + WQy * v28_2_1 + (VT)1.0 * oo2ze * v14_2_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v29_7_0 = QCy * v29_2_0 + WQy * v29_2_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v30_7_0 = QCy * v30_2_0 + WQy * v30_2_1 + (VT)4.0 * oo2ze * v16_2_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v31_7_0 = QCy * v31_2_0 + WQy * v31_2_1 + (VT)3.0 * oo2ze * v17_2_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v32_7_0 = QCy * v32_2_0 + WQy * v32_2_1 + (VT)2.0 * oo2ze * v18_2_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v33_7_0 = QCy * v33_2_0 + WQy * v33_2_1 + (VT)1.0 * oo2ze * v19_2_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v34_7_0 = QCy * v34_2_0 + WQy * v34_2_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
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
            const VT v20_8_0 = QCy * v20_3_0 + WQy * v20_3_1;
            const VT v21_8_0 = QCy * v21_3_0 + WQy * v21_3_1 + (VT)1.0 * oo2ze * v10_3_1;
            const VT v22_8_0 = QCy * v22_3_0 + WQy * v22_3_1;
            const VT v23_8_0 = QCy * v23_3_0 + WQy * v23_3_1 + (VT)2.0 * oo2ze * v11_3_1;
            const VT v24_8_0 = QCy * v24_3_0 + WQy * v24_3_1 + (VT)1.0 * oo2ze * v12_3_1;
            const VT v25_8_0 = QCy * v25_3_0 + WQy * v25_3_1;
            const VT v26_8_0 = QCy * v26_3_0 + WQy * v26_3_1 + (VT)3.0 * oo2ze * v13_3_1;
            const VT v27_8_0 = QCy * v27_3_0 + WQy * v27_3_1 + (VT)2.0 * oo2ze * v15_3_1;
            const VT v28_8_0 = QCy * v28_3_0 + WQy * v28_3_1 + (VT)1.0 * oo2ze * v14_3_1;
            const VT v29_8_0 = QCy * v29_3_0 + WQy * v29_3_1;
            const VT v30_8_0 = QCy * v30_3_0 + WQy * v30_3_1 + (VT)4.0 * oo2ze * v16_3_1;
            const VT v31_8_0 = QCy * v31_3_0 + WQy * v31_3_1 + (VT)3.0 * oo2ze * v17_3_1;
            const VT v32_8_0 = QCy * v32_3_0 + WQy * v32_3_1 + (VT)2.0 * oo2ze * v18_3_1;
            const VT v33_8_0 = QCy * v33_3_0 + WQy * v33_3_1 + (VT)1.0 * oo2ze * v19_3_1;
            const VT v34_8_0 = QCy * v34_3_0 + WQy * v34_3_1;
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
            const VT v20_9_0 = QCz * v20_3_0 + WQz * v20_3_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v21_9_0 = QCz * v21_3_0 + WQz * v21_3_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v22_9_0 = QCz * v22_3_0 + WQz * v22_3_1 + (VT)1.0 * oo2ze * v10_3_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v23_9_0 = QCz * v23_3_0 + WQz * v23_3_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v24_9_0 = QCz * v24_3_0 + WQz * v24_3_1 + (VT)1.0 * oo2ze * v11_3_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v25_9_0 = QCz * v25_3_0 + WQz * v25_3_1 + (VT)2.0 * oo2ze * v12_3_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v26_9_0 = QCz * v26_3_0 + WQz * v26_3_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v27_9_0 = QCz * v27_3_0 + WQz * v27_3_1 + (VT)1.0 * oo2ze * v13_3_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v28_9_0 = QCz * v28_3_0 + WQz * v28_3_1 + (VT)2.0 * oo2ze * v15_3_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v29_9_0 = QCz * v29_3_0 + WQz * v29_3_1 + (VT)3.0 * oo2ze * v14_3_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v30_9_0 = QCz * v30_3_0 + WQz * v30_3_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v31_9_0 = QCz * v31_3_0 + WQz * v31_3_1 + (VT)1.0 * oo2ze * v16_3_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v32_9_0 = QCz * v32_3_0 + WQz * v32_3_1 + (VT)2.0 * oo2ze * v17_3_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v33_9_0 = QCz * v33_3_0 + WQz * v33_3_1 + (VT)3.0 * oo2ze * v18_3_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v34_9_0 = QCz * v34_3_0 + WQz * v34_3_1 + (VT)4.0 * oo2ze * v19_3_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
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
            acc[90] += (double)v20_1_0;
            acc[91] += (double)v20_2_0;
            acc[92] += (double)v20_3_0;
            acc[93] += (double)v20_4_0;
            acc[94] += (double)v20_5_0;
            acc[95] += (double)v20_6_0;
            acc[96] += (double)v20_7_0;
            acc[97] += (double)v20_8_0;
            acc[98] += (double)v20_9_0;
            acc[99] += (double)v21_1_0;
            acc[100] += (double)v21_2_0;
            acc[101] += (double)v21_3_0;
            acc[102] += (double)v21_4_0;
            acc[103] += (double)v21_5_0;
            acc[104] += (double)v21_6_0;
            acc[105] += (double)v21_7_0;
            acc[106] += (double)v21_8_0;
            acc[107] += (double)v21_9_0;
            acc[108] += (double)v22_1_0;
            acc[109] += (double)v22_2_0;
            acc[110] += (double)v22_3_0;
            acc[111] += (double)v22_4_0;
            acc[112] += (double)v22_5_0;
            acc[113] += (double)v22_6_0;
            acc[114] += (double)v22_7_0;
            acc[115] += (double)v22_8_0;
            acc[116] += (double)v22_9_0;
            acc[117] += (double)v23_1_0;
            acc[118] += (double)v23_2_0;
            acc[119] += (double)v23_3_0;
            acc[120] += (double)v23_4_0;
            acc[121] += (double)v23_5_0;
            acc[122] += (double)v23_6_0;
            acc[123] += (double)v23_7_0;
            acc[124] += (double)v23_8_0;
            acc[125] += (double)v23_9_0;
            acc[126] += (double)v24_1_0;
            acc[127] += (double)v24_2_0;
            acc[128] += (double)v24_3_0;
            acc[129] += (double)v24_4_0;
            acc[130] += (double)v24_5_0;
            acc[131] += (double)v24_6_0;
            acc[132] += (double)v24_7_0;
            acc[133] += (double)v24_8_0;
            acc[134] += (double)v24_9_0;
            acc[135] += (double)v25_1_0;
            acc[136] += (double)v25_2_0;
            acc[137] += (double)v25_3_0;
            acc[138] += (double)v25_4_0;
            acc[139] += (double)v25_5_0;
            acc[140] += (double)v25_6_0;
            acc[141] += (double)v25_7_0;
            acc[142] += (double)v25_8_0;
            acc[143] += (double)v25_9_0;
            acc[144] += (double)v26_1_0;
            acc[145] += (double)v26_2_0;
            acc[146] += (double)v26_3_0;
            acc[147] += (double)v26_4_0;
            acc[148] += (double)v26_5_0;
            acc[149] += (double)v26_6_0;
            acc[150] += (double)v26_7_0;
            acc[151] += (double)v26_8_0;
            acc[152] += (double)v26_9_0;
            acc[153] += (double)v27_1_0;
            acc[154] += (double)v27_2_0;
            acc[155] += (double)v27_3_0;
            acc[156] += (double)v27_4_0;
            acc[157] += (double)v27_5_0;
            acc[158] += (double)v27_6_0;
            acc[159] += (double)v27_7_0;
            acc[160] += (double)v27_8_0;
            acc[161] += (double)v27_9_0;
            acc[162] += (double)v28_1_0;
            acc[163] += (double)v28_2_0;
            acc[164] += (double)v28_3_0;
            acc[165] += (double)v28_4_0;
            acc[166] += (double)v28_5_0;
            acc[167] += (double)v28_6_0;
            acc[168] += (double)v28_7_0;
            acc[169] += (double)v28_8_0;
            acc[170] += (double)v28_9_0;
            acc[171] += (double)v29_1_0;
            acc[172] += (double)v29_2_0;
            acc[173] += (double)v29_3_0;
            acc[174] += (double)v29_4_0;
            acc[175] += (double)v29_5_0;
            acc[176] += (double)v29_6_0;
            acc[177] += (double)v29_7_0;
            acc[178] += (double)v29_8_0;
            acc[179] += (double)v29_9_0;
            acc[180] += (double)v30_1_0;
            acc[181] += (double)v30_2_0;
            acc[182] += (double)v30_3_0;
            acc[183] += (double)v30_4_0;
            acc[184] += (double)v30_5_0;
            acc[185] += (double)v30_6_0;
            acc[186] += (double)v30_7_0;
            acc[187] += (double)v30_8_0;
            acc[188] += (double)v30_9_0;
            acc[189] += (double)v31_1_0;
            acc[190] += (double)v31_2_0;
            acc[191] += (double)v31_3_0;
            acc[192] += (double)v31_4_0;
            acc[193] += (double)v31_5_0;
            acc[194] += (double)v31_6_0;
            acc[195] += (double)v31_7_0;
            acc[196] += (double)v31_8_0;
            acc[197] += (double)v31_9_0;
            acc[198] += (double)v32_1_0;
            acc[199] += (double)v32_2_0;
            acc[200] += (double)v32_3_0;
            acc[201] += (double)v32_4_0;
            acc[202] += (double)v32_5_0;
            acc[203] += (double)v32_6_0;
            acc[204] += (double)v32_7_0;
            acc[205] += (double)v32_8_0;
            acc[206] += (double)v32_9_0;
            acc[207] += (double)v33_1_0;
            acc[208] += (double)v33_2_0;
            acc[209] += (double)v33_3_0;
            acc[210] += (double)v33_4_0;
            acc[211] += (double)v33_5_0;
            acc[212] += (double)v33_6_0;
            acc[213] += (double)v33_7_0;
            acc[214] += (double)v33_8_0;
            acc[215] += (double)v33_9_0;
            acc[216] += (double)v34_1_0;
            acc[217] += (double)v34_2_0;
            acc[218] += (double)v34_3_0;
            acc[219] += (double)v34_4_0;
            acc[220] += (double)v34_5_0;
            acc[221] += (double)v34_6_0;
            acc[222] += (double)v34_7_0;
            acc[223] += (double)v34_8_0;
            acc[224] += (double)v34_9_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[270] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_fppp(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h10_1_4 = acc[93] + ABx * acc[3];
    const double h10_1_1 = acc[90] + ABx * acc[0];
    const double k10_1_1_1 = h10_1_4 + CDx * h10_1_1;
    const double h10_1_5 = acc[94] + ABx * acc[4];
    const double k10_1_1_2 = h10_1_5 + CDy * h10_1_1;
    const double h10_1_6 = acc[95] + ABx * acc[5];
    const double k10_1_1_3 = h10_1_6 + CDz * h10_1_1;
    const double h10_1_2 = acc[91] + ABx * acc[1];
    const double k10_1_2_1 = h10_1_5 + CDx * h10_1_2;
    const double h10_1_7 = acc[96] + ABx * acc[6];
    const double k10_1_2_2 = h10_1_7 + CDy * h10_1_2;
    const double h10_1_8 = acc[97] + ABx * acc[7];
    const double k10_1_2_3 = h10_1_8 + CDz * h10_1_2;
    const double h10_1_3 = acc[92] + ABx * acc[2];
    const double k10_1_3_1 = h10_1_6 + CDx * h10_1_3;
    const double k10_1_3_2 = h10_1_8 + CDy * h10_1_3;
    const double h10_1_9 = acc[98] + ABx * acc[8];
    const double k10_1_3_3 = h10_1_9 + CDz * h10_1_3;
    const double h10_2_4 = acc[102] + ABy * acc[3];
    const double h10_2_1 = acc[99] + ABy * acc[0];
    const double k10_2_1_1 = h10_2_4 + CDx * h10_2_1;
    const double h10_2_5 = acc[103] + ABy * acc[4];
    const double k10_2_1_2 = h10_2_5 + CDy * h10_2_1;
    const double h10_2_6 = acc[104] + ABy * acc[5];
    const double k10_2_1_3 = h10_2_6 + CDz * h10_2_1;
    const double h10_2_2 = acc[100] + ABy * acc[1];
    const double k10_2_2_1 = h10_2_5 + CDx * h10_2_2;
    const double h10_2_7 = acc[105] + ABy * acc[6];
    const double k10_2_2_2 = h10_2_7 + CDy * h10_2_2;
    const double h10_2_8 = acc[106] + ABy * acc[7];
    const double k10_2_2_3 = h10_2_8 + CDz * h10_2_2;
    const double h10_2_3 = acc[101] + ABy * acc[2];
    const double k10_2_3_1 = h10_2_6 + CDx * h10_2_3;
    const double k10_2_3_2 = h10_2_8 + CDy * h10_2_3;
    const double h10_2_9 = acc[107] + ABy * acc[8];
    const double k10_2_3_3 = h10_2_9 + CDz * h10_2_3;
    const double h10_3_4 = acc[111] + ABz * acc[3];
    const double h10_3_1 = acc[108] + ABz * acc[0];
    const double k10_3_1_1 = h10_3_4 + CDx * h10_3_1;
    const double h10_3_5 = acc[112] + ABz * acc[4];
    const double k10_3_1_2 = h10_3_5 + CDy * h10_3_1;
    const double h10_3_6 = acc[113] + ABz * acc[5];
    const double k10_3_1_3 = h10_3_6 + CDz * h10_3_1;
    const double h10_3_2 = acc[109] + ABz * acc[1];
    const double k10_3_2_1 = h10_3_5 + CDx * h10_3_2;
    const double h10_3_7 = acc[114] + ABz * acc[6];
    const double k10_3_2_2 = h10_3_7 + CDy * h10_3_2;
    const double h10_3_8 = acc[115] + ABz * acc[7];
    const double k10_3_2_3 = h10_3_8 + CDz * h10_3_2;
    const double h10_3_3 = acc[110] + ABz * acc[2];
    const double k10_3_3_1 = h10_3_6 + CDx * h10_3_3;
    const double k10_3_3_2 = h10_3_8 + CDy * h10_3_3;
    const double h10_3_9 = acc[116] + ABz * acc[8];
    const double k10_3_3_3 = h10_3_9 + CDz * h10_3_3;
    const double h11_1_4 = acc[102] + ABx * acc[12];
    const double h11_1_1 = acc[99] + ABx * acc[9];
    const double k11_1_1_1 = h11_1_4 + CDx * h11_1_1;
    const double h11_1_5 = acc[103] + ABx * acc[13];
    const double k11_1_1_2 = h11_1_5 + CDy * h11_1_1;
    const double h11_1_6 = acc[104] + ABx * acc[14];
    const double k11_1_1_3 = h11_1_6 + CDz * h11_1_1;
    const double h11_1_2 = acc[100] + ABx * acc[10];
    const double k11_1_2_1 = h11_1_5 + CDx * h11_1_2;
    const double h11_1_7 = acc[105] + ABx * acc[15];
    const double k11_1_2_2 = h11_1_7 + CDy * h11_1_2;
    const double h11_1_8 = acc[106] + ABx * acc[16];
    const double k11_1_2_3 = h11_1_8 + CDz * h11_1_2;
    const double h11_1_3 = acc[101] + ABx * acc[11];
    const double k11_1_3_1 = h11_1_6 + CDx * h11_1_3;
    const double k11_1_3_2 = h11_1_8 + CDy * h11_1_3;
    const double h11_1_9 = acc[107] + ABx * acc[17];
    const double k11_1_3_3 = h11_1_9 + CDz * h11_1_3;
    const double h11_2_4 = acc[120] + ABy * acc[12];
    const double h11_2_1 = acc[117] + ABy * acc[9];
    const double k11_2_1_1 = h11_2_4 + CDx * h11_2_1;
    const double h11_2_5 = acc[121] + ABy * acc[13];
    const double k11_2_1_2 = h11_2_5 + CDy * h11_2_1;
    const double h11_2_6 = acc[122] + ABy * acc[14];
    const double k11_2_1_3 = h11_2_6 + CDz * h11_2_1;
    const double h11_2_2 = acc[118] + ABy * acc[10];
    const double k11_2_2_1 = h11_2_5 + CDx * h11_2_2;
    const double h11_2_7 = acc[123] + ABy * acc[15];
    const double k11_2_2_2 = h11_2_7 + CDy * h11_2_2;
    const double h11_2_8 = acc[124] + ABy * acc[16];
    const double k11_2_2_3 = h11_2_8 + CDz * h11_2_2;
    const double h11_2_3 = acc[119] + ABy * acc[11];
    const double k11_2_3_1 = h11_2_6 + CDx * h11_2_3;
    const double k11_2_3_2 = h11_2_8 + CDy * h11_2_3;
    const double h11_2_9 = acc[125] + ABy * acc[17];
    const double k11_2_3_3 = h11_2_9 + CDz * h11_2_3;
    const double h11_3_4 = acc[129] + ABz * acc[12];
    const double h11_3_1 = acc[126] + ABz * acc[9];
    const double k11_3_1_1 = h11_3_4 + CDx * h11_3_1;
    const double h11_3_5 = acc[130] + ABz * acc[13];
    const double k11_3_1_2 = h11_3_5 + CDy * h11_3_1;
    const double h11_3_6 = acc[131] + ABz * acc[14];
    const double k11_3_1_3 = h11_3_6 + CDz * h11_3_1;
    const double h11_3_2 = acc[127] + ABz * acc[10];
    const double k11_3_2_1 = h11_3_5 + CDx * h11_3_2;
    const double h11_3_7 = acc[132] + ABz * acc[15];
    const double k11_3_2_2 = h11_3_7 + CDy * h11_3_2;
    const double h11_3_8 = acc[133] + ABz * acc[16];
    const double k11_3_2_3 = h11_3_8 + CDz * h11_3_2;
    const double h11_3_3 = acc[128] + ABz * acc[11];
    const double k11_3_3_1 = h11_3_6 + CDx * h11_3_3;
    const double k11_3_3_2 = h11_3_8 + CDy * h11_3_3;
    const double h11_3_9 = acc[134] + ABz * acc[17];
    const double k11_3_3_3 = h11_3_9 + CDz * h11_3_3;
    const double h12_1_4 = acc[111] + ABx * acc[21];
    const double h12_1_1 = acc[108] + ABx * acc[18];
    const double k12_1_1_1 = h12_1_4 + CDx * h12_1_1;
    const double h12_1_5 = acc[112] + ABx * acc[22];
    const double k12_1_1_2 = h12_1_5 + CDy * h12_1_1;
    const double h12_1_6 = acc[113] + ABx * acc[23];
    const double k12_1_1_3 = h12_1_6 + CDz * h12_1_1;
    const double h12_1_2 = acc[109] + ABx * acc[19];
    const double k12_1_2_1 = h12_1_5 + CDx * h12_1_2;
    const double h12_1_7 = acc[114] + ABx * acc[24];
    const double k12_1_2_2 = h12_1_7 + CDy * h12_1_2;
    const double h12_1_8 = acc[115] + ABx * acc[25];
    const double k12_1_2_3 = h12_1_8 + CDz * h12_1_2;
    const double h12_1_3 = acc[110] + ABx * acc[20];
    const double k12_1_3_1 = h12_1_6 + CDx * h12_1_3;
    const double k12_1_3_2 = h12_1_8 + CDy * h12_1_3;
    const double h12_1_9 = acc[116] + ABx * acc[26];
    const double k12_1_3_3 = h12_1_9 + CDz * h12_1_3;
    const double h12_2_4 = acc[129] + ABy * acc[21];
    const double h12_2_1 = acc[126] + ABy * acc[18];
    const double k12_2_1_1 = h12_2_4 + CDx * h12_2_1;
    const double h12_2_5 = acc[130] + ABy * acc[22];
    const double k12_2_1_2 = h12_2_5 + CDy * h12_2_1;
    const double h12_2_6 = acc[131] + ABy * acc[23];
    const double k12_2_1_3 = h12_2_6 + CDz * h12_2_1;
    const double h12_2_2 = acc[127] + ABy * acc[19];
    const double k12_2_2_1 = h12_2_5 + CDx * h12_2_2;
    const double h12_2_7 = acc[132] + ABy * acc[24];
    const double k12_2_2_2 = h12_2_7 + CDy * h12_2_2;
    const double h12_2_8 = acc[133] + ABy * acc[25];
    const double k12_2_2_3 = h12_2_8 + CDz * h12_2_2;
    const double h12_2_3 = acc[128] + ABy * acc[20];
    const double k12_2_3_1 = h12_2_6 + CDx * h12_2_3;
    const double k12_2_3_2 = h12_2_8 + CDy * h12_2_3;
    const double h12_2_9 = acc[134] + ABy * acc[26];
    const double k12_2_3_3 = h12_2_9 + CDz * h12_2_3;
    const double h12_3_4 = acc[138] + ABz * acc[21];
    const double h12_3_1 = acc[135] + ABz * acc[18];
    const double k12_3_1_1 = h12_3_4 + CDx * h12_3_1;
    const double h12_3_5 = acc[139] + ABz * acc[22];
    const double k12_3_1_2 = h12_3_5 + CDy * h12_3_1;
    const double h12_3_6 = acc[140] + ABz * acc[23];
    const double k12_3_1_3 = h12_3_6 + CDz * h12_3_1;
    const double h12_3_2 = acc[136] + ABz * acc[19];
    const double k12_3_2_1 = h12_3_5 + CDx * h12_3_2;
    const double h12_3_7 = acc[141] + ABz * acc[24];
    const double k12_3_2_2 = h12_3_7 + CDy * h12_3_2;
    const double h12_3_8 = acc[142] + ABz * acc[25];
    const double k12_3_2_3 = h12_3_8 + CDz * h12_3_2;
    const double h12_3_3 = acc[137] + ABz * acc[20];
    const double k12_3_3_1 = h12_3_6 + CDx * h12_3_3;
    const double k12_3_3_2 = h12_3_8 + CDy * h12_3_3;
    const double h12_3_9 = acc[143] + ABz * acc[26];
    const double k12_3_3_3 = h12_3_9 + CDz * h12_3_3;
    const double h13_1_4 = acc[120] + ABx * acc[30];
    const double h13_1_1 = acc[117] + ABx * acc[27];
    const double k13_1_1_1 = h13_1_4 + CDx * h13_1_1;
    const double h13_1_5 = acc[121] + ABx * acc[31];
    const double k13_1_1_2 = h13_1_5 + CDy * h13_1_1;
    const double h13_1_6 = acc[122] + ABx * acc[32];
    const double k13_1_1_3 = h13_1_6 + CDz * h13_1_1;
    const double h13_1_2 = acc[118] + ABx * acc[28];
    const double k13_1_2_1 = h13_1_5 + CDx * h13_1_2;
    const double h13_1_7 = acc[123] + ABx * acc[33];
    const double k13_1_2_2 = h13_1_7 + CDy * h13_1_2;
    const double h13_1_8 = acc[124] + ABx * acc[34];
    const double k13_1_2_3 = h13_1_8 + CDz * h13_1_2;
    const double h13_1_3 = acc[119] + ABx * acc[29];
    const double k13_1_3_1 = h13_1_6 + CDx * h13_1_3;
    const double k13_1_3_2 = h13_1_8 + CDy * h13_1_3;
    const double h13_1_9 = acc[125] + ABx * acc[35];
    const double k13_1_3_3 = h13_1_9 + CDz * h13_1_3;
    const double h13_2_4 = acc[147] + ABy * acc[30];
    const double h13_2_1 = acc[144] + ABy * acc[27];
    const double k13_2_1_1 = h13_2_4 + CDx * h13_2_1;
    const double h13_2_5 = acc[148] + ABy * acc[31];
    const double k13_2_1_2 = h13_2_5 + CDy * h13_2_1;
    const double h13_2_6 = acc[149] + ABy * acc[32];
    const double k13_2_1_3 = h13_2_6 + CDz * h13_2_1;
    const double h13_2_2 = acc[145] + ABy * acc[28];
    const double k13_2_2_1 = h13_2_5 + CDx * h13_2_2;
    const double h13_2_7 = acc[150] + ABy * acc[33];
    const double k13_2_2_2 = h13_2_7 + CDy * h13_2_2;
    const double h13_2_8 = acc[151] + ABy * acc[34];
    const double k13_2_2_3 = h13_2_8 + CDz * h13_2_2;
    const double h13_2_3 = acc[146] + ABy * acc[29];
    const double k13_2_3_1 = h13_2_6 + CDx * h13_2_3;
    const double k13_2_3_2 = h13_2_8 + CDy * h13_2_3;
    const double h13_2_9 = acc[152] + ABy * acc[35];
    const double k13_2_3_3 = h13_2_9 + CDz * h13_2_3;
    const double h13_3_4 = acc[156] + ABz * acc[30];
    const double h13_3_1 = acc[153] + ABz * acc[27];
    const double k13_3_1_1 = h13_3_4 + CDx * h13_3_1;
    const double h13_3_5 = acc[157] + ABz * acc[31];
    const double k13_3_1_2 = h13_3_5 + CDy * h13_3_1;
    const double h13_3_6 = acc[158] + ABz * acc[32];
    const double k13_3_1_3 = h13_3_6 + CDz * h13_3_1;
    const double h13_3_2 = acc[154] + ABz * acc[28];
    const double k13_3_2_1 = h13_3_5 + CDx * h13_3_2;
    const double h13_3_7 = acc[159] + ABz * acc[33];
    const double k13_3_2_2 = h13_3_7 + CDy * h13_3_2;
    const double h13_3_8 = acc[160] + ABz * acc[34];
    const double k13_3_2_3 = h13_3_8 + CDz * h13_3_2;
    const double h13_3_3 = acc[155] + ABz * acc[29];
    const double k13_3_3_1 = h13_3_6 + CDx * h13_3_3;
    const double k13_3_3_2 = h13_3_8 + CDy * h13_3_3;
    const double h13_3_9 = acc[161] + ABz * acc[35];
    const double k13_3_3_3 = h13_3_9 + CDz * h13_3_3;
    const double h14_1_4 = acc[138] + ABx * acc[39];
    const double h14_1_1 = acc[135] + ABx * acc[36];
    const double k14_1_1_1 = h14_1_4 + CDx * h14_1_1;
    const double h14_1_5 = acc[139] + ABx * acc[40];
    const double k14_1_1_2 = h14_1_5 + CDy * h14_1_1;
    const double h14_1_6 = acc[140] + ABx * acc[41];
    const double k14_1_1_3 = h14_1_6 + CDz * h14_1_1;
    const double h14_1_2 = acc[136] + ABx * acc[37];
    const double k14_1_2_1 = h14_1_5 + CDx * h14_1_2;
    const double h14_1_7 = acc[141] + ABx * acc[42];
    const double k14_1_2_2 = h14_1_7 + CDy * h14_1_2;
    const double h14_1_8 = acc[142] + ABx * acc[43];
    const double k14_1_2_3 = h14_1_8 + CDz * h14_1_2;
    const double h14_1_3 = acc[137] + ABx * acc[38];
    const double k14_1_3_1 = h14_1_6 + CDx * h14_1_3;
    const double k14_1_3_2 = h14_1_8 + CDy * h14_1_3;
    const double h14_1_9 = acc[143] + ABx * acc[44];
    const double k14_1_3_3 = h14_1_9 + CDz * h14_1_3;
    const double h14_2_4 = acc[165] + ABy * acc[39];
    const double h14_2_1 = acc[162] + ABy * acc[36];
    const double k14_2_1_1 = h14_2_4 + CDx * h14_2_1;
    const double h14_2_5 = acc[166] + ABy * acc[40];
    const double k14_2_1_2 = h14_2_5 + CDy * h14_2_1;
    const double h14_2_6 = acc[167] + ABy * acc[41];
    const double k14_2_1_3 = h14_2_6 + CDz * h14_2_1;
    const double h14_2_2 = acc[163] + ABy * acc[37];
    const double k14_2_2_1 = h14_2_5 + CDx * h14_2_2;
    const double h14_2_7 = acc[168] + ABy * acc[42];
    const double k14_2_2_2 = h14_2_7 + CDy * h14_2_2;
    const double h14_2_8 = acc[169] + ABy * acc[43];
    const double k14_2_2_3 = h14_2_8 + CDz * h14_2_2;
    const double h14_2_3 = acc[164] + ABy * acc[38];
    const double k14_2_3_1 = h14_2_6 + CDx * h14_2_3;
    const double k14_2_3_2 = h14_2_8 + CDy * h14_2_3;
    const double h14_2_9 = acc[170] + ABy * acc[44];
    const double k14_2_3_3 = h14_2_9 + CDz * h14_2_3;
    const double h14_3_4 = acc[174] + ABz * acc[39];
    const double h14_3_1 = acc[171] + ABz * acc[36];
    const double k14_3_1_1 = h14_3_4 + CDx * h14_3_1;
    const double h14_3_5 = acc[175] + ABz * acc[40];
    const double k14_3_1_2 = h14_3_5 + CDy * h14_3_1;
    const double h14_3_6 = acc[176] + ABz * acc[41];
    const double k14_3_1_3 = h14_3_6 + CDz * h14_3_1;
    const double h14_3_2 = acc[172] + ABz * acc[37];
    const double k14_3_2_1 = h14_3_5 + CDx * h14_3_2;
    const double h14_3_7 = acc[177] + ABz * acc[42];
    const double k14_3_2_2 = h14_3_7 + CDy * h14_3_2;
    const double h14_3_8 = acc[178] + ABz * acc[43];
    const double k14_3_2_3 = h14_3_8 + CDz * h14_3_2;
    const double h14_3_3 = acc[173] + ABz * acc[38];
    const double k14_3_3_1 = h14_3_6 + CDx * h14_3_3;
    const double k14_3_3_2 = h14_3_8 + CDy * h14_3_3;
    const double h14_3_9 = acc[179] + ABz * acc[44];
    const double k14_3_3_3 = h14_3_9 + CDz * h14_3_3;
    const double h15_1_4 = acc[129] + ABx * acc[48];
    const double h15_1_1 = acc[126] + ABx * acc[45];
    const double k15_1_1_1 = h15_1_4 + CDx * h15_1_1;
    const double h15_1_5 = acc[130] + ABx * acc[49];
    const double k15_1_1_2 = h15_1_5 + CDy * h15_1_1;
    const double h15_1_6 = acc[131] + ABx * acc[50];
    const double k15_1_1_3 = h15_1_6 + CDz * h15_1_1;
    const double h15_1_2 = acc[127] + ABx * acc[46];
    const double k15_1_2_1 = h15_1_5 + CDx * h15_1_2;
    const double h15_1_7 = acc[132] + ABx * acc[51];
    const double k15_1_2_2 = h15_1_7 + CDy * h15_1_2;
    const double h15_1_8 = acc[133] + ABx * acc[52];
    const double k15_1_2_3 = h15_1_8 + CDz * h15_1_2;
    const double h15_1_3 = acc[128] + ABx * acc[47];
    const double k15_1_3_1 = h15_1_6 + CDx * h15_1_3;
    const double k15_1_3_2 = h15_1_8 + CDy * h15_1_3;
    const double h15_1_9 = acc[134] + ABx * acc[53];
    const double k15_1_3_3 = h15_1_9 + CDz * h15_1_3;
    const double h15_2_4 = acc[156] + ABy * acc[48];
    const double h15_2_1 = acc[153] + ABy * acc[45];
    const double k15_2_1_1 = h15_2_4 + CDx * h15_2_1;
    const double h15_2_5 = acc[157] + ABy * acc[49];
    const double k15_2_1_2 = h15_2_5 + CDy * h15_2_1;
    const double h15_2_6 = acc[158] + ABy * acc[50];
    const double k15_2_1_3 = h15_2_6 + CDz * h15_2_1;
    const double h15_2_2 = acc[154] + ABy * acc[46];
    const double k15_2_2_1 = h15_2_5 + CDx * h15_2_2;
    const double h15_2_7 = acc[159] + ABy * acc[51];
    const double k15_2_2_2 = h15_2_7 + CDy * h15_2_2;
    const double h15_2_8 = acc[160] + ABy * acc[52];
    const double k15_2_2_3 = h15_2_8 + CDz * h15_2_2;
    const double h15_2_3 = acc[155] + ABy * acc[47];
    const double k15_2_3_1 = h15_2_6 + CDx * h15_2_3;
    const double k15_2_3_2 = h15_2_8 + CDy * h15_2_3;
    const double h15_2_9 = acc[161] + ABy * acc[53];
    const double k15_2_3_3 = h15_2_9 + CDz * h15_2_3;
    const double h15_3_4 = acc[165] + ABz * acc[48];
    const double h15_3_1 = acc[162] + ABz * acc[45];
    const double k15_3_1_1 = h15_3_4 + CDx * h15_3_1;
    const double h15_3_5 = acc[166] + ABz * acc[49];
    const double k15_3_1_2 = h15_3_5 + CDy * h15_3_1;
    const double h15_3_6 = acc[167] + ABz * acc[50];
    const double k15_3_1_3 = h15_3_6 + CDz * h15_3_1;
    const double h15_3_2 = acc[163] + ABz * acc[46];
    const double k15_3_2_1 = h15_3_5 + CDx * h15_3_2;
    const double h15_3_7 = acc[168] + ABz * acc[51];
    const double k15_3_2_2 = h15_3_7 + CDy * h15_3_2;
    const double h15_3_8 = acc[169] + ABz * acc[52];
    const double k15_3_2_3 = h15_3_8 + CDz * h15_3_2;
    const double h15_3_3 = acc[164] + ABz * acc[47];
    const double k15_3_3_1 = h15_3_6 + CDx * h15_3_3;
    const double k15_3_3_2 = h15_3_8 + CDy * h15_3_3;
    const double h15_3_9 = acc[170] + ABz * acc[53];
    const double k15_3_3_3 = h15_3_9 + CDz * h15_3_3;
    const double h16_1_4 = acc[147] + ABx * acc[57];
    const double h16_1_1 = acc[144] + ABx * acc[54];
    const double k16_1_1_1 = h16_1_4 + CDx * h16_1_1;
    const double h16_1_5 = acc[148] + ABx * acc[58];
    const double k16_1_1_2 = h16_1_5 + CDy * h16_1_1;
    const double h16_1_6 = acc[149] + ABx * acc[59];
    const double k16_1_1_3 = h16_1_6 + CDz * h16_1_1;
    const double h16_1_2 = acc[145] + ABx * acc[55];
    const double k16_1_2_1 = h16_1_5 + CDx * h16_1_2;
    const double h16_1_7 = acc[150] + ABx * acc[60];
    const double k16_1_2_2 = h16_1_7 + CDy * h16_1_2;
    const double h16_1_8 = acc[151] + ABx * acc[61];
    const double k16_1_2_3 = h16_1_8 + CDz * h16_1_2;
    const double h16_1_3 = acc[146] + ABx * acc[56];
    const double k16_1_3_1 = h16_1_6 + CDx * h16_1_3;
    const double k16_1_3_2 = h16_1_8 + CDy * h16_1_3;
    const double h16_1_9 = acc[152] + ABx * acc[62];
    const double k16_1_3_3 = h16_1_9 + CDz * h16_1_3;
    const double h16_2_4 = acc[183] + ABy * acc[57];
    const double h16_2_1 = acc[180] + ABy * acc[54];
    const double k16_2_1_1 = h16_2_4 + CDx * h16_2_1;
    const double h16_2_5 = acc[184] + ABy * acc[58];
    const double k16_2_1_2 = h16_2_5 + CDy * h16_2_1;
    const double h16_2_6 = acc[185] + ABy * acc[59];
    const double k16_2_1_3 = h16_2_6 + CDz * h16_2_1;
    const double h16_2_2 = acc[181] + ABy * acc[55];
    const double k16_2_2_1 = h16_2_5 + CDx * h16_2_2;
    const double h16_2_7 = acc[186] + ABy * acc[60];
    const double k16_2_2_2 = h16_2_7 + CDy * h16_2_2;
    const double h16_2_8 = acc[187] + ABy * acc[61];
    const double k16_2_2_3 = h16_2_8 + CDz * h16_2_2;
    const double h16_2_3 = acc[182] + ABy * acc[56];
    const double k16_2_3_1 = h16_2_6 + CDx * h16_2_3;
    const double k16_2_3_2 = h16_2_8 + CDy * h16_2_3;
    const double h16_2_9 = acc[188] + ABy * acc[62];
    const double k16_2_3_3 = h16_2_9 + CDz * h16_2_3;
    const double h16_3_4 = acc[192] + ABz * acc[57];
    const double h16_3_1 = acc[189] + ABz * acc[54];
    const double k16_3_1_1 = h16_3_4 + CDx * h16_3_1;
    const double h16_3_5 = acc[193] + ABz * acc[58];
    const double k16_3_1_2 = h16_3_5 + CDy * h16_3_1;
    const double h16_3_6 = acc[194] + ABz * acc[59];
    const double k16_3_1_3 = h16_3_6 + CDz * h16_3_1;
    const double h16_3_2 = acc[190] + ABz * acc[55];
    const double k16_3_2_1 = h16_3_5 + CDx * h16_3_2;
    const double h16_3_7 = acc[195] + ABz * acc[60];
    const double k16_3_2_2 = h16_3_7 + CDy * h16_3_2;
    const double h16_3_8 = acc[196] + ABz * acc[61];
    const double k16_3_2_3 = h16_3_8 + CDz * h16_3_2;
    const double h16_3_3 = acc[191] + ABz * acc[56];
    const double k16_3_3_1 = h16_3_6 + CDx * h16_3_3;
    const double k16_3_3_2 = h16_3_8 + CDy * h16_3_3;
    const double h16_3_9 = acc[197] + ABz * acc[62];
    const double k16_3_3_3 = h16_3_9 + CDz * h16_3_3;
    const double h17_1_4 = acc[156] + ABx * acc[66];
    const double h17_1_1 = acc[153] + ABx * acc[63];
    const double k17_1_1_1 = h17_1_4 + CDx * h17_1_1;
    const double h17_1_5 = acc[157] + ABx * acc[67];
    const double k17_1_1_2 = h17_1_5 + CDy * h17_1_1;
    const double h17_1_6 = acc[158] + ABx * acc[68];
    const double k17_1_1_3 = h17_1_6 + CDz * h17_1_1;
    const double h17_1_2 = acc[154] + ABx * acc[64];
    const double k17_1_2_1 = h17_1_5 + CDx * h17_1_2;
    const double h17_1_7 = acc[159] + ABx * acc[69];
    const double k17_1_2_2 = h17_1_7 + CDy * h17_1_2;
    const double h17_1_8 = acc[160] + ABx * acc[70];
    const double k17_1_2_3 = h17_1_8 + CDz * h17_1_2;
    const double h17_1_3 = acc[155] + ABx * acc[65];
    const double k17_1_3_1 = h17_1_6 + CDx * h17_1_3;
    const double k17_1_3_2 = h17_1_8 + CDy * h17_1_3;
    const double h17_1_9 = acc[161] + ABx * acc[71];
    const double k17_1_3_3 = h17_1_9 + CDz * h17_1_3;
    const double h17_2_4 = acc[192] + ABy * acc[66];
    const double h17_2_1 = acc[189] + ABy * acc[63];
    const double k17_2_1_1 = h17_2_4 + CDx * h17_2_1;
    const double h17_2_5 = acc[193] + ABy * acc[67];
    const double k17_2_1_2 = h17_2_5 + CDy * h17_2_1;
    const double h17_2_6 = acc[194] + ABy * acc[68];
    const double k17_2_1_3 = h17_2_6 + CDz * h17_2_1;
    const double h17_2_2 = acc[190] + ABy * acc[64];
    const double k17_2_2_1 = h17_2_5 + CDx * h17_2_2;
    const double h17_2_7 = acc[195] + ABy * acc[69];
    const double k17_2_2_2 = h17_2_7 + CDy * h17_2_2;
    const double h17_2_8 = acc[196] + ABy * acc[70];
    const double k17_2_2_3 = h17_2_8 + CDz * h17_2_2;
    const double h17_2_3 = acc[191] + ABy * acc[65];
    const double k17_2_3_1 = h17_2_6 + CDx * h17_2_3;
    const double k17_2_3_2 = h17_2_8 + CDy * h17_2_3;
    const double h17_2_9 = acc[197] + ABy * acc[71];
    const double k17_2_3_3 = h17_2_9 + CDz * h17_2_3;
    const double h17_3_4 = acc[201] + ABz * acc[66];
    const double h17_3_1 = acc[198] + ABz * acc[63];
    const double k17_3_1_1 = h17_3_4 + CDx * h17_3_1;
    const double h17_3_5 = acc[202] + ABz * acc[67];
    const double k17_3_1_2 = h17_3_5 + CDy * h17_3_1;
    const double h17_3_6 = acc[203] + ABz * acc[68];
    const double k17_3_1_3 = h17_3_6 + CDz * h17_3_1;
    const double h17_3_2 = acc[199] + ABz * acc[64];
    const double k17_3_2_1 = h17_3_5 + CDx * h17_3_2;
    const double h17_3_7 = acc[204] + ABz * acc[69];
    const double k17_3_2_2 = h17_3_7 + CDy * h17_3_2;
    const double h17_3_8 = acc[205] + ABz * acc[70];
    const double k17_3_2_3 = h17_3_8 + CDz * h17_3_2;
    const double h17_3_3 = acc[200] + ABz * acc[65];
    const double k17_3_3_1 = h17_3_6 + CDx * h17_3_3;
    const double k17_3_3_2 = h17_3_8 + CDy * h17_3_3;
    const double h17_3_9 = acc[206] + ABz * acc[71];
    const double k17_3_3_3 = h17_3_9 + CDz * h17_3_3;
    const double h18_1_4 = acc[165] + ABx * acc[75];
    const double h18_1_1 = acc[162] + ABx * acc[72];
    const double k18_1_1_1 = h18_1_4 + CDx * h18_1_1;
    const double h18_1_5 = acc[166] + ABx * acc[76];
    const double k18_1_1_2 = h18_1_5 + CDy * h18_1_1;
    const double h18_1_6 = acc[167] + ABx * acc[77];
    const double k18_1_1_3 = h18_1_6 + CDz * h18_1_1;
    const double h18_1_2 = acc[163] + ABx * acc[73];
    const double k18_1_2_1 = h18_1_5 + CDx * h18_1_2;
    const double h18_1_7 = acc[168] + ABx * acc[78];
    const double k18_1_2_2 = h18_1_7 + CDy * h18_1_2;
    const double h18_1_8 = acc[169] + ABx * acc[79];
    const double k18_1_2_3 = h18_1_8 + CDz * h18_1_2;
    const double h18_1_3 = acc[164] + ABx * acc[74];
    const double k18_1_3_1 = h18_1_6 + CDx * h18_1_3;
    const double k18_1_3_2 = h18_1_8 + CDy * h18_1_3;
    const double h18_1_9 = acc[170] + ABx * acc[80];
    const double k18_1_3_3 = h18_1_9 + CDz * h18_1_3;
    const double h18_2_4 = acc[201] + ABy * acc[75];
    const double h18_2_1 = acc[198] + ABy * acc[72];
    const double k18_2_1_1 = h18_2_4 + CDx * h18_2_1;
    const double h18_2_5 = acc[202] + ABy * acc[76];
    const double k18_2_1_2 = h18_2_5 + CDy * h18_2_1;
    const double h18_2_6 = acc[203] + ABy * acc[77];
    const double k18_2_1_3 = h18_2_6 + CDz * h18_2_1;
    const double h18_2_2 = acc[199] + ABy * acc[73];
    const double k18_2_2_1 = h18_2_5 + CDx * h18_2_2;
    const double h18_2_7 = acc[204] + ABy * acc[78];
    const double k18_2_2_2 = h18_2_7 + CDy * h18_2_2;
    const double h18_2_8 = acc[205] + ABy * acc[79];
    const double k18_2_2_3 = h18_2_8 + CDz * h18_2_2;
    const double h18_2_3 = acc[200] + ABy * acc[74];
    const double k18_2_3_1 = h18_2_6 + CDx * h18_2_3;
    const double k18_2_3_2 = h18_2_8 + CDy * h18_2_3;
    const double h18_2_9 = acc[206] + ABy * acc[80];
    const double k18_2_3_3 = h18_2_9 + CDz * h18_2_3;
    const double h18_3_4 = acc[210] + ABz * acc[75];
    const double h18_3_1 = acc[207] + ABz * acc[72];
    const double k18_3_1_1 = h18_3_4 + CDx * h18_3_1;
    const double h18_3_5 = acc[211] + ABz * acc[76];
    const double k18_3_1_2 = h18_3_5 + CDy * h18_3_1;
    const double h18_3_6 = acc[212] + ABz * acc[77];
    const double k18_3_1_3 = h18_3_6 + CDz * h18_3_1;
    const double h18_3_2 = acc[208] + ABz * acc[73];
    const double k18_3_2_1 = h18_3_5 + CDx * h18_3_2;
    const double h18_3_7 = acc[213] + ABz * acc[78];
    const double k18_3_2_2 = h18_3_7 + CDy * h18_3_2;
    const double h18_3_8 = acc[214] + ABz * acc[79];
    const double k18_3_2_3 = h18_3_8 + CDz * h18_3_2;
    const double h18_3_3 = acc[209] + ABz * acc[74];
    const double k18_3_3_1 = h18_3_6 + CDx * h18_3_3;
    const double k18_3_3_2 = h18_3_8 + CDy * h18_3_3;
    const double h18_3_9 = acc[215] + ABz * acc[80];
    const double k18_3_3_3 = h18_3_9 + CDz * h18_3_3;
    const double h19_1_4 = acc[174] + ABx * acc[84];
    const double h19_1_1 = acc[171] + ABx * acc[81];
    const double k19_1_1_1 = h19_1_4 + CDx * h19_1_1;
    const double h19_1_5 = acc[175] + ABx * acc[85];
    const double k19_1_1_2 = h19_1_5 + CDy * h19_1_1;
    const double h19_1_6 = acc[176] + ABx * acc[86];
    const double k19_1_1_3 = h19_1_6 + CDz * h19_1_1;
    const double h19_1_2 = acc[172] + ABx * acc[82];
    const double k19_1_2_1 = h19_1_5 + CDx * h19_1_2;
    const double h19_1_7 = acc[177] + ABx * acc[87];
    const double k19_1_2_2 = h19_1_7 + CDy * h19_1_2;
    const double h19_1_8 = acc[178] + ABx * acc[88];
    const double k19_1_2_3 = h19_1_8 + CDz * h19_1_2;
    const double h19_1_3 = acc[173] + ABx * acc[83];
    const double k19_1_3_1 = h19_1_6 + CDx * h19_1_3;
    const double k19_1_3_2 = h19_1_8 + CDy * h19_1_3;
    const double h19_1_9 = acc[179] + ABx * acc[89];
    const double k19_1_3_3 = h19_1_9 + CDz * h19_1_3;
    const double h19_2_4 = acc[210] + ABy * acc[84];
    const double h19_2_1 = acc[207] + ABy * acc[81];
    const double k19_2_1_1 = h19_2_4 + CDx * h19_2_1;
    const double h19_2_5 = acc[211] + ABy * acc[85];
    const double k19_2_1_2 = h19_2_5 + CDy * h19_2_1;
    const double h19_2_6 = acc[212] + ABy * acc[86];
    const double k19_2_1_3 = h19_2_6 + CDz * h19_2_1;
    const double h19_2_2 = acc[208] + ABy * acc[82];
    const double k19_2_2_1 = h19_2_5 + CDx * h19_2_2;
    const double h19_2_7 = acc[213] + ABy * acc[87];
    const double k19_2_2_2 = h19_2_7 + CDy * h19_2_2;
    const double h19_2_8 = acc[214] + ABy * acc[88];
    const double k19_2_2_3 = h19_2_8 + CDz * h19_2_2;
    const double h19_2_3 = acc[209] + ABy * acc[83];
    const double k19_2_3_1 = h19_2_6 + CDx * h19_2_3;
    const double k19_2_3_2 = h19_2_8 + CDy * h19_2_3;
    const double h19_2_9 = acc[215] + ABy * acc[89];
    const double k19_2_3_3 = h19_2_9 + CDz * h19_2_3;
    const double h19_3_4 = acc[219] + ABz * acc[84];
    const double h19_3_1 = acc[216] + ABz * acc[81];
    const double k19_3_1_1 = h19_3_4 + CDx * h19_3_1;
    const double h19_3_5 = acc[220] + ABz * acc[85];
    const double k19_3_1_2 = h19_3_5 + CDy * h19_3_1;
    const double h19_3_6 = acc[221] + ABz * acc[86];
    const double k19_3_1_3 = h19_3_6 + CDz * h19_3_1;
    const double h19_3_2 = acc[217] + ABz * acc[82];
    const double k19_3_2_1 = h19_3_5 + CDx * h19_3_2;
    const double h19_3_7 = acc[222] + ABz * acc[87];
    const double k19_3_2_2 = h19_3_7 + CDy * h19_3_2;
    const double h19_3_8 = acc[223] + ABz * acc[88];
    const double k19_3_2_3 = h19_3_8 + CDz * h19_3_2;
    const double h19_3_3 = acc[218] + ABz * acc[83];
    const double k19_3_3_1 = h19_3_6 + CDx * h19_3_3;
    const double k19_3_3_2 = h19_3_8 + CDy * h19_3_3;
    const double h19_3_9 = acc[224] + ABz * acc[89];
    const double k19_3_3_3 = h19_3_9 + CDz * h19_3_3;
    res[0] = k10_1_1_1 * 0.2581988897471611;
    res[1] = k10_1_1_2 * 0.2581988897471611;
    res[2] = k10_1_1_3 * 0.2581988897471611;
    res[3] = k10_1_2_1 * 0.2581988897471611;
    res[4] = k10_1_2_2 * 0.2581988897471611;
    res[5] = k10_1_2_3 * 0.2581988897471611;
    res[6] = k10_1_3_1 * 0.2581988897471611;
    res[7] = k10_1_3_2 * 0.2581988897471611;
    res[8] = k10_1_3_3 * 0.2581988897471611;
    res[9] = k10_2_1_1 * 0.2581988897471611;
    res[10] = k10_2_1_2 * 0.2581988897471611;
    res[11] = k10_2_1_3 * 0.2581988897471611;
    res[12] = k10_2_2_1 * 0.2581988897471611;
    res[13] = k10_2_2_2 * 0.2581988897471611;
    res[14] = k10_2_2_3 * 0.2581988897471611;
    res[15] = k10_2_3_1 * 0.2581988897471611;
    res[16] = k10_2_3_2 * 0.2581988897471611;
    res[17] = k10_2_3_3 * 0.2581988897471611;
    res[18] = k10_3_1_1 * 0.2581988897471611;
    res[19] = k10_3_1_2 * 0.2581988897471611;
    res[20] = k10_3_1_3 * 0.2581988897471611;
    res[21] = k10_3_2_1 * 0.2581988897471611;
    res[22] = k10_3_2_2 * 0.2581988897471611;
    res[23] = k10_3_2_3 * 0.2581988897471611;
    res[24] = k10_3_3_1 * 0.2581988897471611;
    res[25] = k10_3_3_2 * 0.2581988897471611;
    res[26] = k10_3_3_3 * 0.2581988897471611;
    res[27] = k11_1_1_1 * 0.5773502691896258;
    res[28] = k11_1_1_2 * 0.5773502691896258;
    res[29] = k11_1_1_3 * 0.5773502691896258;
    res[30] = k11_1_2_1 * 0.5773502691896258;
    res[31] = k11_1_2_2 * 0.5773502691896258;
    res[32] = k11_1_2_3 * 0.5773502691896258;
    res[33] = k11_1_3_1 * 0.5773502691896258;
    res[34] = k11_1_3_2 * 0.5773502691896258;
    res[35] = k11_1_3_3 * 0.5773502691896258;
    res[36] = k11_2_1_1 * 0.5773502691896258;
    res[37] = k11_2_1_2 * 0.5773502691896258;
    res[38] = k11_2_1_3 * 0.5773502691896258;
    res[39] = k11_2_2_1 * 0.5773502691896258;
    res[40] = k11_2_2_2 * 0.5773502691896258;
    res[41] = k11_2_2_3 * 0.5773502691896258;
    res[42] = k11_2_3_1 * 0.5773502691896258;
    res[43] = k11_2_3_2 * 0.5773502691896258;
    res[44] = k11_2_3_3 * 0.5773502691896258;
    res[45] = k11_3_1_1 * 0.5773502691896258;
    res[46] = k11_3_1_2 * 0.5773502691896258;
    res[47] = k11_3_1_3 * 0.5773502691896258;
    res[48] = k11_3_2_1 * 0.5773502691896258;
    res[49] = k11_3_2_2 * 0.5773502691896258;
    res[50] = k11_3_2_3 * 0.5773502691896258;
    res[51] = k11_3_3_1 * 0.5773502691896258;
    res[52] = k11_3_3_2 * 0.5773502691896258;
    res[53] = k11_3_3_3 * 0.5773502691896258;
    res[54] = k12_1_1_1 * 0.5773502691896258;
    res[55] = k12_1_1_2 * 0.5773502691896258;
    res[56] = k12_1_1_3 * 0.5773502691896258;
    res[57] = k12_1_2_1 * 0.5773502691896258;
    res[58] = k12_1_2_2 * 0.5773502691896258;
    res[59] = k12_1_2_3 * 0.5773502691896258;
    res[60] = k12_1_3_1 * 0.5773502691896258;
    res[61] = k12_1_3_2 * 0.5773502691896258;
    res[62] = k12_1_3_3 * 0.5773502691896258;
    res[63] = k12_2_1_1 * 0.5773502691896258;
    res[64] = k12_2_1_2 * 0.5773502691896258;
    res[65] = k12_2_1_3 * 0.5773502691896258;
    res[66] = k12_2_2_1 * 0.5773502691896258;
    res[67] = k12_2_2_2 * 0.5773502691896258;
    res[68] = k12_2_2_3 * 0.5773502691896258;
    res[69] = k12_2_3_1 * 0.5773502691896258;
    res[70] = k12_2_3_2 * 0.5773502691896258;
    res[71] = k12_2_3_3 * 0.5773502691896258;
    res[72] = k12_3_1_1 * 0.5773502691896258;
    res[73] = k12_3_1_2 * 0.5773502691896258;
    res[74] = k12_3_1_3 * 0.5773502691896258;
    res[75] = k12_3_2_1 * 0.5773502691896258;
    res[76] = k12_3_2_2 * 0.5773502691896258;
    res[77] = k12_3_2_3 * 0.5773502691896258;
    res[78] = k12_3_3_1 * 0.5773502691896258;
    res[79] = k12_3_3_2 * 0.5773502691896258;
    res[80] = k12_3_3_3 * 0.5773502691896258;
    res[81] = k13_1_1_1 * 0.5773502691896258;
    res[82] = k13_1_1_2 * 0.5773502691896258;
    res[83] = k13_1_1_3 * 0.5773502691896258;
    res[84] = k13_1_2_1 * 0.5773502691896258;
    res[85] = k13_1_2_2 * 0.5773502691896258;
    res[86] = k13_1_2_3 * 0.5773502691896258;
    res[87] = k13_1_3_1 * 0.5773502691896258;
    res[88] = k13_1_3_2 * 0.5773502691896258;
    res[89] = k13_1_3_3 * 0.5773502691896258;
    res[90] = k13_2_1_1 * 0.5773502691896258;
    res[91] = k13_2_1_2 * 0.5773502691896258;
    res[92] = k13_2_1_3 * 0.5773502691896258;
    res[93] = k13_2_2_1 * 0.5773502691896258;
    res[94] = k13_2_2_2 * 0.5773502691896258;
    res[95] = k13_2_2_3 * 0.5773502691896258;
    res[96] = k13_2_3_1 * 0.5773502691896258;
    res[97] = k13_2_3_2 * 0.5773502691896258;
    res[98] = k13_2_3_3 * 0.5773502691896258;
    res[99] = k13_3_1_1 * 0.5773502691896258;
    res[100] = k13_3_1_2 * 0.5773502691896258;
    res[101] = k13_3_1_3 * 0.5773502691896258;
    res[102] = k13_3_2_1 * 0.5773502691896258;
    res[103] = k13_3_2_2 * 0.5773502691896258;
    res[104] = k13_3_2_3 * 0.5773502691896258;
    res[105] = k13_3_3_1 * 0.5773502691896258;
    res[106] = k13_3_3_2 * 0.5773502691896258;
    res[107] = k13_3_3_3 * 0.5773502691896258;
    res[108] = k14_1_1_1 * 0.5773502691896258;
    res[109] = k14_1_1_2 * 0.5773502691896258;
    res[110] = k14_1_1_3 * 0.5773502691896258;
    res[111] = k14_1_2_1 * 0.5773502691896258;
    res[112] = k14_1_2_2 * 0.5773502691896258;
    res[113] = k14_1_2_3 * 0.5773502691896258;
    res[114] = k14_1_3_1 * 0.5773502691896258;
    res[115] = k14_1_3_2 * 0.5773502691896258;
    res[116] = k14_1_3_3 * 0.5773502691896258;
    res[117] = k14_2_1_1 * 0.5773502691896258;
    res[118] = k14_2_1_2 * 0.5773502691896258;
    res[119] = k14_2_1_3 * 0.5773502691896258;
    res[120] = k14_2_2_1 * 0.5773502691896258;
    res[121] = k14_2_2_2 * 0.5773502691896258;
    res[122] = k14_2_2_3 * 0.5773502691896258;
    res[123] = k14_2_3_1 * 0.5773502691896258;
    res[124] = k14_2_3_2 * 0.5773502691896258;
    res[125] = k14_2_3_3 * 0.5773502691896258;
    res[126] = k14_3_1_1 * 0.5773502691896258;
    res[127] = k14_3_1_2 * 0.5773502691896258;
    res[128] = k14_3_1_3 * 0.5773502691896258;
    res[129] = k14_3_2_1 * 0.5773502691896258;
    res[130] = k14_3_2_2 * 0.5773502691896258;
    res[131] = k14_3_2_3 * 0.5773502691896258;
    res[132] = k14_3_3_1 * 0.5773502691896258;
    res[133] = k14_3_3_2 * 0.5773502691896258;
    res[134] = k14_3_3_3 * 0.5773502691896258;
    res[135] = k15_1_1_1;
    res[136] = k15_1_1_2;
    res[137] = k15_1_1_3;
    res[138] = k15_1_2_1;
    res[139] = k15_1_2_2;
    res[140] = k15_1_2_3;
    res[141] = k15_1_3_1;
    res[142] = k15_1_3_2;
    res[143] = k15_1_3_3;
    res[144] = k15_2_1_1;
    res[145] = k15_2_1_2;
    res[146] = k15_2_1_3;
    res[147] = k15_2_2_1;
    res[148] = k15_2_2_2;
    res[149] = k15_2_2_3;
    res[150] = k15_2_3_1;
    res[151] = k15_2_3_2;
    res[152] = k15_2_3_3;
    res[153] = k15_3_1_1;
    res[154] = k15_3_1_2;
    res[155] = k15_3_1_3;
    res[156] = k15_3_2_1;
    res[157] = k15_3_2_2;
    res[158] = k15_3_2_3;
    res[159] = k15_3_3_1;
    res[160] = k15_3_3_2;
    res[161] = k15_3_3_3;
    res[162] = k16_1_1_1 * 0.2581988897471611;
    res[163] = k16_1_1_2 * 0.2581988897471611;
    res[164] = k16_1_1_3 * 0.2581988897471611;
    res[165] = k16_1_2_1 * 0.2581988897471611;
    res[166] = k16_1_2_2 * 0.2581988897471611;
    res[167] = k16_1_2_3 * 0.2581988897471611;
    res[168] = k16_1_3_1 * 0.2581988897471611;
    res[169] = k16_1_3_2 * 0.2581988897471611;
    res[170] = k16_1_3_3 * 0.2581988897471611;
    res[171] = k16_2_1_1 * 0.2581988897471611;
    res[172] = k16_2_1_2 * 0.2581988897471611;
    res[173] = k16_2_1_3 * 0.2581988897471611;
    res[174] = k16_2_2_1 * 0.2581988897471611;
    res[175] = k16_2_2_2 * 0.2581988897471611;
    res[176] = k16_2_2_3 * 0.2581988897471611;
    res[177] = k16_2_3_1 * 0.2581988897471611;
    res[178] = k16_2_3_2 * 0.2581988897471611;
    res[179] = k16_2_3_3 * 0.2581988897471611;
    res[180] = k16_3_1_1 * 0.2581988897471611;
    res[181] = k16_3_1_2 * 0.2581988897471611;
    res[182] = k16_3_1_3 * 0.2581988897471611;
    res[183] = k16_3_2_1 * 0.2581988897471611;
    res[184] = k16_3_2_2 * 0.2581988897471611;
    res[185] = k16_3_2_3 * 0.2581988897471611;
    res[186] = k16_3_3_1 * 0.2581988897471611;
    res[187] = k16_3_3_2 * 0.2581988897471611;
    res[188] = k16_3_3_3 * 0.2581988897471611;
    res[189] = k17_1_1_1 * 0.5773502691896258;
    res[190] = k17_1_1_2 * 0.5773502691896258;
    res[191] = k17_1_1_3 * 0.5773502691896258;
    res[192] = k17_1_2_1 * 0.5773502691896258;
    res[193] = k17_1_2_2 * 0.5773502691896258;
    res[194] = k17_1_2_3 * 0.5773502691896258;
    res[195] = k17_1_3_1 * 0.5773502691896258;
    res[196] = k17_1_3_2 * 0.5773502691896258;
    res[197] = k17_1_3_3 * 0.5773502691896258;
    res[198] = k17_2_1_1 * 0.5773502691896258;
    res[199] = k17_2_1_2 * 0.5773502691896258;
    res[200] = k17_2_1_3 * 0.5773502691896258;
    res[201] = k17_2_2_1 * 0.5773502691896258;
    res[202] = k17_2_2_2 * 0.5773502691896258;
    res[203] = k17_2_2_3 * 0.5773502691896258;
    res[204] = k17_2_3_1 * 0.5773502691896258;
    res[205] = k17_2_3_2 * 0.5773502691896258;
    res[206] = k17_2_3_3 * 0.5773502691896258;
    res[207] = k17_3_1_1 * 0.5773502691896258;
    res[208] = k17_3_1_2 * 0.5773502691896258;
    res[209] = k17_3_1_3 * 0.5773502691896258;
    res[210] = k17_3_2_1 * 0.5773502691896258;
    res[211] = k17_3_2_2 * 0.5773502691896258;
    res[212] = k17_3_2_3 * 0.5773502691896258;
    res[213] = k17_3_3_1 * 0.5773502691896258;
    res[214] = k17_3_3_2 * 0.5773502691896258;
    res[215] = k17_3_3_3 * 0.5773502691896258;
    res[216] = k18_1_1_1 * 0.5773502691896258;
    res[217] = k18_1_1_2 * 0.5773502691896258;
    res[218] = k18_1_1_3 * 0.5773502691896258;
    res[219] = k18_1_2_1 * 0.5773502691896258;
    res[220] = k18_1_2_2 * 0.5773502691896258;
    res[221] = k18_1_2_3 * 0.5773502691896258;
    res[222] = k18_1_3_1 * 0.5773502691896258;
    res[223] = k18_1_3_2 * 0.5773502691896258;
    res[224] = k18_1_3_3 * 0.5773502691896258;
    res[225] = k18_2_1_1 * 0.5773502691896258;
    res[226] = k18_2_1_2 * 0.5773502691896258;
    res[227] = k18_2_1_3 * 0.5773502691896258;
    res[228] = k18_2_2_1 * 0.5773502691896258;
    res[229] = k18_2_2_2 * 0.5773502691896258;
    res[230] = k18_2_2_3 * 0.5773502691896258;
    res[231] = k18_2_3_1 * 0.5773502691896258;
    res[232] = k18_2_3_2 * 0.5773502691896258;
    res[233] = k18_2_3_3 * 0.5773502691896258;
    res[234] = k18_3_1_1 * 0.5773502691896258;
    res[235] = k18_3_1_2 * 0.5773502691896258;
    res[236] = k18_3_1_3 * 0.5773502691896258;
    res[237] = k18_3_2_1 * 0.5773502691896258;
    res[238] = k18_3_2_2 * 0.5773502691896258;
    res[239] = k18_3_2_3 * 0.5773502691896258;
    res[240] = k18_3_3_1 * 0.5773502691896258;
    res[241] = k18_3_3_2 * 0.5773502691896258;
    res[242] = k18_3_3_3 * 0.5773502691896258;
    res[243] = k19_1_1_1 * 0.2581988897471611;
    res[244] = k19_1_1_2 * 0.2581988897471611;
    res[245] = k19_1_1_3 * 0.2581988897471611;
    res[246] = k19_1_2_1 * 0.2581988897471611;
    res[247] = k19_1_2_2 * 0.2581988897471611;
    res[248] = k19_1_2_3 * 0.2581988897471611;
    res[249] = k19_1_3_1 * 0.2581988897471611;
    res[250] = k19_1_3_2 * 0.2581988897471611;
    res[251] = k19_1_3_3 * 0.2581988897471611;
    res[252] = k19_2_1_1 * 0.2581988897471611;
    res[253] = k19_2_1_2 * 0.2581988897471611;
    res[254] = k19_2_1_3 * 0.2581988897471611;
    res[255] = k19_2_2_1 * 0.2581988897471611;
    res[256] = k19_2_2_2 * 0.2581988897471611;
    res[257] = k19_2_2_3 * 0.2581988897471611;
    res[258] = k19_2_3_1 * 0.2581988897471611;
    res[259] = k19_2_3_2 * 0.2581988897471611;
    res[260] = k19_2_3_3 * 0.2581988897471611;
    res[261] = k19_3_1_1 * 0.2581988897471611;
    res[262] = k19_3_1_2 * 0.2581988897471611;
    res[263] = k19_3_1_3 * 0.2581988897471611;
    res[264] = k19_3_2_1 * 0.2581988897471611;
    res[265] = k19_3_2_2 * 0.2581988897471611;
    res[266] = k19_3_2_3 * 0.2581988897471611;
    res[267] = k19_3_3_1 * 0.2581988897471611;
    res[268] = k19_3_3_2 * 0.2581988897471611;
    res[269] = k19_3_3_3 * 0.2581988897471611;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[270]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_fppp(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[225];
    vrr_fppp<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 225; ++x) acc_out[x] = acc[x];
    }
    hrr_fppp(P, p, q, acc, res);
}

__device__ __forceinline__ void store_fppp(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
    { const long long ij = ij_0_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_0_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_0_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_0_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_0_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_0_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_0_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_0_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_0_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_0_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_0_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_0_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_0_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_0_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_0_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_0_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_0_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_1_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_1_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_1_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_1_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_1_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_1_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_1_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_1_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_1_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_1_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_1_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_1_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_1_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_1_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_1_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_1_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_1_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_1_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_2_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_2_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_2_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_2_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_2_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_2_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_2_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_2_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_2_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_2_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_2_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_2_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_2_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_2_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_2_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_2_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_2_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_2_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_3_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_3_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_3_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_3_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_3_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_3_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_3_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_3_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_3_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_3_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_3_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_3_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_3_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_3_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
    { const long long ij = ij_3_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[100]; }
    { const long long ij = ij_3_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[101]; }
    { const long long ij = ij_3_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[102]; }
    { const long long ij = ij_3_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[103]; }
    { const long long ij = ij_3_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[104]; }
    { const long long ij = ij_3_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[105]; }
    { const long long ij = ij_3_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[106]; }
    { const long long ij = ij_3_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[107]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[108]; }
    { const long long ij = ij_4_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[109]; }
    { const long long ij = ij_4_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[110]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[111]; }
    { const long long ij = ij_4_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[112]; }
    { const long long ij = ij_4_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[113]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[114]; }
    { const long long ij = ij_4_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[115]; }
    { const long long ij = ij_4_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[116]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[117]; }
    { const long long ij = ij_4_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[118]; }
    { const long long ij = ij_4_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[119]; }
    { const long long ij = ij_4_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[120]; }
    { const long long ij = ij_4_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[121]; }
    { const long long ij = ij_4_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[122]; }
    { const long long ij = ij_4_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[123]; }
    { const long long ij = ij_4_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[124]; }
    { const long long ij = ij_4_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[125]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[126]; }
    { const long long ij = ij_4_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[127]; }
    { const long long ij = ij_4_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[128]; }
    { const long long ij = ij_4_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[129]; }
    { const long long ij = ij_4_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[130]; }
    { const long long ij = ij_4_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[131]; }
    { const long long ij = ij_4_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[132]; }
    { const long long ij = ij_4_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[133]; }
    { const long long ij = ij_4_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[134]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[135]; }
    { const long long ij = ij_5_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[136]; }
    { const long long ij = ij_5_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[137]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[138]; }
    { const long long ij = ij_5_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[139]; }
    { const long long ij = ij_5_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[140]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[141]; }
    { const long long ij = ij_5_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[142]; }
    { const long long ij = ij_5_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[143]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[144]; }
    { const long long ij = ij_5_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[145]; }
    { const long long ij = ij_5_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[146]; }
    { const long long ij = ij_5_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[147]; }
    { const long long ij = ij_5_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[148]; }
    { const long long ij = ij_5_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[149]; }
    { const long long ij = ij_5_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[150]; }
    { const long long ij = ij_5_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[151]; }
    { const long long ij = ij_5_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[152]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[153]; }
    { const long long ij = ij_5_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[154]; }
    { const long long ij = ij_5_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[155]; }
    { const long long ij = ij_5_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[156]; }
    { const long long ij = ij_5_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[157]; }
    { const long long ij = ij_5_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[158]; }
    { const long long ij = ij_5_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[159]; }
    { const long long ij = ij_5_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[160]; }
    { const long long ij = ij_5_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[161]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[162]; }
    { const long long ij = ij_6_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[163]; }
    { const long long ij = ij_6_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[164]; }
    { const long long ij = ij_6_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[165]; }
    { const long long ij = ij_6_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[166]; }
    { const long long ij = ij_6_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[167]; }
    { const long long ij = ij_6_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[168]; }
    { const long long ij = ij_6_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[169]; }
    { const long long ij = ij_6_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[170]; }
    { const long long ij = ij_6_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[171]; }
    { const long long ij = ij_6_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[172]; }
    { const long long ij = ij_6_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[173]; }
    { const long long ij = ij_6_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[174]; }
    { const long long ij = ij_6_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[175]; }
    { const long long ij = ij_6_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[176]; }
    { const long long ij = ij_6_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[177]; }
    { const long long ij = ij_6_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[178]; }
    { const long long ij = ij_6_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[179]; }
    { const long long ij = ij_6_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[180]; }
    { const long long ij = ij_6_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[181]; }
    { const long long ij = ij_6_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[182]; }
    { const long long ij = ij_6_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[183]; }
    { const long long ij = ij_6_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[184]; }
    { const long long ij = ij_6_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[185]; }
    { const long long ij = ij_6_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[186]; }
    { const long long ij = ij_6_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[187]; }
    { const long long ij = ij_6_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[188]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[189]; }
    { const long long ij = ij_7_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[190]; }
    { const long long ij = ij_7_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[191]; }
    { const long long ij = ij_7_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[192]; }
    { const long long ij = ij_7_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[193]; }
    { const long long ij = ij_7_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[194]; }
    { const long long ij = ij_7_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[195]; }
    { const long long ij = ij_7_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[196]; }
    { const long long ij = ij_7_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[197]; }
    { const long long ij = ij_7_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[198]; }
    { const long long ij = ij_7_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[199]; }
    { const long long ij = ij_7_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[200]; }
    { const long long ij = ij_7_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[201]; }
    { const long long ij = ij_7_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[202]; }
    { const long long ij = ij_7_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[203]; }
    { const long long ij = ij_7_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[204]; }
    { const long long ij = ij_7_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[205]; }
    { const long long ij = ij_7_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[206]; }
    { const long long ij = ij_7_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[207]; }
    { const long long ij = ij_7_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[208]; }
    { const long long ij = ij_7_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[209]; }
    { const long long ij = ij_7_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[210]; }
    { const long long ij = ij_7_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[211]; }
    { const long long ij = ij_7_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[212]; }
    { const long long ij = ij_7_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[213]; }
    { const long long ij = ij_7_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[214]; }
    { const long long ij = ij_7_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[215]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[216]; }
    { const long long ij = ij_8_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[217]; }
    { const long long ij = ij_8_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[218]; }
    { const long long ij = ij_8_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[219]; }
    { const long long ij = ij_8_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[220]; }
    { const long long ij = ij_8_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[221]; }
    { const long long ij = ij_8_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[222]; }
    { const long long ij = ij_8_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[223]; }
    { const long long ij = ij_8_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[224]; }
    { const long long ij = ij_8_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[225]; }
    { const long long ij = ij_8_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[226]; }
    { const long long ij = ij_8_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[227]; }
    { const long long ij = ij_8_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[228]; }
    { const long long ij = ij_8_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[229]; }
    { const long long ij = ij_8_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[230]; }
    { const long long ij = ij_8_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[231]; }
    { const long long ij = ij_8_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[232]; }
    { const long long ij = ij_8_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[233]; }
    { const long long ij = ij_8_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[234]; }
    { const long long ij = ij_8_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[235]; }
    { const long long ij = ij_8_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[236]; }
    { const long long ij = ij_8_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[237]; }
    { const long long ij = ij_8_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[238]; }
    { const long long ij = ij_8_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[239]; }
    { const long long ij = ij_8_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[240]; }
    { const long long ij = ij_8_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[241]; }
    { const long long ij = ij_8_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[242]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[243]; }
    { const long long ij = ij_9_0, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[244]; }
    { const long long ij = ij_9_0, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[245]; }
    { const long long ij = ij_9_0, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[246]; }
    { const long long ij = ij_9_0, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[247]; }
    { const long long ij = ij_9_0, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[248]; }
    { const long long ij = ij_9_0, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[249]; }
    { const long long ij = ij_9_0, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[250]; }
    { const long long ij = ij_9_0, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[251]; }
    { const long long ij = ij_9_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[252]; }
    { const long long ij = ij_9_1, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[253]; }
    { const long long ij = ij_9_1, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[254]; }
    { const long long ij = ij_9_1, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[255]; }
    { const long long ij = ij_9_1, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[256]; }
    { const long long ij = ij_9_1, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[257]; }
    { const long long ij = ij_9_1, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[258]; }
    { const long long ij = ij_9_1, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[259]; }
    { const long long ij = ij_9_1, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[260]; }
    { const long long ij = ij_9_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[261]; }
    { const long long ij = ij_9_2, kl = kl_0_1;
      if ((!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[262]; }
    { const long long ij = ij_9_2, kl = kl_0_2;
      if ((!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[263]; }
    { const long long ij = ij_9_2, kl = kl_1_0;
      if ((!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[264]; }
    { const long long ij = ij_9_2, kl = kl_1_1;
      if ((!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[265]; }
    { const long long ij = ij_9_2, kl = kl_1_2;
      if ((!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[266]; }
    { const long long ij = ij_9_2, kl = kl_2_0;
      if ((!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[267]; }
    { const long long ij = ij_9_2, kl = kl_2_1;
      if ((!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[268]; }
    { const long long ij = ij_9_2, kl = kl_2_2;
      if ((!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[269]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_fppp(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 270; ++x) {
        const int ia = x / 27, ibb = (x / 9) % 3, ic = (x / 3) % 3, id = x % 3;
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
__global__ void __launch_bounds__(128) eri_queue_fppp(const EriQueue Q) {
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
        double acc[225];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 225; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_fppp<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_fppp<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 225; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: each leader stores its quartet's whole block at its slot
            if (lead) {
                double res[270];
                hrr_fppp(Q.pairs, p, q, acc, res);
                double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                    (__ldg(&Q.chunk_slot[c]) + base + kq) * (long long)270;
#pragma unroll
                for (int x = 0; x < 270; ++x) dst[x] = res[x];
            }
        } else if (lead) {
            double res[270];
            hrr_fppp(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_fppp(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_fppp(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_fppp(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    constexpr size_t smem = 0;
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_fppp<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_fppp<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_fppp<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_fppp<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_fppp(int mixed) {

    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fppp<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fppp<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

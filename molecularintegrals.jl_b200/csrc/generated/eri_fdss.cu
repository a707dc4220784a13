// Generated by gen_eri.py -- class (fd|ss).  Do not edit.
// VRR entries: 126, contracted block: 46, HRR lines: 129, outputs: 60.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[46], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_fdss(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 46; ++x) acc[x] = 0.0;
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
            const VT v35_0_0 = PAx * v20_0_0 + WPx * v20_0_1 + (VT)4.0 * oo2z * (v10_0_0 - rho_z * v10_0_1);
            const VT v36_0_0 = PAx * v21_0_0 + WPx * v21_0_1 + (VT)3.0 * oo2z * (v11_0_0 - rho_z * v11_0_1);
            const VT v37_0_0 = PAx * v22_0_0 + WPx * v22_0_1 + (VT)3.0 * oo2z * (v12_0_0 - rho_z * v12_0_1);
            const VT v38_0_0 = PAx * v23_0_0 + WPx * v23_0_1 + (VT)2.0 * oo2z * (v13_0_0 - rho_z * v13_0_1);
            const VT v39_0_0 = PAx * v24_0_0 + WPx * v24_0_1 + (VT)2.0 * oo2z * (v15_0_0 - rho_z * v15_0_1);
            const VT v40_0_0 = PAx * v25_0_0 + WPx * v25_0_1 + (VT)2.0 * oo2z * (v14_0_0 - rho_z * v14_0_1);
            const VT v41_0_0 = PAy * v23_0_0 + WPy * v23_0_1 + (VT)2.0 * oo2z * (v11_0_0 - rho_z * v11_0_1);
            const VT v42_0_0 = PAx * v27_0_0 + WPx * v27_0_1 + (VT)1.0 * oo2z * (v17_0_0 - rho_z * v17_0_1);
            const VT v43_0_0 = PAx * v28_0_0 + WPx * v28_0_1 + (VT)1.0 * oo2z * (v18_0_0 - rho_z * v18_0_1);
            const VT v44_0_0 = PAz * v25_0_0 + WPz * v25_0_1 + (VT)2.0 * oo2z * (v12_0_0 - rho_z * v12_0_1);
            const VT v45_0_0 = PAy * v26_0_0 + WPy * v26_0_1 + (VT)3.0 * oo2z * (v13_0_0 - rho_z * v13_0_1);
            const VT v46_0_0 = PAy * v27_0_0 + WPy * v27_0_1 + (VT)2.0 * oo2z * (v15_0_0 - rho_z * v15_0_1);
            const VT v47_0_0 = PAy * v28_0_0 + WPy * v28_0_1 + (VT)1.0 * oo2z * (v14_0_0 - rho_z * v14_0_1);
            const VT v48_0_0 = PAz * v28_0_0 + WPz * v28_0_1 + (VT)2.0 * oo2z * (v15_0_0 - rho_z * v15_0_1);
            const VT v49_0_0 = PAz * v29_0_0 + WPz * v29_0_1 + (VT)3.0 * oo2z * (v14_0_0 - rho_z * v14_0_1);
            const VT v50_0_0 = PAy * v30_0_0 + WPy * v30_0_1 + (VT)4.0 * oo2z * (v16_0_0 - rho_z * v16_0_1);
            const VT v51_0_0 = PAy * v31_0_0 + WPy * v31_0_1 + (VT)3.0 * oo2z * (v17_0_0 - rho_z * v17_0_1);
            const VT v52_0_0 = PAy * v32_0_0 + WPy * v32_0_1 + (VT)2.0 * oo2z * (v18_0_0 - rho_z * v18_0_1);
            const VT v53_0_0 = PAz * v32_0_0 + WPz * v32_0_1 + (VT)2.0 * oo2z * (v17_0_0 - rho_z * v17_0_1);
            const VT v54_0_0 = PAz * v33_0_0 + WPz * v33_0_1 + (VT)3.0 * oo2z * (v18_0_0 - rho_z * v18_0_1);
            const VT v55_0_0 = PAz * v34_0_0 + WPz * v34_0_1 + (VT)4.0 * oo2z * (v19_0_0 - rho_z * v19_0_1);
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
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[60] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_fdss(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h20_1_0 = acc[25] + ABx * acc[10];
    const double h10_1_0 = acc[10] + ABx * acc[0];
    const double h10_4_0 = h20_1_0 + ABx * h10_1_0;
    const double h20_2_0 = acc[26] + ABy * acc[10];
    const double h10_2_0 = acc[11] + ABy * acc[0];
    const double h10_5_0 = h20_2_0 + ABx * h10_2_0;
    const double h20_3_0 = acc[27] + ABz * acc[10];
    const double h10_3_0 = acc[12] + ABz * acc[0];
    const double h10_6_0 = h20_3_0 + ABx * h10_3_0;
    const double h21_2_0 = acc[28] + ABy * acc[11];
    const double h10_7_0 = h21_2_0 + ABy * h10_2_0;
    const double h21_3_0 = acc[29] + ABz * acc[11];
    const double h10_8_0 = h21_3_0 + ABy * h10_3_0;
    const double h22_3_0 = acc[30] + ABz * acc[12];
    const double h10_9_0 = h22_3_0 + ABz * h10_3_0;
    const double h21_1_0 = acc[26] + ABx * acc[11];
    const double h11_1_0 = acc[11] + ABx * acc[1];
    const double h11_4_0 = h21_1_0 + ABx * h11_1_0;
    const double h11_2_0 = acc[13] + ABy * acc[1];
    const double h11_5_0 = h21_2_0 + ABx * h11_2_0;
    const double h11_3_0 = acc[14] + ABz * acc[1];
    const double h11_6_0 = h21_3_0 + ABx * h11_3_0;
    const double h23_2_0 = acc[31] + ABy * acc[13];
    const double h11_7_0 = h23_2_0 + ABy * h11_2_0;
    const double h23_3_0 = acc[32] + ABz * acc[13];
    const double h11_8_0 = h23_3_0 + ABy * h11_3_0;
    const double h24_3_0 = acc[33] + ABz * acc[14];
    const double h11_9_0 = h24_3_0 + ABz * h11_3_0;
    const double h22_1_0 = acc[27] + ABx * acc[12];
    const double h12_1_0 = acc[12] + ABx * acc[2];
    const double h12_4_0 = h22_1_0 + ABx * h12_1_0;
    const double h22_2_0 = acc[29] + ABy * acc[12];
    const double h12_2_0 = acc[14] + ABy * acc[2];
    const double h12_5_0 = h22_2_0 + ABx * h12_2_0;
    const double h12_3_0 = acc[15] + ABz * acc[2];
    const double h12_6_0 = h22_3_0 + ABx * h12_3_0;
    const double h24_2_0 = acc[32] + ABy * acc[14];
    const double h12_7_0 = h24_2_0 + ABy * h12_2_0;
    const double h12_8_0 = h24_3_0 + ABy * h12_3_0;
    const double h25_3_0 = acc[34] + ABz * acc[15];
    const double h12_9_0 = h25_3_0 + ABz * h12_3_0;
    const double h23_1_0 = acc[28] + ABx * acc[13];
    const double h13_1_0 = acc[13] + ABx * acc[3];
    const double h13_4_0 = h23_1_0 + ABx * h13_1_0;
    const double h13_2_0 = acc[16] + ABy * acc[3];
    const double h13_5_0 = h23_2_0 + ABx * h13_2_0;
    const double h13_3_0 = acc[17] + ABz * acc[3];
    const double h13_6_0 = h23_3_0 + ABx * h13_3_0;
    const double h26_2_0 = acc[35] + ABy * acc[16];
    const double h13_7_0 = h26_2_0 + ABy * h13_2_0;
    const double h26_3_0 = acc[36] + ABz * acc[16];
    const double h13_8_0 = h26_3_0 + ABy * h13_3_0;
    const double h27_3_0 = acc[37] + ABz * acc[17];
    const double h13_9_0 = h27_3_0 + ABz * h13_3_0;
    const double h25_1_0 = acc[30] + ABx * acc[15];
    const double h14_1_0 = acc[15] + ABx * acc[4];
    const double h14_4_0 = h25_1_0 + ABx * h14_1_0;
    const double h25_2_0 = acc[33] + ABy * acc[15];
    const double h14_2_0 = acc[18] + ABy * acc[4];
    const double h14_5_0 = h25_2_0 + ABx * h14_2_0;
    const double h14_3_0 = acc[19] + ABz * acc[4];
    const double h14_6_0 = h25_3_0 + ABx * h14_3_0;
    const double h28_2_0 = acc[37] + ABy * acc[18];
    const double h14_7_0 = h28_2_0 + ABy * h14_2_0;
    const double h28_3_0 = acc[38] + ABz * acc[18];
    const double h14_8_0 = h28_3_0 + ABy * h14_3_0;
    const double h29_3_0 = acc[39] + ABz * acc[19];
    const double h14_9_0 = h29_3_0 + ABz * h14_3_0;
    const double h24_1_0 = acc[29] + ABx * acc[14];
    const double h15_1_0 = acc[14] + ABx * acc[5];
    const double h15_4_0 = h24_1_0 + ABx * h15_1_0;
    const double h15_2_0 = acc[17] + ABy * acc[5];
    const double h15_5_0 = h24_2_0 + ABx * h15_2_0;
    const double h15_3_0 = acc[18] + ABz * acc[5];
    const double h15_6_0 = h24_3_0 + ABx * h15_3_0;
    const double h27_2_0 = acc[36] + ABy * acc[17];
    const double h15_7_0 = h27_2_0 + ABy * h15_2_0;
    const double h15_8_0 = h27_3_0 + ABy * h15_3_0;
    const double h15_9_0 = h28_3_0 + ABz * h15_3_0;
    const double h26_1_0 = acc[31] + ABx * acc[16];
    const double h16_1_0 = acc[16] + ABx * acc[6];
    const double h16_4_0 = h26_1_0 + ABx * h16_1_0;
    const double h16_2_0 = acc[20] + ABy * acc[6];
    const double h16_5_0 = h26_2_0 + ABx * h16_2_0;
    const double h16_3_0 = acc[21] + ABz * acc[6];
    const double h16_6_0 = h26_3_0 + ABx * h16_3_0;
    const double h30_2_0 = acc[40] + ABy * acc[20];
    const double h16_7_0 = h30_2_0 + ABy * h16_2_0;
    const double h30_3_0 = acc[41] + ABz * acc[20];
    const double h16_8_0 = h30_3_0 + ABy * h16_3_0;
    const double h31_3_0 = acc[42] + ABz * acc[21];
    const double h16_9_0 = h31_3_0 + ABz * h16_3_0;
    const double h27_1_0 = acc[32] + ABx * acc[17];
    const double h17_1_0 = acc[17] + ABx * acc[7];
    const double h17_4_0 = h27_1_0 + ABx * h17_1_0;
    const double h17_2_0 = acc[21] + ABy * acc[7];
    const double h17_5_0 = h27_2_0 + ABx * h17_2_0;
    const double h17_3_0 = acc[22] + ABz * acc[7];
    const double h17_6_0 = h27_3_0 + ABx * h17_3_0;
    const double h31_2_0 = acc[41] + ABy * acc[21];
    const double h17_7_0 = h31_2_0 + ABy * h17_2_0;
    const double h17_8_0 = h31_3_0 + ABy * h17_3_0;
    const double h32_3_0 = acc[43] + ABz * acc[22];
    const double h17_9_0 = h32_3_0 + ABz * h17_3_0;
    const double h28_1_0 = acc[33] + ABx * acc[18];
    const double h18_1_0 = acc[18] + ABx * acc[8];
    const double h18_4_0 = h28_1_0 + ABx * h18_1_0;
    const double h18_2_0 = acc[22] + ABy * acc[8];
    const double h18_5_0 = h28_2_0 + ABx * h18_2_0;
    const double h18_3_0 = acc[23] + ABz * acc[8];
    const double h18_6_0 = h28_3_0 + ABx * h18_3_0;
    const double h32_2_0 = acc[42] + ABy * acc[22];
    const double h18_7_0 = h32_2_0 + ABy * h18_2_0;
    const double h18_8_0 = h32_3_0 + ABy * h18_3_0;
    const double h33_3_0 = acc[44] + ABz * acc[23];
    const double h18_9_0 = h33_3_0 + ABz * h18_3_0;
    const double h29_1_0 = acc[34] + ABx * acc[19];
    const double h19_1_0 = acc[19] + ABx * acc[9];
    const double h19_4_0 = h29_1_0 + ABx * h19_1_0;
    const double h29_2_0 = acc[38] + ABy * acc[19];
    const double h19_2_0 = acc[23] + ABy * acc[9];
    const double h19_5_0 = h29_2_0 + ABx * h19_2_0;
    const double h19_3_0 = acc[24] + ABz * acc[9];
    const double h19_6_0 = h29_3_0 + ABx * h19_3_0;
    const double h33_2_0 = acc[43] + ABy * acc[23];
    const double h19_7_0 = h33_2_0 + ABy * h19_2_0;
    const double h19_8_0 = h33_3_0 + ABy * h19_3_0;
    const double h34_3_0 = acc[45] + ABz * acc[24];
    const double h19_9_0 = h34_3_0 + ABz * h19_3_0;
    res[0] = h10_4_0 * 0.14907119849998599;
    res[1] = h10_5_0 * 0.2581988897471611;
    res[2] = h10_6_0 * 0.2581988897471611;
    res[3] = h10_7_0 * 0.14907119849998599;
    res[4] = h10_8_0 * 0.2581988897471611;
    res[5] = h10_9_0 * 0.14907119849998599;
    res[6] = h11_4_0 * 0.3333333333333334;
    res[7] = h11_5_0 * 0.5773502691896258;
    res[8] = h11_6_0 * 0.5773502691896258;
    res[9] = h11_7_0 * 0.3333333333333334;
    res[10] = h11_8_0 * 0.5773502691896258;
    res[11] = h11_9_0 * 0.3333333333333334;
    res[12] = h12_4_0 * 0.3333333333333334;
    res[13] = h12_5_0 * 0.5773502691896258;
    res[14] = h12_6_0 * 0.5773502691896258;
    res[15] = h12_7_0 * 0.3333333333333334;
    res[16] = h12_8_0 * 0.5773502691896258;
    res[17] = h12_9_0 * 0.3333333333333334;
    res[18] = h13_4_0 * 0.3333333333333334;
    res[19] = h13_5_0 * 0.5773502691896258;
    res[20] = h13_6_0 * 0.5773502691896258;
    res[21] = h13_7_0 * 0.3333333333333334;
    res[22] = h13_8_0 * 0.5773502691896258;
    res[23] = h13_9_0 * 0.3333333333333334;
    res[24] = h14_4_0 * 0.3333333333333334;
    res[25] = h14_5_0 * 0.5773502691896258;
    res[26] = h14_6_0 * 0.5773502691896258;
    res[27] = h14_7_0 * 0.3333333333333334;
    res[28] = h14_8_0 * 0.5773502691896258;
    res[29] = h14_9_0 * 0.3333333333333334;
    res[30] = h15_4_0 * 0.5773502691896258;
    res[31] = h15_5_0;
    res[32] = h15_6_0;
    res[33] = h15_7_0 * 0.5773502691896258;
    res[34] = h15_8_0;
    res[35] = h15_9_0 * 0.5773502691896258;
    res[36] = h16_4_0 * 0.14907119849998599;
    res[37] = h16_5_0 * 0.2581988897471611;
    res[38] = h16_6_0 * 0.2581988897471611;
    res[39] = h16_7_0 * 0.14907119849998599;
    res[40] = h16_8_0 * 0.2581988897471611;
    res[41] = h16_9_0 * 0.14907119849998599;
    res[42] = h17_4_0 * 0.3333333333333334;
    res[43] = h17_5_0 * 0.5773502691896258;
    res[44] = h17_6_0 * 0.5773502691896258;
    res[45] = h17_7_0 * 0.3333333333333334;
    res[46] = h17_8_0 * 0.5773502691896258;
    res[47] = h17_9_0 * 0.3333333333333334;
    res[48] = h18_4_0 * 0.3333333333333334;
    res[49] = h18_5_0 * 0.5773502691896258;
    res[50] = h18_6_0 * 0.5773502691896258;
    res[51] = h18_7_0 * 0.3333333333333334;
    res[52] = h18_8_0 * 0.5773502691896258;
    res[53] = h18_9_0 * 0.3333333333333334;
    res[54] = h19_4_0 * 0.14907119849998599;
    res[55] = h19_5_0 * 0.2581988897471611;
    res[56] = h19_6_0 * 0.2581988897471611;
    res[57] = h19_7_0 * 0.14907119849998599;
    res[58] = h19_8_0 * 0.2581988897471611;
    res[59] = h19_9_0 * 0.14907119849998599;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[60]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_fdss(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[46];
    vrr_fdss<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 46; ++x) acc_out[x] = acc[x];
    }
    hrr_fdss(P, p, q, acc, res);
}

__device__ __forceinline__ void store_fdss(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
    { const long long ij = ij_0_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_1_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_1_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_1_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_2_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_2_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_2_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_3_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_3_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_3_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_4_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_4_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_4_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_5_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_5_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_5_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_6_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_6_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_6_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_6_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_6_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_6_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_7_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_7_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_7_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_7_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_7_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_7_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_8_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_8_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_8_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_8_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_8_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_8_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_9_0, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_9_1, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_9_2, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_9_3, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_9_4, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_9_5, kl = kl_0_0;
      if ((!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_fdss(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 60; ++x) {
        const int ia = x / 6, ibb = (x / 1) % 6, ic = (x / 1) % 1, id = x % 1;
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
__global__ void __launch_bounds__(128) eri_queue_fdss(const EriQueue Q) {
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
        double acc[46];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 46; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_fdss<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_fdss<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 46; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 60 doubles (launch_eri_fdss)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 60);
            if (lead) hrr_fdss(Q.pairs, p, q, acc, sb + kq * 60);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)60;
            for (int t = lane; t < nlive * 60; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[60];
            hrr_fdss(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_fdss(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_fdss(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (61440 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_fdss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_fdss<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 61440);
        cudaFuncSetAttribute(eri_queue_fdss<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 61440);
        done[dev] = true;
    }
}

void launch_eri_fdss(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 61440 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 61440 : 0;
    if (smem) eri_prepare_fdss();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_fdss<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_fdss<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_fdss<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_fdss<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_fdss(int mixed) {
    eri_prepare_fdss();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fdss<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_fdss<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

// Generated by gen_eri.py -- class (dd|dp).  Do not edit.
// VRR entries: 1175, contracted block: 496, HRR lines: 1912, outputs: 648.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[496], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_dddp(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 496; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[8];
            boys_fm<7>(T, B, F);
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
            const VT v1_0_0 = PAx * v0_0_0 + WPx * v0_0_1;
            const VT v1_0_1 = PAx * v0_0_1 + WPx * v0_0_2;
            const VT v1_0_2 = PAx * v0_0_2 + WPx * v0_0_3;
            const VT v1_0_3 = PAx * v0_0_3 + WPx * v0_0_4;
            const VT v1_0_4 = PAx * v0_0_4 + WPx * v0_0_5;
            const VT v1_0_5 = PAx * v0_0_5 + WPx * v0_0_6;
            const VT v1_0_6 = PAx * v0_0_6 + WPx * v0_0_7;
            const VT v2_0_0 = PAy * v0_0_0 + WPy * v0_0_1;
            const VT v2_0_1 = PAy * v0_0_1 + WPy * v0_0_2;
            const VT v2_0_2 = PAy * v0_0_2 + WPy * v0_0_3;
            const VT v2_0_3 = PAy * v0_0_3 + WPy * v0_0_4;
            const VT v2_0_4 = PAy * v0_0_4 + WPy * v0_0_5;
            const VT v2_0_5 = PAy * v0_0_5 + WPy * v0_0_6;
            const VT v2_0_6 = PAy * v0_0_6 + WPy * v0_0_7;
            const VT v3_0_0 = PAz * v0_0_0 + WPz * v0_0_1;
            const VT v3_0_1 = PAz * v0_0_1 + WPz * v0_0_2;
            const VT v3_0_2 = PAz * v0_0_2 + WPz * v0_0_3;
            const VT v3_0_3 = PAz * v0_0_3 + WPz * v0_0_4;
            const VT v3_0_4 = PAz * v0_0_4 + WPz * v0_0_5;
            const VT v3_0_5 = PAz * v0_0_5 + WPz * v0_0_6;
            const VT v3_0_6 = PAz * v0_0_6 + WPz * v0_0_7;
            const VT v4_0_0 = PAx * v1_0_0 + WPx * v1_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v4_0_1 = PAx * v1_0_1 + WPx * v1_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v4_0_2 = PAx * v1_0_2 + WPx * v1_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v4_0_3 = PAx * v1_0_3 + WPx * v1_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v4_0_4 = PAx * v1_0_4 + WPx * v1_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v4_0_5 = PAx * v1_0_5 + WPx * v1_0_6 + (VT)1.0 * oo2z * (v0_0_5 - rho_z * v0_0_6);
            const VT v5_0_0 = PAx * v2_0_0 + WPx * v2_0_1;
            const VT v5_0_1 = PAx * v2_0_1 + WPx * v2_0_2;
            const VT v5_0_2 = PAx * v2_0_2 + WPx * v2_0_3;
            const VT v5_0_3 = PAx * v2_0_3 + WPx * v2_0_4;
            const VT v5_0_4 = PAx * v2_0_4 + WPx * v2_0_5;
            const VT v5_0_5 = PAx * v2_0_5 + WPx * v2_0_6;
            const VT v6_0_0 = PAx * v3_0_0 + WPx * v3_0_1;
            const VT v6_0_1 = PAx * v3_0_1 + WPx * v3_0_2;
            const VT v6_0_2 = PAx * v3_0_2 + WPx * v3_0_3;
            const VT v6_0_3 = PAx * v3_0_3 + WPx * v3_0_4;
            const VT v6_0_4 = PAx * v3_0_4 + WPx * v3_0_5;
            const VT v6_0_5 = PAx * v3_0_5 + WPx * v3_0_6;
            const VT v7_0_0 = PAy * v2_0_0 + WPy * v2_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v7_0_1 = PAy * v2_0_1 + WPy * v2_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v7_0_2 = PAy * v2_0_2 + WPy * v2_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v7_0_3 = PAy * v2_0_3 + WPy * v2_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v7_0_4 = PAy * v2_0_4 + WPy * v2_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v7_0_5 = PAy * v2_0_5 + WPy * v2_0_6 + (VT)1.0 * oo2z * (v0_0_5 - rho_z * v0_0_6);
            const VT v8_0_0 = PAy * v3_0_0 + WPy * v3_0_1;
            const VT v8_0_1 = PAy * v3_0_1 + WPy * v3_0_2;
            const VT v8_0_2 = PAy * v3_0_2 + WPy * v3_0_3;
            const VT v8_0_3 = PAy * v3_0_3 + WPy * v3_0_4;
            const VT v8_0_4 = PAy * v3_0_4 + WPy * v3_0_5;
            const VT v8_0_5 = PAy * v3_0_5 + WPy * v3_0_6;
            const VT v9_0_0 = PAz * v3_0_0 + WPz * v3_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v9_0_1 = PAz * v3_0_1 + WPz * v3_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v9_0_2 = PAz * v3_0_2 + WPz * v3_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v9_0_3 = PAz * v3_0_3 + WPz * v3_0_4 + (VT)1.0 * oo2z * (v0_0_3 - rho_z * v0_0_4);
            const VT v9_0_4 = PAz * v3_0_4 + WPz * v3_0_5 + (VT)1.0 * oo2z * (v0_0_4 - rho_z * v0_0_5);
            const VT v9_0_5 = PAz * v3_0_5 + WPz * v3_0_6 + (VT)1.0 * oo2z * (v0_0_5 - rho_z * v0_0_6);
            const VT v10_0_0 = PAx * v4_0_0 + WPx * v4_0_1 + (VT)2.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v10_0_1 = PAx * v4_0_1 + WPx * v4_0_2 + (VT)2.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v10_0_2 = PAx * v4_0_2 + WPx * v4_0_3 + (VT)2.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v10_0_3 = PAx * v4_0_3 + WPx * v4_0_4 + (VT)2.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v10_0_4 = PAx * v4_0_4 + WPx * v4_0_5 + (VT)2.0 * oo2z * (v1_0_4 - rho_z * v1_0_5);
            const VT v11_0_0 = PAx * v5_0_0 + WPx * v5_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v11_0_1 = PAx * v5_0_1 + WPx * v5_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v11_0_2 = PAx * v5_0_2 + WPx * v5_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v11_0_3 = PAx * v5_0_3 + WPx * v5_0_4 + (VT)1.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v11_0_4 = PAx * v5_0_4 + WPx * v5_0_5 + (VT)1.0 * oo2z * (v2_0_4 - rho_z * v2_0_5);
            const VT v12_0_0 = PAx * v6_0_0 + WPx * v6_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v12_0_1 = PAx * v6_0_1 + WPx * v6_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v12_0_2 = PAx * v6_0_2 + WPx * v6_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v12_0_3 = PAx * v6_0_3 + WPx * v6_0_4 + (VT)1.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v12_0_4 = PAx * v6_0_4 + WPx * v6_0_5 + (VT)1.0 * oo2z * (v3_0_4 - rho_z * v3_0_5);
            const VT v13_0_0 = PAy * v5_0_0 + WPy * v5_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v13_0_1 = PAy * v5_0_1 + WPy * v5_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v13_0_2 = PAy * v5_0_2 + WPy * v5_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v13_0_3 = PAy * v5_0_3 + WPy * v5_0_4 + (VT)1.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v13_0_4 = PAy * v5_0_4 + WPy * v5_0_5 + (VT)1.0 * oo2z * (v1_0_4 - rho_z * v1_0_5);
            const VT v14_0_0 = PAz * v6_0_0 + WPz * v6_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v14_0_1 = PAz * v6_0_1 + WPz * v6_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v14_0_2 = PAz * v6_0_2 + WPz * v6_0_3 + (VT)1.0 * oo2z * (v1_0_2 - rho_z * v1_0_3);
            const VT v14_0_3 = PAz * v6_0_3 + WPz * v6_0_4 + (VT)1.0 * oo2z * (v1_0_3 - rho_z * v1_0_4);
            const VT v14_0_4 = PAz * v6_0_4 + WPz * v6_0_5 + (VT)1.0 * oo2z * (v1_0_4 - rho_z * v1_0_5);
            const VT v15_0_0 = PAx * v8_0_0 + WPx * v8_0_1;
            const VT v15_0_1 = PAx * v8_0_1 + WPx * v8_0_2;
            const VT v15_0_2 = PAx * v8_0_2 + WPx * v8_0_3;
            const VT v15_0_3 = PAx * v8_0_3 + WPx * v8_0_4;
            const VT v15_0_4 = PAx * v8_0_4 + WPx * v8_0_5;
            const VT v16_0_0 = PAy * v7_0_0 + WPy * v7_0_1 + (VT)2.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v16_0_1 = PAy * v7_0_1 + WPy * v7_0_2 + (VT)2.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v16_0_2 = PAy * v7_0_2 + WPy * v7_0_3 + (VT)2.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v16_0_3 = PAy * v7_0_3 + WPy * v7_0_4 + (VT)2.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v16_0_4 = PAy * v7_0_4 + WPy * v7_0_5 + (VT)2.0 * oo2z * (v2_0_4 - rho_z * v2_0_5);
            const VT v17_0_0 = PAy * v8_0_0 + WPy * v8_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v17_0_1 = PAy * v8_0_1 + WPy * v8_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v17_0_2 = PAy * v8_0_2 + WPy * v8_0_3 + (VT)1.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v17_0_3 = PAy * v8_0_3 + WPy * v8_0_4 + (VT)1.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v17_0_4 = PAy * v8_0_4 + WPy * v8_0_5 + (VT)1.0 * oo2z * (v3_0_4 - rho_z * v3_0_5);
            const VT v18_0_0 = PAz * v8_0_0 + WPz * v8_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v18_0_1 = PAz * v8_0_1 + WPz * v8_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v18_0_2 = PAz * v8_0_2 + WPz * v8_0_3 + (VT)1.0 * oo2z * (v2_0_2 - rho_z * v2_0_3);
            const VT v18_0_3 = PAz * v8_0_3 + WPz * v8_0_4 + (VT)1.0 * oo2z * (v2_0_3 - rho_z * v2_0_4);
            const VT v18_0_4 = PAz * v8_0_4 + WPz * v8_0_5 + (VT)1.0 * oo2z * (v2_0_4 - rho_z * v2_0_5);
            const VT v19_0_0 = PAz * v9_0_0 + WPz * v9_0_1 + (VT)2.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v19_0_1 = PAz * v9_0_1 + WPz * v9_0_2 + (VT)2.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v19_0_2 = PAz * v9_0_2 + WPz * v9_0_3 + (VT)2.0 * oo2z * (v3_0_2 - rho_z * v3_0_3);
            const VT v19_0_3 = PAz * v9_0_3 + WPz * v9_0_4 + (VT)2.0 * oo2z * (v3_0_3 - rho_z * v3_0_4);
            const VT v19_0_4 = PAz * v9_0_4 + WPz * v9_0_5 + (VT)2.0 * oo2z * (v3_0_4 - rho_z * v3_0_5);
            const VT v20_0_0 = PAx * v10_0_0 + WPx * v10_0_1 + (VT)3.0 * oo2z * (v4_0_0 - rho_z * v4_0_1);
            const VT v20_0_1 = PAx * v10_0_1 + WPx * v10_0_2 + (VT)3.0 * oo2z * (v4_0_1 - rho_z * v4_0_2);
            const VT v20_0_2 = PAx * v10_0_2 + WPx * v10_0_3 + (VT)3.0 * oo2z * (v4_0_2 - rho_z * v4_0_3);
            const VT v20_0_3 = PAx * v10_0_3 + WPx * v10_0_4 + (VT)3.0 * oo2z * (v4_0_3 - rho_z * v4_0_4);
            const VT v21_0_0 = PAx * v11_0_0 + WPx * v11_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v21_0_1 = PAx * v11_0_1 + WPx * v11_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v21_0_2 = PAx * v11_0_2 + WPx * v11_0_3 + (VT)2.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v21_0_3 = PAx * v11_0_3 + WPx * v11_0_4 + (VT)2.0 * oo2z * (v5_0_3 - rho_z * v5_0_4);
            const VT v22_0_0 = PAx * v12_0_0 + WPx * v12_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v22_0_1 = PAx * v12_0_1 + WPx * v12_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v22_0_2 = PAx * v12_0_2 + WPx * v12_0_3 + (VT)2.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v22_0_3 = PAx * v12_0_3 + WPx * v12_0_4 + (VT)2.0 * oo2z * (v6_0_3 - rho_z * v6_0_4);
            const VT v23_0_0 = PAx * v13_0_0 + WPx * v13_0_1 + (VT)1.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v23_0_1 = PAx * v13_0_1 + WPx * v13_0_2 + (VT)1.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v23_0_2 = PAx * v13_0_2 + WPx * v13_0_3 + (VT)1.0 * oo2z * (v7_0_2 - rho_z * v7_0_3);
            const VT v23_0_3 = PAx * v13_0_3 + WPx * v13_0_4 + (VT)1.0 * oo2z * (v7_0_3 - rho_z * v7_0_4);
            const VT v24_0_0 = PAx * v15_0_0 + WPx * v15_0_1 + (VT)1.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v24_0_1 = PAx * v15_0_1 + WPx * v15_0_2 + (VT)1.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v24_0_2 = PAx * v15_0_2 + WPx * v15_0_3 + (VT)1.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v24_0_3 = PAx * v15_0_3 + WPx * v15_0_4 + (VT)1.0 * oo2z * (v8_0_3 - rho_z * v8_0_4);
            const VT v25_0_0 = PAx * v14_0_0 + WPx * v14_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v25_0_1 = PAx * v14_0_1 + WPx * v14_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v25_0_2 = PAx * v14_0_2 + WPx * v14_0_3 + (VT)1.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v25_0_3 = PAx * v14_0_3 + WPx * v14_0_4 + (VT)1.0 * oo2z * (v9_0_3 - rho_z * v9_0_4);
            const VT v26_0_0 = PAy * v13_0_0 + WPy * v13_0_1 + (VT)2.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v26_0_1 = PAy * v13_0_1 + WPy * v13_0_2 + (VT)2.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v26_0_2 = PAy * v13_0_2 + WPy * v13_0_3 + (VT)2.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v26_0_3 = PAy * v13_0_3 + WPy * v13_0_4 + (VT)2.0 * oo2z * (v5_0_3 - rho_z * v5_0_4);
            const VT v27_0_0 = PAy * v15_0_0 + WPy * v15_0_1 + (VT)1.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v27_0_1 = PAy * v15_0_1 + WPy * v15_0_2 + (VT)1.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v27_0_2 = PAy * v15_0_2 + WPy * v15_0_3 + (VT)1.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v27_0_3 = PAy * v15_0_3 + WPy * v15_0_4 + (VT)1.0 * oo2z * (v6_0_3 - rho_z * v6_0_4);
            const VT v28_0_0 = PAz * v15_0_0 + WPz * v15_0_1 + (VT)1.0 * oo2z * (v5_0_0 - rho_z * v5_0_1);
            const VT v28_0_1 = PAz * v15_0_1 + WPz * v15_0_2 + (VT)1.0 * oo2z * (v5_0_1 - rho_z * v5_0_2);
            const VT v28_0_2 = PAz * v15_0_2 + WPz * v15_0_3 + (VT)1.0 * oo2z * (v5_0_2 - rho_z * v5_0_3);
            const VT v28_0_3 = PAz * v15_0_3 + WPz * v15_0_4 + (VT)1.0 * oo2z * (v5_0_3 - rho_z * v5_0_4);
            const VT v29_0_0 = PAz * v14_0_0 + WPz * v14_0_1 + (VT)2.0 * oo2z * (v6_0_0 - rho_z * v6_0_1);
            const VT v29_0_1 = PAz * v14_0_1 + WPz * v14_0_2 + (VT)2.0 * oo2z * (v6_0_1 - rho_z * v6_0_2);
            const VT v29_0_2 = PAz * v14_0_2 + WPz * v14_0_3 + (VT)2.0 * oo2z * (v6_0_2 - rho_z * v6_0_3);
            const VT v29_0_3 = PAz * v14_0_3 + WPz * v14_0_4 + (VT)2.0 * oo2z * (v6_0_3 - rho_z * v6_0_4);
            const VT v30_0_0 = PAy * v16_0_0 + WPy * v16_0_1 + (VT)3.0 * oo2z * (v7_0_0 - rho_z * v7_0_1);
            const VT v30_0_1 = PAy * v16_0_1 + WPy * v16_0_2 + (VT)3.0 * oo2z * (v7_0_1 - rho_z * v7_0_2);
            const VT v30_0_2 = PAy * v16_0_2 + WPy * v16_0_3 + (VT)3.0 * oo2z * (v7_0_2 - rho_z * v7_0_3);
            const VT v30_0_3 = PAy * v16_0_3 + WPy * v16_0_4 + (VT)3.0 * oo2z * (v7_0_3 - rho_z * v7_0_4);
            const VT v31_0_0 = PAy * v17_0_0 + WPy * v17_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v31_0_1 = PAy * v17_0_1 + WPy * v17_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v31_0_2 = PAy * v17_0_2 + WPy * v17_0_3 + (VT)2.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v31_0_3 = PAy * v17_0_3 + WPy * v17_0_4 + (VT)2.0 * oo2z * (v8_0_3 - rho_z * v8_0_4);
            const VT v32_0_0 = PAy * v18_0_0 + WPy * v18_0_1 + (VT)1.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v32_0_1 = PAy * v18_0_1 + WPy * v18_0_2 + (VT)1.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v32_0_2 = PAy * v18_0_2 + WPy * v18_0_3 + (VT)1.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v32_0_3 = PAy * v18_0_3 + WPy * v18_0_4 + (VT)1.0 * oo2z * (v9_0_3 - rho_z * v9_0_4);
            const VT v33_0_0 = PAz * v18_0_0 + WPz * v18_0_1 + (VT)2.0 * oo2z * (v8_0_0 - rho_z * v8_0_1);
            const VT v33_0_1 = PAz * v18_0_1 + WPz * v18_0_2 + (VT)2.0 * oo2z * (v8_0_1 - rho_z * v8_0_2);
            const VT v33_0_2 = PAz * v18_0_2 + WPz * v18_0_3 + (VT)2.0 * oo2z * (v8_0_2 - rho_z * v8_0_3);
            const VT v33_0_3 = PAz * v18_0_3 + WPz * v18_0_4 + (VT)2.0 * oo2z * (v8_0_3 - rho_z * v8_0_4);
            const VT v34_0_0 = PAz * v19_0_0 + WPz * v19_0_1 + (VT)3.0 * oo2z * (v9_0_0 - rho_z * v9_0_1);
            const VT v34_0_1 = PAz * v19_0_1 + WPz * v19_0_2 + (VT)3.0 * oo2z * (v9_0_1 - rho_z * v9_0_2);
            const VT v34_0_2 = PAz * v19_0_2 + WPz * v19_0_3 + (VT)3.0 * oo2z * (v9_0_2 - rho_z * v9_0_3);
            const VT v34_0_3 = PAz * v19_0_3 + WPz * v19_0_4 + (VT)3.0 * oo2z * (v9_0_3 - rho_z * v9_0_4);
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
            const VT v20_1_0 = QCx * v20_0_0 + WQx * v20_0_1 + (VT)4.0 * oo2ze * v10_0_1;
            const VT v20_1_1 = QCx * v20_0_1 + WQx * v20_0_2 + (VT)4.0 * oo2ze * v10_0_2;
            const VT v20_1_2 = QCx * v20_0_2 + WQx * v20_0_3 + (VT)4.0 * oo2ze * v10_0_3;
            const VT v21_1_0 = QCx * v21_0_0 + WQx * v21_0_1 + (VT)3.0 * oo2ze * v11_0_1;
            const VT v21_1_1 = QCx * v21_0_1 + WQx * v21_0_2 + (VT)3.0 * oo2ze * v11_0_2;
            const VT v21_1_2 = QCx * v21_0_2 + WQx * v21_0_3 + (VT)3.0 * oo2ze * v11_0_3;
            const VT v22_1_0 = QCx * v22_0_0 + WQx * v22_0_1 + (VT)3.0 * oo2ze * v12_0_1;
            const VT v22_1_1 = QCx * v22_0_1 + WQx * v22_0_2 + (VT)3.0 * oo2ze * v12_0_2;
            const VT v22_1_2 = QCx * v22_0_2 + WQx * v22_0_3 + (VT)3.0 * oo2ze * v12_0_3;
            const VT v23_1_0 = QCx * v23_0_0 + WQx * v23_0_1 + (VT)2.0 * oo2ze * v13_0_1;
            const VT v23_1_1 = QCx * v23_0_1 + WQx * v23_0_2 + (VT)2.0 * oo2ze * v13_0_2;
            const VT v23_1_2 = QCx * v23_0_2 + WQx * v23_0_3 + (VT)2.0 * oo2ze * v13_0_3;
            const VT v24_1_0 = QCx * v24_0_0 + WQx * v24_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v24_1_1 = QCx * v24_0_1 + WQx * v24_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v24_1_2 = QCx * v24_0_2 + WQx * v24_0_3 + (VT)2.0 * oo2ze * v15_0_3;
            const VT v25_1_0 = QCx * v25_0_0 + WQx * v25_0_1 + (VT)2.0 * oo2ze * v14_0_1;
            const VT v25_1_1 = QCx * v25_0_1 + WQx * v25_0_2 + (VT)2.0 * oo2ze * v14_0_2;
            const VT v25_1_2 = QCx * v25_0_2 + WQx * v25_0_3 + (VT)2.0 * oo2ze * v14_0_3;
            const VT v26_1_0 = QCx * v26_0_0 + WQx * v26_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v26_1_1 = QCx * v26_0_1 + WQx * v26_0_2 + (VT)1.0 * oo2ze * v16_0_2;
            const VT v26_1_2 = QCx * v26_0_2 + WQx * v26_0_3 + (VT)1.0 * oo2ze * v16_0_3;
            const VT v27_1_0 = QCx * v27_0_0 + WQx * v27_0_1 + (VT)1.0 * oo2ze * v17_0_1;
            const VT v27_1_1 = QCx * v27_0_1 + WQx * v27_0_2 + (VT)1.0 * oo2ze * v17_0_2;
            const VT v27_1_2 = QCx * v27_0_2 + WQx * v27_0_3 + (VT)1.0 * oo2ze * v17_0_3;
            const VT v28_1_0 = QCx * v28_0_0 + WQx * v28_0_1 + (VT)1.0 * oo2ze * v18_0_1;
            const VT v28_1_1 = QCx * v28_0_1 + WQx * v28_0_2 + (VT)1.0 * oo2ze * v18_0_2;
            const VT v28_1_2 = QCx * v28_0_2 + WQx * v28_0_3 + (VT)1.0 * oo2ze * v18_0_3;
            const VT v29_1_0 = QCx * v29_0_0 + WQx * v29_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v29_1_1 = QCx * v29_0_1 + WQx * v29_0_2 + (VT)1.0 * oo2ze * v19_0_2;
            const VT v29_1_2 = QCx * v29_0_2 + WQx * v29_0_3 + (VT)1.0 * oo2ze * v19_0_3;
            const VT v30_1_0 = QCx * v30_0_0 + WQx * v30_0_1;
            const VT v30_1_1 = QCx * v30_0_1 + WQx * v30_0_2;
            const VT v30_1_2 = QCx * v30_0_2 + WQx * v30_0_3;
            const VT v31_1_0 = QCx * v31_0_0 + WQx * v31_0_1;
            const VT v31_1_1 = QCx * v31_0_1 + WQx * v31_0_2;
            const VT v31_1_2 = QCx * v31_0_2 + WQx * v31_0_3;
            const VT v32_1_0 = QCx * v32_0_0 + WQx * v32_0_1;
            const VT v32_1_1 = QCx * v32_0_1 + WQx * v32_0_2;
            const VT v32_1_2 = QCx * v32_0_2 + WQx * v32_0_3;
            const VT v33_1_0 = QCx * v33_0_0 + WQx * v33_0_1;
            const VT v33_1_1 = QCx * v33_0_1 + WQx * v33_0_2;
            const VT v33_1_2 = QCx * v33_0_2 + WQx * v33_0_3;
            const VT v34_1_0 = QCx * v34_0_0 + WQx * v34_0_1;
            const VT v34_1_1 = QCx * v34_0_1 + WQx * v34_0_2;
            const VT v34_1_2 = QCx * v34_0_2 + WQx * v34_0_3;
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
            const VT v20_2_0 = QCy * v20_0_0 + WQy * v20_0_1;
            const VT v20_2_1 = QCy * v20_0_1 + WQy * v20_0_2;
            const VT v20_2_2 = QCy * v20_0_2 + WQy * v20_0_3;
            const VT v21_2_0 = QCy * v21_0_0 + WQy * v21_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v21_2_1 = QCy * v21_0_1 + WQy * v21_0_2 + (VT)1.0 * oo2ze * v10_0_2;
            const VT v21_2_2 = QCy * v21_0_2 + WQy * v21_0_3 + (VT)1.0 * oo2ze * v10_0_3;
            const VT v22_2_0 = QCy * v22_0_0 + WQy * v22_0_1;
            const VT v22_2_1 = QCy * v22_0_1 + WQy * v22_0_2;
            const VT v22_2_2 = QCy * v22_0_2 + WQy * v22_0_3;
            const VT v23_2_0 = QCy * v23_0_0 + WQy * v23_0_1 + (VT)2.0 * oo2ze * v11_0_1;
            const VT v23_2_1 = QCy * v23_0_1 + WQy * v23_0_2 + (VT)2.0 * oo2ze * v11_0_2;
            const VT v23_2_2 = QCy * v23_0_2 + WQy * v23_0_3 + (VT)2.0 * oo2ze * v11_0_3;
            const VT v24_2_0 = QCy * v24_0_0 + WQy * v24_0_1 + (VT)1.0 * oo2ze * v12_0_1;
            const VT v24_2_1 = QCy * v24_0_1 + WQy * v24_0_2 + (VT)1.0 * oo2ze * v12_0_2;
            const VT v24_2_2 = QCy * v24_0_2 + WQy * v24_0_3 + (VT)1.0 * oo2ze * v12_0_3;
            const VT v25_2_0 = QCy * v25_0_0 + WQy * v25_0_1;
            const VT v25_2_1 = QCy * v25_0_1 + WQy * v25_0_2;
            const VT v25_2_2 = QCy * v25_0_2 + WQy * v25_0_3;
            const VT v26_2_0 = QCy * v26_0_0 + WQy * v26_0_1 + (VT)3.0 * oo2ze * v13_0_1;
            const VT v26_2_1 = QCy * v26_0_1 + WQy * v26_0_2 + (VT)3.0 * oo2ze * v13_0_2;
            const VT v26_2_2 = QCy * v26_0_2 + WQy * v26_0_3 + (VT)3.0 * oo2ze * v13_0_3;
            const VT v27_2_0 = QCy * v27_0_0 + WQy * v27_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v27_2_1 = QCy * v27_0_1 + WQy * v27_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v27_2_2 = QCy * v27_0_2 + WQy * v27_0_3 + (VT)2.0 * oo2ze * v15_0_3;
            const VT v28_2_0 = QCy * v28_0_0 + WQy * v28_0_1 + (VT)1.0 * oo2ze * v14_0_1;
            const VT v28_2_1 = QCy * v28_0_1 + WQy * v28_0_2 + (VT)1.0 * oo2ze * v14_0_2;
            const VT v28_2_2 = QCy * v28_0_2 + WQy * v28_0_3 + (VT)1.0 * oo2ze * v14_0_3;
            const VT v29_2_0 = QCy * v29_0_0 + WQy * v29_0_1;
            const VT v29_2_1 = QCy * v29_0_1 + WQy * v29_0_2;
            const VT v29_2_2 = QCy * v29_0_2 + WQy * v29_0_3;
            const VT v30_2_0 = QCy * v30_0_0 + WQy * v30_0_1 + (VT)4.0 * oo2ze * v16_0_1;
            const VT v30_2_1 = QCy * v30_0_1 + WQy * v30_0_2 + (VT)4.0 * oo2ze * v16_0_2;
            const VT v30_2_2 = QCy * v30_0_2 + WQy * v30_0_3 + (VT)4.0 * oo2ze * v16_0_3;
            const VT v31_2_0 = QCy * v31_0_0 + WQy * v31_0_1 + (VT)3.0 * oo2ze * v17_0_1;
            const VT v31_2_1 = QCy * v31_0_1 + WQy * v31_0_2 + (VT)3.0 * oo2ze * v17_0_2;
            const VT v31_2_2 = QCy * v31_0_2 + WQy * v31_0_3 + (VT)3.0 * oo2ze * v17_0_3;
            const VT v32_2_0 = QCy * v32_0_0 + WQy * v32_0_1 + (VT)2.0 * oo2ze * v18_0_1;
            const VT v32_2_1 = QCy * v32_0_1 + WQy * v32_0_2 + (VT)2.0 * oo2ze * v18_0_2;
            const VT v32_2_2 = QCy * v32_0_2 + WQy * v32_0_3 + (VT)2.0 * oo2ze * v18_0_3;
            const VT v33_2_0 = QCy * v33_0_0 + WQy * v33_0_1 + (VT)1.0 * oo2ze * v19_0_1;
            const VT v33_2_1 = QCy * v33_0_1 + WQy * v33_0_2 + (VT)1.0 * oo2ze * v19_0_2;
            const VT v33_2_2 = QCy * v33_0_2 + WQy * v33_0_3 + (VT)1.0 * oo2ze * v19_0_3;
            const VT v34_2_0 = QCy * v34_0_0 + WQy * v34_0_1;
            const VT v34_2_1 = QCy * v34_0_1 + WQy * v34_0_2;
            const VT v34_2_2 = QCy * v34_0_2 + WQy * v34_0_3;
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
            const VT v20_3_0 = QCz * v20_0_0 + WQz * v20_0_1;
            const VT v20_3_1 = QCz * v20_0_1 + WQz * v20_0_2;
            const VT v20_3_2 = QCz * v20_0_2 + WQz * v20_0_3;
            const VT v21_3_0 = QCz * v21_0_0 + WQz * v21_0_1;
            const VT v21_3_1 = QCz * v21_0_1 + WQz * v21_0_2;
            const VT v21_3_2 = QCz * v21_0_2 + WQz * v21_0_3;
            const VT v22_3_0 = QCz * v22_0_0 + WQz * v22_0_1 + (VT)1.0 * oo2ze * v10_0_1;
            const VT v22_3_1 = QCz * v22_0_1 + WQz * v22_0_2 + (VT)1.0 * oo2ze * v10_0_2;
            const VT v22_3_2 = QCz * v22_0_2 + WQz * v22_0_3 + (VT)1.0 * oo2ze * v10_0_3;
            const VT v23_3_0 = QCz * v23_0_0 + WQz * v23_0_1;
            const VT v23_3_1 = QCz * v23_0_1 + WQz * v23_0_2;
            const VT v23_3_2 = QCz * v23_0_2 + WQz * v23_0_3;
            const VT v24_3_0 = QCz * v24_0_0 + WQz * v24_0_1 + (VT)1.0 * oo2ze * v11_0_1;
            const VT v24_3_1 = QCz * v24_0_1 + WQz * v24_0_2 + (VT)1.0 * oo2ze * v11_0_2;
            const VT v24_3_2 = QCz * v24_0_2 + WQz * v24_0_3 + (VT)1.0 * oo2ze * v11_0_3;
            const VT v25_3_0 = QCz * v25_0_0 + WQz * v25_0_1 + (VT)2.0 * oo2ze * v12_0_1;
            const VT v25_3_1 = QCz * v25_0_1 + WQz * v25_0_2 + (VT)2.0 * oo2ze * v12_0_2;
            const VT v25_3_2 = QCz * v25_0_2 + WQz * v25_0_3 + (VT)2.0 * oo2ze * v12_0_3;
            const VT v26_3_0 = QCz * v26_0_0 + WQz * v26_0_1;
            const VT v26_3_1 = QCz * v26_0_1 + WQz * v26_0_2;
            const VT v26_3_2 = QCz * v26_0_2 + WQz * v26_0_3;
            const VT v27_3_0 = QCz * v27_0_0 + WQz * v27_0_1 + (VT)1.0 * oo2ze * v13_0_1;
            const VT v27_3_1 = QCz * v27_0_1 + WQz * v27_0_2 + (VT)1.0 * oo2ze * v13_0_2;
            const VT v27_3_2 = QCz * v27_0_2 + WQz * v27_0_3 + (VT)1.0 * oo2ze * v13_0_3;
            const VT v28_3_0 = QCz * v28_0_0 + WQz * v28_0_1 + (VT)2.0 * oo2ze * v15_0_1;
            const VT v28_3_1 = QCz * v28_0_1 + WQz * v28_0_2 + (VT)2.0 * oo2ze * v15_0_2;
            const VT v28_3_2 = QCz * v28_0_2 + WQz * v28_0_3 + (VT)2.0 * oo2ze * v15_0_3;
            const VT v29_3_0 = QCz * v29_0_0 + WQz * v29_0_1 + (VT)3.0 * oo2ze * v14_0_1;
            const VT v29_3_1 = QCz * v29_0_1 + WQz * v29_0_2 + (VT)3.0 * oo2ze * v14_0_2;
            const VT v29_3_2 = QCz * v29_0_2 + WQz * v29_0_3 + (VT)3.0 * oo2ze * v14_0_3;
            const VT v30_3_0 = QCz * v30_0_0 + WQz * v30_0_1;
            const VT v30_3_1 = QCz * v30_0_1 + WQz * v30_0_2;
            const VT v30_3_2 = QCz * v30_0_2 + WQz * v30_0_3;
            const VT v31_3_0 = QCz * v31_0_0 + WQz * v31_0_1 + (VT)1.0 * oo2ze * v16_0_1;
            const VT v31_3_1 = QCz * v31_0_1 + WQz * v31_0_2 + (VT)1.0 * oo2ze * v16_0_2;
            const VT v31_3_2 = QCz * v31_0_2 + WQz * v31_0_3 + (VT)1.0 * oo2ze * v16_0_3;
            const VT v32_3_0 = QCz * v32_0_0 + WQz * v32_0_1 + (VT)2.0 * oo2ze * v17_0_1;
            const VT v32_3_1 = QCz * v32_0_1 + WQz * v32_0_2 + (VT)2.0 * oo2ze * v17_0_2;
            const VT v32_3_2 = QCz * v32_0_2 + WQz * v32_0_3 + (VT)2.0 * oo2ze * v17_0_3;
            const VT v33_3_0 = QCz * v33_0_0 + WQz * v33_0_1 + (VT)3.0 * oo2ze * v18_0_1;
            const VT v33_3_1 = QCz * v33_0_1 + WQz * v33_0_2 + (VT)3.0 * oo2ze * v18_0_2;
            const VT v33_3_2 = QCz * v33_0_2 + WQz * v33_0_3 + (VT)3.0 * oo2ze * v18_0_3;
            const VT v34_3_0 = QCz * v34_0_0 + WQz * v34_0_1 + (VT)4.0 * oo2ze * v19_0_1;
            const VT v34_3_1 = QCz * v34_0_1 + WQz * v34_0_2 + (VT)4.0 * oo2ze * v19_0_2;
            const VT v34_3_2 = QCz * v34_0_2 + WQz * v34_0_3 + (VT)4.0 * oo2ze * v19_0_3;
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
            const VT v20_4_0 = QCx * v20_1_0 + WQx * v20_1_1 + (VT)4.0 * oo2ze * v10_1_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v20_4_1 = QCx * v20_1_1 + WQx * v20_1_2 + (VT)4.0 * oo2ze * v10_1_2 + (VT)1.0 * oo2e * (v20_0_1 - rho_e * v20_0_2);
            const VT v21_4_0 = QCx * v21_1_0 + WQx * v21_1_1 + (VT)3.0 * oo2ze * v11_1_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v21_4_1 = QCx * v21_1_1 + WQx * v21_1_2 + (VT)3.0 * oo2ze * v11_1_2 + (VT)1.0 * oo2e * (v21_0_1 - rho_e * v21_0_2);
            const VT v22_4_0 = QCx * v22_1_0 + WQx * v22_1_1 + (VT)3.0 * oo2ze * v12_1_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v22_4_1 = QCx * v22_1_1 + WQx * v22_1_2 + (VT)3.0 * oo2ze * v12_1_2 + (VT)1.0 * oo2e * (v22_0_1 - rho_e * v22_0_2);
            const VT v23_4_0 = QCx * v23_1_0 + WQx * v23_1_1 + (VT)2.0 * oo2ze * v13_1_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v23_4_1 = QCx * v23_1_1 + WQx * v23_1_2 + (VT)2.0 * oo2ze * v13_1_2 + (VT)1.0 * oo2e * (v23_0_1 - rho_e * v23_0_2);
            const VT v24_4_0 = QCx * v24_1_0 + WQx * v24_1_1 + (VT)2.0 * oo2ze * v15_1_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v24_4_1 = QCx * v24_1_1 + WQx * v24_1_2 + (VT)2.0 * oo2ze * v15_1_2 + (VT)1.0 * oo2e * (v24_0_1 - rho_e * v24_0_2);
            const VT v25_4_0 = QCx * v25_1_0 + WQx * v25_1_1 + (VT)2.0 * oo2ze * v14_1_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v25_4_1 = QCx * v25_1_1 + WQx * v25_1_2 + (VT)2.0 * oo2ze * v14_1_2 + (VT)1.0 * oo2e * (v25_0_1 - rho_e * v25_0_2);
            const VT v26_4_0 = QCx * v26_1_0 + WQx * v26_1_1 + (VT)1.0 * oo2ze * v16_1_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v26_4_1 = QCx * v26_1_1 + WQx * v26_1_2 + (VT)1.0 * oo2ze * v16_1_2 + (VT)1.0 * oo2e * (v26_0_1 - rho_e * v26_0_2);
            const VT v27_4_0 = QCx * v27_1_0 + WQx * v27_1_1 + (VT)1.0 * oo2ze * v17_1_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v27_4_1 = QCx * v27_1_1 + WQx * v27_1_2 + (VT)1.0 * oo2ze * v17_1_2 + (VT)1.0 * oo2e * (v27_0_1 - rho_e * v27_0_2);
            const VT v28_4_0 = QCx * v28_1_0 + WQx * v28_1_1 + (VT)1.0 * oo2ze * v18_1_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v28_4_1 = QCx * v28_1_1 + WQx * v28_1_2 + (VT)1.0 * oo2ze * v18_1_2 + (VT)1.0 * oo2e * (v28_0_1 - rho_e * v28_0_2);
            const VT v29_4_0 = QCx * v29_1_0 + WQx * v29_1_1 + (VT)1.0 * oo2ze * v19_1_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v29_4_1 = QCx * v29_1_1 + WQx * v29_1_2 + (VT)1.0 * oo2ze * v19_1_2 + (VT)1.0 * oo2e * (v29_0_1 - rho_e * v29_0_2);
            const VT v30_4_0 = QCx * v30_1_0 + WQx * v30_1_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v30_4_1 = QCx * v30_1_1 + WQx * v30_1_2 + (VT)1.0 * oo2e * (v30_0_1 - rho_e * v30_0_2);
            const VT v31_4_0 = QCx * v31_1_0 + WQx * v31_1_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v31_4_1 = QCx * v31_1_1 + WQx * v31_1_2 + (VT)1.0 * oo2e * (v31_0_1 - rho_e * v31_0_2);
            const VT v32_4_0 = QCx * v32_1_0 + WQx * v32_1_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v32_4_1 = QCx * v32_1_1 + WQx * v32_1_2 + (VT)1.0 * oo2e * (v32_0_1 - rho_e * v32_0_2);
            const VT v33_4_0 = QCx * v33_1_0 + WQx * v33_1_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v33_4_1 = QCx * v33_1_1 + WQx * v33_1_2 + (VT)1.0 * oo2e * (v33_0_1 - rho_e * v33_0_2);
            const VT v34_4_0 = QCx * v34_1_0 + WQx * v34_1_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
            const VT v34_4_1 = QCx * v34_1_1 + WQx * v34_1_2 + (VT)1.0 * oo2e * (v34_0_1 - rho_e * v34_0_2);
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
            const VT v20_5_0 = QCx * v20_2_0 + WQx * v20_2_1 + (VT)4.0 * oo2ze * v10_2_1;
            const VT v20_5_1 = QCx * v20_2_1 + WQx * v20_2_2 + (VT)4.0 * oo2ze * v10_2_2;
            const VT v21_5_0 = QCx * v21_2_0 + WQx * v21_2_1 + (VT)3.0 * oo2ze * v11_2_1;
            const VT v21_5_1 = QCx * v21_2_1 + WQx * v21_2_2 + (VT)3.0 * oo2ze * v11_2_2;
            const VT v22_5_0 = QCx * v22_2_0 + WQx * v22_2_1 + (VT)3.0 * oo2ze * v12_2_1;
            const VT v22_5_1 = QCx * v22_2_1 + WQx * v22_2_2 + (VT)3.0 * oo2ze * v12_2_2;
            const VT v23_5_0 = QCx * v23_2_0 + WQx * v23_2_1 + (VT)2.0 * oo2ze * v13_2_1;
            const VT v23_5_1 = QCx * v23_2_1 + WQx * v23_2_2 + (VT)2.0 * oo2ze * v13_2_2;
            const VT v24_5_0 = QCx * v24_2_0 + WQx * v24_2_1 + (VT)2.0 * oo2ze * v15_2_1;
            const VT v24_5_1 = QCx * v24_2_1 + WQx * v24_2_2 + (VT)2.0 * oo2ze * v15_2_2;
            const VT v25_5_0 = QCx * v25_2_0 + WQx * v25_2_1 + (VT)2.0 * oo2ze * v14_2_1;
            const VT v25_5_1 = QCx * v25_2_1 + WQx * v25_2_2 + (VT)2.0 * oo2ze * v14_2_2;
            const VT v26_5_0 = QCx * v26_2_0 + WQx * v26_2_1 + (VT)1.0 * oo2ze * v16_2_1;
            const VT v26_5_1 = QCx * v26_2_1 + WQx * v26_2_2 + (VT)1.0 * oo2ze * v16_2_2;
            const VT v27_5_0 = QCx * v27_2_0 + WQx * v27_2_1 + (VT)1.0 * oo2ze * v17_2_1;
            const VT v27_5_1 = QCx * v27_2_1 + WQx * v27_2_2 + (VT)1.0 * oo2ze * v17_2_2;
            const VT v28_5_0 = QCx * v28_2_0 + WQx * v28_2_1 + (VT)1.0 * oo2ze * v18_2_1;
            const VT v28_5_1 = QCx * v28_2_1 + WQx * v28_2_2 + (VT)1.0 * oo2ze * v18_2_2;
            const VT v29_5_0 = QCx * v29_2_0 + WQx * v29_2_1 + (VT)1.0 * oo2ze * v19_2_1;
            const VT v29_5_1 = QCx * v29_2_1 + WQx * v29_2_2 + (VT)1.0 * oo2ze * v19_2_2;
            const VT v30_5_0 = QCx * v30_2_0 + WQx * v30_2_1;
            const VT v30_5_1 = QCx * v30_2_1 + WQx * v30_2_2;
            const VT v31_5_0 = QCx * v31_2_0 + WQx * v31_2_1;
            const VT v31_5_1 = QCx * v31_2_1 + WQx * v31_2_2;
            const VT v32_5_0 = QCx * v32_2_0 + WQx * v32_2_1;
            const VT v32_5_1 = QCx * v32_2_1 + WQx * v32_2_2;
            const VT v33_5_0 = QCx * v33_2_0 + WQx * v33_2_1;
            const VT v33_5_1 = QCx * v33_2_1 + WQx * v33_2_2;
            const VT v34_5_0 = QCx * v34_2_0 + WQx * v34_2_1;
            const VT v34_5_1 = QCx * v34_2_1 + WQx * v34_2_2;
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
            const VT v20_6_0 = QCx * v20_3_0 + WQx * v20_3_1 + (VT)4.0 * oo2ze * v10_3_1;
            const VT v20_6_1 = QCx * v20_3_1 + WQx * v20_3_2 + (VT)4.0 * oo2ze * v10_3_2;
            const VT v21_6_0 = QCx * v21_3_0 + WQx * v21_3_1 + (VT)3.0 * oo2ze * v11_3_1;
            const VT v21_6_1 = QCx * v21_3_1 + WQx * v21_3_2 + (VT)3.0 * oo2ze * v11_3_2;
            const VT v22_6_0 = QCx * v22_3_0 + WQx * v22_3_1 + (VT)3.0 * oo2ze * v12_3_1;
            const VT v22_6_1 = QCx * v22_3_1 + WQx * v22_3_2 + (VT)3.0 * oo2ze * v12_3_2;
            const VT v23_6_0 = QCx * v23_3_0 + WQx * v23_3_1 + (VT)2.0 * oo2ze * v13_3_1;
            const VT v23_6_1 = QCx * v23_3_1 + WQx * v23_3_2 + (VT)2.0 * oo2ze * v13_3_2;
            const VT v24_6_0 = QCx * v24_3_0 + WQx * v24_3_1 + (VT)2.0 * oo2ze * v15_3_1;
            const VT v24_6_1 = QCx * v24_3_1 + WQx * v24_3_2 + (VT)2.0 * oo2ze * v15_3_2;
            const VT v25_6_0 = QCx * v25_3_0 + WQx * v25_3_1 + (VT)2.0 * oo2ze * v14_3_1;
            const VT v25_6_1 = QCx * v25_3_1 + WQx * v25_3_2 + (VT)2.0 * oo2ze * v14_3_2;
            const VT v26_6_0 = QCx * v26_3_0 + WQx * v26_3_1 + (VT)1.0 * oo2ze * v16_3_1;
            const VT v26_6_1 = QCx * v26_3_1 + WQx * v26_3_2 + (VT)1.0 * oo2ze * v16_3_2;
            const VT v27_6_0 = QCx * v27_3_0 + WQx * v27_3_1 + (VT)1.0 * oo2ze * v17_3_1;
            const VT v27_6_1 = QCx * v27_3_1 + WQx * v27_3_2 + (VT)1.0 * oo2ze * v17_3_2;
            const VT v28_6_0 = QCx * v28_3_0 + WQx * v28_3_1 + (VT)1.0 * oo2ze * v18_3_1;
            const VT v28_6_1 = QCx * v28_3_1 + WQx * v28_3_2 + (VT)1.0 * oo2ze * v18_3_2;
            const VT v29_6_0 = QCx * v29_3_0 + WQx * v29_3_1 + (VT)1.0 * oo2ze * v19_3_1;
            const VT v29_6_1 = QCx * v29_3_1 + WQx * v29_3_2 + (VT)1.0 * oo2ze * v19_3_2;
            const VT v30_6_0 = QCx * v30_3_0 + WQx * v30_3_1;
            const VT v30_6_1 = QCx * v30_3_1 + WQx * v30_3_2;
            const VT v31_6_0 = QCx * v31_3_0 + WQx * v31_3_1;
            const VT v31_6_1 = QCx * v31_3_1 + WQx * v31_3_2;
            const VT v32_6_0 = QCx * v32_3_0 + WQx * v32_3_1;
            const VT v32_6_1 = QCx * v32_3_1 + WQx * v32_3_2;
            const VT v33_6_0 = QCx * v33_3_0 + WQx * v33_3_1;
            const VT v33_6_1 = QCx * v33_3_1 + WQx * v33_3_2;
            const VT v34_6_0 = QCx * v34_3_0 + WQx * v34_3_1;
            const VT v34_6_1 = QCx * v34_3_1 + WQx * v34_3_2;
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
            const VT v20_7_0 = QCy * v20_2_0 + WQy * v20_2_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v20_7_1 = QCy * v20_2_1 + WQy * v20_2_2 + (VT)1.0 * oo2e * (v20_0_1 - rho_e * v20_0_2);
            const VT v21_7_0 = QCy * v21_2_0 + WQy * v21_2_1 + (VT)1.0 * oo2ze * v10_2_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v21_7_1 = QCy * v21_2_1 + WQy * v21_2_2 + (VT)1.0 * oo2ze * v10_2_2 + (VT)1.0 * oo2e * (v21_0_1 - rho_e * v21_0_2);
            const VT v22_7_0 = QCy * v22_2_0 + WQy * v22_2_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v22_7_1 = QCy * v22_2_1 + WQy * v22_2_2 + (VT)1.0 * oo2e * (v22_0_1 - rho_e * v22_0_2);
            const VT v23_7_0 = QCy * v23_2_0 + WQy * v23_2_1 + (VT)2.0 * oo2ze * v11_2_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v23_7_1 = QCy * v23_2_1 + WQy * v23_2_2 + (VT)2.0 * oo2ze * v11_2_2 + (VT)1.0 * oo2e * (v23_0_1 - rho_e * v23_0_2);
            const VT v24_7_0 = QCy * v24_2_0 + WQy * v24_2_1 + (VT)1.0 * oo2ze * v12_2_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v24_7_1 = QCy * v24_2_1 + WQy * v24_2_2 + (VT)1.0 * oo2ze * v12_2_2 + (VT)1.0 * oo2e * (v24_0_1 - rho_e * v24_0_2);
            const VT v25_7_0 = QCy * v25_2_0 + WQy * v25_2_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v25_7_1 = QCy * v25_2_1 + WQy * v25_2_2 + (VT)1.0 * oo2e * (v25_0_1 - rho_e * v25_0_2);
            const VT v26_7_0 = QCy * v26_2_0 + WQy * v26_2_1 + (VT)3.0 * oo2ze * v13_2_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v26_7_1 = QCy * v26_2_1 + WQy * v26_2_2 + (VT)3.0 * oo2ze * v13_2_2 + (VT)1.0 * oo2e * (v26_0_1 - rho_e * v26_0_2);
            const VT v27_7_0 = QCy * v27_2_0 + WQy * v27_2_1 + (VT)2.0 * oo2ze * v15_2_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v27_7_1 = QCy * v27_2_1 + WQy * v27_2_2 + (VT)2.0 * oo2ze * v15_2_2 + (VT)1.0 * oo2e * (v27_0_1 - rho_e * v27_0_2);
            const VT v28_7_0 = QCy * v28_2_0 + WQy * v28_2_1 + (VT)1.0 * oo2ze * v14_2_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v28_7_1 = QCy * v28_2_1 + WQy * v28_2_2 + (VT)1.0 * oo2ze * v14_2_2 + (VT)1.0 * oo2e * (v28_0_1 - rho_e * v28_0_2);
            const VT v29_7_0 = QCy * v29_2_0 + WQy * v29_2_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v29_7_1 = QCy * v29_2_1 + WQy * v29_2_2 + (VT)1.0 * oo2e * (v29_0_1 - rho_e * v29_0_2);
            const VT v30_7_0 = QCy * v30_2_0 + WQy * v30_2_1 + (VT)4.0 * oo2ze * v16_2_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v30_7_1 = QCy * v30_2_1 + WQy * v30_2_2 + (VT)4.0 * oo2ze * v16_2_2 + (VT)1.0 * oo2e * (v30_0_1 - rho_e * v30_0_2);
            const VT v31_7_0 = QCy * v31_2_0 + WQy * v31_2_1 + (VT)3.0 * oo2ze * v17_2_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v31_7_1 = QCy * v31_2_1 + WQy * v31_2_2 + (VT)3.0 * oo2ze * v17_2_2 + (VT)1.0 * oo2e * (v31_0_1 - rho_e * v31_0_2);
            const VT v32_7_0 = QCy * v32_2_0 + WQy * v32_2_1 + (VT)2.0 * oo2ze * v18_2_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v32_7_1 = QCy * v32_2_1 + WQy * v32_2_2 + (VT)2.0 * oo2ze * v18_2_2 + (VT)1.0 * oo2e * (v32_0_1 - rho_e * v32_0_2);
            const VT v33_7_0 = QCy * v33_2_0 + WQy * v33_2_1 + (VT)1.0 * oo2ze * v19_2_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v33_7_1 = QCy * v33_2_1 + WQy * v33_2_2 + (VT)1.0 * oo2ze * v19_2_2 + (VT)1.0 * oo2e * (v33_0_1 - rho_e * v33_0_2);
            const VT v34_7_0 = QCy * v34_2_0 + WQy * v34_2_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
            const VT v34_7_1 = QCy * v34_2_1 + WQy * v34_2_2 + (VT)1.0 * oo2e * (v34_0_1 - rho_e * v34_0_2);
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
            const VT v20_8_0 = QCy * v20_3_0 + WQy * v20_3_1;
            const VT v20_8_1 = QCy * v20_3_1 + WQy * v20_3_2;
            const VT v21_8_0 = QCy * v21_3_0 + WQy * v21_3_1 + (VT)1.0 * oo2ze * v10_3_1;
            const VT v21_8_1 = QCy * v21_3_1 + WQy * v21_3_2 + (VT)1.0 * oo2ze * v10_3_2;
            const VT v22_8_0 = QCy * v22_3_0 + WQy * v22_3_1;
            const VT v22_8_1 = QCy * v22_3_1 + WQy * v22_3_2;
            const VT v23_8_0 = QCy * v23_3_0 + WQy * v23_3_1 + (VT)2.0 * oo2ze * v11_3_1;
            const VT v23_8_1 = QCy * v23_3_1 + WQy * v23_3_2 + (VT)2.0 * oo2ze * v11_3_2;
            const VT v24_8_0 = QCy * v24_3_0 + WQy * v24_3_1 + (VT)1.0 * oo2ze * v12_3_1;
            const VT v24_8_1 = QCy * v24_3_1 + WQy * v24_3_2 + (VT)1.0 * oo2ze * v12_3_2;
            const VT v25_8_0 = QCy * v25_3_0 + WQy * v25_3_1;
            const VT v25_8_1 = QCy * v25_3_1 + WQy * v25_3_2;
            const VT v26_8_0 = QCy * v26_3_0 + WQy * v26_3_1 + (VT)3.0 * oo2ze * v13_3_1;
            const VT v26_8_1 = QCy * v26_3_1 + WQy * v26_3_2 + (VT)3.0 * oo2ze * v13_3_2;
            const VT v27_8_0 = QCy * v27_3_0 + WQy * v27_3_1 + (VT)2.0 * oo2ze * v15_3_1;
            const VT v27_8_1 = QCy * v27_3_1 + WQy * v27_3_2 + (VT)2.0 * oo2ze * v15_3_2;
            const VT v28_8_0 = QCy * v28_3_0 + WQy * v28_3_1 + (VT)1.0 * oo2ze * v14_3_1;
            const VT v28_8_1 = QCy * v28_3_1 + WQy * v28_3_2 + (VT)1.0 * oo2ze * v14_3_2;
            const VT v29_8_0 = QCy * v29_3_0 + WQy * v29_3_1;
            const VT v29_8_1 = QCy * v29_3_1 + WQy * v29_3_2;
            const VT v30_8_0 = QCy * v30_3_0 + WQy * v30_3_1 + (VT)4.0 * oo2ze * v16_3_1;
            const VT v30_8_1 = QCy * v30_3_1 + WQy * v30_3_2 + (VT)4.0 * oo2ze * v16_3_2;
            const VT v31_8_0 = QCy * v31_3_0 + WQy * v31_3_1 + (VT)3.0 * oo2ze * v17_3_1;
            const VT v31_8_1 = QCy * v31_3_1 + WQy * v31_3_2 + (VT)3.0 * oo2ze * v17_3_2;
            const VT v32_8_0 = QCy * v32_3_0 + WQy * v32_3_1 + (VT)2.0 * oo2ze * v18_3_1;
            const VT v32_8_1 = QCy * v32_3_1 + WQy * v32_3_2 + (VT)2.0 * oo2ze * v18_3_2;
            const VT v33_8_0 = QCy * v33_3_0 + WQy * v33_3_1 + (VT)1.0 * oo2ze * v19_3_1;
            const VT v33_8_1 = QCy * v33_3_1 + WQy * v33_3_2 + (VT)1.0 * oo2ze * v19_3_2;
            const VT v34_8_0 = QCy * v34_3_0 + WQy * v34_3_1;
            const VT v34_8_1 = QCy * v34_3_1 + WQy * v34_3_2;
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
            const VT v20_9_0 = QCz * v20_3_0 + WQz * v20_3_1 + (VT)1.0 * oo2e * (v20_0_0 - rho_e * v20_0_1);
            const VT v20_9_1 = QCz * v20_3_1 + WQz * v20_3_2 + (VT)1.0 * oo2e * (v20_0_1 - rho_e * v20_0_2);
            const VT v21_9_0 = QCz * v21_3_0 + WQz * v21_3_1 + (VT)1.0 * oo2e * (v21_0_0 - rho_e * v21_0_1);
            const VT v21_9_1 = QCz * v21_3_1 + WQz * v21_3_2 + (VT)1.0 * oo2e * (v21_0_1 - rho_e * v21_0_2);
            const VT v22_9_0 = QCz * v22_3_0 + WQz * v22_3_1 + (VT)1.0 * oo2ze * v10_3_1 + (VT)1.0 * oo2e * (v22_0_0 - rho_e * v22_0_1);
            const VT v22_9_1 = QCz * v22_3_1 + WQz * v22_3_2 + (VT)1.0 * oo2ze * v10_3_2 + (VT)1.0 * oo2e * (v22_0_1 - rho_e * v22_0_2);
            const VT v23_9_0 = QCz * v23_3_0 + WQz * v23_3_1 + (VT)1.0 * oo2e * (v23_0_0 - rho_e * v23_0_1);
            const VT v23_9_1 = QCz * v23_3_1 + WQz * v23_3_2 + (VT)1.0 * oo2e * (v23_0_1 - rho_e * v23_0_2);
            const VT v24_9_0 = QCz * v24_3_0 + WQz * v24_3_1 + (VT)1.0 * oo2ze * v11_3_1 + (VT)1.0 * oo2e * (v24_0_0 - rho_e * v24_0_1);
            const VT v24_9_1 = QCz * v24_3_1 + WQz * v24_3_2 + (VT)1.0 * oo2ze * v11_3_2 + (VT)1.0 * oo2e * (v24_0_1 - rho_e * v24_0_2);
            const VT v25_9_0 = QCz * v25_3_0 + WQz * v25_3_1 + (VT)2.0 * oo2ze * v12_3_1 + (VT)1.0 * oo2e * (v25_0_0 - rho_e * v25_0_1);
            const VT v25_9_1 = QCz * v25_3_1 + WQz * v25_3_2 + (VT)2.0 * oo2ze * v12_3_2 + (VT)1.0 * oo2e * (v25_0_1 - rho_e * v25_0_2);
            const VT v26_9_0 = QCz * v26_3_0 + WQz * v26_3_1 + (VT)1.0 * oo2e * (v26_0_0 - rho_e * v26_0_1);
            const VT v26_9_1 = QCz * v26_3_1 + WQz * v26_3_2 + (VT)1.0 * oo2e * (v26_0_1 - rho_e * v26_0_2);
            const VT v27_9_0 = QCz * v27_3_0 + WQz * v27_3_1 + (VT)1.0 * oo2ze * v13_3_1 + (VT)1.0 * oo2e * (v27_0_0 - rho_e * v27_0_1);
            const VT v27_9_1 = QCz * v27_3_1 + WQz * v27_3_2 + (VT)1.0 * oo2ze * v13_3_2 + (VT)1.0 * oo2e * (v27_0_1 - rho_e * v27_0_2);
            const VT v28_9_0 = QCz * v28_3_0 + WQz * v28_3_1 + (VT)2.0 * oo2ze * v15_3_1 + (VT)1.0 * oo2e * (v28_0_0 - rho_e * v28_0_1);
            const VT v28_9_1 = QCz * v28_3_1 + WQz * v28_3_2 + (VT)2.0 * oo2ze * v15_3_2 + (VT)1.0 * oo2e * (v28_0_1 - rho_e * v28_0_2);
            const VT v29_9_0 = QCz * v29_3_0 + WQz * v29_3_1 + (VT)3.0 * oo2ze * v14_3_1 + (VT)1.0 * oo2e * (v29_0_0 - rho_e * v29_0_1);
            const VT v29_9_1 = QCz * v29_3_1 + WQz * v29_3_2 + (VT)3.0 * oo2ze * v14_3_2 + (VT)1.0 * oo2e * (v29_0_1 - rho_e * v29_0_2);
            const VT v30_9_0 = QCz * v30_3_0 + WQz * v30_3_1 + (VT)1.0 * oo2e * (v30_0_0 - rho_e * v30_0_1);
            const VT v30_9_1 = QCz * v30_3_1 + WQz * v30_3_2 + (VT)1.0 * oo2e * (v30_0_1 - rho_e * v30_0_2);
            const VT v31_9_0 = QCz * v31_3_0 + WQz * v31_3_1 + (VT)1.0 * oo2ze * v16_3_1 + (VT)1.0 * oo2e * (v31_0_0 - rho_e * v31_0_1);
            const VT v31_9_1 = QCz * v31_3_1 + WQz * v31_3_2 + (VT)1.0 * oo2ze * v16_3_2 + (VT)1.0 * oo2e * (v31_0_1 - rho_e * v31_0_2);
            const VT v32_9_0 = QCz * v32_3_0 + WQz * v32_3_1 + (VT)2.0 * oo2ze * v17_3_1 + (VT)1.0 * oo2e * (v32_0_0 - rho_e * v32_0_1);
            const VT v32_9_1 = QCz * v32_3_1 + WQz * v32_3_2 + (VT)2.0 * oo2ze * v17_3_2 + (VT)1.0 * oo2e * (v32_0_1 - rho_e * v32_0_2);
            const VT v33_9_0 = QCz * v33_3_0 + WQz * v33_3_1 + (VT)3.0 * oo2ze * v18_3_1 + (VT)1.0 * oo2e * (v33_0_0 - rho_e * v33_0_1);
            const VT v33_9_1 = QCz * v33_3_1 + WQz * v33_3_2 + (VT)3.0 * oo2ze * v18_3_2 + (VT)1.0 * oo2e * (v33_0_1 - rho_e * v33_0_2);
            const VT v34_9_0 = QCz * v34_3_0 + WQz * v34_3_1 + (VT)4.0 * oo2ze * v19_3_1 + (VT)1.0 * oo2e * (v34_0_0 - rho_e * v34_0_1);
            const VT v34_9_1 = QCz * v34_3_1 + WQz * v34_3_2 + (VT)4.0 * oo2ze * v19_3_2 + (VT)1.0 * oo2e * (v34_0_1 - rho_e * v34_0_2);
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
            const VT v20_10_0 = QCx * v20_4_0 + WQx * v20_4_1 + (VT)4.0 * oo2ze * v10_4_1 + (VT)2.0 * oo2e * (v20_1_0 - rho_e * v20_1_1);
            const VT v21_10_0 = QCx * v21_4_0 + WQx * v21_4_1 + (VT)3.0 * oo2ze * v11_4_1 + (VT)2.0 * oo2e * (v21_1_0 - rho_e * v21_1_1);
            const VT v22_10_0 = QCx * v22_4_0 + WQx * v22_4_1 + (VT)3.0 * oo2ze * v12_4_1 + (VT)2.0 * oo2e * (v22_1_0 - rho_e * v22_1_1);
            const VT v23_10_0 = QCx * v23_4_0 + WQx * v23_4_1 + (VT)2.0 * oo2ze * v13_4_1 + (VT)2.0 * oo2e * (v23_1_0 - rho_e * v23_1_1);
            const VT v24_10_0 = QCx * v24_4_0 + WQx * v24_4_1 + (VT)2.0 * oo2ze * v15_4_1 + (VT)2.0 * oo2e * (v24_1_0 - rho_e * v24_1_1);
            const VT v25_10_0 = QCx * v25_4_0 + WQx * v25_4_1 + (VT)2.0 * oo2ze * v14_4_1 + (VT)2.0 * oo2e * (v25_1_0 - rho_e * v25_1_1);
            const VT v26_10_0 = QCx * v26_4_0 + WQx * v26_4_1 + (VT)1.0 * oo2ze * v16_4_1 + (VT)2.0 * oo2e * (v26_1_0 - rho_e * v26_1_1);
            const VT v27_10_0 = QCx * v27_4_0 + WQx * v27_4_1 + (VT)1.0 * oo2ze * v17_4_1 + (VT)2.0 * oo2e * (v27_1_0 - rho_e * v27_1_1);
            const VT v28_10_0 = QCx * v28_4_0 + WQx * v28_4_1 + (VT)1.0 * oo2ze * v18_4_1 + (VT)2.0 * oo2e * (v28_1_0 - rho_e * v28_1_1);
            const VT v29_10_0 = QCx * v29_4_0 + WQx * v29_4_1 + (VT)1.0 * oo2ze * v19_4_1 + (VT)2.0 * oo2e * (v29_1_0 - rho_e * v29_1_1);
            const VT v30_10_0 = QCx * v30_4_0 + WQx * v30_4_1 + (VT)2.0 * oo2e * (v30_1_0 - rho_e * v30_1_1);
            const VT v31_10_0 = QCx * v31_4_0 + WQx * v31_4_1 + (VT)2.0 * oo2e * (v31_1_0 - rho_e * v31_1_1);
            const VT v32_10_0 = QCx * v32_4_0 + WQx * v32_4_1 + (VT)2.0 * oo2e * (v32_1_0 - rho_e * v32_1_1);
            const VT v33_10_0 = QCx * v33_4_0 + WQx * v33_4_1 + (VT)2.0 * oo2e * (v33_1_0 - rho_e * v33_1_1);
            const VT v34_10_0 = QCx * v34_4_0 + WQx * v34_4_1 + (VT)2.0 * oo2e * (v34_1_0 - rho_e * v34_1_1);
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
            const VT v20_11_0 = QCx * v20_5_0 + WQx * v20_5_1 + (VT)4.0 * oo2ze * v10_5_1 + (VT)1.0 * oo2e * (v20_2_0 - rho_e * v20_2_1);
            const VT v21_11_0 = QCx * v21_5_0 + WQx * v21_5_1 + (VT)3.0 * oo2ze * v11_5_1 + (VT)1.0 * oo2e * (v21_2_0 - rho_e * v21_2_1);
            const VT v22_11_0 = QCx * v22_5_0 + WQx * v22_5_1 + (VT)3.0 * oo2ze * v12_5_1 + (VT)1.0 * oo2e * (v22_2_0 - rho_e * v22_2_1);
            const VT v23_11_0 = QCx * v23_5_0 + WQx * v23_5_1 + (VT)2.0 * oo2ze * v13_5_1 + (VT)1.0 * oo2e * (v23_2_0 - rho_e * v23_2_1);
            const VT v24_11_0 = QCx * v24_5_0 + WQx * v24_5_1 + (VT)2.0 * oo2ze * v15_5_1 + (VT)1.0 * oo2e * (v24_2_0 - rho_e * v24_2_1);
            const VT v25_11_0 = QCx * v25_5_0 + WQx * v25_5_1 + (VT)2.0 * oo2ze * v14_5_1 + (VT)1.0 * oo2e * (v25_2_0 - rho_e * v25_2_1);
            const VT v26_11_0 = QCx * v26_5_0 + WQx * v26_5_1 + (VT)1.0 * oo2ze * v16_5_1 + (VT)1.0 * oo2e * (v26_2_0 - rho_e * v26_2_1);
            const VT v27_11_0 = QCx * v27_5_0 + WQx * v27_5_1 + (VT)1.0 * oo2ze * v17_5_1 + (VT)1.0 * oo2e * (v27_2_0 - rho_e * v27_2_1);
            const VT v28_11_0 = QCx * v28_5_0 + WQx * v28_5_1 + (VT)1.0 * oo2ze * v18_5_1 + (VT)1.0 * oo2e * (v28_2_0 - rho_e * v28_2_1);
            const VT v29_11_0 = QCx * v29_5_0 + WQx * v29_5_1 + (VT)1.0 * oo2ze * v19_5_1 + (VT)1.0 * oo2e * (v29_2_0 - rho_e * v29_2_1);
            const VT v30_11_0 = QCx * v30_5_0 + WQx * v30_5_1 + (VT)1.0 * oo2e * (v30_2_0 - rho_e * v30_2_1);
            const VT v31_11_0 = QCx * v31_5_0 + WQx * v31_5_1 + (VT)1.0 * oo2e * (v31_2_0 - rho_e * v31_2_1);
            const VT v32_11_0 = QCx * v32_5_0 + WQx * v32_5_1 + (VT)1.0 * oo2e * (v32_2_0 - rho_e * v32_2_1);
            const VT v33_11_0 = QCx * v33_5_0 + WQx * v33_5_1 + (VT)1.0 * oo2e * (v33_2_0 - rho_e * v33_2_1);
            const VT v34_11_0 = QCx * v34_5_0 + WQx * v34_5_1 + (VT)1.0 * oo2e * (v34_2_0 - rho_e * v34_2_1);
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
            const VT v20_12_0 = QCx * v20_6_0 + WQx * v20_6_1 + (VT)4.0 * oo2ze * v10_6_1 + (VT)1.0 * oo2e * (v20_3_0 - rho_e * v20_3_1);
            const VT v21_12_0 = QCx * v21_6_0 + WQx * v21_6_1 + (VT)3.0 * oo2ze * v11_6_1 + (VT)1.0 * oo2e * (v21_3_0 - rho_e * v21_3_1);
            const VT v22_12_0 = QCx * v22_6_0 + WQx * v22_6_1 + (VT)3.0 * oo2ze * v12_6_1 + (VT)1.0 * oo2e * (v22_3_0 - rho_e * v22_3_1);
            const VT v23_12_0 = QCx * v23_6_0 + WQx * v23_6_1 + (VT)2.0 * oo2ze * v13_6_1 + (VT)1.0 * oo2e * (v23_3_0 - rho_e * v23_3_1);
            const VT v24_12_0 = QCx * v24_6_0 + WQx * v24_6_1 + (VT)2.0 * oo2ze * v15_6_1 + (VT)1.0 * oo2e * (v24_3_0 - rho_e * v24_3_1);
            const VT v25_12_0 = QCx * v25_6_0 + WQx * v25_6_1 + (VT)2.0 * oo2ze * v14_6_1 + (VT)1.0 * oo2e * (v25_3_0 - rho_e * v25_3_1);
            const VT v26_12_0 = QCx * v26_6_0 + WQx * v26_6_1 + (VT)1.0 * oo2ze * v16_6_1 + (VT)1.0 * oo2e * (v26_3_0 - rho_e * v26_3_1);
            const VT v27_12_0 = QCx * v27_6_0 + WQx * v27_6_1 + (VT)1.0 * oo2ze * v17_6_1 + (VT)1.0 * oo2e * (v27_3_0 - rho_e * v27_3_1);
            const VT v28_12_0 = QCx * v28_6_0 + WQx * v28_6_1 + (VT)1.0 * oo2ze * v18_6_1 + (VT)1.0 * oo2e * (v28_3_0 - rho_e * v28_3_1);
            const VT v29_12_0 = QCx * v29_6_0 + WQx * v29_6_1 + (VT)1.0 * oo2ze * v19_6_1 + (VT)1.0 * oo2e * (v29_3_0 - rho_e * v29_3_1);
            const VT v30_12_0 = QCx * v30_6_0 + WQx * v30_6_1 + (VT)1.0 * oo2e * (v30_3_0 - rho_e * v30_3_1);
            const VT v31_12_0 = QCx * v31_6_0 + WQx * v31_6_1 + (VT)1.0 * oo2e * (v31_3_0 - rho_e * v31_3_1);
            const VT v32_12_0 = QCx * v32_6_0 + WQx * v32_6_1 + (VT)1.0 * oo2e * (v32_3_0 - rho_e * v32_3_1);
            const VT v33_12_0 = QCx * v33_6_0 + WQx * v33_6_1 + (VT)1.0 * oo2e * (v33_3_0 - rho_e * v33_3_1);
            const VT v34_12_0 = QCx * v34_6_0 + WQx * v34_6_1 + (VT)1.0 * oo2e * (v34_3_0 - rho_e * v34_3_1);
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
            const VT v20_13_0 = QCy * v20_5_0 + WQy * v20_5_1 + (VT)1.0 * oo2e * (v20_1_0 - rho_e * v20_1_1);
            const VT v21_13_0 = QCy * v21_5_0 + WQy * v21_5_1 + (VT)1.0 * oo2ze * v10_5_1 + (VT)1.0 * oo2e * (v21_1_0 - rho_e * v21_1_1);
            const VT v22_13_0 = QCy * v22_5_0 + WQy * v22_5_1 + (VT)1.0 * oo2e * (v22_1_0 - rho_e * v22_1_1);
            const VT v23_13_0 = QCy * v23_5_0 + WQy * v23_5_1 + (VT)2.0 * oo2ze * v11_5_1 + (VT)1.0 * oo2e * (v23_1_0 - rho_e * v23_1_1);
            const VT v24_13_0 = QCy * v24_5_0 + WQy * v24_5_1 + (VT)1.0 * oo2ze * v12_5_1 + (VT)1.0 * oo2e * (v24_1_0 - rho_e * v24_1_1);
            const VT v25_13_0 = QCy * v25_5_0 + WQy * v25_5_1 + (VT)1.0 * oo2e * (v25_1_0 - rho_e * v25_1_1);
            const VT v26_13_0 = QCy * v26_5_0 + WQy * v26_5_1 + (VT)3.0 * oo2ze * v13_5_1 + (VT)1.0 * oo2e * (v26_1_0 - rho_e * v26_1_1);
            const VT v27_13_0 = QCy * v27_5_0 + WQy * v27_5_1 + (VT)2.0 * oo2ze * v15_5_1 + (VT)1.0 * oo2e * (v27_1_0 - rho_e * v27_1_1);
            const VT v28_13_0 = QCy * v28_5_0 + WQy * v28_5_1 + (VT)1.0 * oo2ze * v14_5_1 + (VT)1.0 * oo2e * (v28_1_0 - rho_e * v28_1_1);
            const VT v29_13_0 = QCy * v29_5_0 + WQy * v29_5_1 + (VT)1.0 * oo2e * (v29_1_0 - rho_e * v29_1_1);
            const VT v30_13_0 = QCy * v30_5_0 + WQy * v30_5_1 + (VT)4.0 * oo2ze * v16_5_1 + (VT)1.0 * oo2e * (v30_1_0 - rho_e * v30_1_1);
            const VT v31_13_0 = QCy * v31_5_0 + WQy * v31_5_1 + (VT)3.0 * oo2ze * v17_5_1 + (VT)1.0 * oo2e * (v31_1_0 - rho_e * v31_1_1);
            const VT v32_13_0 = QCy * v32_5_0 + WQy * v32_5_1 + (VT)2.0 * oo2ze * v18_5_1 + (VT)1.0 * oo2e * (v32_1_0 - rho_e * v32_1_1);
            const VT v33_13_0 = QCy * v33_5_0 + WQy * v33_5_1 + (VT)1.0 * oo2ze * v19_5_1 + (VT)1.0 * oo2e * (v33_1_0 - rho_e * v33_1_1);
            const VT v34_13_0 = QCy * v34_5_0 + WQy * v34_5_1 + (VT)1.0 * oo2e * (v34_1_0 - rho_e * v34_1_1);
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
            const VT v20_14_0 = QCz * v20_6_0 + WQz * v20_6_1 + (VT)1.0 * oo2e * (v20_1_0 - rho_e * v20_1_1);
            const VT v21_14_0 = QCz * v21_6_0 + WQz * v21_6_1 + (VT)1.0 * oo2e * (v21_1_0 - rho_e * v21_1_1);
            const VT v22_14_0 = QCz * v22_6_0 + WQz * v22_6_1 + (VT)1.0 * oo2ze * v10_6_1 + (VT)1.0 * oo2e * (v22_1_0 - rho_e * v22_1_1);
            const VT v23_14_0 = QCz * v23_6_0 + WQz * v23_6_1 + (VT)1.0 * oo2e * (v23_1_0 - rho_e * v23_1_1);
            const VT v24_14_0 = QCz * v24_6_0 + WQz * v24_6_1 + (VT)1.0 * oo2ze * v11_6_1 + (VT)1.0 * oo2e * (v24_1_0 - rho_e * v24_1_1);
            const VT v25_14_0 = QCz * v25_6_0 + WQz * v25_6_1 + (VT)2.0 * oo2ze * v12_6_1 + (VT)1.0 * oo2e * (v25_1_0 - rho_e * v25_1_1);
            const VT v26_14_0 = QCz * v26_6_0 + WQz * v26_6_1 + (VT)1.0 * oo2e * (v26_1_0 - rho_e * v26_1_1);
            const VT v27_14_0 = QCz * v27_6_0 + WQz * v27_6_1 + (VT)1.0 * oo2ze * v13_6_1 + (VT)1.0 * oo2e * (v27_1_0 - rho_e * v27_1_1);
            const VT v28_14_0 = QCz * v28_6_0 + WQz * v28_6_1 + (VT)2.0 * oo2ze * v15_6_1 + (VT)1.0 * oo2e * (v28_1_0 - rho_e * v28_1_1);
            const VT v29_14_0 = QCz * v29_6_0 + WQz * v29_6_1 + (VT)3.0 * oo2ze * v14_6_1 + (VT)1.0 * oo2e * (v29_1_0 - rho_e * v29_1_1);
            const VT v30_14_0 = QCz * v30_6_0 + WQz * v30_6_1 + (VT)1.0 * oo2e * (v30_1_0 - rho_e * v30_1_1);
            const VT v31_14_0 = QCz * v31_6_0 + WQz * v31_6_1 + (VT)1.0 * oo2ze * v16_6_1 + (VT)1.0 * oo2e * (v31_1_0 - rho_e * v31_1_1);
            const VT v32_14_0 = QCz * v32_6_0 + WQz * v32_6_1 + (VT)2.0 * oo2ze * v17_6_1 + (VT)1.0 * oo2e * (v32_1_0 - rho_e * v32_1_1);
            const VT v33_14_0 = QCz * v33_6_0 + WQz * v33_6_1 + (VT)3.0 * oo2ze * v18_6_1 + (VT)1.0 * oo2e * (v33_1_0 - rho_e * v33_1_1);
            const VT v34_14_0 = QCz * v34_6_0 + WQz * v34_6_1 + (VT)4.0 * oo2ze * v19_6_1 + (VT)1.0 * oo2e * (v34_1_0 - rho_e * v34_1_1);
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
            const VT v20_15_0 = QCx * v20_8_0 + WQx * v20_8_1 + (VT)4.0 * oo2ze * v10_8_1;
            const VT v21_15_0 = QCx * v21_8_0 + WQx * v21_8_1 + (VT)3.0 * oo2ze * v11_8_1;
            const VT v22_15_0 = QCx * v22_8_0 + WQx * v22_8_1 + (VT)3.0 * oo2ze * v12_8_1;
            const VT v23_15_0 = QCx * v23_8_0 + WQx * v23_8_1 + (VT)2.0 * oo2ze * v13_8_1;
            const VT v24_15_0 = QCx * v24_8_0 + WQx * v24_8_1 + (VT)2.0 * oo2ze * v15_8_1;
            const VT v25_15_0 = QCx * v25_8_0 + WQx * v25_8_1 + (VT)2.0 * oo2ze * v14_8_1;
            const VT v26_15_0 = QCx * v26_8_0 + WQx * v26_8_1 + (VT)1.0 * oo2ze * v16_8_1;
            const VT v27_15_0 = QCx * v27_8_0 + WQx * v27_8_1 + (VT)1.0 * oo2ze * v17_8_1;
            const VT v28_15_0 = QCx * v28_8_0 + WQx * v28_8_1 + (VT)1.0 * oo2ze * v18_8_1;
            const VT v29_15_0 = QCx * v29_8_0 + WQx * v29_8_1 + (VT)1.0 * oo2ze * v19_8_1;
            const VT v30_15_0 = QCx * v30_8_0 + WQx * v30_8_1;
            const VT v31_15_0 = QCx * v31_8_0 + WQx * v31_8_1;
            const VT v32_15_0 = QCx * v32_8_0 + WQx * v32_8_1;
            const VT v33_15_0 = QCx * v33_8_0 + WQx * v33_8_1;
            const VT v34_15_0 = QCx * v34_8_0 + WQx * v34_8_1;
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
            const VT v20_16_0 = QCy * v20_7_0 + WQy * v20_7_1 + (VT)2.0 * oo2e * (v20_2_0 - rho_e * v20_2_1);
            const VT v21_16_0 = QCy * v21_7_0 + WQy * v21_7_1 + (VT)1.0 * oo2ze * v10_7_1 + (VT)2.0 * oo2e * (v21_2_0 - rho_e * v21_2_1);
            const VT v22_16_0 = QCy * v22_7_0 + WQy * v22_7_1 + (VT)2.0 * oo2e * (v22_2_0 - rho_e * v22_2_1);
            const VT v23_16_0 = QCy * v23_7_0 + WQy * v23_7_1 + (VT)2.0 * oo2ze * v11_7_1 + (VT)2.0 * oo2e * (v23_2_0 - rho_e * v23_2_1);
            const VT v24_16_0 = QCy * v24_7_0 + WQy * v24_7_1 + (VT)1.0 * oo2ze * v12_7_1 + (VT)2.0 * oo2e * (v24_2_0 - rho_e * v24_2_1);
            const VT v25_16_0 = QCy * v25_7_0 + WQy * v25_7_1 + (VT)2.0 * oo2e * (v25_2_0 - rho_e * v25_2_1);
            const VT v26_16_0 = QCy * v26_7_0 + WQy * v26_7_1 + (VT)3.0 * oo2ze * v13_7_1 + (VT)2.0 * oo2e * (v26_2_0 - rho_e * v26_2_1);
            const VT v27_16_0 = QCy * v27_7_0 + WQy * v27_7_1 + (VT)2.0 * oo2ze * v15_7_1 + (VT)2.0 * oo2e * (v27_2_0 - rho_e * v27_2_1);
            const VT v28_16_0 = QCy * v28_7_0 + WQy * v28_7_1 + (VT)1.0 * oo2ze * v14_7_1 + (VT)2.0 * oo2e * (v28_2_0 - rho_e * v28_2_1);
            const VT v29_16_0 = QCy * v29_7_0 + WQy * v29_7_1 + (VT)2.0 * oo2e * (v29_2_0 - rho_e * v29_2_1);
            const VT v30_16_0 = QCy * v30_7_0 + WQy * v30_7_1 + (VT)4.0 * oo2ze * v16_7_1 + (VT)2.0 * oo2e * (v30_2_0 - rho_e * v30_2_1);
            const VT v31_16_0 = QCy * v31_7_0 + WQy * v31_7_1 + (VT)3.0 * oo2ze * v17_7_1 + (VT)2.0 * oo2e * (v31_2_0 - rho_e * v31_2_1);
            const VT v32_16_0 = QCy * v32_7_0 + WQy * v32_7_1 + (VT)2.0 * oo2ze * v18_7_1 + (VT)2.0 * oo2e * (v32_2_0 - rho_e * v32_2_1);
            const VT v33_16_0 = QCy * v33_7_0 + WQy * v33_7_1 + (VT)1.0 * oo2ze * v19_7_1 + (VT)2.0 * oo2e * (v33_2_0 - rho_e * v33_2_1);
            const VT v34_16_0 = QCy * v34_7_0 + WQy * v34_7_1 + (VT)2.0 * oo2e * (v34_2_0 - rho_e * v34_2_1);
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
            const VT v20_17_0 = QCy * v20_8_0 + WQy * v20_8_1 + (VT)1.0 * oo2e * (v20_3_0 - rho_e * v20_3_1);
            const VT v21_17_0 = QCy * v21_8_0 + WQy * v21_8_1 + (VT)1.0 * oo2ze * v10_8_1 + (VT)1.0 * oo2e * (v21_3_0 - rho_e * v21_3_1);
            const VT v22_17_0 = QCy * v22_8_0 + WQy * v22_8_1 + (VT)1.0 * oo2e * (v22_3_0 - rho_e * v22_3_1);
            const VT v23_17_0 = QCy * v23_8_0 + WQy * v23_8_1 + (VT)2.0 * oo2ze * v11_8_1 + (VT)1.0 * oo2e * (v23_3_0 - rho_e * v23_3_1);
            const VT v24_17_0 = QCy * v24_8_0 + WQy * v24_8_1 + (VT)1.0 * oo2ze * v12_8_1 + (VT)1.0 * oo2e * (v24_3_0 - rho_e * v24_3_1);
            const VT v25_17_0 = QCy * v25_8_0 + WQy * v25_8_1 + (VT)1.0 * oo2e * (v25_3_0 - rho_e * v25_3_1);
            const VT v26_17_0 = QCy * v26_8_0 + WQy * v26_8_1 + (VT)3.0 * oo2ze * v13_8_1 + (VT)1.0 * oo2e * (v26_3_0 - rho_e * v26_3_1);
            const VT v27_17_0 = QCy * v27_8_0 + WQy * v27_8_1 + (VT)2.0 * oo2ze * v15_8_1 + (VT)1.0 * oo2e * (v27_3_0 - rho_e * v27_3_1);
            const VT v28_17_0 = QCy * v28_8_0 + WQy * v28_8_1 + (VT)1.0 * oo2ze * v14_8_1 + (VT)1.0 * oo2e * (v28_3_0 - rho_e * v28_3_1);
            const VT v29_17_0 = QCy * v29_8_0 + WQy * v29_8_1 + (VT)1.0 * oo2e * (v29_3_0 - rho_e * v29_3_1);
            const VT v30_17_0 = QCy * v30_8_0 + WQy * v30_8_1 + (VT)4.0 * oo2ze * v16_8_1 + (VT)1.0 * oo2e * (v30_3_0 - rho_e * v30_3_1);
            const VT v31_17_0 = QCy * v31_8_0 + WQy * v31_8_1 + (VT)3.0 * oo2ze * v17_8_1 + (VT)1.0 * oo2e * (v31_3_0 - rho_e * v31_3_1);
            const VT v32_17_0 = QCy * v32_8_0 + WQy * v32_8_1 + (VT)2.0 * oo2ze * v18_8_1 + (VT)1.0 * oo2e * (v32_3_0 - rho_e * v32_3_1);
            const VT v33_17_0 = QCy * v33_8_0 + WQy * v33_8_1 + (VT)1.0 * oo2ze * v19_8_1 + (VT)1.0 * oo2e * (v33_3_0 - rho_e * v33_3_1);
            const VT v34_17_0 = QCy * v34_8_0 + WQy * v34_8_1 + (VT)1.0 * oo2e * (v34_3_0 - rho_e * v34_3_1);
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
            const VT v20_18_0 = QCz * v20_8_0 + WQz * v20_8_1 + (VT)1.0 * oo2e * (v20_2_0 - rho_e * v20_2_1);
            const VT v21_18_0 = QCz * v21_8_0 + WQz * v21_8_1 + (VT)1.0 * oo2e * (v21_2_0 - rho_e * v21_2_1);
            const VT v22_18_0 = QCz * v22_8_0 + WQz * v22_8_1 + (VT)1.0 * oo2ze * v10_8_1 + (VT)1.0 * oo2e * (v22_2_0 - rho_e * v22_2_1);
            const VT v23_18_0 = QCz * v23_8_0 + WQz * v23_8_1 + (VT)1.0 * oo2e * (v23_2_0 - rho_e * v23_2_1);
            const VT v24_18_0 = QCz * v24_8_0 + WQz * v24_8_1 + (VT)1.0 * oo2ze * v11_8_1 + (VT)1.0 * oo2e * (v24_2_0 - rho_e * v24_2_1);
            const VT v25_18_0 = QCz * v25_8_0 + WQz * v25_8_1 + (VT)2.0 * oo2ze * v12_8_1 + (VT)1.0 * oo2e * (v25_2_0 - rho_e * v25_2_1);
            const VT v26_18_0 = QCz * v26_8_0 + WQz * v26_8_1 + (VT)1.0 * oo2e * (v26_2_0 - rho_e * v26_2_1);
            const VT v27_18_0 = QCz * v27_8_0 + WQz * v27_8_1 + (VT)1.0 * oo2ze * v13_8_1 + (VT)1.0 * oo2e * (v27_2_0 - rho_e * v27_2_1);
            const VT v28_18_0 = QCz * v28_8_0 + WQz * v28_8_1 + (VT)2.0 * oo2ze * v15_8_1 + (VT)1.0 * oo2e * (v28_2_0 - rho_e * v28_2_1);
            const VT v29_18_0 = QCz * v29_8_0 + WQz * v29_8_1 + (VT)3.0 * oo2ze * v14_8_1 + (VT)1.0 * oo2e * (v29_2_0 - rho_e * v29_2_1);
            const VT v30_18_0 = QCz * v30_8_0 + WQz * v30_8_1 + (VT)1.0 * oo2e * (v30_2_0 - rho_e * v30_2_1);
            const VT v31_18_0 = QCz * v31_8_0 + WQz * v31_8_1 + (VT)1.0 * oo2ze * v16_8_1 + (VT)1.0 * oo2e * (v31_2_0 - rho_e * v31_2_1);
            const VT v32_18_0 = QCz * v32_8_0 + WQz * v32_8_1 + (VT)2.0 * oo2ze * v17_8_1 + (VT)1.0 * oo2e * (v32_2_0 - rho_e * v32_2_1);
            const VT v33_18_0 = QCz * v33_8_0 + WQz * v33_8_1 + (VT)3.0 * oo2ze * v18_8_1 + (VT)1.0 * oo2e * (v33_2_0 - rho_e * v33_2_1);
            const VT v34_18_0 = QCz * v34_8_0 + WQz * v34_8_1 + (VT)4.0 * oo2ze * v19_8_1 + (VT)1.0 * oo2e * (v34_2_0 - rho_e * v34_2_1);
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
            const VT v20_19_0 = QCz * v20_9_0 + WQz * v20_9_1 + (VT)2.0 * oo2e * (v20_3_0 - rho_e * v20_3_1);
            const VT v21_19_0 = QCz * v21_9_0 + WQz * v21_9_1 + (VT)2.0 * oo2e * (v21_3_0 - rho_e * v21_3_1);
            const VT v22_19_0 = QCz * v22_9_0 + WQz * v22_9_1 + (VT)1.0 * oo2ze * v10_9_1 + (VT)2.0 * oo2e * (v22_3_0 - rho_e * v22_3_1);
            const VT v23_19_0 = QCz * v23_9_0 + WQz * v23_9_1 + (VT)2.0 * oo2e * (v23_3_0 - rho_e * v23_3_1);
            const VT v24_19_0 = QCz * v24_9_0 + WQz * v24_9_1 + (VT)1.0 * oo2ze * v11_9_1 + (VT)2.0 * oo2e * (v24_3_0 - rho_e * v24_3_1);
            const VT v25_19_0 = QCz * v25_9_0 + WQz * v25_9_1 + (VT)2.0 * oo2ze * v12_9_1 + (VT)2.0 * oo2e * (v25_3_0 - rho_e * v25_3_1);
            const VT v26_19_0 = QCz * v26_9_0 + WQz * v26_9_1 + (VT)2.0 * oo2e * (v26_3_0 - rho_e * v26_3_1);
            const VT v27_19_0 = QCz * v27_9_0 + WQz * v27_9_1 + (VT)1.0 * oo2ze * v13_9_1 + (VT)2.0 * oo2e * (v27_3_0 - rho_e * v27_3_1);
            const VT v28_19_0 = QCz * v28_9_0 + WQz * v28_9_1 + (VT)2.0 * oo2ze * v15_9_1 + (VT)2.0 * oo2e * (v28_3_0 - rho_e * v28_3_1);
            const VT v29_19_0 = QCz * v29_9_0 + WQz * v29_9_1 + (VT)3.0 * oo2ze * v14_9_1 + (VT)2.0 * oo2e * (v29_3_0 - rho_e * v29_3_1);
            const VT v30_19_0 = QCz * v30_9_0 + WQz * v30_9_1 + (VT)2.0 * oo2e * (v30_3_0 - rho_e * v30_3_1);
            const VT v31_19_0 = QCz * v31_9_0 + WQz * v31_9_1 + (VT)1.0 * oo2ze * v16_9_1 + (VT)2.0 * oo2e * (v31_3_0 - rho_e * v31_3_1);
            const VT v32_19_0 = QCz * v32_9_0 + WQz * v32_9_1 + (VT)2.0 * oo2ze * v17_9_1 + (VT)2.0 * oo2e * (v32_3_0 - rho_e * v32_3_1);
            const VT v33_19_0 = QCz * v33_9_0 + WQz * v33_9_1 + (VT)3.0 * oo2ze * v18_9_1 + (VT)2.0 * oo2e * (v33_3_0 - rho_e * v33_3_1);
            const VT v34_19_0 = QCz * v34_9_0 + WQz * v34_9_1 + (VT)4.0 * oo2ze * v19_9_1 + (VT)2.0 * oo2e * (v34_3_0 - rho_e * v34_3_1);
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
            acc[256] += (double)v20_4_0;
            acc[257] += (double)v20_5_0;
            acc[258] += (double)v20_6_0;
            acc[259] += (double)v20_7_0;
            acc[260] += (double)v20_8_0;
            acc[261] += (double)v20_9_0;
            acc[262] += (double)v20_10_0;
            acc[263] += (double)v20_11_0;
            acc[264] += (double)v20_12_0;
            acc[265] += (double)v20_13_0;
            acc[266] += (double)v20_14_0;
            acc[267] += (double)v20_15_0;
            acc[268] += (double)v20_16_0;
            acc[269] += (double)v20_17_0;
            acc[270] += (double)v20_18_0;
            acc[271] += (double)v20_19_0;
            acc[272] += (double)v21_4_0;
            acc[273] += (double)v21_5_0;
            acc[274] += (double)v21_6_0;
            acc[275] += (double)v21_7_0;
            acc[276] += (double)v21_8_0;
            acc[277] += (double)v21_9_0;
            acc[278] += (double)v21_10_0;
            acc[279] += (double)v21_11_0;
            acc[280] += (double)v21_12_0;
            acc[281] += (double)v21_13_0;
            acc[282] += (double)v21_14_0;
            acc[283] += (double)v21_15_0;
            acc[284] += (double)v21_16_0;
            acc[285] += (double)v21_17_0;
            acc[286] += (double)v21_18_0;
            acc[287] += (double)v21_19_0;
            acc[288] += (double)v22_4_0;
            acc[289] += (double)v22_5_0;
            acc[290] += (double)v22_6_0;
            acc[291] += (double)v22_7_0;
            acc[292] += (double)v22_8_0;
            acc[293] += (double)v22_9_0;
            acc[294] += (double)v22_10_0;
            acc[295] += (double)v22_11_0;
            acc[296] += (double)v22_12_0;
            acc[297] += (double)v22_13_0;
            acc[298] += (double)v22_14_0;
            acc[299] += (double)v22_15_0;
            acc[300] += (double)v22_16_0;
            acc[301] += (double)v22_17_0;
            acc[302] += (double)v22_18_0;
            acc[303] += (double)v22_19_0;
            acc[304] += (double)v23_4_0;
            acc[305] += (double)v23_5_0;
            acc[306] += (double)v23_6_0;
            acc[307] += (double)v23_7_0;
            acc[308] += (double)v23_8_0;
            acc[309] += (double)v23_9_0;
            acc[310] += (double)v23_10_0;
            acc[311] += (double)v23_11_0;
            acc[312] += (double)v23_12_0;
            acc[313] += (double)v23_13_0;
            acc[314] += (double)v23_14_0;
            acc[315] += (double)v23_15_0;
            acc[316] += (double)v23_16_0;
            acc[317] += (double)v23_17_0;
            acc[318] += (double)v23_18_0;
            acc[319] += (double)v23_19_0;
            acc[320] += (double)v24_4_0;
            acc[321] += (double)v24_5_0;
            acc[322] += (double)v24_6_0;
            acc[323] += (double)v24_7_0;
            acc[324] += (double)v24_8_0;
            acc[325] += (double)v24_9_0;
            acc[326] += (double)v24_10_0;
            acc[327] += (double)v24_11_0;
            acc[328] += (double)v24_12_0;
            acc[329] += (double)v24_13_0;
            acc[330] += (double)v24_14_0;
            acc[331] += (double)v24_15_0;
            acc[332] += (double)v24_16_0;
            acc[333] += (double)v24_17_0;
            acc[334] += (double)v24_18_0;
            acc[335] += (double)v24_19_0;
            acc[336] += (double)v25_4_0;
            acc[337] += (double)v25_5_0;
            acc[338] += (double)v25_6_0;
            acc[339] += (double)v25_7_0;
            acc[340] += (double)v25_8_0;
            acc[341] += (double)v25_9_0;
            acc[342] += (double)v25_10_0;
            acc[343] += (double)v25_11_0;
            acc[344] += (double)v25_12_0;
            acc[345] += (double)v25_13_0;
            acc[346] += (double)v25_14_0;
            acc[347] += (double)v25_15_0;
            acc[348] += (double)v25_16_0;
            acc[349] += (double)v25_17_0;
            acc[350] += (double)v25_18_0;
            acc[351] += (double)v25_19_0;
            acc[352] += (double)v26_4_0;
            acc[353] += (double)v26_5_0;
            acc[354] += (double)v26_6_0;
            acc[355] += (double)v26_7_0;
            acc[356] += (double)v26_8_0;
            acc[357] += (double)v26_9_0;
            acc[358] += (double)v26_10_0;
            acc[359] += (double)v26_11_0;
            acc[360] += (double)v26_12_0;
            acc[361] += (double)v26_13_0;
            acc[362] += (double)v26_14_0;
            acc[363] += (double)v26_15_0;
            acc[364] += (double)v26_16_0;
            acc[365] += (double)v26_17_0;
            acc[366] += (double)v26_18_0;
            acc[367] += (double)v26_19_0;
            acc[368] += (double)v27_4_0;
            acc[369] += (double)v27_5_0;
            acc[370] += (double)v27_6_0;
            acc[371] += (double)v27_7_0;
            acc[372] += (double)v27_8_0;
            acc[373] += (double)v27_9_0;
            acc[374] += (double)v27_10_0;
            acc[375] += (double)v27_11_0;
            acc[376] += (double)v27_12_0;
            acc[377] += (double)v27_13_0;
            acc[378] += (double)v27_14_0;
            acc[379] += (double)v27_15_0;
            acc[380] += (double)v27_16_0;
            acc[381] += (double)v27_17_0;
            acc[382] += (double)v27_18_0;
            acc[383] += (double)v27_19_0;
            acc[384] += (double)v28_4_0;
            acc[385] += (double)v28_5_0;
            acc[386] += (double)v28_6_0;
            acc[387] += (double)v28_7_0;
            acc[388] += (double)v28_8_0;
            acc[389] += (double)v28_9_0;
            acc[390] += (double)v28_10_0;
            acc[391] += (double)v28_11_0;
            acc[392] += (double)v28_12_0;
            acc[393] += (double)v28_13_0;
            acc[394] += (double)v28_14_0;
            acc[395] += (double)v28_15_0;
            acc[396] += (double)v28_16_0;
            acc[397] += (double)v28_17_0;
            acc[398] += (double)v28_18_0;
            acc[399] += (double)v28_19_0;
            acc[400] += (double)v29_4_0;
            acc[401] += (double)v29_5_0;
            acc[402] += (double)v29_6_0;
            acc[403] += (double)v29_7_0;
            acc[404] += (double)v29_8_0;
            acc[405] += (double)v29_9_0;
            acc[406] += (double)v29_10_0;
            acc[407] += (double)v29_11_0;
            acc[408] += (double)v29_12_0;
            acc[409] += (double)v29_13_0;
            acc[410] += (double)v29_14_0;
            acc[411] += (double)v29_15_0;
            acc[412] += (double)v29_16_0;
            acc[413] += (double)v29_17_0;
            acc[414] += (double)v29_18_0;
            acc[415] += (double)v29_19_0;
            acc[416] += (double)v30_4_0;
            acc[417] += (double)v30_5_0;
            acc[418] += (double)v30_6_0;
            acc[419] += (double)v30_7_0;
            acc[420] += (double)v30_8_0;
            acc[421] += (double)v30_9_0;
            acc[422] += (double)v30_10_0;
            acc[423] += (double)v30_11_0;
            acc[424] += (double)v30_12_0;
            acc[425] += (double)v30_13_0;
            acc[426] += (double)v30_14_0;
            acc[427] += (double)v30_15_0;
            acc[428] += (double)v30_16_0;
            acc[429] += (double)v30_17_0;
            acc[430] += (double)v30_18_0;
            acc[431] += (double)v30_19_0;
            acc[432] += (double)v31_4_0;
            acc[433] += (double)v31_5_0;
            acc[434] += (double)v31_6_0;
            acc[435] += (double)v31_7_0;
            acc[436] += (double)v31_8_0;
            acc[437] += (double)v31_9_0;
            acc[438] += (double)v31_10_0;
            acc[439] += (double)v31_11_0;
            acc[440] += (double)v31_12_0;
            acc[441] += (double)v31_13_0;
            acc[442] += (double)v31_14_0;
            acc[443] += (double)v31_15_0;
            acc[444] += (double)v31_16_0;
            acc[445] += (double)v31_17_0;
            acc[446] += (double)v31_18_0;
            acc[447] += (double)v31_19_0;
            acc[448] += (double)v32_4_0;
            acc[449] += (double)v32_5_0;
            acc[450] += (double)v32_6_0;
            acc[451] += (double)v32_7_0;
            acc[452] += (double)v32_8_0;
            acc[453] += (double)v32_9_0;
            acc[454] += (double)v32_10_0;
            acc[455] += (double)v32_11_0;
            acc[456] += (double)v32_12_0;
            acc[457] += (double)v32_13_0;
            acc[458] += (double)v32_14_0;
            acc[459] += (double)v32_15_0;
            acc[460] += (double)v32_16_0;
            acc[461] += (double)v32_17_0;
            acc[462] += (double)v32_18_0;
            acc[463] += (double)v32_19_0;
            acc[464] += (double)v33_4_0;
            acc[465] += (double)v33_5_0;
            acc[466] += (double)v33_6_0;
            acc[467] += (double)v33_7_0;
            acc[468] += (double)v33_8_0;
            acc[469] += (double)v33_9_0;
            acc[470] += (double)v33_10_0;
            acc[471] += (double)v33_11_0;
            acc[472] += (double)v33_12_0;
            acc[473] += (double)v33_13_0;
            acc[474] += (double)v33_14_0;
            acc[475] += (double)v33_15_0;
            acc[476] += (double)v33_16_0;
            acc[477] += (double)v33_17_0;
            acc[478] += (double)v33_18_0;
            acc[479] += (double)v33_19_0;
            acc[480] += (double)v34_4_0;
            acc[481] += (double)v34_5_0;
            acc[482] += (double)v34_6_0;
            acc[483] += (double)v34_7_0;
            acc[484] += (double)v34_8_0;
            acc[485] += (double)v34_9_0;
            acc[486] += (double)v34_10_0;
            acc[487] += (double)v34_11_0;
            acc[488] += (double)v34_12_0;
            acc[489] += (double)v34_13_0;
            acc[490] += (double)v34_14_0;
            acc[491] += (double)v34_15_0;
            acc[492] += (double)v34_16_0;
            acc[493] += (double)v34_17_0;
            acc[494] += (double)v34_18_0;
            acc[495] += (double)v34_19_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[648] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_dddp(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h10_1_10 = acc[262] + ABx * acc[102];
    const double h4_1_10 = acc[102] + ABx * acc[6];
    const double h4_4_10 = h10_1_10 + ABx * h4_1_10;
    const double h10_1_4 = acc[256] + ABx * acc[96];
    const double h4_1_4 = acc[96] + ABx * acc[0];
    const double h4_4_4 = h10_1_4 + ABx * h4_1_4;
    const double k4_4_4_1 = h4_4_10 + CDx * h4_4_4;
    const double h10_1_11 = acc[263] + ABx * acc[103];
    const double h4_1_11 = acc[103] + ABx * acc[7];
    const double h4_4_11 = h10_1_11 + ABx * h4_1_11;
    const double k4_4_4_2 = h4_4_11 + CDy * h4_4_4;
    const double h10_1_12 = acc[264] + ABx * acc[104];
    const double h4_1_12 = acc[104] + ABx * acc[8];
    const double h4_4_12 = h10_1_12 + ABx * h4_1_12;
    const double k4_4_4_3 = h4_4_12 + CDz * h4_4_4;
    const double h10_1_5 = acc[257] + ABx * acc[97];
    const double h4_1_5 = acc[97] + ABx * acc[1];
    const double h4_4_5 = h10_1_5 + ABx * h4_1_5;
    const double k4_4_5_1 = h4_4_11 + CDx * h4_4_5;
    const double h10_1_13 = acc[265] + ABx * acc[105];
    const double h4_1_13 = acc[105] + ABx * acc[9];
    const double h4_4_13 = h10_1_13 + ABx * h4_1_13;
    const double k4_4_5_2 = h4_4_13 + CDy * h4_4_5;
    const double h10_1_15 = acc[267] + ABx * acc[107];
    const double h4_1_15 = acc[107] + ABx * acc[11];
    const double h4_4_15 = h10_1_15 + ABx * h4_1_15;
    const double k4_4_5_3 = h4_4_15 + CDz * h4_4_5;
    const double h10_1_6 = acc[258] + ABx * acc[98];
    const double h4_1_6 = acc[98] + ABx * acc[2];
    const double h4_4_6 = h10_1_6 + ABx * h4_1_6;
    const double k4_4_6_1 = h4_4_12 + CDx * h4_4_6;
    const double k4_4_6_2 = h4_4_15 + CDy * h4_4_6;
    const double h10_1_14 = acc[266] + ABx * acc[106];
    const double h4_1_14 = acc[106] + ABx * acc[10];
    const double h4_4_14 = h10_1_14 + ABx * h4_1_14;
    const double k4_4_6_3 = h4_4_14 + CDz * h4_4_6;
    const double h10_1_7 = acc[259] + ABx * acc[99];
    const double h4_1_7 = acc[99] + ABx * acc[3];
    const double h4_4_7 = h10_1_7 + ABx * h4_1_7;
    const double k4_4_7_1 = h4_4_13 + CDx * h4_4_7;
    const double h10_1_16 = acc[268] + ABx * acc[108];
    const double h4_1_16 = acc[108] + ABx * acc[12];
    const double h4_4_16 = h10_1_16 + ABx * h4_1_16;
    const double k4_4_7_2 = h4_4_16 + CDy * h4_4_7;
    const double h10_1_17 = acc[269] + ABx * acc[109];
    const double h4_1_17 = acc[109] + ABx * acc[13];
    const double h4_4_17 = h10_1_17 + ABx * h4_1_17;
    const double k4_4_7_3 = h4_4_17 + CDz * h4_4_7;
    const double h10_1_8 = acc[260] + ABx * acc[100];
    const double h4_1_8 = acc[100] + ABx * acc[4];
    const double h4_4_8 = h10_1_8 + ABx * h4_1_8;
    const double k4_4_8_1 = h4_4_15 + CDx * h4_4_8;
    const double k4_4_8_2 = h4_4_17 + CDy * h4_4_8;
    const double h10_1_18 = acc[270] + ABx * acc[110];
    const double h4_1_18 = acc[110] + ABx * acc[14];
    const double h4_4_18 = h10_1_18 + ABx * h4_1_18;
    const double k4_4_8_3 = h4_4_18 + CDz * h4_4_8;
    const double h10_1_9 = acc[261] + ABx * acc[101];
    const double h4_1_9 = acc[101] + ABx * acc[5];
    const double h4_4_9 = h10_1_9 + ABx * h4_1_9;
    const double k4_4_9_1 = h4_4_14 + CDx * h4_4_9;
    const double k4_4_9_2 = h4_4_18 + CDy * h4_4_9;
    const double h10_1_19 = acc[271] + ABx * acc[111];
    const double h4_1_19 = acc[111] + ABx * acc[15];
    const double h4_4_19 = h10_1_19 + ABx * h4_1_19;
    const double k4_4_9_3 = h4_4_19 + CDz * h4_4_9;
    const double h10_2_10 = acc[278] + ABy * acc[102];
    const double h4_2_10 = acc[118] + ABy * acc[6];
    const double h4_5_10 = h10_2_10 + ABx * h4_2_10;
    const double h10_2_4 = acc[272] + ABy * acc[96];
    const double h4_2_4 = acc[112] + ABy * acc[0];
    const double h4_5_4 = h10_2_4 + ABx * h4_2_4;
    const double k4_5_4_1 = h4_5_10 + CDx * h4_5_4;
    const double h10_2_11 = acc[279] + ABy * acc[103];
    const double h4_2_11 = acc[119] + ABy * acc[7];
    const double h4_5_11 = h10_2_11 + ABx * h4_2_11;
    const double k4_5_4_2 = h4_5_11 + CDy * h4_5_4;
    const double h10_2_12 = acc[280] + ABy * acc[104];
    const double h4_2_12 = acc[120] + ABy * acc[8];
    const double h4_5_12 = h10_2_12 + ABx * h4_2_12;
    const double k4_5_4_3 = h4_5_12 + CDz * h4_5_4;
    const double h10_2_5 = acc[273] + ABy * acc[97];
    const double h4_2_5 = acc[113] + ABy * acc[1];
    const double h4_5_5 = h10_2_5 + ABx * h4_2_5;
    const double k4_5_5_1 = h4_5_11 + CDx * h4_5_5;
    const double h10_2_13 = acc[281] + ABy * acc[105];
    const double h4_2_13 = acc[121] + ABy * acc[9];
    const double h4_5_13 = h10_2_13 + ABx * h4_2_13;
    const double k4_5_5_2 = h4_5_13 + CDy * h4_5_5;
    const double h10_2_15 = acc[283] + ABy * acc[107];
    const double h4_2_15 = acc[123] + ABy * acc[11];
    const double h4_5_15 = h10_2_15 + ABx * h4_2_15;
    const double k4_5_5_3 = h4_5_15 + CDz * h4_5_5;
    const double h10_2_6 = acc[274] + ABy * acc[98];
    const double h4_2_6 = acc[114] + ABy * acc[2];
    const double h4_5_6 = h10_2_6 + ABx * h4_2_6;
    const double k4_5_6_1 = h4_5_12 + CDx * h4_5_6;
    const double k4_5_6_2 = h4_5_15 + CDy * h4_5_6;
    const double h10_2_14 = acc[282] + ABy * acc[106];
    const double h4_2_14 = acc[122] + ABy * acc[10];
    const double h4_5_14 = h10_2_14 + ABx * h4_2_14;
    const double k4_5_6_3 = h4_5_14 + CDz * h4_5_6;
    const double h10_2_7 = acc[275] + ABy * acc[99];
    const double h4_2_7 = acc[115] + ABy * acc[3];
    const double h4_5_7 = h10_2_7 + ABx * h4_2_7;
    const double k4_5_7_1 = h4_5_13 + CDx * h4_5_7;
    const double h10_2_16 = acc[284] + ABy * acc[108];
    const double h4_2_16 = acc[124] + ABy * acc[12];
    const double h4_5_16 = h10_2_16 + ABx * h4_2_16;
    const double k4_5_7_2 = h4_5_16 + CDy * h4_5_7;
    const double h10_2_17 = acc[285] + ABy * acc[109];
    const double h4_2_17 = acc[125] + ABy * acc[13];
    const double h4_5_17 = h10_2_17 + ABx * h4_2_17;
    const double k4_5_7_3 = h4_5_17 + CDz * h4_5_7;
    const double h10_2_8 = acc[276] + ABy * acc[100];
    const double h4_2_8 = acc[116] + ABy * acc[4];
    const double h4_5_8 = h10_2_8 + ABx * h4_2_8;
    const double k4_5_8_1 = h4_5_15 + CDx * h4_5_8;
    const double k4_5_8_2 = h4_5_17 + CDy * h4_5_8;
    const double h10_2_18 = acc[286] + ABy * acc[110];
    const double h4_2_18 = acc[126] + ABy * acc[14];
    const double h4_5_18 = h10_2_18 + ABx * h4_2_18;
    const double k4_5_8_3 = h4_5_18 + CDz * h4_5_8;
    const double h10_2_9 = acc[277] + ABy * acc[101];
    const double h4_2_9 = acc[117] + ABy * acc[5];
    const double h4_5_9 = h10_2_9 + ABx * h4_2_9;
    const double k4_5_9_1 = h4_5_14 + CDx * h4_5_9;
    const double k4_5_9_2 = h4_5_18 + CDy * h4_5_9;
    const double h10_2_19 = acc[287] + ABy * acc[111];
    const double h4_2_19 = acc[127] + ABy * acc[15];
    const double h4_5_19 = h10_2_19 + ABx * h4_2_19;
    const double k4_5_9_3 = h4_5_19 + CDz * h4_5_9;
    const double h10_3_10 = acc[294] + ABz * acc[102];
    const double h4_3_10 = acc[134] + ABz * acc[6];
    const double h4_6_10 = h10_3_10 + ABx * h4_3_10;
    const double h10_3_4 = acc[288] + ABz * acc[96];
    const double h4_3_4 = acc[128] + ABz * acc[0];
    const double h4_6_4 = h10_3_4 + ABx * h4_3_4;
    const double k4_6_4_1 = h4_6_10 + CDx * h4_6_4;
    const double h10_3_11 = acc[295] + ABz * acc[103];
    const double h4_3_11 = acc[135] + ABz * acc[7];
    const double h4_6_11 = h10_3_11 + ABx * h4_3_11;
    const double k4_6_4_2 = h4_6_11 + CDy * h4_6_4;
    const double h10_3_12 = acc[296] + ABz * acc[104];
    const double h4_3_12 = acc[136] + ABz * acc[8];
    const double h4_6_12 = h10_3_12 + ABx * h4_3_12;
    const double k4_6_4_3 = h4_6_12 + CDz * h4_6_4;
    const double h10_3_5 = acc[289] + ABz * acc[97];
    const double h4_3_5 = acc[129] + ABz * acc[1];
    const double h4_6_5 = h10_3_5 + ABx * h4_3_5;
    const double k4_6_5_1 = h4_6_11 + CDx * h4_6_5;
    const double h10_3_13 = acc[297] + ABz * acc[105];
    const double h4_3_13 = acc[137] + ABz * acc[9];
    const double h4_6_13 = h10_3_13 + ABx * h4_3_13;
    const double k4_6_5_2 = h4_6_13 + CDy * h4_6_5;
    const double h10_3_15 = acc[299] + ABz * acc[107];
    const double h4_3_15 = acc[139] + ABz * acc[11];
    const double h4_6_15 = h10_3_15 + ABx * h4_3_15;
    const double k4_6_5_3 = h4_6_15 + CDz * h4_6_5;
    const double h10_3_6 = acc[290] + ABz * acc[98];
    const double h4_3_6 = acc[130] + ABz * acc[2];
    const double h4_6_6 = h10_3_6 + ABx * h4_3_6;
    const double k4_6_6_1 = h4_6_12 + CDx * h4_6_6;
    const double k4_6_6_2 = h4_6_15 + CDy * h4_6_6;
    const double h10_3_14 = acc[298] + ABz * acc[106];
    const double h4_3_14 = acc[138] + ABz * acc[10];
    const double h4_6_14 = h10_3_14 + ABx * h4_3_14;
    const double k4_6_6_3 = h4_6_14 + CDz * h4_6_6;
    const double h10_3_7 = acc[291] + ABz * acc[99];
    const double h4_3_7 = acc[131] + ABz * acc[3];
    const double h4_6_7 = h10_3_7 + ABx * h4_3_7;
    const double k4_6_7_1 = h4_6_13 + CDx * h4_6_7;
    const double h10_3_16 = acc[300] + ABz * acc[108];
    const double h4_3_16 = acc[140] + ABz * acc[12];
    const double h4_6_16 = h10_3_16 + ABx * h4_3_16;
    const double k4_6_7_2 = h4_6_16 + CDy * h4_6_7;
    const double h10_3_17 = acc[301] + ABz * acc[109];
    const double h4_3_17 = acc[141] + ABz * acc[13];
    const double h4_6_17 = h10_3_17 + ABx * h4_3_17;
    const double k4_6_7_3 = h4_6_17 + CDz * h4_6_7;
    const double h10_3_8 = acc[292] + ABz * acc[100];
    const double h4_3_8 = acc[132] + ABz * acc[4];
    const double h4_6_8 = h10_3_8 + ABx * h4_3_8;
    const double k4_6_8_1 = h4_6_15 + CDx * h4_6_8;
    const double k4_6_8_2 = h4_6_17 + CDy * h4_6_8;
    const double h10_3_18 = acc[302] + ABz * acc[110];
    const double h4_3_18 = acc[142] + ABz * acc[14];
    const double h4_6_18 = h10_3_18 + ABx * h4_3_18;
    const double k4_6_8_3 = h4_6_18 + CDz * h4_6_8;
    const double h10_3_9 = acc[293] + ABz * acc[101];
    const double h4_3_9 = acc[133] + ABz * acc[5];
    const double h4_6_9 = h10_3_9 + ABx * h4_3_9;
    const double k4_6_9_1 = h4_6_14 + CDx * h4_6_9;
    const double k4_6_9_2 = h4_6_18 + CDy * h4_6_9;
    const double h10_3_19 = acc[303] + ABz * acc[111];
    const double h4_3_19 = acc[143] + ABz * acc[15];
    const double h4_6_19 = h10_3_19 + ABx * h4_3_19;
    const double k4_6_9_3 = h4_6_19 + CDz * h4_6_9;
    const double h11_2_10 = acc[310] + ABy * acc[118];
    const double h4_7_10 = h11_2_10 + ABy * h4_2_10;
    const double h11_2_4 = acc[304] + ABy * acc[112];
    const double h4_7_4 = h11_2_4 + ABy * h4_2_4;
    const double k4_7_4_1 = h4_7_10 + CDx * h4_7_4;
    const double h11_2_11 = acc[311] + ABy * acc[119];
    const double h4_7_11 = h11_2_11 + ABy * h4_2_11;
    const double k4_7_4_2 = h4_7_11 + CDy * h4_7_4;
    const double h11_2_12 = acc[312] + ABy * acc[120];
    const double h4_7_12 = h11_2_12 + ABy * h4_2_12;
    const double k4_7_4_3 = h4_7_12 + CDz * h4_7_4;
    const double h11_2_5 = acc[305] + ABy * acc[113];
    const double h4_7_5 = h11_2_5 + ABy * h4_2_5;
    const double k4_7_5_1 = h4_7_11 + CDx * h4_7_5;
    const double h11_2_13 = acc[313] + ABy * acc[121];
    const double h4_7_13 = h11_2_13 + ABy * h4_2_13;
    const double k4_7_5_2 = h4_7_13 + CDy * h4_7_5;
    const double h11_2_15 = acc[315] + ABy * acc[123];
    const double h4_7_15 = h11_2_15 + ABy * h4_2_15;
    const double k4_7_5_3 = h4_7_15 + CDz * h4_7_5;
    const double h11_2_6 = acc[306] + ABy * acc[114];
    const double h4_7_6 = h11_2_6 + ABy * h4_2_6;
    const double k4_7_6_1 = h4_7_12 + CDx * h4_7_6;
    const double k4_7_6_2 = h4_7_15 + CDy * h4_7_6;
    const double h11_2_14 = acc[314] + ABy * acc[122];
    const double h4_7_14 = h11_2_14 + ABy * h4_2_14;
    const double k4_7_6_3 = h4_7_14 + CDz * h4_7_6;
    const double h11_2_7 = acc[307] + ABy * acc[115];
    const double h4_7_7 = h11_2_7 + ABy * h4_2_7;
    const double k4_7_7_1 = h4_7_13 + CDx * h4_7_7;
    const double h11_2_16 = acc[316] + ABy * acc[124];
    const double h4_7_16 = h11_2_16 + ABy * h4_2_16;
    const double k4_7_7_2 = h4_7_16 + CDy * h4_7_7;
    const double h11_2_17 = acc[317] + ABy * acc[125];
    const double h4_7_17 = h11_2_17 + ABy * h4_2_17;
    const double k4_7_7_3 = h4_7_17 + CDz * h4_7_7;
    const double h11_2_8 = acc[308] + ABy * acc[116];
    const double h4_7_8 = h11_2_8 + ABy * h4_2_8;
    const double k4_7_8_1 = h4_7_15 + CDx * h4_7_8;
    const double k4_7_8_2 = h4_7_17 + CDy * h4_7_8;
    const double h11_2_18 = acc[318] + ABy * acc[126];
    const double h4_7_18 = h11_2_18 + ABy * h4_2_18;
    const double k4_7_8_3 = h4_7_18 + CDz * h4_7_8;
    const double h11_2_9 = acc[309] + ABy * acc[117];
    const double h4_7_9 = h11_2_9 + ABy * h4_2_9;
    const double k4_7_9_1 = h4_7_14 + CDx * h4_7_9;
    const double k4_7_9_2 = h4_7_18 + CDy * h4_7_9;
    const double h11_2_19 = acc[319] + ABy * acc[127];
    const double h4_7_19 = h11_2_19 + ABy * h4_2_19;
    const double k4_7_9_3 = h4_7_19 + CDz * h4_7_9;
    const double h11_3_10 = acc[326] + ABz * acc[118];
    const double h4_8_10 = h11_3_10 + ABy * h4_3_10;
    const double h11_3_4 = acc[320] + ABz * acc[112];
    const double h4_8_4 = h11_3_4 + ABy * h4_3_4;
    const double k4_8_4_1 = h4_8_10 + CDx * h4_8_4;
    const double h11_3_11 = acc[327] + ABz * acc[119];
    const double h4_8_11 = h11_3_11 + ABy * h4_3_11;
    const double k4_8_4_2 = h4_8_11 + CDy * h4_8_4;
    const double h11_3_12 = acc[328] + ABz * acc[120];
    const double h4_8_12 = h11_3_12 + ABy * h4_3_12;
    const double k4_8_4_3 = h4_8_12 + CDz * h4_8_4;
    const double h11_3_5 = acc[321] + ABz * acc[113];
    const double h4_8_5 = h11_3_5 + ABy * h4_3_5;
    const double k4_8_5_1 = h4_8_11 + CDx * h4_8_5;
    const double h11_3_13 = acc[329] + ABz * acc[121];
    const double h4_8_13 = h11_3_13 + ABy * h4_3_13;
    const double k4_8_5_2 = h4_8_13 + CDy * h4_8_5;
    const double h11_3_15 = acc[331] + ABz * acc[123];
    const double h4_8_15 = h11_3_15 + ABy * h4_3_15;
    const double k4_8_5_3 = h4_8_15 + CDz * h4_8_5;
    const double h11_3_6 = acc[322] + ABz * acc[114];
    const double h4_8_6 = h11_3_6 + ABy * h4_3_6;
    const double k4_8_6_1 = h4_8_12 + CDx * h4_8_6;
    const double k4_8_6_2 = h4_8_15 + CDy * h4_8_6;
    const double h11_3_14 = acc[330] + ABz * acc[122];
    const double h4_8_14 = h11_3_14 + ABy * h4_3_14;
    const double k4_8_6_3 = h4_8_14 + CDz * h4_8_6;
    const double h11_3_7 = acc[323] + ABz * acc[115];
    const double h4_8_7 = h11_3_7 + ABy * h4_3_7;
    const double k4_8_7_1 = h4_8_13 + CDx * h4_8_7;
    const double h11_3_16 = acc[332] + ABz * acc[124];
    const double h4_8_16 = h11_3_16 + ABy * h4_3_16;
    const double k4_8_7_2 = h4_8_16 + CDy * h4_8_7;
    const double h11_3_17 = acc[333] + ABz * acc[125];
    const double h4_8_17 = h11_3_17 + ABy * h4_3_17;
    const double k4_8_7_3 = h4_8_17 + CDz * h4_8_7;
    const double h11_3_8 = acc[324] + ABz * acc[116];
    const double h4_8_8 = h11_3_8 + ABy * h4_3_8;
    const double k4_8_8_1 = h4_8_15 + CDx * h4_8_8;
    const double k4_8_8_2 = h4_8_17 + CDy * h4_8_8;
    const double h11_3_18 = acc[334] + ABz * acc[126];
    const double h4_8_18 = h11_3_18 + ABy * h4_3_18;
    const double k4_8_8_3 = h4_8_18 + CDz * h4_8_8;
    const double h11_3_9 = acc[325] + ABz * acc[117];
    const double h4_8_9 = h11_3_9 + ABy * h4_3_9;
    const double k4_8_9_1 = h4_8_14 + CDx * h4_8_9;
    const double k4_8_9_2 = h4_8_18 + CDy * h4_8_9;
    const double h11_3_19 = acc[335] + ABz * acc[127];
    const double h4_8_19 = h11_3_19 + ABy * h4_3_19;
    const double k4_8_9_3 = h4_8_19 + CDz * h4_8_9;
    const double h12_3_10 = acc[342] + ABz * acc[134];
    const double h4_9_10 = h12_3_10 + ABz * h4_3_10;
    const double h12_3_4 = acc[336] + ABz * acc[128];
    const double h4_9_4 = h12_3_4 + ABz * h4_3_4;
    const double k4_9_4_1 = h4_9_10 + CDx * h4_9_4;
    const double h12_3_11 = acc[343] + ABz * acc[135];
    const double h4_9_11 = h12_3_11 + ABz * h4_3_11;
    const double k4_9_4_2 = h4_9_11 + CDy * h4_9_4;
    const double h12_3_12 = acc[344] + ABz * acc[136];
    const double h4_9_12 = h12_3_12 + ABz * h4_3_12;
    const double k4_9_4_3 = h4_9_12 + CDz * h4_9_4;
    const double h12_3_5 = acc[337] + ABz * acc[129];
    const double h4_9_5 = h12_3_5 + ABz * h4_3_5;
    const double k4_9_5_1 = h4_9_11 + CDx * h4_9_5;
    const double h12_3_13 = acc[345] + ABz * acc[137];
    const double h4_9_13 = h12_3_13 + ABz * h4_3_13;
    const double k4_9_5_2 = h4_9_13 + CDy * h4_9_5;
    const double h12_3_15 = acc[347] + ABz * acc[139];
    const double h4_9_15 = h12_3_15 + ABz * h4_3_15;
    const double k4_9_5_3 = h4_9_15 + CDz * h4_9_5;
    const double h12_3_6 = acc[338] + ABz * acc[130];
    const double h4_9_6 = h12_3_6 + ABz * h4_3_6;
    const double k4_9_6_1 = h4_9_12 + CDx * h4_9_6;
    const double k4_9_6_2 = h4_9_15 + CDy * h4_9_6;
    const double h12_3_14 = acc[346] + ABz * acc[138];
    const double h4_9_14 = h12_3_14 + ABz * h4_3_14;
    const double k4_9_6_3 = h4_9_14 + CDz * h4_9_6;
    const double h12_3_7 = acc[339] + ABz * acc[131];
    const double h4_9_7 = h12_3_7 + ABz * h4_3_7;
    const double k4_9_7_1 = h4_9_13 + CDx * h4_9_7;
    const double h12_3_16 = acc[348] + ABz * acc[140];
    const double h4_9_16 = h12_3_16 + ABz * h4_3_16;
    const double k4_9_7_2 = h4_9_16 + CDy * h4_9_7;
    const double h12_3_17 = acc[349] + ABz * acc[141];
    const double h4_9_17 = h12_3_17 + ABz * h4_3_17;
    const double k4_9_7_3 = h4_9_17 + CDz * h4_9_7;
    const double h12_3_8 = acc[340] + ABz * acc[132];
    const double h4_9_8 = h12_3_8 + ABz * h4_3_8;
    const double k4_9_8_1 = h4_9_15 + CDx * h4_9_8;
    const double k4_9_8_2 = h4_9_17 + CDy * h4_9_8;
    const double h12_3_18 = acc[350] + ABz * acc[142];
    const double h4_9_18 = h12_3_18 + ABz * h4_3_18;
    const double k4_9_8_3 = h4_9_18 + CDz * h4_9_8;
    const double h12_3_9 = acc[341] + ABz * acc[133];
    const double h4_9_9 = h12_3_9 + ABz * h4_3_9;
    const double k4_9_9_1 = h4_9_14 + CDx * h4_9_9;
    const double k4_9_9_2 = h4_9_18 + CDy * h4_9_9;
    const double h12_3_19 = acc[351] + ABz * acc[143];
    const double h4_9_19 = h12_3_19 + ABz * h4_3_19;
    const double k4_9_9_3 = h4_9_19 + CDz * h4_9_9;
    const double h11_1_10 = acc[278] + ABx * acc[118];
    const double h5_1_10 = acc[118] + ABx * acc[22];
    const double h5_4_10 = h11_1_10 + ABx * h5_1_10;
    const double h11_1_4 = acc[272] + ABx * acc[112];
    const double h5_1_4 = acc[112] + ABx * acc[16];
    const double h5_4_4 = h11_1_4 + ABx * h5_1_4;
    const double k5_4_4_1 = h5_4_10 + CDx * h5_4_4;
    const double h11_1_11 = acc[279] + ABx * acc[119];
    const double h5_1_11 = acc[119] + ABx * acc[23];
    const double h5_4_11 = h11_1_11 + ABx * h5_1_11;
    const double k5_4_4_2 = h5_4_11 + CDy * h5_4_4;
    const double h11_1_12 = acc[280] + ABx * acc[120];
    const double h5_1_12 = acc[120] + ABx * acc[24];
    const double h5_4_12 = h11_1_12 + ABx * h5_1_12;
    const double k5_4_4_3 = h5_4_12 + CDz * h5_4_4;
    const double h11_1_5 = acc[273] + ABx * acc[113];
    const double h5_1_5 = acc[113] + ABx * acc[17];
    const double h5_4_5 = h11_1_5 + ABx * h5_1_5;
    const double k5_4_5_1 = h5_4_11 + CDx * h5_4_5;
    const double h11_1_13 = acc[281] + ABx * acc[121];
    const double h5_1_13 = acc[121] + ABx * acc[25];
    const double h5_4_13 = h11_1_13 + ABx * h5_1_13;
    const double k5_4_5_2 = h5_4_13 + CDy * h5_4_5;
    const double h11_1_15 = acc[283] + ABx * acc[123];
    const double h5_1_15 = acc[123] + ABx * acc[27];
    const double h5_4_15 = h11_1_15 + ABx * h5_1_15;
    const double k5_4_5_3 = h5_4_15 + CDz * h5_4_5;
    const double h11_1_6 = acc[274] + ABx * acc[114];
    const double h5_1_6 = acc[114] + ABx * acc[18];
    const double h5_4_6 = h11_1_6 + ABx * h5_1_6;
    const double k5_4_6_1 = h5_4_12 + CDx * h5_4_6;
    const double k5_4_6_2 = h5_4_15 + CDy * h5_4_6;
    const double h11_1_14 = acc[282] + ABx * acc[122];
    const double h5_1_14 = acc[122] + ABx * acc[26];
    const double h5_4_14 = h11_1_14 + ABx * h5_1_14;
    const double k5_4_6_3 = h5_4_14 + CDz * h5_4_6;
    const double h11_1_7 = acc[275] + ABx * acc[115];
    const double h5_1_7 = acc[115] + ABx * acc[19];
    const double h5_4_7 = h11_1_7 + ABx * h5_1_7;
    const double k5_4_7_1 = h5_4_13 + CDx * h5_4_7;
    const double h11_1_16 = acc[284] + ABx * acc[124];
    const double h5_1_16 = acc[124] + ABx * acc[28];
    const double h5_4_16 = h11_1_16 + ABx * h5_1_16;
    const double k5_4_7_2 = h5_4_16 + CDy * h5_4_7;
    const double h11_1_17 = acc[285] + ABx * acc[125];
    const double h5_1_17 = acc[125] + ABx * acc[29];
    const double h5_4_17 = h11_1_17 + ABx * h5_1_17;
    const double k5_4_7_3 = h5_4_17 + CDz * h5_4_7;
    const double h11_1_8 = acc[276] + ABx * acc[116];
    const double h5_1_8 = acc[116] + ABx * acc[20];
    const double h5_4_8 = h11_1_8 + ABx * h5_1_8;
    const double k5_4_8_1 = h5_4_15 + CDx * h5_4_8;
    const double k5_4_8_2 = h5_4_17 + CDy * h5_4_8;
    const double h11_1_18 = acc[286] + ABx * acc[126];
    const double h5_1_18 = acc[126] + ABx * acc[30];
    const double h5_4_18 = h11_1_18 + ABx * h5_1_18;
    const double k5_4_8_3 = h5_4_18 + CDz * h5_4_8;
    const double h11_1_9 = acc[277] + ABx * acc[117];
    const double h5_1_9 = acc[117] + ABx * acc[21];
    const double h5_4_9 = h11_1_9 + ABx * h5_1_9;
    const double k5_4_9_1 = h5_4_14 + CDx * h5_4_9;
    const double k5_4_9_2 = h5_4_18 + CDy * h5_4_9;
    const double h11_1_19 = acc[287] + ABx * acc[127];
    const double h5_1_19 = acc[127] + ABx * acc[31];
    const double h5_4_19 = h11_1_19 + ABx * h5_1_19;
    const double k5_4_9_3 = h5_4_19 + CDz * h5_4_9;
    const double h5_2_10 = acc[150] + ABy * acc[22];
    const double h5_5_10 = h11_2_10 + ABx * h5_2_10;
    const double h5_2_4 = acc[144] + ABy * acc[16];
    const double h5_5_4 = h11_2_4 + ABx * h5_2_4;
    const double k5_5_4_1 = h5_5_10 + CDx * h5_5_4;
    const double h5_2_11 = acc[151] + ABy * acc[23];
    const double h5_5_11 = h11_2_11 + ABx * h5_2_11;
    const double k5_5_4_2 = h5_5_11 + CDy * h5_5_4;
    const double h5_2_12 = acc[152] + ABy * acc[24];
    const double h5_5_12 = h11_2_12 + ABx * h5_2_12;
    const double k5_5_4_3 = h5_5_12 + CDz * h5_5_4;
    const double h5_2_5 = acc[145] + ABy * acc[17];
    const double h5_5_5 = h11_2_5 + ABx * h5_2_5;
    const double k5_5_5_1 = h5_5_11 + CDx * h5_5_5;
    const double h5_2_13 = acc[153] + ABy * acc[25];
    const double h5_5_13 = h11_2_13 + ABx * h5_2_13;
    const double k5_5_5_2 = h5_5_13 + CDy * h5_5_5;
    const double h5_2_15 = acc[155] + ABy * acc[27];
    const double h5_5_15 = h11_2_15 + ABx * h5_2_15;
    const double k5_5_5_3 = h5_5_15 + CDz * h5_5_5;
    const double h5_2_6 = acc[146] + ABy * acc[18];
    const double h5_5_6 = h11_2_6 + ABx * h5_2_6;
    const double k5_5_6_1 = h5_5_12 + CDx * h5_5_6;
    const double k5_5_6_2 = h5_5_15 + CDy * h5_5_6;
    const double h5_2_14 = acc[154] + ABy * acc[26];
    const double h5_5_14 = h11_2_14 + ABx * h5_2_14;
    const double k5_5_6_3 = h5_5_14 + CDz * h5_5_6;
    const double h5_2_7 = acc[147] + ABy * acc[19];
    const double h5_5_7 = h11_2_7 + ABx * h5_2_7;
    const double k5_5_7_1 = h5_5_13 + CDx * h5_5_7;
    const double h5_2_16 = acc[156] + ABy * acc[28];
    const double h5_5_16 = h11_2_16 + ABx * h5_2_16;
    const double k5_5_7_2 = h5_5_16 + CDy * h5_5_7;
    const double h5_2_17 = acc[157] + ABy * acc[29];
    const double h5_5_17 = h11_2_17 + ABx * h5_2_17;
    const double k5_5_7_3 = h5_5_17 + CDz * h5_5_7;
    const double h5_2_8 = acc[148] + ABy * acc[20];
    const double h5_5_8 = h11_2_8 + ABx * h5_2_8;
    const double k5_5_8_1 = h5_5_15 + CDx * h5_5_8;
    const double k5_5_8_2 = h5_5_17 + CDy * h5_5_8;
    const double h5_2_18 = acc[158] + ABy * acc[30];
    const double h5_5_18 = h11_2_18 + ABx * h5_2_18;
    const double k5_5_8_3 = h5_5_18 + CDz * h5_5_8;
    const double h5_2_9 = acc[149] + ABy * acc[21];
    const double h5_5_9 = h11_2_9 + ABx * h5_2_9;
    const double k5_5_9_1 = h5_5_14 + CDx * h5_5_9;
    const double k5_5_9_2 = h5_5_18 + CDy * h5_5_9;
    const double h5_2_19 = acc[159] + ABy * acc[31];
    const double h5_5_19 = h11_2_19 + ABx * h5_2_19;
    const double k5_5_9_3 = h5_5_19 + CDz * h5_5_9;
    const double h5_3_10 = acc[182] + ABz * acc[22];
    const double h5_6_10 = h11_3_10 + ABx * h5_3_10;
    const double h5_3_4 = acc[176] + ABz * acc[16];
    const double h5_6_4 = h11_3_4 + ABx * h5_3_4;
    const double k5_6_4_1 = h5_6_10 + CDx * h5_6_4;
    const double h5_3_11 = acc[183] + ABz * acc[23];
    const double h5_6_11 = h11_3_11 + ABx * h5_3_11;
    const double k5_6_4_2 = h5_6_11 + CDy * h5_6_4;
    const double h5_3_12 = acc[184] + ABz * acc[24];
    const double h5_6_12 = h11_3_12 + ABx * h5_3_12;
    const double k5_6_4_3 = h5_6_12 + CDz * h5_6_4;
    const double h5_3_5 = acc[177] + ABz * acc[17];
    const double h5_6_5 = h11_3_5 + ABx * h5_3_5;
    const double k5_6_5_1 = h5_6_11 + CDx * h5_6_5;
    const double h5_3_13 = acc[185] + ABz * acc[25];
    const double h5_6_13 = h11_3_13 + ABx * h5_3_13;
    const double k5_6_5_2 = h5_6_13 + CDy * h5_6_5;
    const double h5_3_15 = acc[187] + ABz * acc[27];
    const double h5_6_15 = h11_3_15 + ABx * h5_3_15;
    const double k5_6_5_3 = h5_6_15 + CDz * h5_6_5;
    const double h5_3_6 = acc[178] + ABz * acc[18];
    const double h5_6_6 = h11_3_6 + ABx * h5_3_6;
    const double k5_6_6_1 = h5_6_12 + CDx * h5_6_6;
    const double k5_6_6_2 = h5_6_15 + CDy * h5_6_6;
    const double h5_3_14 = acc[186] + ABz * acc[26];
    const double h5_6_14 = h11_3_14 + ABx * h5_3_14;
    const double k5_6_6_3 = h5_6_14 + CDz * h5_6_6;
    const double h5_3_7 = acc[179] + ABz * acc[19];
    const double h5_6_7 = h11_3_7 + ABx * h5_3_7;
    const double k5_6_7_1 = h5_6_13 + CDx * h5_6_7;
    const double h5_3_16 = acc[188] + ABz * acc[28];
    const double h5_6_16 = h11_3_16 + ABx * h5_3_16;
    const double k5_6_7_2 = h5_6_16 + CDy * h5_6_7;
    const double h5_3_17 = acc[189] + ABz * acc[29];
    const double h5_6_17 = h11_3_17 + ABx * h5_3_17;
    const double k5_6_7_3 = h5_6_17 + CDz * h5_6_7;
    const double h5_3_8 = acc[180] + ABz * acc[20];
    const double h5_6_8 = h11_3_8 + ABx * h5_3_8;
    const double k5_6_8_1 = h5_6_15 + CDx * h5_6_8;
    const double k5_6_8_2 = h5_6_17 + CDy * h5_6_8;
    const double h5_3_18 = acc[190] + ABz * acc[30];
    const double h5_6_18 = h11_3_18 + ABx * h5_3_18;
    const double k5_6_8_3 = h5_6_18 + CDz * h5_6_8;
    const double h5_3_9 = acc[181] + ABz * acc[21];
    const double h5_6_9 = h11_3_9 + ABx * h5_3_9;
    const double k5_6_9_1 = h5_6_14 + CDx * h5_6_9;
    const double k5_6_9_2 = h5_6_18 + CDy * h5_6_9;
    const double h5_3_19 = acc[191] + ABz * acc[31];
    const double h5_6_19 = h11_3_19 + ABx * h5_3_19;
    const double k5_6_9_3 = h5_6_19 + CDz * h5_6_9;
    const double h13_2_10 = acc[358] + ABy * acc[150];
    const double h5_7_10 = h13_2_10 + ABy * h5_2_10;
    const double h13_2_4 = acc[352] + ABy * acc[144];
    const double h5_7_4 = h13_2_4 + ABy * h5_2_4;
    const double k5_7_4_1 = h5_7_10 + CDx * h5_7_4;
    const double h13_2_11 = acc[359] + ABy * acc[151];
    const double h5_7_11 = h13_2_11 + ABy * h5_2_11;
    const double k5_7_4_2 = h5_7_11 + CDy * h5_7_4;
    const double h13_2_12 = acc[360] + ABy * acc[152];
    const double h5_7_12 = h13_2_12 + ABy * h5_2_12;
    const double k5_7_4_3 = h5_7_12 + CDz * h5_7_4;
    const double h13_2_5 = acc[353] + ABy * acc[145];
    const double h5_7_5 = h13_2_5 + ABy * h5_2_5;
    const double k5_7_5_1 = h5_7_11 + CDx * h5_7_5;
    const double h13_2_13 = acc[361] + ABy * acc[153];
    const double h5_7_13 = h13_2_13 + ABy * h5_2_13;
    const double k5_7_5_2 = h5_7_13 + CDy * h5_7_5;
    const double h13_2_15 = acc[363] + ABy * acc[155];
    const double h5_7_15 = h13_2_15 + ABy * h5_2_15;
    const double k5_7_5_3 = h5_7_15 + CDz * h5_7_5;
    const double h13_2_6 = acc[354] + ABy * acc[146];
    const double h5_7_6 = h13_2_6 + ABy * h5_2_6;
    const double k5_7_6_1 = h5_7_12 + CDx * h5_7_6;
    const double k5_7_6_2 = h5_7_15 + CDy * h5_7_6;
    const double h13_2_14 = acc[362] + ABy * acc[154];
    const double h5_7_14 = h13_2_14 + ABy * h5_2_14;
    const double k5_7_6_3 = h5_7_14 + CDz * h5_7_6;
    const double h13_2_7 = acc[355] + ABy * acc[147];
    const double h5_7_7 = h13_2_7 + ABy * h5_2_7;
    const double k5_7_7_1 = h5_7_13 + CDx * h5_7_7;
    const double h13_2_16 = acc[364] + ABy * acc[156];
    const double h5_7_16 = h13_2_16 + ABy * h5_2_16;
    const double k5_7_7_2 = h5_7_16 + CDy * h5_7_7;
    const double h13_2_17 = acc[365] + ABy * acc[157];
    const double h5_7_17 = h13_2_17 + ABy * h5_2_17;
    const double k5_7_7_3 = h5_7_17 + CDz * h5_7_7;
    const double h13_2_8 = acc[356] + ABy * acc[148];
    const double h5_7_8 = h13_2_8 + ABy * h5_2_8;
    const double k5_7_8_1 = h5_7_15 + CDx * h5_7_8;
    const double k5_7_8_2 = h5_7_17 + CDy * h5_7_8;
    const double h13_2_18 = acc[366] + ABy * acc[158];
    const double h5_7_18 = h13_2_18 + ABy * h5_2_18;
    const double k5_7_8_3 = h5_7_18 + CDz * h5_7_8;
    const double h13_2_9 = acc[357] + ABy * acc[149];
    const double h5_7_9 = h13_2_9 + ABy * h5_2_9;
    const double k5_7_9_1 = h5_7_14 + CDx * h5_7_9;
    const double k5_7_9_2 = h5_7_18 + CDy * h5_7_9;
    const double h13_2_19 = acc[367] + ABy * acc[159];
    const double h5_7_19 = h13_2_19 + ABy * h5_2_19;
    const double k5_7_9_3 = h5_7_19 + CDz * h5_7_9;
    const double h13_3_10 = acc[374] + ABz * acc[150];
    const double h5_8_10 = h13_3_10 + ABy * h5_3_10;
    const double h13_3_4 = acc[368] + ABz * acc[144];
    const double h5_8_4 = h13_3_4 + ABy * h5_3_4;
    const double k5_8_4_1 = h5_8_10 + CDx * h5_8_4;
    const double h13_3_11 = acc[375] + ABz * acc[151];
    const double h5_8_11 = h13_3_11 + ABy * h5_3_11;
    const double k5_8_4_2 = h5_8_11 + CDy * h5_8_4;
    const double h13_3_12 = acc[376] + ABz * acc[152];
    const double h5_8_12 = h13_3_12 + ABy * h5_3_12;
    const double k5_8_4_3 = h5_8_12 + CDz * h5_8_4;
    const double h13_3_5 = acc[369] + ABz * acc[145];
    const double h5_8_5 = h13_3_5 + ABy * h5_3_5;
    const double k5_8_5_1 = h5_8_11 + CDx * h5_8_5;
    const double h13_3_13 = acc[377] + ABz * acc[153];
    const double h5_8_13 = h13_3_13 + ABy * h5_3_13;
    const double k5_8_5_2 = h5_8_13 + CDy * h5_8_5;
    const double h13_3_15 = acc[379] + ABz * acc[155];
    const double h5_8_15 = h13_3_15 + ABy * h5_3_15;
    const double k5_8_5_3 = h5_8_15 + CDz * h5_8_5;
    const double h13_3_6 = acc[370] + ABz * acc[146];
    const double h5_8_6 = h13_3_6 + ABy * h5_3_6;
    const double k5_8_6_1 = h5_8_12 + CDx * h5_8_6;
    const double k5_8_6_2 = h5_8_15 + CDy * h5_8_6;
    const double h13_3_14 = acc[378] + ABz * acc[154];
    const double h5_8_14 = h13_3_14 + ABy * h5_3_14;
    const double k5_8_6_3 = h5_8_14 + CDz * h5_8_6;
    const double h13_3_7 = acc[371] + ABz * acc[147];
    const double h5_8_7 = h13_3_7 + ABy * h5_3_7;
    const double k5_8_7_1 = h5_8_13 + CDx * h5_8_7;
    const double h13_3_16 = acc[380] + ABz * acc[156];
    const double h5_8_16 = h13_3_16 + ABy * h5_3_16;
    const double k5_8_7_2 = h5_8_16 + CDy * h5_8_7;
    const double h13_3_17 = acc[381] + ABz * acc[157];
    const double h5_8_17 = h13_3_17 + ABy * h5_3_17;
    const double k5_8_7_3 = h5_8_17 + CDz * h5_8_7;
    const double h13_3_8 = acc[372] + ABz * acc[148];
    const double h5_8_8 = h13_3_8 + ABy * h5_3_8;
    const double k5_8_8_1 = h5_8_15 + CDx * h5_8_8;
    const double k5_8_8_2 = h5_8_17 + CDy * h5_8_8;
    const double h13_3_18 = acc[382] + ABz * acc[158];
    const double h5_8_18 = h13_3_18 + ABy * h5_3_18;
    const double k5_8_8_3 = h5_8_18 + CDz * h5_8_8;
    const double h13_3_9 = acc[373] + ABz * acc[149];
    const double h5_8_9 = h13_3_9 + ABy * h5_3_9;
    const double k5_8_9_1 = h5_8_14 + CDx * h5_8_9;
    const double k5_8_9_2 = h5_8_18 + CDy * h5_8_9;
    const double h13_3_19 = acc[383] + ABz * acc[159];
    const double h5_8_19 = h13_3_19 + ABy * h5_3_19;
    const double k5_8_9_3 = h5_8_19 + CDz * h5_8_9;
    const double h15_3_10 = acc[390] + ABz * acc[182];
    const double h5_9_10 = h15_3_10 + ABz * h5_3_10;
    const double h15_3_4 = acc[384] + ABz * acc[176];
    const double h5_9_4 = h15_3_4 + ABz * h5_3_4;
    const double k5_9_4_1 = h5_9_10 + CDx * h5_9_4;
    const double h15_3_11 = acc[391] + ABz * acc[183];
    const double h5_9_11 = h15_3_11 + ABz * h5_3_11;
    const double k5_9_4_2 = h5_9_11 + CDy * h5_9_4;
    const double h15_3_12 = acc[392] + ABz * acc[184];
    const double h5_9_12 = h15_3_12 + ABz * h5_3_12;
    const double k5_9_4_3 = h5_9_12 + CDz * h5_9_4;
    const double h15_3_5 = acc[385] + ABz * acc[177];
    const double h5_9_5 = h15_3_5 + ABz * h5_3_5;
    const double k5_9_5_1 = h5_9_11 + CDx * h5_9_5;
    const double h15_3_13 = acc[393] + ABz * acc[185];
    const double h5_9_13 = h15_3_13 + ABz * h5_3_13;
    const double k5_9_5_2 = h5_9_13 + CDy * h5_9_5;
    const double h15_3_15 = acc[395] + ABz * acc[187];
    const double h5_9_15 = h15_3_15 + ABz * h5_3_15;
    const double k5_9_5_3 = h5_9_15 + CDz * h5_9_5;
    const double h15_3_6 = acc[386] + ABz * acc[178];
    const double h5_9_6 = h15_3_6 + ABz * h5_3_6;
    const double k5_9_6_1 = h5_9_12 + CDx * h5_9_6;
    const double k5_9_6_2 = h5_9_15 + CDy * h5_9_6;
    const double h15_3_14 = acc[394] + ABz * acc[186];
    const double h5_9_14 = h15_3_14 + ABz * h5_3_14;
    const double k5_9_6_3 = h5_9_14 + CDz * h5_9_6;
    const double h15_3_7 = acc[387] + ABz * acc[179];
    const double h5_9_7 = h15_3_7 + ABz * h5_3_7;
    const double k5_9_7_1 = h5_9_13 + CDx * h5_9_7;
    const double h15_3_16 = acc[396] + ABz * acc[188];
    const double h5_9_16 = h15_3_16 + ABz * h5_3_16;
    const double k5_9_7_2 = h5_9_16 + CDy * h5_9_7;
    const double h15_3_17 = acc[397] + ABz * acc[189];
    const double h5_9_17 = h15_3_17 + ABz * h5_3_17;
    const double k5_9_7_3 = h5_9_17 + CDz * h5_9_7;
    const double h15_3_8 = acc[388] + ABz * acc[180];
    const double h5_9_8 = h15_3_8 + ABz * h5_3_8;
    const double k5_9_8_1 = h5_9_15 + CDx * h5_9_8;
    const double k5_9_8_2 = h5_9_17 + CDy * h5_9_8;
    const double h15_3_18 = acc[398] + ABz * acc[190];
    const double h5_9_18 = h15_3_18 + ABz * h5_3_18;
    const double k5_9_8_3 = h5_9_18 + CDz * h5_9_8;
    const double h15_3_9 = acc[389] + ABz * acc[181];
    const double h5_9_9 = h15_3_9 + ABz * h5_3_9;
    const double k5_9_9_1 = h5_9_14 + CDx * h5_9_9;
    const double k5_9_9_2 = h5_9_18 + CDy * h5_9_9;
    const double h15_3_19 = acc[399] + ABz * acc[191];
    const double h5_9_19 = h15_3_19 + ABz * h5_3_19;
    const double k5_9_9_3 = h5_9_19 + CDz * h5_9_9;
    const double h12_1_10 = acc[294] + ABx * acc[134];
    const double h6_1_10 = acc[134] + ABx * acc[38];
    const double h6_4_10 = h12_1_10 + ABx * h6_1_10;
    const double h12_1_4 = acc[288] + ABx * acc[128];
    const double h6_1_4 = acc[128] + ABx * acc[32];
    const double h6_4_4 = h12_1_4 + ABx * h6_1_4;
    const double k6_4_4_1 = h6_4_10 + CDx * h6_4_4;
    const double h12_1_11 = acc[295] + ABx * acc[135];
    const double h6_1_11 = acc[135] + ABx * acc[39];
    const double h6_4_11 = h12_1_11 + ABx * h6_1_11;
    const double k6_4_4_2 = h6_4_11 + CDy * h6_4_4;
    const double h12_1_12 = acc[296] + ABx * acc[136];
    const double h6_1_12 = acc[136] + ABx * acc[40];
    const double h6_4_12 = h12_1_12 + ABx * h6_1_12;
    const double k6_4_4_3 = h6_4_12 + CDz * h6_4_4;
    const double h12_1_5 = acc[289] + ABx * acc[129];
    const double h6_1_5 = acc[129] + ABx * acc[33];
    const double h6_4_5 = h12_1_5 + ABx * h6_1_5;
    const double k6_4_5_1 = h6_4_11 + CDx * h6_4_5;
    const double h12_1_13 = acc[297] + ABx * acc[137];
    const double h6_1_13 = acc[137] + ABx * acc[41];
    const double h6_4_13 = h12_1_13 + ABx * h6_1_13;
    const double k6_4_5_2 = h6_4_13 + CDy * h6_4_5;
    const double h12_1_15 = acc[299] + ABx * acc[139];
    const double h6_1_15 = acc[139] + ABx * acc[43];
    const double h6_4_15 = h12_1_15 + ABx * h6_1_15;
    const double k6_4_5_3 = h6_4_15 + CDz * h6_4_5;
    const double h12_1_6 = acc[290] + ABx * acc[130];
    const double h6_1_6 = acc[130] + ABx * acc[34];
    const double h6_4_6 = h12_1_6 + ABx * h6_1_6;
    const double k6_4_6_1 = h6_4_12 + CDx * h6_4_6;
    const double k6_4_6_2 = h6_4_15 + CDy * h6_4_6;
    const double h12_1_14 = acc[298] + ABx * acc[138];
    const double h6_1_14 = acc[138] + ABx * acc[42];
    const double h6_4_14 = h12_1_14 + ABx * h6_1_14;
    const double k6_4_6_3 = h6_4_14 + CDz * h6_4_6;
    const double h12_1_7 = acc[291] + ABx * acc[131];
    const double h6_1_7 = acc[131] + ABx * acc[35];
    const double h6_4_7 = h12_1_7 + ABx * h6_1_7;
    const double k6_4_7_1 = h6_4_13 + CDx * h6_4_7;
    const double h12_1_16 = acc[300] + ABx * acc[140];
    const double h6_1_16 = acc[140] + ABx * acc[44];
    const double h6_4_16 = h12_1_16 + ABx * h6_1_16;
    const double k6_4_7_2 = h6_4_16 + CDy * h6_4_7;
    const double h12_1_17 = acc[301] + ABx * acc[141];
    const double h6_1_17 = acc[141] + ABx * acc[45];
    const double h6_4_17 = h12_1_17 + ABx * h6_1_17;
    const double k6_4_7_3 = h6_4_17 + CDz * h6_4_7;
    const double h12_1_8 = acc[292] + ABx * acc[132];
    const double h6_1_8 = acc[132] + ABx * acc[36];
    const double h6_4_8 = h12_1_8 + ABx * h6_1_8;
    const double k6_4_8_1 = h6_4_15 + CDx * h6_4_8;
    const double k6_4_8_2 = h6_4_17 + CDy * h6_4_8;
    const double h12_1_18 = acc[302] + ABx * acc[142];
    const double h6_1_18 = acc[142] + ABx * acc[46];
    const double h6_4_18 = h12_1_18 + ABx * h6_1_18;
    const double k6_4_8_3 = h6_4_18 + CDz * h6_4_8;
    const double h12_1_9 = acc[293] + ABx * acc[133];
    const double h6_1_9 = acc[133] + ABx * acc[37];
    const double h6_4_9 = h12_1_9 + ABx * h6_1_9;
    const double k6_4_9_1 = h6_4_14 + CDx * h6_4_9;
    const double k6_4_9_2 = h6_4_18 + CDy * h6_4_9;
    const double h12_1_19 = acc[303] + ABx * acc[143];
    const double h6_1_19 = acc[143] + ABx * acc[47];
    const double h6_4_19 = h12_1_19 + ABx * h6_1_19;
    const double k6_4_9_3 = h6_4_19 + CDz * h6_4_9;
    const double h12_2_10 = acc[326] + ABy * acc[134];
    const double h6_2_10 = acc[182] + ABy * acc[38];
    const double h6_5_10 = h12_2_10 + ABx * h6_2_10;
    const double h12_2_4 = acc[320] + ABy * acc[128];
    const double h6_2_4 = acc[176] + ABy * acc[32];
    const double h6_5_4 = h12_2_4 + ABx * h6_2_4;
    const double k6_5_4_1 = h6_5_10 + CDx * h6_5_4;
    const double h12_2_11 = acc[327] + ABy * acc[135];
    const double h6_2_11 = acc[183] + ABy * acc[39];
    const double h6_5_11 = h12_2_11 + ABx * h6_2_11;
    const double k6_5_4_2 = h6_5_11 + CDy * h6_5_4;
    const double h12_2_12 = acc[328] + ABy * acc[136];
    const double h6_2_12 = acc[184] + ABy * acc[40];
    const double h6_5_12 = h12_2_12 + ABx * h6_2_12;
    const double k6_5_4_3 = h6_5_12 + CDz * h6_5_4;
    const double h12_2_5 = acc[321] + ABy * acc[129];
    const double h6_2_5 = acc[177] + ABy * acc[33];
    const double h6_5_5 = h12_2_5 + ABx * h6_2_5;
    const double k6_5_5_1 = h6_5_11 + CDx * h6_5_5;
    const double h12_2_13 = acc[329] + ABy * acc[137];
    const double h6_2_13 = acc[185] + ABy * acc[41];
    const double h6_5_13 = h12_2_13 + ABx * h6_2_13;
    const double k6_5_5_2 = h6_5_13 + CDy * h6_5_5;
    const double h12_2_15 = acc[331] + ABy * acc[139];
    const double h6_2_15 = acc[187] + ABy * acc[43];
    const double h6_5_15 = h12_2_15 + ABx * h6_2_15;
    const double k6_5_5_3 = h6_5_15 + CDz * h6_5_5;
    const double h12_2_6 = acc[322] + ABy * acc[130];
    const double h6_2_6 = acc[178] + ABy * acc[34];
    const double h6_5_6 = h12_2_6 + ABx * h6_2_6;
    const double k6_5_6_1 = h6_5_12 + CDx * h6_5_6;
    const double k6_5_6_2 = h6_5_15 + CDy * h6_5_6;
    const double h12_2_14 = acc[330] + ABy * acc[138];
    const double h6_2_14 = acc[186] + ABy * acc[42];
    const double h6_5_14 = h12_2_14 + ABx * h6_2_14;
    const double k6_5_6_3 = h6_5_14 + CDz * h6_5_6;
    const double h12_2_7 = acc[323] + ABy * acc[131];
    const double h6_2_7 = acc[179] + ABy * acc[35];
    const double h6_5_7 = h12_2_7 + ABx * h6_2_7;
    const double k6_5_7_1 = h6_5_13 + CDx * h6_5_7;
    const double h12_2_16 = acc[332] + ABy * acc[140];
    const double h6_2_16 = acc[188] + ABy * acc[44];
    const double h6_5_16 = h12_2_16 + ABx * h6_2_16;
    const double k6_5_7_2 = h6_5_16 + CDy * h6_5_7;
    const double h12_2_17 = acc[333] + ABy * acc[141];
    const double h6_2_17 = acc[189] + ABy * acc[45];
    const double h6_5_17 = h12_2_17 + ABx * h6_2_17;
    const double k6_5_7_3 = h6_5_17 + CDz * h6_5_7;
    const double h12_2_8 = acc[324] + ABy * acc[132];
    const double h6_2_8 = acc[180] + ABy * acc[36];
    const double h6_5_8 = h12_2_8 + ABx * h6_2_8;
    const double k6_5_8_1 = h6_5_15 + CDx * h6_5_8;
    const double k6_5_8_2 = h6_5_17 + CDy * h6_5_8;
    const double h12_2_18 = acc[334] + ABy * acc[142];
    const double h6_2_18 = acc[190] + ABy * acc[46];
    const double h6_5_18 = h12_2_18 + ABx * h6_2_18;
    const double k6_5_8_3 = h6_5_18 + CDz * h6_5_8;
    const double h12_2_9 = acc[325] + ABy * acc[133];
    const double h6_2_9 = acc[181] + ABy * acc[37];
    const double h6_5_9 = h12_2_9 + ABx * h6_2_9;
    const double k6_5_9_1 = h6_5_14 + CDx * h6_5_9;
    const double k6_5_9_2 = h6_5_18 + CDy * h6_5_9;
    const double h12_2_19 = acc[335] + ABy * acc[143];
    const double h6_2_19 = acc[191] + ABy * acc[47];
    const double h6_5_19 = h12_2_19 + ABx * h6_2_19;
    const double k6_5_9_3 = h6_5_19 + CDz * h6_5_9;
    const double h6_3_10 = acc[166] + ABz * acc[38];
    const double h6_6_10 = h12_3_10 + ABx * h6_3_10;
    const double h6_3_4 = acc[160] + ABz * acc[32];
    const double h6_6_4 = h12_3_4 + ABx * h6_3_4;
    const double k6_6_4_1 = h6_6_10 + CDx * h6_6_4;
    const double h6_3_11 = acc[167] + ABz * acc[39];
    const double h6_6_11 = h12_3_11 + ABx * h6_3_11;
    const double k6_6_4_2 = h6_6_11 + CDy * h6_6_4;
    const double h6_3_12 = acc[168] + ABz * acc[40];
    const double h6_6_12 = h12_3_12 + ABx * h6_3_12;
    const double k6_6_4_3 = h6_6_12 + CDz * h6_6_4;
    const double h6_3_5 = acc[161] + ABz * acc[33];
    const double h6_6_5 = h12_3_5 + ABx * h6_3_5;
    const double k6_6_5_1 = h6_6_11 + CDx * h6_6_5;
    const double h6_3_13 = acc[169] + ABz * acc[41];
    const double h6_6_13 = h12_3_13 + ABx * h6_3_13;
    const double k6_6_5_2 = h6_6_13 + CDy * h6_6_5;
    const double h6_3_15 = acc[171] + ABz * acc[43];
    const double h6_6_15 = h12_3_15 + ABx * h6_3_15;
    const double k6_6_5_3 = h6_6_15 + CDz * h6_6_5;
    const double h6_3_6 = acc[162] + ABz * acc[34];
    const double h6_6_6 = h12_3_6 + ABx * h6_3_6;
    const double k6_6_6_1 = h6_6_12 + CDx * h6_6_6;
    const double k6_6_6_2 = h6_6_15 + CDy * h6_6_6;
    const double h6_3_14 = acc[170] + ABz * acc[42];
    const double h6_6_14 = h12_3_14 + ABx * h6_3_14;
    const double k6_6_6_3 = h6_6_14 + CDz * h6_6_6;
    const double h6_3_7 = acc[163] + ABz * acc[35];
    const double h6_6_7 = h12_3_7 + ABx * h6_3_7;
    const double k6_6_7_1 = h6_6_13 + CDx * h6_6_7;
    const double h6_3_16 = acc[172] + ABz * acc[44];
    const double h6_6_16 = h12_3_16 + ABx * h6_3_16;
    const double k6_6_7_2 = h6_6_16 + CDy * h6_6_7;
    const double h6_3_17 = acc[173] + ABz * acc[45];
    const double h6_6_17 = h12_3_17 + ABx * h6_3_17;
    const double k6_6_7_3 = h6_6_17 + CDz * h6_6_7;
    const double h6_3_8 = acc[164] + ABz * acc[36];
    const double h6_6_8 = h12_3_8 + ABx * h6_3_8;
    const double k6_6_8_1 = h6_6_15 + CDx * h6_6_8;
    const double k6_6_8_2 = h6_6_17 + CDy * h6_6_8;
    const double h6_3_18 = acc[174] + ABz * acc[46];
    const double h6_6_18 = h12_3_18 + ABx * h6_3_18;
    const double k6_6_8_3 = h6_6_18 + CDz * h6_6_8;
    const double h6_3_9 = acc[165] + ABz * acc[37];
    const double h6_6_9 = h12_3_9 + ABx * h6_3_9;
    const double k6_6_9_1 = h6_6_14 + CDx * h6_6_9;
    const double k6_6_9_2 = h6_6_18 + CDy * h6_6_9;
    const double h6_3_19 = acc[175] + ABz * acc[47];
    const double h6_6_19 = h12_3_19 + ABx * h6_3_19;
    const double k6_6_9_3 = h6_6_19 + CDz * h6_6_9;
    const double h15_2_10 = acc[374] + ABy * acc[182];
    const double h6_7_10 = h15_2_10 + ABy * h6_2_10;
    const double h15_2_4 = acc[368] + ABy * acc[176];
    const double h6_7_4 = h15_2_4 + ABy * h6_2_4;
    const double k6_7_4_1 = h6_7_10 + CDx * h6_7_4;
    const double h15_2_11 = acc[375] + ABy * acc[183];
    const double h6_7_11 = h15_2_11 + ABy * h6_2_11;
    const double k6_7_4_2 = h6_7_11 + CDy * h6_7_4;
    const double h15_2_12 = acc[376] + ABy * acc[184];
    const double h6_7_12 = h15_2_12 + ABy * h6_2_12;
    const double k6_7_4_3 = h6_7_12 + CDz * h6_7_4;
    const double h15_2_5 = acc[369] + ABy * acc[177];
    const double h6_7_5 = h15_2_5 + ABy * h6_2_5;
    const double k6_7_5_1 = h6_7_11 + CDx * h6_7_5;
    const double h15_2_13 = acc[377] + ABy * acc[185];
    const double h6_7_13 = h15_2_13 + ABy * h6_2_13;
    const double k6_7_5_2 = h6_7_13 + CDy * h6_7_5;
    const double h15_2_15 = acc[379] + ABy * acc[187];
    const double h6_7_15 = h15_2_15 + ABy * h6_2_15;
    const double k6_7_5_3 = h6_7_15 + CDz * h6_7_5;
    const double h15_2_6 = acc[370] + ABy * acc[178];
    const double h6_7_6 = h15_2_6 + ABy * h6_2_6;
    const double k6_7_6_1 = h6_7_12 + CDx * h6_7_6;
    const double k6_7_6_2 = h6_7_15 + CDy * h6_7_6;
    const double h15_2_14 = acc[378] + ABy * acc[186];
    const double h6_7_14 = h15_2_14 + ABy * h6_2_14;
    const double k6_7_6_3 = h6_7_14 + CDz * h6_7_6;
    const double h15_2_7 = acc[371] + ABy * acc[179];
    const double h6_7_7 = h15_2_7 + ABy * h6_2_7;
    const double k6_7_7_1 = h6_7_13 + CDx * h6_7_7;
    const double h15_2_16 = acc[380] + ABy * acc[188];
    const double h6_7_16 = h15_2_16 + ABy * h6_2_16;
    const double k6_7_7_2 = h6_7_16 + CDy * h6_7_7;
    const double h15_2_17 = acc[381] + ABy * acc[189];
    const double h6_7_17 = h15_2_17 + ABy * h6_2_17;
    const double k6_7_7_3 = h6_7_17 + CDz * h6_7_7;
    const double h15_2_8 = acc[372] + ABy * acc[180];
    const double h6_7_8 = h15_2_8 + ABy * h6_2_8;
    const double k6_7_8_1 = h6_7_15 + CDx * h6_7_8;
    const double k6_7_8_2 = h6_7_17 + CDy * h6_7_8;
    const double h15_2_18 = acc[382] + ABy * acc[190];
    const double h6_7_18 = h15_2_18 + ABy * h6_2_18;
    const double k6_7_8_3 = h6_7_18 + CDz * h6_7_8;
    const double h15_2_9 = acc[373] + ABy * acc[181];
    const double h6_7_9 = h15_2_9 + ABy * h6_2_9;
    const double k6_7_9_1 = h6_7_14 + CDx * h6_7_9;
    const double k6_7_9_2 = h6_7_18 + CDy * h6_7_9;
    const double h15_2_19 = acc[383] + ABy * acc[191];
    const double h6_7_19 = h15_2_19 + ABy * h6_2_19;
    const double k6_7_9_3 = h6_7_19 + CDz * h6_7_9;
    const double h6_8_10 = h15_3_10 + ABy * h6_3_10;
    const double h6_8_4 = h15_3_4 + ABy * h6_3_4;
    const double k6_8_4_1 = h6_8_10 + CDx * h6_8_4;
    const double h6_8_11 = h15_3_11 + ABy * h6_3_11;
    const double k6_8_4_2 = h6_8_11 + CDy * h6_8_4;
    const double h6_8_12 = h15_3_12 + ABy * h6_3_12;
    const double k6_8_4_3 = h6_8_12 + CDz * h6_8_4;
    const double h6_8_5 = h15_3_5 + ABy * h6_3_5;
    const double k6_8_5_1 = h6_8_11 + CDx * h6_8_5;
    const double h6_8_13 = h15_3_13 + ABy * h6_3_13;
    const double k6_8_5_2 = h6_8_13 + CDy * h6_8_5;
    const double h6_8_15 = h15_3_15 + ABy * h6_3_15;
    const double k6_8_5_3 = h6_8_15 + CDz * h6_8_5;
    const double h6_8_6 = h15_3_6 + ABy * h6_3_6;
    const double k6_8_6_1 = h6_8_12 + CDx * h6_8_6;
    const double k6_8_6_2 = h6_8_15 + CDy * h6_8_6;
    const double h6_8_14 = h15_3_14 + ABy * h6_3_14;
    const double k6_8_6_3 = h6_8_14 + CDz * h6_8_6;
    const double h6_8_7 = h15_3_7 + ABy * h6_3_7;
    const double k6_8_7_1 = h6_8_13 + CDx * h6_8_7;
    const double h6_8_16 = h15_3_16 + ABy * h6_3_16;
    const double k6_8_7_2 = h6_8_16 + CDy * h6_8_7;
    const double h6_8_17 = h15_3_17 + ABy * h6_3_17;
    const double k6_8_7_3 = h6_8_17 + CDz * h6_8_7;
    const double h6_8_8 = h15_3_8 + ABy * h6_3_8;
    const double k6_8_8_1 = h6_8_15 + CDx * h6_8_8;
    const double k6_8_8_2 = h6_8_17 + CDy * h6_8_8;
    const double h6_8_18 = h15_3_18 + ABy * h6_3_18;
    const double k6_8_8_3 = h6_8_18 + CDz * h6_8_8;
    const double h6_8_9 = h15_3_9 + ABy * h6_3_9;
    const double k6_8_9_1 = h6_8_14 + CDx * h6_8_9;
    const double k6_8_9_2 = h6_8_18 + CDy * h6_8_9;
    const double h6_8_19 = h15_3_19 + ABy * h6_3_19;
    const double k6_8_9_3 = h6_8_19 + CDz * h6_8_9;
    const double h14_3_10 = acc[406] + ABz * acc[166];
    const double h6_9_10 = h14_3_10 + ABz * h6_3_10;
    const double h14_3_4 = acc[400] + ABz * acc[160];
    const double h6_9_4 = h14_3_4 + ABz * h6_3_4;
    const double k6_9_4_1 = h6_9_10 + CDx * h6_9_4;
    const double h14_3_11 = acc[407] + ABz * acc[167];
    const double h6_9_11 = h14_3_11 + ABz * h6_3_11;
    const double k6_9_4_2 = h6_9_11 + CDy * h6_9_4;
    const double h14_3_12 = acc[408] + ABz * acc[168];
    const double h6_9_12 = h14_3_12 + ABz * h6_3_12;
    const double k6_9_4_3 = h6_9_12 + CDz * h6_9_4;
    const double h14_3_5 = acc[401] + ABz * acc[161];
    const double h6_9_5 = h14_3_5 + ABz * h6_3_5;
    const double k6_9_5_1 = h6_9_11 + CDx * h6_9_5;
    const double h14_3_13 = acc[409] + ABz * acc[169];
    const double h6_9_13 = h14_3_13 + ABz * h6_3_13;
    const double k6_9_5_2 = h6_9_13 + CDy * h6_9_5;
    const double h14_3_15 = acc[411] + ABz * acc[171];
    const double h6_9_15 = h14_3_15 + ABz * h6_3_15;
    const double k6_9_5_3 = h6_9_15 + CDz * h6_9_5;
    const double h14_3_6 = acc[402] + ABz * acc[162];
    const double h6_9_6 = h14_3_6 + ABz * h6_3_6;
    const double k6_9_6_1 = h6_9_12 + CDx * h6_9_6;
    const double k6_9_6_2 = h6_9_15 + CDy * h6_9_6;
    const double h14_3_14 = acc[410] + ABz * acc[170];
    const double h6_9_14 = h14_3_14 + ABz * h6_3_14;
    const double k6_9_6_3 = h6_9_14 + CDz * h6_9_6;
    const double h14_3_7 = acc[403] + ABz * acc[163];
    const double h6_9_7 = h14_3_7 + ABz * h6_3_7;
    const double k6_9_7_1 = h6_9_13 + CDx * h6_9_7;
    const double h14_3_16 = acc[412] + ABz * acc[172];
    const double h6_9_16 = h14_3_16 + ABz * h6_3_16;
    const double k6_9_7_2 = h6_9_16 + CDy * h6_9_7;
    const double h14_3_17 = acc[413] + ABz * acc[173];
    const double h6_9_17 = h14_3_17 + ABz * h6_3_17;
    const double k6_9_7_3 = h6_9_17 + CDz * h6_9_7;
    const double h14_3_8 = acc[404] + ABz * acc[164];
    const double h6_9_8 = h14_3_8 + ABz * h6_3_8;
    const double k6_9_8_1 = h6_9_15 + CDx * h6_9_8;
    const double k6_9_8_2 = h6_9_17 + CDy * h6_9_8;
    const double h14_3_18 = acc[414] + ABz * acc[174];
    const double h6_9_18 = h14_3_18 + ABz * h6_3_18;
    const double k6_9_8_3 = h6_9_18 + CDz * h6_9_8;
    const double h14_3_9 = acc[405] + ABz * acc[165];
    const double h6_9_9 = h14_3_9 + ABz * h6_3_9;
    const double k6_9_9_1 = h6_9_14 + CDx * h6_9_9;
    const double k6_9_9_2 = h6_9_18 + CDy * h6_9_9;
    const double h14_3_19 = acc[415] + ABz * acc[175];
    const double h6_9_19 = h14_3_19 + ABz * h6_3_19;
    const double k6_9_9_3 = h6_9_19 + CDz * h6_9_9;
    const double h13_1_10 = acc[310] + ABx * acc[150];
    const double h7_1_10 = acc[150] + ABx * acc[54];
    const double h7_4_10 = h13_1_10 + ABx * h7_1_10;
    const double h13_1_4 = acc[304] + ABx * acc[144];
    const double h7_1_4 = acc[144] + ABx * acc[48];
    const double h7_4_4 = h13_1_4 + ABx * h7_1_4;
    const double k7_4_4_1 = h7_4_10 + CDx * h7_4_4;
    const double h13_1_11 = acc[311] + ABx * acc[151];
    const double h7_1_11 = acc[151] + ABx * acc[55];
    const double h7_4_11 = h13_1_11 + ABx * h7_1_11;
    const double k7_4_4_2 = h7_4_11 + CDy * h7_4_4;
    const double h13_1_12 = acc[312] + ABx * acc[152];
    const double h7_1_12 = acc[152] + ABx * acc[56];
    const double h7_4_12 = h13_1_12 + ABx * h7_1_12;
    const double k7_4_4_3 = h7_4_12 + CDz * h7_4_4;
    const double h13_1_5 = acc[305] + ABx * acc[145];
    const double h7_1_5 = acc[145] + ABx * acc[49];
    const double h7_4_5 = h13_1_5 + ABx * h7_1_5;
    const double k7_4_5_1 = h7_4_11 + CDx * h7_4_5;
    const double h13_1_13 = acc[313] + ABx * acc[153];
    const double h7_1_13 = acc[153] + ABx * acc[57];
    const double h7_4_13 = h13_1_13 + ABx * h7_1_13;
    const double k7_4_5_2 = h7_4_13 + CDy * h7_4_5;
    const double h13_1_15 = acc[315] + ABx * acc[155];
    const double h7_1_15 = acc[155] + ABx * acc[59];
    const double h7_4_15 = h13_1_15 + ABx * h7_1_15;
    const double k7_4_5_3 = h7_4_15 + CDz * h7_4_5;
    const double h13_1_6 = acc[306] + ABx * acc[146];
    const double h7_1_6 = acc[146] + ABx * acc[50];
    const double h7_4_6 = h13_1_6 + ABx * h7_1_6;
    const double k7_4_6_1 = h7_4_12 + CDx * h7_4_6;
    const double k7_4_6_2 = h7_4_15 + CDy * h7_4_6;
    const double h13_1_14 = acc[314] + ABx * acc[154];
    const double h7_1_14 = acc[154] + ABx * acc[58];
    const double h7_4_14 = h13_1_14 + ABx * h7_1_14;
    const double k7_4_6_3 = h7_4_14 + CDz * h7_4_6;
    const double h13_1_7 = acc[307] + ABx * acc[147];
    const double h7_1_7 = acc[147] + ABx * acc[51];
    const double h7_4_7 = h13_1_7 + ABx * h7_1_7;
    const double k7_4_7_1 = h7_4_13 + CDx * h7_4_7;
    const double h13_1_16 = acc[316] + ABx * acc[156];
    const double h7_1_16 = acc[156] + ABx * acc[60];
    const double h7_4_16 = h13_1_16 + ABx * h7_1_16;
    const double k7_4_7_2 = h7_4_16 + CDy * h7_4_7;
    const double h13_1_17 = acc[317] + ABx * acc[157];
    const double h7_1_17 = acc[157] + ABx * acc[61];
    const double h7_4_17 = h13_1_17 + ABx * h7_1_17;
    const double k7_4_7_3 = h7_4_17 + CDz * h7_4_7;
    const double h13_1_8 = acc[308] + ABx * acc[148];
    const double h7_1_8 = acc[148] + ABx * acc[52];
    const double h7_4_8 = h13_1_8 + ABx * h7_1_8;
    const double k7_4_8_1 = h7_4_15 + CDx * h7_4_8;
    const double k7_4_8_2 = h7_4_17 + CDy * h7_4_8;
    const double h13_1_18 = acc[318] + ABx * acc[158];
    const double h7_1_18 = acc[158] + ABx * acc[62];
    const double h7_4_18 = h13_1_18 + ABx * h7_1_18;
    const double k7_4_8_3 = h7_4_18 + CDz * h7_4_8;
    const double h13_1_9 = acc[309] + ABx * acc[149];
    const double h7_1_9 = acc[149] + ABx * acc[53];
    const double h7_4_9 = h13_1_9 + ABx * h7_1_9;
    const double k7_4_9_1 = h7_4_14 + CDx * h7_4_9;
    const double k7_4_9_2 = h7_4_18 + CDy * h7_4_9;
    const double h13_1_19 = acc[319] + ABx * acc[159];
    const double h7_1_19 = acc[159] + ABx * acc[63];
    const double h7_4_19 = h13_1_19 + ABx * h7_1_19;
    const double k7_4_9_3 = h7_4_19 + CDz * h7_4_9;
    const double h7_2_10 = acc[198] + ABy * acc[54];
    const double h7_5_10 = h13_2_10 + ABx * h7_2_10;
    const double h7_2_4 = acc[192] + ABy * acc[48];
    const double h7_5_4 = h13_2_4 + ABx * h7_2_4;
    const double k7_5_4_1 = h7_5_10 + CDx * h7_5_4;
    const double h7_2_11 = acc[199] + ABy * acc[55];
    const double h7_5_11 = h13_2_11 + ABx * h7_2_11;
    const double k7_5_4_2 = h7_5_11 + CDy * h7_5_4;
    const double h7_2_12 = acc[200] + ABy * acc[56];
    const double h7_5_12 = h13_2_12 + ABx * h7_2_12;
    const double k7_5_4_3 = h7_5_12 + CDz * h7_5_4;
    const double h7_2_5 = acc[193] + ABy * acc[49];
    const double h7_5_5 = h13_2_5 + ABx * h7_2_5;
    const double k7_5_5_1 = h7_5_11 + CDx * h7_5_5;
    const double h7_2_13 = acc[201] + ABy * acc[57];
    const double h7_5_13 = h13_2_13 + ABx * h7_2_13;
    const double k7_5_5_2 = h7_5_13 + CDy * h7_5_5;
    const double h7_2_15 = acc[203] + ABy * acc[59];
    const double h7_5_15 = h13_2_15 + ABx * h7_2_15;
    const double k7_5_5_3 = h7_5_15 + CDz * h7_5_5;
    const double h7_2_6 = acc[194] + ABy * acc[50];
    const double h7_5_6 = h13_2_6 + ABx * h7_2_6;
    const double k7_5_6_1 = h7_5_12 + CDx * h7_5_6;
    const double k7_5_6_2 = h7_5_15 + CDy * h7_5_6;
    const double h7_2_14 = acc[202] + ABy * acc[58];
    const double h7_5_14 = h13_2_14 + ABx * h7_2_14;
    const double k7_5_6_3 = h7_5_14 + CDz * h7_5_6;
    const double h7_2_7 = acc[195] + ABy * acc[51];
    const double h7_5_7 = h13_2_7 + ABx * h7_2_7;
    const double k7_5_7_1 = h7_5_13 + CDx * h7_5_7;
    const double h7_2_16 = acc[204] + ABy * acc[60];
    const double h7_5_16 = h13_2_16 + ABx * h7_2_16;
    const double k7_5_7_2 = h7_5_16 + CDy * h7_5_7;
    const double h7_2_17 = acc[205] + ABy * acc[61];
    const double h7_5_17 = h13_2_17 + ABx * h7_2_17;
    const double k7_5_7_3 = h7_5_17 + CDz * h7_5_7;
    const double h7_2_8 = acc[196] + ABy * acc[52];
    const double h7_5_8 = h13_2_8 + ABx * h7_2_8;
    const double k7_5_8_1 = h7_5_15 + CDx * h7_5_8;
    const double k7_5_8_2 = h7_5_17 + CDy * h7_5_8;
    const double h7_2_18 = acc[206] + ABy * acc[62];
    const double h7_5_18 = h13_2_18 + ABx * h7_2_18;
    const double k7_5_8_3 = h7_5_18 + CDz * h7_5_8;
    const double h7_2_9 = acc[197] + ABy * acc[53];
    const double h7_5_9 = h13_2_9 + ABx * h7_2_9;
    const double k7_5_9_1 = h7_5_14 + CDx * h7_5_9;
    const double k7_5_9_2 = h7_5_18 + CDy * h7_5_9;
    const double h7_2_19 = acc[207] + ABy * acc[63];
    const double h7_5_19 = h13_2_19 + ABx * h7_2_19;
    const double k7_5_9_3 = h7_5_19 + CDz * h7_5_9;
    const double h7_3_10 = acc[214] + ABz * acc[54];
    const double h7_6_10 = h13_3_10 + ABx * h7_3_10;
    const double h7_3_4 = acc[208] + ABz * acc[48];
    const double h7_6_4 = h13_3_4 + ABx * h7_3_4;
    const double k7_6_4_1 = h7_6_10 + CDx * h7_6_4;
    const double h7_3_11 = acc[215] + ABz * acc[55];
    const double h7_6_11 = h13_3_11 + ABx * h7_3_11;
    const double k7_6_4_2 = h7_6_11 + CDy * h7_6_4;
    const double h7_3_12 = acc[216] + ABz * acc[56];
    const double h7_6_12 = h13_3_12 + ABx * h7_3_12;
    const double k7_6_4_3 = h7_6_12 + CDz * h7_6_4;
    const double h7_3_5 = acc[209] + ABz * acc[49];
    const double h7_6_5 = h13_3_5 + ABx * h7_3_5;
    const double k7_6_5_1 = h7_6_11 + CDx * h7_6_5;
    const double h7_3_13 = acc[217] + ABz * acc[57];
    const double h7_6_13 = h13_3_13 + ABx * h7_3_13;
    const double k7_6_5_2 = h7_6_13 + CDy * h7_6_5;
    const double h7_3_15 = acc[219] + ABz * acc[59];
    const double h7_6_15 = h13_3_15 + ABx * h7_3_15;
    const double k7_6_5_3 = h7_6_15 + CDz * h7_6_5;
    const double h7_3_6 = acc[210] + ABz * acc[50];
    const double h7_6_6 = h13_3_6 + ABx * h7_3_6;
    const double k7_6_6_1 = h7_6_12 + CDx * h7_6_6;
    const double k7_6_6_2 = h7_6_15 + CDy * h7_6_6;
    const double h7_3_14 = acc[218] + ABz * acc[58];
    const double h7_6_14 = h13_3_14 + ABx * h7_3_14;
    const double k7_6_6_3 = h7_6_14 + CDz * h7_6_6;
    const double h7_3_7 = acc[211] + ABz * acc[51];
    const double h7_6_7 = h13_3_7 + ABx * h7_3_7;
    const double k7_6_7_1 = h7_6_13 + CDx * h7_6_7;
    const double h7_3_16 = acc[220] + ABz * acc[60];
    const double h7_6_16 = h13_3_16 + ABx * h7_3_16;
    const double k7_6_7_2 = h7_6_16 + CDy * h7_6_7;
    const double h7_3_17 = acc[221] + ABz * acc[61];
    const double h7_6_17 = h13_3_17 + ABx * h7_3_17;
    const double k7_6_7_3 = h7_6_17 + CDz * h7_6_7;
    const double h7_3_8 = acc[212] + ABz * acc[52];
    const double h7_6_8 = h13_3_8 + ABx * h7_3_8;
    const double k7_6_8_1 = h7_6_15 + CDx * h7_6_8;
    const double k7_6_8_2 = h7_6_17 + CDy * h7_6_8;
    const double h7_3_18 = acc[222] + ABz * acc[62];
    const double h7_6_18 = h13_3_18 + ABx * h7_3_18;
    const double k7_6_8_3 = h7_6_18 + CDz * h7_6_8;
    const double h7_3_9 = acc[213] + ABz * acc[53];
    const double h7_6_9 = h13_3_9 + ABx * h7_3_9;
    const double k7_6_9_1 = h7_6_14 + CDx * h7_6_9;
    const double k7_6_9_2 = h7_6_18 + CDy * h7_6_9;
    const double h7_3_19 = acc[223] + ABz * acc[63];
    const double h7_6_19 = h13_3_19 + ABx * h7_3_19;
    const double k7_6_9_3 = h7_6_19 + CDz * h7_6_9;
    const double h16_2_10 = acc[422] + ABy * acc[198];
    const double h7_7_10 = h16_2_10 + ABy * h7_2_10;
    const double h16_2_4 = acc[416] + ABy * acc[192];
    const double h7_7_4 = h16_2_4 + ABy * h7_2_4;
    const double k7_7_4_1 = h7_7_10 + CDx * h7_7_4;
    const double h16_2_11 = acc[423] + ABy * acc[199];
    const double h7_7_11 = h16_2_11 + ABy * h7_2_11;
    const double k7_7_4_2 = h7_7_11 + CDy * h7_7_4;
    const double h16_2_12 = acc[424] + ABy * acc[200];
    const double h7_7_12 = h16_2_12 + ABy * h7_2_12;
    const double k7_7_4_3 = h7_7_12 + CDz * h7_7_4;
    const double h16_2_5 = acc[417] + ABy * acc[193];
    const double h7_7_5 = h16_2_5 + ABy * h7_2_5;
    const double k7_7_5_1 = h7_7_11 + CDx * h7_7_5;
    const double h16_2_13 = acc[425] + ABy * acc[201];
    const double h7_7_13 = h16_2_13 + ABy * h7_2_13;
    const double k7_7_5_2 = h7_7_13 + CDy * h7_7_5;
    const double h16_2_15 = acc[427] + ABy * acc[203];
    const double h7_7_15 = h16_2_15 + ABy * h7_2_15;
    const double k7_7_5_3 = h7_7_15 + CDz * h7_7_5;
    const double h16_2_6 = acc[418] + ABy * acc[194];
    const double h7_7_6 = h16_2_6 + ABy * h7_2_6;
    const double k7_7_6_1 = h7_7_12 + CDx * h7_7_6;
    const double k7_7_6_2 = h7_7_15 + CDy * h7_7_6;
    const double h16_2_14 = acc[426] + ABy * acc[202];
    const double h7_7_14 = h16_2_14 + ABy * h7_2_14;
    const double k7_7_6_3 = h7_7_14 + CDz * h7_7_6;
    const double h16_2_7 = acc[419] + ABy * acc[195];
    const double h7_7_7 = h16_2_7 + ABy * h7_2_7;
    const double k7_7_7_1 = h7_7_13 + CDx * h7_7_7;
    const double h16_2_16 = acc[428] + ABy * acc[204];
    const double h7_7_16 = h16_2_16 + ABy * h7_2_16;
    const double k7_7_7_2 = h7_7_16 + CDy * h7_7_7;
    const double h16_2_17 = acc[429] + ABy * acc[205];
    const double h7_7_17 = h16_2_17 + ABy * h7_2_17;
    const double k7_7_7_3 = h7_7_17 + CDz * h7_7_7;
    const double h16_2_8 = acc[420] + ABy * acc[196];
    const double h7_7_8 = h16_2_8 + ABy * h7_2_8;
    const double k7_7_8_1 = h7_7_15 + CDx * h7_7_8;
    const double k7_7_8_2 = h7_7_17 + CDy * h7_7_8;
    const double h16_2_18 = acc[430] + ABy * acc[206];
    const double h7_7_18 = h16_2_18 + ABy * h7_2_18;
    const double k7_7_8_3 = h7_7_18 + CDz * h7_7_8;
    const double h16_2_9 = acc[421] + ABy * acc[197];
    const double h7_7_9 = h16_2_9 + ABy * h7_2_9;
    const double k7_7_9_1 = h7_7_14 + CDx * h7_7_9;
    const double k7_7_9_2 = h7_7_18 + CDy * h7_7_9;
    const double h16_2_19 = acc[431] + ABy * acc[207];
    const double h7_7_19 = h16_2_19 + ABy * h7_2_19;
    const double k7_7_9_3 = h7_7_19 + CDz * h7_7_9;
    const double h16_3_10 = acc[438] + ABz * acc[198];
    const double h7_8_10 = h16_3_10 + ABy * h7_3_10;
    const double h16_3_4 = acc[432] + ABz * acc[192];
    const double h7_8_4 = h16_3_4 + ABy * h7_3_4;
    const double k7_8_4_1 = h7_8_10 + CDx * h7_8_4;
    const double h16_3_11 = acc[439] + ABz * acc[199];
    const double h7_8_11 = h16_3_11 + ABy * h7_3_11;
    const double k7_8_4_2 = h7_8_11 + CDy * h7_8_4;
    const double h16_3_12 = acc[440] + ABz * acc[200];
    const double h7_8_12 = h16_3_12 + ABy * h7_3_12;
    const double k7_8_4_3 = h7_8_12 + CDz * h7_8_4;
    const double h16_3_5 = acc[433] + ABz * acc[193];
    const double h7_8_5 = h16_3_5 + ABy * h7_3_5;
    const double k7_8_5_1 = h7_8_11 + CDx * h7_8_5;
    const double h16_3_13 = acc[441] + ABz * acc[201];
    const double h7_8_13 = h16_3_13 + ABy * h7_3_13;
    const double k7_8_5_2 = h7_8_13 + CDy * h7_8_5;
    const double h16_3_15 = acc[443] + ABz * acc[203];
    const double h7_8_15 = h16_3_15 + ABy * h7_3_15;
    const double k7_8_5_3 = h7_8_15 + CDz * h7_8_5;
    const double h16_3_6 = acc[434] + ABz * acc[194];
    const double h7_8_6 = h16_3_6 + ABy * h7_3_6;
    const double k7_8_6_1 = h7_8_12 + CDx * h7_8_6;
    const double k7_8_6_2 = h7_8_15 + CDy * h7_8_6;
    const double h16_3_14 = acc[442] + ABz * acc[202];
    const double h7_8_14 = h16_3_14 + ABy * h7_3_14;
    const double k7_8_6_3 = h7_8_14 + CDz * h7_8_6;
    const double h16_3_7 = acc[435] + ABz * acc[195];
    const double h7_8_7 = h16_3_7 + ABy * h7_3_7;
    const double k7_8_7_1 = h7_8_13 + CDx * h7_8_7;
    const double h16_3_16 = acc[444] + ABz * acc[204];
    const double h7_8_16 = h16_3_16 + ABy * h7_3_16;
    const double k7_8_7_2 = h7_8_16 + CDy * h7_8_7;
    const double h16_3_17 = acc[445] + ABz * acc[205];
    const double h7_8_17 = h16_3_17 + ABy * h7_3_17;
    const double k7_8_7_3 = h7_8_17 + CDz * h7_8_7;
    const double h16_3_8 = acc[436] + ABz * acc[196];
    const double h7_8_8 = h16_3_8 + ABy * h7_3_8;
    const double k7_8_8_1 = h7_8_15 + CDx * h7_8_8;
    const double k7_8_8_2 = h7_8_17 + CDy * h7_8_8;
    const double h16_3_18 = acc[446] + ABz * acc[206];
    const double h7_8_18 = h16_3_18 + ABy * h7_3_18;
    const double k7_8_8_3 = h7_8_18 + CDz * h7_8_8;
    const double h16_3_9 = acc[437] + ABz * acc[197];
    const double h7_8_9 = h16_3_9 + ABy * h7_3_9;
    const double k7_8_9_1 = h7_8_14 + CDx * h7_8_9;
    const double k7_8_9_2 = h7_8_18 + CDy * h7_8_9;
    const double h16_3_19 = acc[447] + ABz * acc[207];
    const double h7_8_19 = h16_3_19 + ABy * h7_3_19;
    const double k7_8_9_3 = h7_8_19 + CDz * h7_8_9;
    const double h17_3_10 = acc[454] + ABz * acc[214];
    const double h7_9_10 = h17_3_10 + ABz * h7_3_10;
    const double h17_3_4 = acc[448] + ABz * acc[208];
    const double h7_9_4 = h17_3_4 + ABz * h7_3_4;
    const double k7_9_4_1 = h7_9_10 + CDx * h7_9_4;
    const double h17_3_11 = acc[455] + ABz * acc[215];
    const double h7_9_11 = h17_3_11 + ABz * h7_3_11;
    const double k7_9_4_2 = h7_9_11 + CDy * h7_9_4;
    const double h17_3_12 = acc[456] + ABz * acc[216];
    const double h7_9_12 = h17_3_12 + ABz * h7_3_12;
    const double k7_9_4_3 = h7_9_12 + CDz * h7_9_4;
    const double h17_3_5 = acc[449] + ABz * acc[209];
    const double h7_9_5 = h17_3_5 + ABz * h7_3_5;
    const double k7_9_5_1 = h7_9_11 + CDx * h7_9_5;
    const double h17_3_13 = acc[457] + ABz * acc[217];
    const double h7_9_13 = h17_3_13 + ABz * h7_3_13;
    const double k7_9_5_2 = h7_9_13 + CDy * h7_9_5;
    const double h17_3_15 = acc[459] + ABz * acc[219];
    const double h7_9_15 = h17_3_15 + ABz * h7_3_15;
    const double k7_9_5_3 = h7_9_15 + CDz * h7_9_5;
    const double h17_3_6 = acc[450] + ABz * acc[210];
    const double h7_9_6 = h17_3_6 + ABz * h7_3_6;
    const double k7_9_6_1 = h7_9_12 + CDx * h7_9_6;
    const double k7_9_6_2 = h7_9_15 + CDy * h7_9_6;
    const double h17_3_14 = acc[458] + ABz * acc[218];
    const double h7_9_14 = h17_3_14 + ABz * h7_3_14;
    const double k7_9_6_3 = h7_9_14 + CDz * h7_9_6;
    const double h17_3_7 = acc[451] + ABz * acc[211];
    const double h7_9_7 = h17_3_7 + ABz * h7_3_7;
    const double k7_9_7_1 = h7_9_13 + CDx * h7_9_7;
    const double h17_3_16 = acc[460] + ABz * acc[220];
    const double h7_9_16 = h17_3_16 + ABz * h7_3_16;
    const double k7_9_7_2 = h7_9_16 + CDy * h7_9_7;
    const double h17_3_17 = acc[461] + ABz * acc[221];
    const double h7_9_17 = h17_3_17 + ABz * h7_3_17;
    const double k7_9_7_3 = h7_9_17 + CDz * h7_9_7;
    const double h17_3_8 = acc[452] + ABz * acc[212];
    const double h7_9_8 = h17_3_8 + ABz * h7_3_8;
    const double k7_9_8_1 = h7_9_15 + CDx * h7_9_8;
    const double k7_9_8_2 = h7_9_17 + CDy * h7_9_8;
    const double h17_3_18 = acc[462] + ABz * acc[222];
    const double h7_9_18 = h17_3_18 + ABz * h7_3_18;
    const double k7_9_8_3 = h7_9_18 + CDz * h7_9_8;
    const double h17_3_9 = acc[453] + ABz * acc[213];
    const double h7_9_9 = h17_3_9 + ABz * h7_3_9;
    const double k7_9_9_1 = h7_9_14 + CDx * h7_9_9;
    const double k7_9_9_2 = h7_9_18 + CDy * h7_9_9;
    const double h17_3_19 = acc[463] + ABz * acc[223];
    const double h7_9_19 = h17_3_19 + ABz * h7_3_19;
    const double k7_9_9_3 = h7_9_19 + CDz * h7_9_9;
    const double h15_1_10 = acc[326] + ABx * acc[182];
    const double h8_1_10 = acc[182] + ABx * acc[70];
    const double h8_4_10 = h15_1_10 + ABx * h8_1_10;
    const double h15_1_4 = acc[320] + ABx * acc[176];
    const double h8_1_4 = acc[176] + ABx * acc[64];
    const double h8_4_4 = h15_1_4 + ABx * h8_1_4;
    const double k8_4_4_1 = h8_4_10 + CDx * h8_4_4;
    const double h15_1_11 = acc[327] + ABx * acc[183];
    const double h8_1_11 = acc[183] + ABx * acc[71];
    const double h8_4_11 = h15_1_11 + ABx * h8_1_11;
    const double k8_4_4_2 = h8_4_11 + CDy * h8_4_4;
    const double h15_1_12 = acc[328] + ABx * acc[184];
    const double h8_1_12 = acc[184] + ABx * acc[72];
    const double h8_4_12 = h15_1_12 + ABx * h8_1_12;
    const double k8_4_4_3 = h8_4_12 + CDz * h8_4_4;
    const double h15_1_5 = acc[321] + ABx * acc[177];
    const double h8_1_5 = acc[177] + ABx * acc[65];
    const double h8_4_5 = h15_1_5 + ABx * h8_1_5;
    const double k8_4_5_1 = h8_4_11 + CDx * h8_4_5;
    const double h15_1_13 = acc[329] + ABx * acc[185];
    const double h8_1_13 = acc[185] + ABx * acc[73];
    const double h8_4_13 = h15_1_13 + ABx * h8_1_13;
    const double k8_4_5_2 = h8_4_13 + CDy * h8_4_5;
    const double h15_1_15 = acc[331] + ABx * acc[187];
    const double h8_1_15 = acc[187] + ABx * acc[75];
    const double h8_4_15 = h15_1_15 + ABx * h8_1_15;
    const double k8_4_5_3 = h8_4_15 + CDz * h8_4_5;
    const double h15_1_6 = acc[322] + ABx * acc[178];
    const double h8_1_6 = acc[178] + ABx * acc[66];
    const double h8_4_6 = h15_1_6 + ABx * h8_1_6;
    const double k8_4_6_1 = h8_4_12 + CDx * h8_4_6;
    const double k8_4_6_2 = h8_4_15 + CDy * h8_4_6;
    const double h15_1_14 = acc[330] + ABx * acc[186];
    const double h8_1_14 = acc[186] + ABx * acc[74];
    const double h8_4_14 = h15_1_14 + ABx * h8_1_14;
    const double k8_4_6_3 = h8_4_14 + CDz * h8_4_6;
    const double h15_1_7 = acc[323] + ABx * acc[179];
    const double h8_1_7 = acc[179] + ABx * acc[67];
    const double h8_4_7 = h15_1_7 + ABx * h8_1_7;
    const double k8_4_7_1 = h8_4_13 + CDx * h8_4_7;
    const double h15_1_16 = acc[332] + ABx * acc[188];
    const double h8_1_16 = acc[188] + ABx * acc[76];
    const double h8_4_16 = h15_1_16 + ABx * h8_1_16;
    const double k8_4_7_2 = h8_4_16 + CDy * h8_4_7;
    const double h15_1_17 = acc[333] + ABx * acc[189];
    const double h8_1_17 = acc[189] + ABx * acc[77];
    const double h8_4_17 = h15_1_17 + ABx * h8_1_17;
    const double k8_4_7_3 = h8_4_17 + CDz * h8_4_7;
    const double h15_1_8 = acc[324] + ABx * acc[180];
    const double h8_1_8 = acc[180] + ABx * acc[68];
    const double h8_4_8 = h15_1_8 + ABx * h8_1_8;
    const double k8_4_8_1 = h8_4_15 + CDx * h8_4_8;
    const double k8_4_8_2 = h8_4_17 + CDy * h8_4_8;
    const double h15_1_18 = acc[334] + ABx * acc[190];
    const double h8_1_18 = acc[190] + ABx * acc[78];
    const double h8_4_18 = h15_1_18 + ABx * h8_1_18;
    const double k8_4_8_3 = h8_4_18 + CDz * h8_4_8;
    const double h15_1_9 = acc[325] + ABx * acc[181];
    const double h8_1_9 = acc[181] + ABx * acc[69];
    const double h8_4_9 = h15_1_9 + ABx * h8_1_9;
    const double k8_4_9_1 = h8_4_14 + CDx * h8_4_9;
    const double k8_4_9_2 = h8_4_18 + CDy * h8_4_9;
    const double h15_1_19 = acc[335] + ABx * acc[191];
    const double h8_1_19 = acc[191] + ABx * acc[79];
    const double h8_4_19 = h15_1_19 + ABx * h8_1_19;
    const double k8_4_9_3 = h8_4_19 + CDz * h8_4_9;
    const double h8_2_10 = acc[214] + ABy * acc[70];
    const double h8_5_10 = h15_2_10 + ABx * h8_2_10;
    const double h8_2_4 = acc[208] + ABy * acc[64];
    const double h8_5_4 = h15_2_4 + ABx * h8_2_4;
    const double k8_5_4_1 = h8_5_10 + CDx * h8_5_4;
    const double h8_2_11 = acc[215] + ABy * acc[71];
    const double h8_5_11 = h15_2_11 + ABx * h8_2_11;
    const double k8_5_4_2 = h8_5_11 + CDy * h8_5_4;
    const double h8_2_12 = acc[216] + ABy * acc[72];
    const double h8_5_12 = h15_2_12 + ABx * h8_2_12;
    const double k8_5_4_3 = h8_5_12 + CDz * h8_5_4;
    const double h8_2_5 = acc[209] + ABy * acc[65];
    const double h8_5_5 = h15_2_5 + ABx * h8_2_5;
    const double k8_5_5_1 = h8_5_11 + CDx * h8_5_5;
    const double h8_2_13 = acc[217] + ABy * acc[73];
    const double h8_5_13 = h15_2_13 + ABx * h8_2_13;
    const double k8_5_5_2 = h8_5_13 + CDy * h8_5_5;
    const double h8_2_15 = acc[219] + ABy * acc[75];
    const double h8_5_15 = h15_2_15 + ABx * h8_2_15;
    const double k8_5_5_3 = h8_5_15 + CDz * h8_5_5;
    const double h8_2_6 = acc[210] + ABy * acc[66];
    const double h8_5_6 = h15_2_6 + ABx * h8_2_6;
    const double k8_5_6_1 = h8_5_12 + CDx * h8_5_6;
    const double k8_5_6_2 = h8_5_15 + CDy * h8_5_6;
    const double h8_2_14 = acc[218] + ABy * acc[74];
    const double h8_5_14 = h15_2_14 + ABx * h8_2_14;
    const double k8_5_6_3 = h8_5_14 + CDz * h8_5_6;
    const double h8_2_7 = acc[211] + ABy * acc[67];
    const double h8_5_7 = h15_2_7 + ABx * h8_2_7;
    const double k8_5_7_1 = h8_5_13 + CDx * h8_5_7;
    const double h8_2_16 = acc[220] + ABy * acc[76];
    const double h8_5_16 = h15_2_16 + ABx * h8_2_16;
    const double k8_5_7_2 = h8_5_16 + CDy * h8_5_7;
    const double h8_2_17 = acc[221] + ABy * acc[77];
    const double h8_5_17 = h15_2_17 + ABx * h8_2_17;
    const double k8_5_7_3 = h8_5_17 + CDz * h8_5_7;
    const double h8_2_8 = acc[212] + ABy * acc[68];
    const double h8_5_8 = h15_2_8 + ABx * h8_2_8;
    const double k8_5_8_1 = h8_5_15 + CDx * h8_5_8;
    const double k8_5_8_2 = h8_5_17 + CDy * h8_5_8;
    const double h8_2_18 = acc[222] + ABy * acc[78];
    const double h8_5_18 = h15_2_18 + ABx * h8_2_18;
    const double k8_5_8_3 = h8_5_18 + CDz * h8_5_8;
    const double h8_2_9 = acc[213] + ABy * acc[69];
    const double h8_5_9 = h15_2_9 + ABx * h8_2_9;
    const double k8_5_9_1 = h8_5_14 + CDx * h8_5_9;
    const double k8_5_9_2 = h8_5_18 + CDy * h8_5_9;
    const double h8_2_19 = acc[223] + ABy * acc[79];
    const double h8_5_19 = h15_2_19 + ABx * h8_2_19;
    const double k8_5_9_3 = h8_5_19 + CDz * h8_5_9;
    const double h8_3_10 = acc[230] + ABz * acc[70];
    const double h8_6_10 = h15_3_10 + ABx * h8_3_10;
    const double h8_3_4 = acc[224] + ABz * acc[64];
    const double h8_6_4 = h15_3_4 + ABx * h8_3_4;
    const double k8_6_4_1 = h8_6_10 + CDx * h8_6_4;
    const double h8_3_11 = acc[231] + ABz * acc[71];
    const double h8_6_11 = h15_3_11 + ABx * h8_3_11;
    const double k8_6_4_2 = h8_6_11 + CDy * h8_6_4;
    const double h8_3_12 = acc[232] + ABz * acc[72];
    const double h8_6_12 = h15_3_12 + ABx * h8_3_12;
    const double k8_6_4_3 = h8_6_12 + CDz * h8_6_4;
    const double h8_3_5 = acc[225] + ABz * acc[65];
    const double h8_6_5 = h15_3_5 + ABx * h8_3_5;
    const double k8_6_5_1 = h8_6_11 + CDx * h8_6_5;
    const double h8_3_13 = acc[233] + ABz * acc[73];
    const double h8_6_13 = h15_3_13 + ABx * h8_3_13;
    const double k8_6_5_2 = h8_6_13 + CDy * h8_6_5;
    const double h8_3_15 = acc[235] + ABz * acc[75];
    const double h8_6_15 = h15_3_15 + ABx * h8_3_15;
    const double k8_6_5_3 = h8_6_15 + CDz * h8_6_5;
    const double h8_3_6 = acc[226] + ABz * acc[66];
    const double h8_6_6 = h15_3_6 + ABx * h8_3_6;
    const double k8_6_6_1 = h8_6_12 + CDx * h8_6_6;
    const double k8_6_6_2 = h8_6_15 + CDy * h8_6_6;
    const double h8_3_14 = acc[234] + ABz * acc[74];
    const double h8_6_14 = h15_3_14 + ABx * h8_3_14;
    const double k8_6_6_3 = h8_6_14 + CDz * h8_6_6;
    const double h8_3_7 = acc[227] + ABz * acc[67];
    const double h8_6_7 = h15_3_7 + ABx * h8_3_7;
    const double k8_6_7_1 = h8_6_13 + CDx * h8_6_7;
    const double h8_3_16 = acc[236] + ABz * acc[76];
    const double h8_6_16 = h15_3_16 + ABx * h8_3_16;
    const double k8_6_7_2 = h8_6_16 + CDy * h8_6_7;
    const double h8_3_17 = acc[237] + ABz * acc[77];
    const double h8_6_17 = h15_3_17 + ABx * h8_3_17;
    const double k8_6_7_3 = h8_6_17 + CDz * h8_6_7;
    const double h8_3_8 = acc[228] + ABz * acc[68];
    const double h8_6_8 = h15_3_8 + ABx * h8_3_8;
    const double k8_6_8_1 = h8_6_15 + CDx * h8_6_8;
    const double k8_6_8_2 = h8_6_17 + CDy * h8_6_8;
    const double h8_3_18 = acc[238] + ABz * acc[78];
    const double h8_6_18 = h15_3_18 + ABx * h8_3_18;
    const double k8_6_8_3 = h8_6_18 + CDz * h8_6_8;
    const double h8_3_9 = acc[229] + ABz * acc[69];
    const double h8_6_9 = h15_3_9 + ABx * h8_3_9;
    const double k8_6_9_1 = h8_6_14 + CDx * h8_6_9;
    const double k8_6_9_2 = h8_6_18 + CDy * h8_6_9;
    const double h8_3_19 = acc[239] + ABz * acc[79];
    const double h8_6_19 = h15_3_19 + ABx * h8_3_19;
    const double k8_6_9_3 = h8_6_19 + CDz * h8_6_9;
    const double h17_2_10 = acc[438] + ABy * acc[214];
    const double h8_7_10 = h17_2_10 + ABy * h8_2_10;
    const double h17_2_4 = acc[432] + ABy * acc[208];
    const double h8_7_4 = h17_2_4 + ABy * h8_2_4;
    const double k8_7_4_1 = h8_7_10 + CDx * h8_7_4;
    const double h17_2_11 = acc[439] + ABy * acc[215];
    const double h8_7_11 = h17_2_11 + ABy * h8_2_11;
    const double k8_7_4_2 = h8_7_11 + CDy * h8_7_4;
    const double h17_2_12 = acc[440] + ABy * acc[216];
    const double h8_7_12 = h17_2_12 + ABy * h8_2_12;
    const double k8_7_4_3 = h8_7_12 + CDz * h8_7_4;
    const double h17_2_5 = acc[433] + ABy * acc[209];
    const double h8_7_5 = h17_2_5 + ABy * h8_2_5;
    const double k8_7_5_1 = h8_7_11 + CDx * h8_7_5;
    const double h17_2_13 = acc[441] + ABy * acc[217];
    const double h8_7_13 = h17_2_13 + ABy * h8_2_13;
    const double k8_7_5_2 = h8_7_13 + CDy * h8_7_5;
    const double h17_2_15 = acc[443] + ABy * acc[219];
    const double h8_7_15 = h17_2_15 + ABy * h8_2_15;
    const double k8_7_5_3 = h8_7_15 + CDz * h8_7_5;
    const double h17_2_6 = acc[434] + ABy * acc[210];
    const double h8_7_6 = h17_2_6 + ABy * h8_2_6;
    const double k8_7_6_1 = h8_7_12 + CDx * h8_7_6;
    const double k8_7_6_2 = h8_7_15 + CDy * h8_7_6;
    const double h17_2_14 = acc[442] + ABy * acc[218];
    const double h8_7_14 = h17_2_14 + ABy * h8_2_14;
    const double k8_7_6_3 = h8_7_14 + CDz * h8_7_6;
    const double h17_2_7 = acc[435] + ABy * acc[211];
    const double h8_7_7 = h17_2_7 + ABy * h8_2_7;
    const double k8_7_7_1 = h8_7_13 + CDx * h8_7_7;
    const double h17_2_16 = acc[444] + ABy * acc[220];
    const double h8_7_16 = h17_2_16 + ABy * h8_2_16;
    const double k8_7_7_2 = h8_7_16 + CDy * h8_7_7;
    const double h17_2_17 = acc[445] + ABy * acc[221];
    const double h8_7_17 = h17_2_17 + ABy * h8_2_17;
    const double k8_7_7_3 = h8_7_17 + CDz * h8_7_7;
    const double h17_2_8 = acc[436] + ABy * acc[212];
    const double h8_7_8 = h17_2_8 + ABy * h8_2_8;
    const double k8_7_8_1 = h8_7_15 + CDx * h8_7_8;
    const double k8_7_8_2 = h8_7_17 + CDy * h8_7_8;
    const double h17_2_18 = acc[446] + ABy * acc[222];
    const double h8_7_18 = h17_2_18 + ABy * h8_2_18;
    const double k8_7_8_3 = h8_7_18 + CDz * h8_7_8;
    const double h17_2_9 = acc[437] + ABy * acc[213];
    const double h8_7_9 = h17_2_9 + ABy * h8_2_9;
    const double k8_7_9_1 = h8_7_14 + CDx * h8_7_9;
    const double k8_7_9_2 = h8_7_18 + CDy * h8_7_9;
    const double h17_2_19 = acc[447] + ABy * acc[223];
    const double h8_7_19 = h17_2_19 + ABy * h8_2_19;
    const double k8_7_9_3 = h8_7_19 + CDz * h8_7_9;
    const double h8_8_10 = h17_3_10 + ABy * h8_3_10;
    const double h8_8_4 = h17_3_4 + ABy * h8_3_4;
    const double k8_8_4_1 = h8_8_10 + CDx * h8_8_4;
    const double h8_8_11 = h17_3_11 + ABy * h8_3_11;
    const double k8_8_4_2 = h8_8_11 + CDy * h8_8_4;
    const double h8_8_12 = h17_3_12 + ABy * h8_3_12;
    const double k8_8_4_3 = h8_8_12 + CDz * h8_8_4;
    const double h8_8_5 = h17_3_5 + ABy * h8_3_5;
    const double k8_8_5_1 = h8_8_11 + CDx * h8_8_5;
    const double h8_8_13 = h17_3_13 + ABy * h8_3_13;
    const double k8_8_5_2 = h8_8_13 + CDy * h8_8_5;
    const double h8_8_15 = h17_3_15 + ABy * h8_3_15;
    const double k8_8_5_3 = h8_8_15 + CDz * h8_8_5;
    const double h8_8_6 = h17_3_6 + ABy * h8_3_6;
    const double k8_8_6_1 = h8_8_12 + CDx * h8_8_6;
    const double k8_8_6_2 = h8_8_15 + CDy * h8_8_6;
    const double h8_8_14 = h17_3_14 + ABy * h8_3_14;
    const double k8_8_6_3 = h8_8_14 + CDz * h8_8_6;
    const double h8_8_7 = h17_3_7 + ABy * h8_3_7;
    const double k8_8_7_1 = h8_8_13 + CDx * h8_8_7;
    const double h8_8_16 = h17_3_16 + ABy * h8_3_16;
    const double k8_8_7_2 = h8_8_16 + CDy * h8_8_7;
    const double h8_8_17 = h17_3_17 + ABy * h8_3_17;
    const double k8_8_7_3 = h8_8_17 + CDz * h8_8_7;
    const double h8_8_8 = h17_3_8 + ABy * h8_3_8;
    const double k8_8_8_1 = h8_8_15 + CDx * h8_8_8;
    const double k8_8_8_2 = h8_8_17 + CDy * h8_8_8;
    const double h8_8_18 = h17_3_18 + ABy * h8_3_18;
    const double k8_8_8_3 = h8_8_18 + CDz * h8_8_8;
    const double h8_8_9 = h17_3_9 + ABy * h8_3_9;
    const double k8_8_9_1 = h8_8_14 + CDx * h8_8_9;
    const double k8_8_9_2 = h8_8_18 + CDy * h8_8_9;
    const double h8_8_19 = h17_3_19 + ABy * h8_3_19;
    const double k8_8_9_3 = h8_8_19 + CDz * h8_8_9;
    const double h18_3_10 = acc[470] + ABz * acc[230];
    const double h8_9_10 = h18_3_10 + ABz * h8_3_10;
    const double h18_3_4 = acc[464] + ABz * acc[224];
    const double h8_9_4 = h18_3_4 + ABz * h8_3_4;
    const double k8_9_4_1 = h8_9_10 + CDx * h8_9_4;
    const double h18_3_11 = acc[471] + ABz * acc[231];
    const double h8_9_11 = h18_3_11 + ABz * h8_3_11;
    const double k8_9_4_2 = h8_9_11 + CDy * h8_9_4;
    const double h18_3_12 = acc[472] + ABz * acc[232];
    const double h8_9_12 = h18_3_12 + ABz * h8_3_12;
    const double k8_9_4_3 = h8_9_12 + CDz * h8_9_4;
    const double h18_3_5 = acc[465] + ABz * acc[225];
    const double h8_9_5 = h18_3_5 + ABz * h8_3_5;
    const double k8_9_5_1 = h8_9_11 + CDx * h8_9_5;
    const double h18_3_13 = acc[473] + ABz * acc[233];
    const double h8_9_13 = h18_3_13 + ABz * h8_3_13;
    const double k8_9_5_2 = h8_9_13 + CDy * h8_9_5;
    const double h18_3_15 = acc[475] + ABz * acc[235];
    const double h8_9_15 = h18_3_15 + ABz * h8_3_15;
    const double k8_9_5_3 = h8_9_15 + CDz * h8_9_5;
    const double h18_3_6 = acc[466] + ABz * acc[226];
    const double h8_9_6 = h18_3_6 + ABz * h8_3_6;
    const double k8_9_6_1 = h8_9_12 + CDx * h8_9_6;
    const double k8_9_6_2 = h8_9_15 + CDy * h8_9_6;
    const double h18_3_14 = acc[474] + ABz * acc[234];
    const double h8_9_14 = h18_3_14 + ABz * h8_3_14;
    const double k8_9_6_3 = h8_9_14 + CDz * h8_9_6;
    const double h18_3_7 = acc[467] + ABz * acc[227];
    const double h8_9_7 = h18_3_7 + ABz * h8_3_7;
    const double k8_9_7_1 = h8_9_13 + CDx * h8_9_7;
    const double h18_3_16 = acc[476] + ABz * acc[236];
    const double h8_9_16 = h18_3_16 + ABz * h8_3_16;
    const double k8_9_7_2 = h8_9_16 + CDy * h8_9_7;
    const double h18_3_17 = acc[477] + ABz * acc[237];
    const double h8_9_17 = h18_3_17 + ABz * h8_3_17;
    const double k8_9_7_3 = h8_9_17 + CDz * h8_9_7;
    const double h18_3_8 = acc[468] + ABz * acc[228];
    const double h8_9_8 = h18_3_8 + ABz * h8_3_8;
    const double k8_9_8_1 = h8_9_15 + CDx * h8_9_8;
    const double k8_9_8_2 = h8_9_17 + CDy * h8_9_8;
    const double h18_3_18 = acc[478] + ABz * acc[238];
    const double h8_9_18 = h18_3_18 + ABz * h8_3_18;
    const double k8_9_8_3 = h8_9_18 + CDz * h8_9_8;
    const double h18_3_9 = acc[469] + ABz * acc[229];
    const double h8_9_9 = h18_3_9 + ABz * h8_3_9;
    const double k8_9_9_1 = h8_9_14 + CDx * h8_9_9;
    const double k8_9_9_2 = h8_9_18 + CDy * h8_9_9;
    const double h18_3_19 = acc[479] + ABz * acc[239];
    const double h8_9_19 = h18_3_19 + ABz * h8_3_19;
    const double k8_9_9_3 = h8_9_19 + CDz * h8_9_9;
    const double h14_1_10 = acc[342] + ABx * acc[166];
    const double h9_1_10 = acc[166] + ABx * acc[86];
    const double h9_4_10 = h14_1_10 + ABx * h9_1_10;
    const double h14_1_4 = acc[336] + ABx * acc[160];
    const double h9_1_4 = acc[160] + ABx * acc[80];
    const double h9_4_4 = h14_1_4 + ABx * h9_1_4;
    const double k9_4_4_1 = h9_4_10 + CDx * h9_4_4;
    const double h14_1_11 = acc[343] + ABx * acc[167];
    const double h9_1_11 = acc[167] + ABx * acc[87];
    const double h9_4_11 = h14_1_11 + ABx * h9_1_11;
    const double k9_4_4_2 = h9_4_11 + CDy * h9_4_4;
    const double h14_1_12 = acc[344] + ABx * acc[168];
    const double h9_1_12 = acc[168] + ABx * acc[88];
    const double h9_4_12 = h14_1_12 + ABx * h9_1_12;
    const double k9_4_4_3 = h9_4_12 + CDz * h9_4_4;
    const double h14_1_5 = acc[337] + ABx * acc[161];
    const double h9_1_5 = acc[161] + ABx * acc[81];
    const double h9_4_5 = h14_1_5 + ABx * h9_1_5;
    const double k9_4_5_1 = h9_4_11 + CDx * h9_4_5;
    const double h14_1_13 = acc[345] + ABx * acc[169];
    const double h9_1_13 = acc[169] + ABx * acc[89];
    const double h9_4_13 = h14_1_13 + ABx * h9_1_13;
    const double k9_4_5_2 = h9_4_13 + CDy * h9_4_5;
    const double h14_1_15 = acc[347] + ABx * acc[171];
    const double h9_1_15 = acc[171] + ABx * acc[91];
    const double h9_4_15 = h14_1_15 + ABx * h9_1_15;
    const double k9_4_5_3 = h9_4_15 + CDz * h9_4_5;
    const double h14_1_6 = acc[338] + ABx * acc[162];
    const double h9_1_6 = acc[162] + ABx * acc[82];
    const double h9_4_6 = h14_1_6 + ABx * h9_1_6;
    const double k9_4_6_1 = h9_4_12 + CDx * h9_4_6;
    const double k9_4_6_2 = h9_4_15 + CDy * h9_4_6;
    const double h14_1_14 = acc[346] + ABx * acc[170];
    const double h9_1_14 = acc[170] + ABx * acc[90];
    const double h9_4_14 = h14_1_14 + ABx * h9_1_14;
    const double k9_4_6_3 = h9_4_14 + CDz * h9_4_6;
    const double h14_1_7 = acc[339] + ABx * acc[163];
    const double h9_1_7 = acc[163] + ABx * acc[83];
    const double h9_4_7 = h14_1_7 + ABx * h9_1_7;
    const double k9_4_7_1 = h9_4_13 + CDx * h9_4_7;
    const double h14_1_16 = acc[348] + ABx * acc[172];
    const double h9_1_16 = acc[172] + ABx * acc[92];
    const double h9_4_16 = h14_1_16 + ABx * h9_1_16;
    const double k9_4_7_2 = h9_4_16 + CDy * h9_4_7;
    const double h14_1_17 = acc[349] + ABx * acc[173];
    const double h9_1_17 = acc[173] + ABx * acc[93];
    const double h9_4_17 = h14_1_17 + ABx * h9_1_17;
    const double k9_4_7_3 = h9_4_17 + CDz * h9_4_7;
    const double h14_1_8 = acc[340] + ABx * acc[164];
    const double h9_1_8 = acc[164] + ABx * acc[84];
    const double h9_4_8 = h14_1_8 + ABx * h9_1_8;
    const double k9_4_8_1 = h9_4_15 + CDx * h9_4_8;
    const double k9_4_8_2 = h9_4_17 + CDy * h9_4_8;
    const double h14_1_18 = acc[350] + ABx * acc[174];
    const double h9_1_18 = acc[174] + ABx * acc[94];
    const double h9_4_18 = h14_1_18 + ABx * h9_1_18;
    const double k9_4_8_3 = h9_4_18 + CDz * h9_4_8;
    const double h14_1_9 = acc[341] + ABx * acc[165];
    const double h9_1_9 = acc[165] + ABx * acc[85];
    const double h9_4_9 = h14_1_9 + ABx * h9_1_9;
    const double k9_4_9_1 = h9_4_14 + CDx * h9_4_9;
    const double k9_4_9_2 = h9_4_18 + CDy * h9_4_9;
    const double h14_1_19 = acc[351] + ABx * acc[175];
    const double h9_1_19 = acc[175] + ABx * acc[95];
    const double h9_4_19 = h14_1_19 + ABx * h9_1_19;
    const double k9_4_9_3 = h9_4_19 + CDz * h9_4_9;
    const double h14_2_10 = acc[390] + ABy * acc[166];
    const double h9_2_10 = acc[230] + ABy * acc[86];
    const double h9_5_10 = h14_2_10 + ABx * h9_2_10;
    const double h14_2_4 = acc[384] + ABy * acc[160];
    const double h9_2_4 = acc[224] + ABy * acc[80];
    const double h9_5_4 = h14_2_4 + ABx * h9_2_4;
    const double k9_5_4_1 = h9_5_10 + CDx * h9_5_4;
    const double h14_2_11 = acc[391] + ABy * acc[167];
    const double h9_2_11 = acc[231] + ABy * acc[87];
    const double h9_5_11 = h14_2_11 + ABx * h9_2_11;
    const double k9_5_4_2 = h9_5_11 + CDy * h9_5_4;
    const double h14_2_12 = acc[392] + ABy * acc[168];
    const double h9_2_12 = acc[232] + ABy * acc[88];
    const double h9_5_12 = h14_2_12 + ABx * h9_2_12;
    const double k9_5_4_3 = h9_5_12 + CDz * h9_5_4;
    const double h14_2_5 = acc[385] + ABy * acc[161];
    const double h9_2_5 = acc[225] + ABy * acc[81];
    const double h9_5_5 = h14_2_5 + ABx * h9_2_5;
    const double k9_5_5_1 = h9_5_11 + CDx * h9_5_5;
    const double h14_2_13 = acc[393] + ABy * acc[169];
    const double h9_2_13 = acc[233] + ABy * acc[89];
    const double h9_5_13 = h14_2_13 + ABx * h9_2_13;
    const double k9_5_5_2 = h9_5_13 + CDy * h9_5_5;
    const double h14_2_15 = acc[395] + ABy * acc[171];
    const double h9_2_15 = acc[235] + ABy * acc[91];
    const double h9_5_15 = h14_2_15 + ABx * h9_2_15;
    const double k9_5_5_3 = h9_5_15 + CDz * h9_5_5;
    const double h14_2_6 = acc[386] + ABy * acc[162];
    const double h9_2_6 = acc[226] + ABy * acc[82];
    const double h9_5_6 = h14_2_6 + ABx * h9_2_6;
    const double k9_5_6_1 = h9_5_12 + CDx * h9_5_6;
    const double k9_5_6_2 = h9_5_15 + CDy * h9_5_6;
    const double h14_2_14 = acc[394] + ABy * acc[170];
    const double h9_2_14 = acc[234] + ABy * acc[90];
    const double h9_5_14 = h14_2_14 + ABx * h9_2_14;
    const double k9_5_6_3 = h9_5_14 + CDz * h9_5_6;
    const double h14_2_7 = acc[387] + ABy * acc[163];
    const double h9_2_7 = acc[227] + ABy * acc[83];
    const double h9_5_7 = h14_2_7 + ABx * h9_2_7;
    const double k9_5_7_1 = h9_5_13 + CDx * h9_5_7;
    const double h14_2_16 = acc[396] + ABy * acc[172];
    const double h9_2_16 = acc[236] + ABy * acc[92];
    const double h9_5_16 = h14_2_16 + ABx * h9_2_16;
    const double k9_5_7_2 = h9_5_16 + CDy * h9_5_7;
    const double h14_2_17 = acc[397] + ABy * acc[173];
    const double h9_2_17 = acc[237] + ABy * acc[93];
    const double h9_5_17 = h14_2_17 + ABx * h9_2_17;
    const double k9_5_7_3 = h9_5_17 + CDz * h9_5_7;
    const double h14_2_8 = acc[388] + ABy * acc[164];
    const double h9_2_8 = acc[228] + ABy * acc[84];
    const double h9_5_8 = h14_2_8 + ABx * h9_2_8;
    const double k9_5_8_1 = h9_5_15 + CDx * h9_5_8;
    const double k9_5_8_2 = h9_5_17 + CDy * h9_5_8;
    const double h14_2_18 = acc[398] + ABy * acc[174];
    const double h9_2_18 = acc[238] + ABy * acc[94];
    const double h9_5_18 = h14_2_18 + ABx * h9_2_18;
    const double k9_5_8_3 = h9_5_18 + CDz * h9_5_8;
    const double h14_2_9 = acc[389] + ABy * acc[165];
    const double h9_2_9 = acc[229] + ABy * acc[85];
    const double h9_5_9 = h14_2_9 + ABx * h9_2_9;
    const double k9_5_9_1 = h9_5_14 + CDx * h9_5_9;
    const double k9_5_9_2 = h9_5_18 + CDy * h9_5_9;
    const double h14_2_19 = acc[399] + ABy * acc[175];
    const double h9_2_19 = acc[239] + ABy * acc[95];
    const double h9_5_19 = h14_2_19 + ABx * h9_2_19;
    const double k9_5_9_3 = h9_5_19 + CDz * h9_5_9;
    const double h9_3_10 = acc[246] + ABz * acc[86];
    const double h9_6_10 = h14_3_10 + ABx * h9_3_10;
    const double h9_3_4 = acc[240] + ABz * acc[80];
    const double h9_6_4 = h14_3_4 + ABx * h9_3_4;
    const double k9_6_4_1 = h9_6_10 + CDx * h9_6_4;
    const double h9_3_11 = acc[247] + ABz * acc[87];
    const double h9_6_11 = h14_3_11 + ABx * h9_3_11;
    const double k9_6_4_2 = h9_6_11 + CDy * h9_6_4;
    const double h9_3_12 = acc[248] + ABz * acc[88];
    const double h9_6_12 = h14_3_12 + ABx * h9_3_12;
    const double k9_6_4_3 = h9_6_12 + CDz * h9_6_4;
    const double h9_3_5 = acc[241] + ABz * acc[81];
    const double h9_6_5 = h14_3_5 + ABx * h9_3_5;
    const double k9_6_5_1 = h9_6_11 + CDx * h9_6_5;
    const double h9_3_13 = acc[249] + ABz * acc[89];
    const double h9_6_13 = h14_3_13 + ABx * h9_3_13;
    const double k9_6_5_2 = h9_6_13 + CDy * h9_6_5;
    const double h9_3_15 = acc[251] + ABz * acc[91];
    const double h9_6_15 = h14_3_15 + ABx * h9_3_15;
    const double k9_6_5_3 = h9_6_15 + CDz * h9_6_5;
    const double h9_3_6 = acc[242] + ABz * acc[82];
    const double h9_6_6 = h14_3_6 + ABx * h9_3_6;
    const double k9_6_6_1 = h9_6_12 + CDx * h9_6_6;
    const double k9_6_6_2 = h9_6_15 + CDy * h9_6_6;
    const double h9_3_14 = acc[250] + ABz * acc[90];
    const double h9_6_14 = h14_3_14 + ABx * h9_3_14;
    const double k9_6_6_3 = h9_6_14 + CDz * h9_6_6;
    const double h9_3_7 = acc[243] + ABz * acc[83];
    const double h9_6_7 = h14_3_7 + ABx * h9_3_7;
    const double k9_6_7_1 = h9_6_13 + CDx * h9_6_7;
    const double h9_3_16 = acc[252] + ABz * acc[92];
    const double h9_6_16 = h14_3_16 + ABx * h9_3_16;
    const double k9_6_7_2 = h9_6_16 + CDy * h9_6_7;
    const double h9_3_17 = acc[253] + ABz * acc[93];
    const double h9_6_17 = h14_3_17 + ABx * h9_3_17;
    const double k9_6_7_3 = h9_6_17 + CDz * h9_6_7;
    const double h9_3_8 = acc[244] + ABz * acc[84];
    const double h9_6_8 = h14_3_8 + ABx * h9_3_8;
    const double k9_6_8_1 = h9_6_15 + CDx * h9_6_8;
    const double k9_6_8_2 = h9_6_17 + CDy * h9_6_8;
    const double h9_3_18 = acc[254] + ABz * acc[94];
    const double h9_6_18 = h14_3_18 + ABx * h9_3_18;
    const double k9_6_8_3 = h9_6_18 + CDz * h9_6_8;
    const double h9_3_9 = acc[245] + ABz * acc[85];
    const double h9_6_9 = h14_3_9 + ABx * h9_3_9;
    const double k9_6_9_1 = h9_6_14 + CDx * h9_6_9;
    const double k9_6_9_2 = h9_6_18 + CDy * h9_6_9;
    const double h9_3_19 = acc[255] + ABz * acc[95];
    const double h9_6_19 = h14_3_19 + ABx * h9_3_19;
    const double k9_6_9_3 = h9_6_19 + CDz * h9_6_9;
    const double h18_2_10 = acc[454] + ABy * acc[230];
    const double h9_7_10 = h18_2_10 + ABy * h9_2_10;
    const double h18_2_4 = acc[448] + ABy * acc[224];
    const double h9_7_4 = h18_2_4 + ABy * h9_2_4;
    const double k9_7_4_1 = h9_7_10 + CDx * h9_7_4;
    const double h18_2_11 = acc[455] + ABy * acc[231];
    const double h9_7_11 = h18_2_11 + ABy * h9_2_11;
    const double k9_7_4_2 = h9_7_11 + CDy * h9_7_4;
    const double h18_2_12 = acc[456] + ABy * acc[232];
    const double h9_7_12 = h18_2_12 + ABy * h9_2_12;
    const double k9_7_4_3 = h9_7_12 + CDz * h9_7_4;
    const double h18_2_5 = acc[449] + ABy * acc[225];
    const double h9_7_5 = h18_2_5 + ABy * h9_2_5;
    const double k9_7_5_1 = h9_7_11 + CDx * h9_7_5;
    const double h18_2_13 = acc[457] + ABy * acc[233];
    const double h9_7_13 = h18_2_13 + ABy * h9_2_13;
    const double k9_7_5_2 = h9_7_13 + CDy * h9_7_5;
    const double h18_2_15 = acc[459] + ABy * acc[235];
    const double h9_7_15 = h18_2_15 + ABy * h9_2_15;
    const double k9_7_5_3 = h9_7_15 + CDz * h9_7_5;
    const double h18_2_6 = acc[450] + ABy * acc[226];
    const double h9_7_6 = h18_2_6 + ABy * h9_2_6;
    const double k9_7_6_1 = h9_7_12 + CDx * h9_7_6;
    const double k9_7_6_2 = h9_7_15 + CDy * h9_7_6;
    const double h18_2_14 = acc[458] + ABy * acc[234];
    const double h9_7_14 = h18_2_14 + ABy * h9_2_14;
    const double k9_7_6_3 = h9_7_14 + CDz * h9_7_6;
    const double h18_2_7 = acc[451] + ABy * acc[227];
    const double h9_7_7 = h18_2_7 + ABy * h9_2_7;
    const double k9_7_7_1 = h9_7_13 + CDx * h9_7_7;
    const double h18_2_16 = acc[460] + ABy * acc[236];
    const double h9_7_16 = h18_2_16 + ABy * h9_2_16;
    const double k9_7_7_2 = h9_7_16 + CDy * h9_7_7;
    const double h18_2_17 = acc[461] + ABy * acc[237];
    const double h9_7_17 = h18_2_17 + ABy * h9_2_17;
    const double k9_7_7_3 = h9_7_17 + CDz * h9_7_7;
    const double h18_2_8 = acc[452] + ABy * acc[228];
    const double h9_7_8 = h18_2_8 + ABy * h9_2_8;
    const double k9_7_8_1 = h9_7_15 + CDx * h9_7_8;
    const double k9_7_8_2 = h9_7_17 + CDy * h9_7_8;
    const double h18_2_18 = acc[462] + ABy * acc[238];
    const double h9_7_18 = h18_2_18 + ABy * h9_2_18;
    const double k9_7_8_3 = h9_7_18 + CDz * h9_7_8;
    const double h18_2_9 = acc[453] + ABy * acc[229];
    const double h9_7_9 = h18_2_9 + ABy * h9_2_9;
    const double k9_7_9_1 = h9_7_14 + CDx * h9_7_9;
    const double k9_7_9_2 = h9_7_18 + CDy * h9_7_9;
    const double h18_2_19 = acc[463] + ABy * acc[239];
    const double h9_7_19 = h18_2_19 + ABy * h9_2_19;
    const double k9_7_9_3 = h9_7_19 + CDz * h9_7_9;
    const double h9_8_10 = h18_3_10 + ABy * h9_3_10;
    const double h9_8_4 = h18_3_4 + ABy * h9_3_4;
    const double k9_8_4_1 = h9_8_10 + CDx * h9_8_4;
    const double h9_8_11 = h18_3_11 + ABy * h9_3_11;
    const double k9_8_4_2 = h9_8_11 + CDy * h9_8_4;
    const double h9_8_12 = h18_3_12 + ABy * h9_3_12;
    const double k9_8_4_3 = h9_8_12 + CDz * h9_8_4;
    const double h9_8_5 = h18_3_5 + ABy * h9_3_5;
    const double k9_8_5_1 = h9_8_11 + CDx * h9_8_5;
    const double h9_8_13 = h18_3_13 + ABy * h9_3_13;
    const double k9_8_5_2 = h9_8_13 + CDy * h9_8_5;
    const double h9_8_15 = h18_3_15 + ABy * h9_3_15;
    const double k9_8_5_3 = h9_8_15 + CDz * h9_8_5;
    const double h9_8_6 = h18_3_6 + ABy * h9_3_6;
    const double k9_8_6_1 = h9_8_12 + CDx * h9_8_6;
    const double k9_8_6_2 = h9_8_15 + CDy * h9_8_6;
    const double h9_8_14 = h18_3_14 + ABy * h9_3_14;
    const double k9_8_6_3 = h9_8_14 + CDz * h9_8_6;
    const double h9_8_7 = h18_3_7 + ABy * h9_3_7;
    const double k9_8_7_1 = h9_8_13 + CDx * h9_8_7;
    const double h9_8_16 = h18_3_16 + ABy * h9_3_16;
    const double k9_8_7_2 = h9_8_16 + CDy * h9_8_7;
    const double h9_8_17 = h18_3_17 + ABy * h9_3_17;
    const double k9_8_7_3 = h9_8_17 + CDz * h9_8_7;
    const double h9_8_8 = h18_3_8 + ABy * h9_3_8;
    const double k9_8_8_1 = h9_8_15 + CDx * h9_8_8;
    const double k9_8_8_2 = h9_8_17 + CDy * h9_8_8;
    const double h9_8_18 = h18_3_18 + ABy * h9_3_18;
    const double k9_8_8_3 = h9_8_18 + CDz * h9_8_8;
    const double h9_8_9 = h18_3_9 + ABy * h9_3_9;
    const double k9_8_9_1 = h9_8_14 + CDx * h9_8_9;
    const double k9_8_9_2 = h9_8_18 + CDy * h9_8_9;
    const double h9_8_19 = h18_3_19 + ABy * h9_3_19;
    const double k9_8_9_3 = h9_8_19 + CDz * h9_8_9;
    const double h19_3_10 = acc[486] + ABz * acc[246];
    const double h9_9_10 = h19_3_10 + ABz * h9_3_10;
    const double h19_3_4 = acc[480] + ABz * acc[240];
    const double h9_9_4 = h19_3_4 + ABz * h9_3_4;
    const double k9_9_4_1 = h9_9_10 + CDx * h9_9_4;
    const double h19_3_11 = acc[487] + ABz * acc[247];
    const double h9_9_11 = h19_3_11 + ABz * h9_3_11;
    const double k9_9_4_2 = h9_9_11 + CDy * h9_9_4;
    const double h19_3_12 = acc[488] + ABz * acc[248];
    const double h9_9_12 = h19_3_12 + ABz * h9_3_12;
    const double k9_9_4_3 = h9_9_12 + CDz * h9_9_4;
    const double h19_3_5 = acc[481] + ABz * acc[241];
    const double h9_9_5 = h19_3_5 + ABz * h9_3_5;
    const double k9_9_5_1 = h9_9_11 + CDx * h9_9_5;
    const double h19_3_13 = acc[489] + ABz * acc[249];
    const double h9_9_13 = h19_3_13 + ABz * h9_3_13;
    const double k9_9_5_2 = h9_9_13 + CDy * h9_9_5;
    const double h19_3_15 = acc[491] + ABz * acc[251];
    const double h9_9_15 = h19_3_15 + ABz * h9_3_15;
    const double k9_9_5_3 = h9_9_15 + CDz * h9_9_5;
    const double h19_3_6 = acc[482] + ABz * acc[242];
    const double h9_9_6 = h19_3_6 + ABz * h9_3_6;
    const double k9_9_6_1 = h9_9_12 + CDx * h9_9_6;
    const double k9_9_6_2 = h9_9_15 + CDy * h9_9_6;
    const double h19_3_14 = acc[490] + ABz * acc[250];
    const double h9_9_14 = h19_3_14 + ABz * h9_3_14;
    const double k9_9_6_3 = h9_9_14 + CDz * h9_9_6;
    const double h19_3_7 = acc[483] + ABz * acc[243];
    const double h9_9_7 = h19_3_7 + ABz * h9_3_7;
    const double k9_9_7_1 = h9_9_13 + CDx * h9_9_7;
    const double h19_3_16 = acc[492] + ABz * acc[252];
    const double h9_9_16 = h19_3_16 + ABz * h9_3_16;
    const double k9_9_7_2 = h9_9_16 + CDy * h9_9_7;
    const double h19_3_17 = acc[493] + ABz * acc[253];
    const double h9_9_17 = h19_3_17 + ABz * h9_3_17;
    const double k9_9_7_3 = h9_9_17 + CDz * h9_9_7;
    const double h19_3_8 = acc[484] + ABz * acc[244];
    const double h9_9_8 = h19_3_8 + ABz * h9_3_8;
    const double k9_9_8_1 = h9_9_15 + CDx * h9_9_8;
    const double k9_9_8_2 = h9_9_17 + CDy * h9_9_8;
    const double h19_3_18 = acc[494] + ABz * acc[254];
    const double h9_9_18 = h19_3_18 + ABz * h9_3_18;
    const double k9_9_8_3 = h9_9_18 + CDz * h9_9_8;
    const double h19_3_9 = acc[485] + ABz * acc[245];
    const double h9_9_9 = h19_3_9 + ABz * h9_3_9;
    const double k9_9_9_1 = h9_9_14 + CDx * h9_9_9;
    const double k9_9_9_2 = h9_9_18 + CDy * h9_9_9;
    const double h19_3_19 = acc[495] + ABz * acc[255];
    const double h9_9_19 = h19_3_19 + ABz * h9_3_19;
    const double k9_9_9_3 = h9_9_19 + CDz * h9_9_9;
    res[0] = k4_4_4_1 * 0.19245008972987535;
    res[1] = k4_4_4_2 * 0.19245008972987535;
    res[2] = k4_4_4_3 * 0.19245008972987535;
    res[3] = k4_4_5_1 * 0.3333333333333334;
    res[4] = k4_4_5_2 * 0.3333333333333334;
    res[5] = k4_4_5_3 * 0.3333333333333334;
    res[6] = k4_4_6_1 * 0.3333333333333334;
    res[7] = k4_4_6_2 * 0.3333333333333334;
    res[8] = k4_4_6_3 * 0.3333333333333334;
    res[9] = k4_4_7_1 * 0.19245008972987535;
    res[10] = k4_4_7_2 * 0.19245008972987535;
    res[11] = k4_4_7_3 * 0.19245008972987535;
    res[12] = k4_4_8_1 * 0.3333333333333334;
    res[13] = k4_4_8_2 * 0.3333333333333334;
    res[14] = k4_4_8_3 * 0.3333333333333334;
    res[15] = k4_4_9_1 * 0.19245008972987535;
    res[16] = k4_4_9_2 * 0.19245008972987535;
    res[17] = k4_4_9_3 * 0.19245008972987535;
    res[18] = k4_5_4_1 * 0.3333333333333334;
    res[19] = k4_5_4_2 * 0.3333333333333334;
    res[20] = k4_5_4_3 * 0.3333333333333334;
    res[21] = k4_5_5_1 * 0.5773502691896258;
    res[22] = k4_5_5_2 * 0.5773502691896258;
    res[23] = k4_5_5_3 * 0.5773502691896258;
    res[24] = k4_5_6_1 * 0.5773502691896258;
    res[25] = k4_5_6_2 * 0.5773502691896258;
    res[26] = k4_5_6_3 * 0.5773502691896258;
    res[27] = k4_5_7_1 * 0.3333333333333334;
    res[28] = k4_5_7_2 * 0.3333333333333334;
    res[29] = k4_5_7_3 * 0.3333333333333334;
    res[30] = k4_5_8_1 * 0.5773502691896258;
    res[31] = k4_5_8_2 * 0.5773502691896258;
    res[32] = k4_5_8_3 * 0.5773502691896258;
    res[33] = k4_5_9_1 * 0.3333333333333334;
    res[34] = k4_5_9_2 * 0.3333333333333334;
    res[35] = k4_5_9_3 * 0.3333333333333334;
    res[36] = k4_6_4_1 * 0.3333333333333334;
    res[37] = k4_6_4_2 * 0.3333333333333334;
    res[38] = k4_6_4_3 * 0.3333333333333334;
    res[39] = k4_6_5_1 * 0.5773502691896258;
    res[40] = k4_6_5_2 * 0.5773502691896258;
    res[41] = k4_6_5_3 * 0.5773502691896258;
    res[42] = k4_6_6_1 * 0.5773502691896258;
    res[43] = k4_6_6_2 * 0.5773502691896258;
    res[44] = k4_6_6_3 * 0.5773502691896258;
    res[45] = k4_6_7_1 * 0.3333333333333334;
    res[46] = k4_6_7_2 * 0.3333333333333334;
    res[47] = k4_6_7_3 * 0.3333333333333334;
    res[48] = k4_6_8_1 * 0.5773502691896258;
    res[49] = k4_6_8_2 * 0.5773502691896258;
    res[50] = k4_6_8_3 * 0.5773502691896258;
    res[51] = k4_6_9_1 * 0.3333333333333334;
    res[52] = k4_6_9_2 * 0.3333333333333334;
    res[53] = k4_6_9_3 * 0.3333333333333334;
    res[54] = k4_7_4_1 * 0.19245008972987535;
    res[55] = k4_7_4_2 * 0.19245008972987535;
    res[56] = k4_7_4_3 * 0.19245008972987535;
    res[57] = k4_7_5_1 * 0.3333333333333334;
    res[58] = k4_7_5_2 * 0.3333333333333334;
    res[59] = k4_7_5_3 * 0.3333333333333334;
    res[60] = k4_7_6_1 * 0.3333333333333334;
    res[61] = k4_7_6_2 * 0.3333333333333334;
    res[62] = k4_7_6_3 * 0.3333333333333334;
    res[63] = k4_7_7_1 * 0.19245008972987535;
    res[64] = k4_7_7_2 * 0.19245008972987535;
    res[65] = k4_7_7_3 * 0.19245008972987535;
    res[66] = k4_7_8_1 * 0.3333333333333334;
    res[67] = k4_7_8_2 * 0.3333333333333334;
    res[68] = k4_7_8_3 * 0.3333333333333334;
    res[69] = k4_7_9_1 * 0.19245008972987535;
    res[70] = k4_7_9_2 * 0.19245008972987535;
    res[71] = k4_7_9_3 * 0.19245008972987535;
    res[72] = k4_8_4_1 * 0.3333333333333334;
    res[73] = k4_8_4_2 * 0.3333333333333334;
    res[74] = k4_8_4_3 * 0.3333333333333334;
    res[75] = k4_8_5_1 * 0.5773502691896258;
    res[76] = k4_8_5_2 * 0.5773502691896258;
    res[77] = k4_8_5_3 * 0.5773502691896258;
    res[78] = k4_8_6_1 * 0.5773502691896258;
    res[79] = k4_8_6_2 * 0.5773502691896258;
    res[80] = k4_8_6_3 * 0.5773502691896258;
    res[81] = k4_8_7_1 * 0.3333333333333334;
    res[82] = k4_8_7_2 * 0.3333333333333334;
    res[83] = k4_8_7_3 * 0.3333333333333334;
    res[84] = k4_8_8_1 * 0.5773502691896258;
    res[85] = k4_8_8_2 * 0.5773502691896258;
    res[86] = k4_8_8_3 * 0.5773502691896258;
    res[87] = k4_8_9_1 * 0.3333333333333334;
    res[88] = k4_8_9_2 * 0.3333333333333334;
    res[89] = k4_8_9_3 * 0.3333333333333334;
    res[90] = k4_9_4_1 * 0.19245008972987535;
    res[91] = k4_9_4_2 * 0.19245008972987535;
    res[92] = k4_9_4_3 * 0.19245008972987535;
    res[93] = k4_9_5_1 * 0.3333333333333334;
    res[94] = k4_9_5_2 * 0.3333333333333334;
    res[95] = k4_9_5_3 * 0.3333333333333334;
    res[96] = k4_9_6_1 * 0.3333333333333334;
    res[97] = k4_9_6_2 * 0.3333333333333334;
    res[98] = k4_9_6_3 * 0.3333333333333334;
    res[99] = k4_9_7_1 * 0.19245008972987535;
    res[100] = k4_9_7_2 * 0.19245008972987535;
    res[101] = k4_9_7_3 * 0.19245008972987535;
    res[102] = k4_9_8_1 * 0.3333333333333334;
    res[103] = k4_9_8_2 * 0.3333333333333334;
    res[104] = k4_9_8_3 * 0.3333333333333334;
    res[105] = k4_9_9_1 * 0.19245008972987535;
    res[106] = k4_9_9_2 * 0.19245008972987535;
    res[107] = k4_9_9_3 * 0.19245008972987535;
    res[108] = k5_4_4_1 * 0.3333333333333334;
    res[109] = k5_4_4_2 * 0.3333333333333334;
    res[110] = k5_4_4_3 * 0.3333333333333334;
    res[111] = k5_4_5_1 * 0.5773502691896258;
    res[112] = k5_4_5_2 * 0.5773502691896258;
    res[113] = k5_4_5_3 * 0.5773502691896258;
    res[114] = k5_4_6_1 * 0.5773502691896258;
    res[115] = k5_4_6_2 * 0.5773502691896258;
    res[116] = k5_4_6_3 * 0.5773502691896258;
    res[117] = k5_4_7_1 * 0.3333333333333334;
    res[118] = k5_4_7_2 * 0.3333333333333334;
    res[119] = k5_4_7_3 * 0.3333333333333334;
    res[120] = k5_4_8_1 * 0.5773502691896258;
    res[121] = k5_4_8_2 * 0.5773502691896258;
    res[122] = k5_4_8_3 * 0.5773502691896258;
    res[123] = k5_4_9_1 * 0.3333333333333334;
    res[124] = k5_4_9_2 * 0.3333333333333334;
    res[125] = k5_4_9_3 * 0.3333333333333334;
    res[126] = k5_5_4_1 * 0.5773502691896258;
    res[127] = k5_5_4_2 * 0.5773502691896258;
    res[128] = k5_5_4_3 * 0.5773502691896258;
    res[129] = k5_5_5_1;
    res[130] = k5_5_5_2;
    res[131] = k5_5_5_3;
    res[132] = k5_5_6_1;
    res[133] = k5_5_6_2;
    res[134] = k5_5_6_3;
    res[135] = k5_5_7_1 * 0.5773502691896258;
    res[136] = k5_5_7_2 * 0.5773502691896258;
    res[137] = k5_5_7_3 * 0.5773502691896258;
    res[138] = k5_5_8_1;
    res[139] = k5_5_8_2;
    res[140] = k5_5_8_3;
    res[141] = k5_5_9_1 * 0.5773502691896258;
    res[142] = k5_5_9_2 * 0.5773502691896258;
    res[143] = k5_5_9_3 * 0.5773502691896258;
    res[144] = k5_6_4_1 * 0.5773502691896258;
    res[145] = k5_6_4_2 * 0.5773502691896258;
    res[146] = k5_6_4_3 * 0.5773502691896258;
    res[147] = k5_6_5_1;
    res[148] = k5_6_5_2;
    res[149] = k5_6_5_3;
    res[150] = k5_6_6_1;
    res[151] = k5_6_6_2;
    res[152] = k5_6_6_3;
    res[153] = k5_6_7_1 * 0.5773502691896258;
    res[154] = k5_6_7_2 * 0.5773502691896258;
    res[155] = k5_6_7_3 * 0.5773502691896258;
    res[156] = k5_6_8_1;
    res[157] = k5_6_8_2;
    res[158] = k5_6_8_3;
    res[159] = k5_6_9_1 * 0.5773502691896258;
    res[160] = k5_6_9_2 * 0.5773502691896258;
    res[161] = k5_6_9_3 * 0.5773502691896258;
    res[162] = k5_7_4_1 * 0.3333333333333334;
    res[163] = k5_7_4_2 * 0.3333333333333334;
    res[164] = k5_7_4_3 * 0.3333333333333334;
    res[165] = k5_7_5_1 * 0.5773502691896258;
    res[166] = k5_7_5_2 * 0.5773502691896258;
    res[167] = k5_7_5_3 * 0.5773502691896258;
    res[168] = k5_7_6_1 * 0.5773502691896258;
    res[169] = k5_7_6_2 * 0.5773502691896258;
    res[170] = k5_7_6_3 * 0.5773502691896258;
    res[171] = k5_7_7_1 * 0.3333333333333334;
    res[172] = k5_7_7_2 * 0.3333333333333334;
    res[173] = k5_7_7_3 * 0.3333333333333334;
    res[174] = k5_7_8_1 * 0.5773502691896258;
    res[175] = k5_7_8_2 * 0.5773502691896258;
    res[176] = k5_7_8_3 * 0.5773502691896258;
    res[177] = k5_7_9_1 * 0.3333333333333334;
    res[178] = k5_7_9_2 * 0.3333333333333334;
    res[179] = k5_7_9_3 * 0.3333333333333334;
    res[180] = k5_8_4_1 * 0.5773502691896258;
    res[181] = k5_8_4_2 * 0.5773502691896258;
    res[182] = k5_8_4_3 * 0.5773502691896258;
    res[183] = k5_8_5_1;
    res[184] = k5_8_5_2;
    res[185] = k5_8_5_3;
    res[186] = k5_8_6_1;
    res[187] = k5_8_6_2;
    res[188] = k5_8_6_3;
    res[189] = k5_8_7_1 * 0.5773502691896258;
    res[190] = k5_8_7_2 * 0.5773502691896258;
    res[191] = k5_8_7_3 * 0.5773502691896258;
    res[192] = k5_8_8_1;
    res[193] = k5_8_8_2;
    res[194] = k5_8_8_3;
    res[195] = k5_8_9_1 * 0.5773502691896258;
    res[196] = k5_8_9_2 * 0.5773502691896258;
    res[197] = k5_8_9_3 * 0.5773502691896258;
    res[198] = k5_9_4_1 * 0.3333333333333334;
    res[199] = k5_9_4_2 * 0.3333333333333334;
    res[200] = k5_9_4_3 * 0.3333333333333334;
    res[201] = k5_9_5_1 * 0.5773502691896258;
    res[202] = k5_9_5_2 * 0.5773502691896258;
    res[203] = k5_9_5_3 * 0.5773502691896258;
    res[204] = k5_9_6_1 * 0.5773502691896258;
    res[205] = k5_9_6_2 * 0.5773502691896258;
    res[206] = k5_9_6_3 * 0.5773502691896258;
    res[207] = k5_9_7_1 * 0.3333333333333334;
    res[208] = k5_9_7_2 * 0.3333333333333334;
    res[209] = k5_9_7_3 * 0.3333333333333334;
    res[210] = k5_9_8_1 * 0.5773502691896258;
    res[211] = k5_9_8_2 * 0.5773502691896258;
    res[212] = k5_9_8_3 * 0.5773502691896258;
    res[213] = k5_9_9_1 * 0.3333333333333334;
    res[214] = k5_9_9_2 * 0.3333333333333334;
    res[215] = k5_9_9_3 * 0.3333333333333334;
    res[216] = k6_4_4_1 * 0.3333333333333334;
    res[217] = k6_4_4_2 * 0.3333333333333334;
    res[218] = k6_4_4_3 * 0.3333333333333334;
    res[219] = k6_4_5_1 * 0.5773502691896258;
    res[220] = k6_4_5_2 * 0.5773502691896258;
    res[221] = k6_4_5_3 * 0.5773502691896258;
    res[222] = k6_4_6_1 * 0.5773502691896258;
    res[223] = k6_4_6_2 * 0.5773502691896258;
    res[224] = k6_4_6_3 * 0.5773502691896258;
    res[225] = k6_4_7_1 * 0.3333333333333334;
    res[226] = k6_4_7_2 * 0.3333333333333334;
    res[227] = k6_4_7_3 * 0.3333333333333334;
    res[228] = k6_4_8_1 * 0.5773502691896258;
    res[229] = k6_4_8_2 * 0.5773502691896258;
    res[230] = k6_4_8_3 * 0.5773502691896258;
    res[231] = k6_4_9_1 * 0.3333333333333334;
    res[232] = k6_4_9_2 * 0.3333333333333334;
    res[233] = k6_4_9_3 * 0.3333333333333334;
    res[234] = k6_5_4_1 * 0.5773502691896258;
    res[235] = k6_5_4_2 * 0.5773502691896258;
    res[236] = k6_5_4_3 * 0.5773502691896258;
    res[237] = k6_5_5_1;
    res[238] = k6_5_5_2;
    res[239] = k6_5_5_3;
    res[240] = k6_5_6_1;
    res[241] = k6_5_6_2;
    res[242] = k6_5_6_3;
    res[243] = k6_5_7_1 * 0.5773502691896258;
    res[244] = k6_5_7_2 * 0.5773502691896258;
    res[245] = k6_5_7_3 * 0.5773502691896258;
    res[246] = k6_5_8_1;
    res[247] = k6_5_8_2;
    res[248] = k6_5_8_3;
    res[249] = k6_5_9_1 * 0.5773502691896258;
    res[250] = k6_5_9_2 * 0.5773502691896258;
    res[251] = k6_5_9_3 * 0.5773502691896258;
    res[252] = k6_6_4_1 * 0.5773502691896258;
    res[253] = k6_6_4_2 * 0.5773502691896258;
    res[254] = k6_6_4_3 * 0.5773502691896258;
    res[255] = k6_6_5_1;
    res[256] = k6_6_5_2;
    res[257] = k6_6_5_3;
    res[258] = k6_6_6_1;
    res[259] = k6_6_6_2;
    res[260] = k6_6_6_3;
    res[261] = k6_6_7_1 * 0.5773502691896258;
    res[262] = k6_6_7_2 * 0.5773502691896258;
    res[263] = k6_6_7_3 * 0.5773502691896258;
    res[264] = k6_6_8_1;
    res[265] = k6_6_8_2;
    res[266] = k6_6_8_3;
    res[267] = k6_6_9_1 * 0.5773502691896258;
    res[268] = k6_6_9_2 * 0.5773502691896258;
    res[269] = k6_6_9_3 * 0.5773502691896258;
    res[270] = k6_7_4_1 * 0.3333333333333334;
    res[271] = k6_7_4_2 * 0.3333333333333334;
    res[272] = k6_7_4_3 * 0.3333333333333334;
    res[273] = k6_7_5_1 * 0.5773502691896258;
    res[274] = k6_7_5_2 * 0.5773502691896258;
    res[275] = k6_7_5_3 * 0.5773502691896258;
    res[276] = k6_7_6_1 * 0.5773502691896258;
    res[277] = k6_7_6_2 * 0.5773502691896258;
    res[278] = k6_7_6_3 * 0.5773502691896258;
    res[279] = k6_7_7_1 * 0.3333333333333334;
    res[280] = k6_7_7_2 * 0.3333333333333334;
    res[281] = k6_7_7_3 * 0.3333333333333334;
    res[282] = k6_7_8_1 * 0.5773502691896258;
    res[283] = k6_7_8_2 * 0.5773502691896258;
    res[284] = k6_7_8_3 * 0.5773502691896258;
    res[285] = k6_7_9_1 * 0.3333333333333334;
    res[286] = k6_7_9_2 * 0.3333333333333334;
    res[287] = k6_7_9_3 * 0.3333333333333334;
    res[288] = k6_8_4_1 * 0.5773502691896258;
    res[289] = k6_8_4_2 * 0.5773502691896258;
    res[290] = k6_8_4_3 * 0.5773502691896258;
    res[291] = k6_8_5_1;
    res[292] = k6_8_5_2;
    res[293] = k6_8_5_3;
    res[294] = k6_8_6_1;
    res[295] = k6_8_6_2;
    res[296] = k6_8_6_3;
    res[297] = k6_8_7_1 * 0.5773502691896258;
    res[298] = k6_8_7_2 * 0.5773502691896258;
    res[299] = k6_8_7_3 * 0.5773502691896258;
    res[300] = k6_8_8_1;
    res[301] = k6_8_8_2;
    res[302] = k6_8_8_3;
    res[303] = k6_8_9_1 * 0.5773502691896258;
    res[304] = k6_8_9_2 * 0.5773502691896258;
    res[305] = k6_8_9_3 * 0.5773502691896258;
    res[306] = k6_9_4_1 * 0.3333333333333334;
    res[307] = k6_9_4_2 * 0.3333333333333334;
    res[308] = k6_9_4_3 * 0.3333333333333334;
    res[309] = k6_9_5_1 * 0.5773502691896258;
    res[310] = k6_9_5_2 * 0.5773502691896258;
    res[311] = k6_9_5_3 * 0.5773502691896258;
    res[312] = k6_9_6_1 * 0.5773502691896258;
    res[313] = k6_9_6_2 * 0.5773502691896258;
    res[314] = k6_9_6_3 * 0.5773502691896258;
    res[315] = k6_9_7_1 * 0.3333333333333334;
    res[316] = k6_9_7_2 * 0.3333333333333334;
    res[317] = k6_9_7_3 * 0.3333333333333334;
    res[318] = k6_9_8_1 * 0.5773502691896258;
    res[319] = k6_9_8_2 * 0.5773502691896258;
    res[320] = k6_9_8_3 * 0.5773502691896258;
    res[321] = k6_9_9_1 * 0.3333333333333334;
    res[322] = k6_9_9_2 * 0.3333333333333334;
    res[323] = k6_9_9_3 * 0.3333333333333334;
    res[324] = k7_4_4_1 * 0.19245008972987535;
    res[325] = k7_4_4_2 * 0.19245008972987535;
    res[326] = k7_4_4_3 * 0.19245008972987535;
    res[327] = k7_4_5_1 * 0.3333333333333334;
    res[328] = k7_4_5_2 * 0.3333333333333334;
    res[329] = k7_4_5_3 * 0.3333333333333334;
    res[330] = k7_4_6_1 * 0.3333333333333334;
    res[331] = k7_4_6_2 * 0.3333333333333334;
    res[332] = k7_4_6_3 * 0.3333333333333334;
    res[333] = k7_4_7_1 * 0.19245008972987535;
    res[334] = k7_4_7_2 * 0.19245008972987535;
    res[335] = k7_4_7_3 * 0.19245008972987535;
    res[336] = k7_4_8_1 * 0.3333333333333334;
    res[337] = k7_4_8_2 * 0.3333333333333334;
    res[338] = k7_4_8_3 * 0.3333333333333334;
    res[339] = k7_4_9_1 * 0.19245008972987535;
    res[340] = k7_4_9_2 * 0.19245008972987535;
    res[341] = k7_4_9_3 * 0.19245008972987535;
    res[342] = k7_5_4_1 * 0.3333333333333334;
    res[343] = k7_5_4_2 * 0.3333333333333334;
    res[344] = k7_5_4_3 * 0.3333333333333334;
    res[345] = k7_5_5_1 * 0.5773502691896258;
    res[346] = k7_5_5_2 * 0.5773502691896258;
    res[347] = k7_5_5_3 * 0.5773502691896258;
    res[348] = k7_5_6_1 * 0.5773502691896258;
    res[349] = k7_5_6_2 * 0.5773502691896258;
    res[350] = k7_5_6_3 * 0.5773502691896258;
    res[351] = k7_5_7_1 * 0.3333333333333334;
    res[352] = k7_5_7_2 * 0.3333333333333334;
    res[353] = k7_5_7_3 * 0.3333333333333334;
    res[354] = k7_5_8_1 * 0.5773502691896258;
    res[355] = k7_5_8_2 * 0.5773502691896258;
    res[356] = k7_5_8_3 * 0.5773502691896258;
    res[357] = k7_5_9_1 * 0.3333333333333334;
    res[358] = k7_5_9_2 * 0.3333333333333334;
    res[359] = k7_5_9_3 * 0.3333333333333334;
    res[360] = k7_6_4_1 * 0.3333333333333334;
    res[361] = k7_6_4_2 * 0.3333333333333334;
    res[362] = k7_6_4_3 * 0.3333333333333334;
    res[363] = k7_6_5_1 * 0.5773502691896258;
    res[364] = k7_6_5_2 * 0.5773502691896258;
    res[365] = k7_6_5_3 * 0.5773502691896258;
    res[366] = k7_6_6_1 * 0.5773502691896258;
    res[367] = k7_6_6_2 * 0.5773502691896258;
    res[368] = k7_6_6_3 * 0.5773502691896258;
    res[369] = k7_6_7_1 * 0.3333333333333334;
    res[370] = k7_6_7_2 * 0.3333333333333334;
    res[371] = k7_6_7_3 * 0.3333333333333334;
    res[372] = k7_6_8_1 * 0.5773502691896258;
    res[373] = k7_6_8_2 * 0.5773502691896258;
    res[374] = k7_6_8_3 * 0.5773502691896258;
    res[375] = k7_6_9_1 * 0.3333333333333334;
    res[376] = k7_6_9_2 * 0.3333333333333334;
    res[377] = k7_6_9_3 * 0.3333333333333334;
    res[378] = k7_7_4_1 * 0.19245008972987535;
    res[379] = k7_7_4_2 * 0.19245008972987535;
    res[380] = k7_7_4_3 * 0.19245008972987535;
    res[381] = k7_7_5_1 * 0.3333333333333334;
    res[382] = k7_7_5_2 * 0.3333333333333334;
    res[383] = k7_7_5_3 * 0.3333333333333334;
    res[384] = k7_7_6_1 * 0.3333333333333334;
    res[385] = k7_7_6_2 * 0.3333333333333334;
    res[386] = k7_7_6_3 * 0.3333333333333334;
    res[387] = k7_7_7_1 * 0.19245008972987535;
    res[388] = k7_7_7_2 * 0.19245008972987535;
    res[389] = k7_7_7_3 * 0.19245008972987535;
    res[390] = k7_7_8_1 * 0.3333333333333334;
    res[391] = k7_7_8_2 * 0.3333333333333334;
    res[392] = k7_7_8_3 * 0.3333333333333334;
    res[393] = k7_7_9_1 * 0.19245008972987535;
    res[394] = k7_7_9_2 * 0.19245008972987535;
    res[395] = k7_7_9_3 * 0.19245008972987535;
    res[396] = k7_8_4_1 * 0.3333333333333334;
    res[397] = k7_8_4_2 * 0.3333333333333334;
    res[398] = k7_8_4_3 * 0.3333333333333334;
    res[399] = k7_8_5_1 * 0.5773502691896258;
    res[400] = k7_8_5_2 * 0.5773502691896258;
    res[401] = k7_8_5_3 * 0.5773502691896258;
    res[402] = k7_8_6_1 * 0.5773502691896258;
    res[403] = k7_8_6_2 * 0.5773502691896258;
    res[404] = k7_8_6_3 * 0.5773502691896258;
    res[405] = k7_8_7_1 * 0.3333333333333334;
    res[406] = k7_8_7_2 * 0.3333333333333334;
    res[407] = k7_8_7_3 * 0.3333333333333334;
    res[408] = k7_8_8_1 * 0.5773502691896258;
    res[409] = k7_8_8_2 * 0.5773502691896258;
    res[410] = k7_8_8_3 * 0.5773502691896258;
    res[411] = k7_8_9_1 * 0.3333333333333334;
    res[412] = k7_8_9_2 * 0.3333333333333334;
    res[413] = k7_8_9_3 * 0.3333333333333334;
    res[414] = k7_9_4_1 * 0.19245008972987535;
    res[415] = k7_9_4_2 * 0.19245008972987535;
    res[416] = k7_9_4_3 * 0.19245008972987535;
    res[417] = k7_9_5_1 * 0.3333333333333334;
    res[418] = k7_9_5_2 * 0.3333333333333334;
    res[419] = k7_9_5_3 * 0.3333333333333334;
    res[420] = k7_9_6_1 * 0.3333333333333334;
    res[421] = k7_9_6_2 * 0.3333333333333334;
    res[422] = k7_9_6_3 * 0.3333333333333334;
    res[423] = k7_9_7_1 * 0.19245008972987535;
    res[424] = k7_9_7_2 * 0.19245008972987535;
    res[425] = k7_9_7_3 * 0.19245008972987535;
    res[426] = k7_9_8_1 * 0.3333333333333334;
    res[427] = k7_9_8_2 * 0.3333333333333334;
    res[428] = k7_9_8_3 * 0.3333333333333334;
    res[429] = k7_9_9_1 * 0.19245008972987535;
    res[430] = k7_9_9_2 * 0.19245008972987535;
    res[431] = k7_9_9_3 * 0.19245008972987535;
    res[432] = k8_4_4_1 * 0.3333333333333334;
    res[433] = k8_4_4_2 * 0.3333333333333334;
    res[434] = k8_4_4_3 * 0.3333333333333334;
    res[435] = k8_4_5_1 * 0.5773502691896258;
    res[436] = k8_4_5_2 * 0.5773502691896258;
    res[437] = k8_4_5_3 * 0.5773502691896258;
    res[438] = k8_4_6_1 * 0.5773502691896258;
    res[439] = k8_4_6_2 * 0.5773502691896258;
    res[440] = k8_4_6_3 * 0.5773502691896258;
    res[441] = k8_4_7_1 * 0.3333333333333334;
    res[442] = k8_4_7_2 * 0.3333333333333334;
    res[443] = k8_4_7_3 * 0.3333333333333334;
    res[444] = k8_4_8_1 * 0.5773502691896258;
    res[445] = k8_4_8_2 * 0.5773502691896258;
    res[446] = k8_4_8_3 * 0.5773502691896258;
    res[447] = k8_4_9_1 * 0.3333333333333334;
    res[448] = k8_4_9_2 * 0.3333333333333334;
    res[449] = k8_4_9_3 * 0.3333333333333334;
    res[450] = k8_5_4_1 * 0.5773502691896258;
    res[451] = k8_5_4_2 * 0.5773502691896258;
    res[452] = k8_5_4_3 * 0.5773502691896258;
    res[453] = k8_5_5_1;
    res[454] = k8_5_5_2;
    res[455] = k8_5_5_3;
    res[456] = k8_5_6_1;
    res[457] = k8_5_6_2;
    res[458] = k8_5_6_3;
    res[459] = k8_5_7_1 * 0.5773502691896258;
    res[460] = k8_5_7_2 * 0.5773502691896258;
    res[461] = k8_5_7_3 * 0.5773502691896258;
    res[462] = k8_5_8_1;
    res[463] = k8_5_8_2;
    res[464] = k8_5_8_3;
    res[465] = k8_5_9_1 * 0.5773502691896258;
    res[466] = k8_5_9_2 * 0.5773502691896258;
    res[467] = k8_5_9_3 * 0.5773502691896258;
    res[468] = k8_6_4_1 * 0.5773502691896258;
    res[469] = k8_6_4_2 * 0.5773502691896258;
    res[470] = k8_6_4_3 * 0.5773502691896258;
    res[471] = k8_6_5_1;
    res[472] = k8_6_5_2;
    res[473] = k8_6_5_3;
    res[474] = k8_6_6_1;
    res[475] = k8_6_6_2;
    res[476] = k8_6_6_3;
    res[477] = k8_6_7_1 * 0.5773502691896258;
    res[478] = k8_6_7_2 * 0.5773502691896258;
    res[479] = k8_6_7_3 * 0.5773502691896258;
    res[480] = k8_6_8_1;
    res[481] = k8_6_8_2;
    res[482] = k8_6_8_3;
    res[483] = k8_6_9_1 * 0.5773502691896258;
    res[484] = k8_6_9_2 * 0.5773502691896258;
    res[485] = k8_6_9_3 * 0.5773502691896258;
    res[486] = k8_7_4_1 * 0.3333333333333334;
    res[487] = k8_7_4_2 * 0.3333333333333334;
    res[488] = k8_7_4_3 * 0.3333333333333334;
    res[489] = k8_7_5_1 * 0.5773502691896258;
    res[490] = k8_7_5_2 * 0.5773502691896258;
    res[491] = k8_7_5_3 * 0.5773502691896258;
    res[492] = k8_7_6_1 * 0.5773502691896258;
    res[493] = k8_7_6_2 * 0.5773502691896258;
    res[494] = k8_7_6_3 * 0.5773502691896258;
    res[495] = k8_7_7_1 * 0.3333333333333334;
    res[496] = k8_7_7_2 * 0.3333333333333334;
    res[497] = k8_7_7_3 * 0.3333333333333334;
    res[498] = k8_7_8_1 * 0.5773502691896258;
    res[499] = k8_7_8_2 * 0.5773502691896258;
    res[500] = k8_7_8_3 * 0.5773502691896258;
    res[501] = k8_7_9_1 * 0.3333333333333334;
    res[502] = k8_7_9_2 * 0.3333333333333334;
    res[503] = k8_7_9_3 * 0.3333333333333334;
    res[504] = k8_8_4_1 * 0.5773502691896258;
    res[505] = k8_8_4_2 * 0.5773502691896258;
    res[506] = k8_8_4_3 * 0.5773502691896258;
    res[507] = k8_8_5_1;
    res[508] = k8_8_5_2;
    res[509] = k8_8_5_3;
    res[510] = k8_8_6_1;
    res[511] = k8_8_6_2;
    res[512] = k8_8_6_3;
    res[513] = k8_8_7_1 * 0.5773502691896258;
    res[514] = k8_8_7_2 * 0.5773502691896258;
    res[515] = k8_8_7_3 * 0.5773502691896258;
    res[516] = k8_8_8_1;
    res[517] = k8_8_8_2;
    res[518] = k8_8_8_3;
    res[519] = k8_8_9_1 * 0.5773502691896258;
    res[520] = k8_8_9_2 * 0.5773502691896258;
    res[521] = k8_8_9_3 * 0.5773502691896258;
    res[522] = k8_9_4_1 * 0.3333333333333334;
    res[523] = k8_9_4_2 * 0.3333333333333334;
    res[524] = k8_9_4_3 * 0.3333333333333334;
    res[525] = k8_9_5_1 * 0.5773502691896258;
    res[526] = k8_9_5_2 * 0.5773502691896258;
    res[527] = k8_9_5_3 * 0.5773502691896258;
    res[528] = k8_9_6_1 * 0.5773502691896258;
    res[529] = k8_9_6_2 * 0.5773502691896258;
    res[530] = k8_9_6_3 * 0.5773502691896258;
    res[531] = k8_9_7_1 * 0.3333333333333334;
    res[532] = k8_9_7_2 * 0.3333333333333334;
    res[533] = k8_9_7_3 * 0.3333333333333334;
    res[534] = k8_9_8_1 * 0.5773502691896258;
    res[535] = k8_9_8_2 * 0.5773502691896258;
    res[536] = k8_9_8_3 * 0.5773502691896258;
    res[537] = k8_9_9_1 * 0.3333333333333334;
    res[538] = k8_9_9_2 * 0.3333333333333334;
    res[539] = k8_9_9_3 * 0.3333333333333334;
    res[540] = k9_4_4_1 * 0.19245008972987535;
    res[541] = k9_4_4_2 * 0.19245008972987535;
    res[542] = k9_4_4_3 * 0.19245008972987535;
    res[543] = k9_4_5_1 * 0.3333333333333334;
    res[544] = k9_4_5_2 * 0.3333333333333334;
    res[545] = k9_4_5_3 * 0.3333333333333334;
    res[546] = k9_4_6_1 * 0.3333333333333334;
    res[547] = k9_4_6_2 * 0.3333333333333334;
    res[548] = k9_4_6_3 * 0.3333333333333334;
    res[549] = k9_4_7_1 * 0.19245008972987535;
    res[550] = k9_4_7_2 * 0.19245008972987535;
    res[551] = k9_4_7_3 * 0.19245008972987535;
    res[552] = k9_4_8_1 * 0.3333333333333334;
    res[553] = k9_4_8_2 * 0.3333333333333334;
    res[554] = k9_4_8_3 * 0.3333333333333334;
    res[555] = k9_4_9_1 * 0.19245008972987535;
    res[556] = k9_4_9_2 * 0.19245008972987535;
    res[557] = k9_4_9_3 * 0.19245008972987535;
    res[558] = k9_5_4_1 * 0.3333333333333334;
    res[559] = k9_5_4_2 * 0.3333333333333334;
    res[560] = k9_5_4_3 * 0.3333333333333334;
    res[561] = k9_5_5_1 * 0.5773502691896258;
    res[562] = k9_5_5_2 * 0.5773502691896258;
    res[563] = k9_5_5_3 * 0.5773502691896258;
    res[564] = k9_5_6_1 * 0.5773502691896258;
    res[565] = k9_5_6_2 * 0.5773502691896258;
    res[566] = k9_5_6_3 * 0.5773502691896258;
    res[567] = k9_5_7_1 * 0.3333333333333334;
    res[568] = k9_5_7_2 * 0.3333333333333334;
    res[569] = k9_5_7_3 * 0.3333333333333334;
    res[570] = k9_5_8_1 * 0.5773502691896258;
    res[571] = k9_5_8_2 * 0.5773502691896258;
    res[572] = k9_5_8_3 * 0.5773502691896258;
    res[573] = k9_5_9_1 * 0.3333333333333334;
    res[574] = k9_5_9_2 * 0.3333333333333334;
    res[575] = k9_5_9_3 * 0.3333333333333334;
    res[576] = k9_6_4_1 * 0.3333333333333334;
    res[577] = k9_6_4_2 * 0.3333333333333334;
    res[578] = k9_6_4_3 * 0.3333333333333334;
    res[579] = k9_6_5_1 * 0.5773502691896258;
    res[580] = k9_6_5_2 * 0.5773502691896258;
    res[581] = k9_6_5_3 * 0.5773502691896258;
    res[582] = k9_6_6_1 * 0.5773502691896258;
    res[583] = k9_6_6_2 * 0.5773502691896258;
    res[584] = k9_6_6_3 * 0.5773502691896258;
    res[585] = k9_6_7_1 * 0.3333333333333334;
    res[586] = k9_6_7_2 * 0.3333333333333334;
    res[587] = k9_6_7_3 * 0.3333333333333334;
    res[588] = k9_6_8_1 * 0.5773502691896258;
    res[589] = k9_6_8_2 * 0.5773502691896258;
    res[590] = k9_6_8_3 * 0.5773502691896258;
    res[591] = k9_6_9_1 * 0.3333333333333334;
    res[592] = k9_6_9_2 * 0.3333333333333334;
    res[593] = k9_6_9_3 * 0.3333333333333334;
    res[594] = k9_7_4_1 * 0.19245008972987535;
    res[595] = k9_7_4_2 * 0.19245008972987535;
    res[596] = k9_7_4_3 * 0.19245008972987535;
    res[597] = k9_7_5_1 * 0.3333333333333334;
    res[598] = k9_7_5_2 * 0.3333333333333334;
    res[599] = k9_7_5_3 * 0.3333333333333334;
    res[600] = k9_7_6_1 * 0.3333333333333334;
    res[601] = k9_7_6_2 * 0.3333333333333334;
    res[602] = k9_7_6_3 * 0.3333333333333334;
    res[603] = k9_7_7_1 * 0.19245008972987535;
    res[604] = k9_7_7_2 * 0.19245008972987535;
    res[605] = k9_7_7_3 * 0.19245008972987535;
    res[606] = k9_7_8_1 * 0.3333333333333334;
    res[607] = k9_7_8_2 * 0.3333333333333334;
    res[608] = k9_7_8_3 * 0.3333333333333334;
    res[609] = k9_7_9_1 * 0.19245008972987535;
    res[610] = k9_7_9_2 * 0.19245008972987535;
    res[611] = k9_7_9_3 * 0.19245008972987535;
    res[612] = k9_8_4_1 * 0.3333333333333334;
    res[613] = k9_8_4_2 * 0.3333333333333334;
    res[614] = k9_8_4_3 * 0.3333333333333334;
    res[615] = k9_8_5_1 * 0.5773502691896258;
    res[616] = k9_8_5_2 * 0.5773502691896258;
    res[617] = k9_8_5_3 * 0.5773502691896258;
    res[618] = k9_8_6_1 * 0.5773502691896258;
    res[619] = k9_8_6_2 * 0.5773502691896258;
    res[620] = k9_8_6_3 * 0.5773502691896258;
    res[621] = k9_8_7_1 * 0.3333333333333334;
    res[622] = k9_8_7_2 * 0.3333333333333334;
    res[623] = k9_8_7_3 * 0.3333333333333334;
    res[624] = k9_8_8_1 * 0.5773502691896258;
    res[625] = k9_8_8_2 * 0.5773502691896258;
    res[626] = k9_8_8_3 * 0.5773502691896258;
    res[627] = k9_8_9_1 * 0.3333333333333334;
    res[628] = k9_8_9_2 * 0.3333333333333334;
    res[629] = k9_8_9_3 * 0.3333333333333334;
    res[630] = k9_9_4_1 * 0.19245008972987535;
    res[631] = k9_9_4_2 * 0.19245008972987535;
    res[632] = k9_9_4_3 * 0.19245008972987535;
    res[633] = k9_9_5_1 * 0.3333333333333334;
    res[634] = k9_9_5_2 * 0.3333333333333334;
    res[635] = k9_9_5_3 * 0.3333333333333334;
    res[636] = k9_9_6_1 * 0.3333333333333334;
    res[637] = k9_9_6_2 * 0.3333333333333334;
    res[638] = k9_9_6_3 * 0.3333333333333334;
    res[639] = k9_9_7_1 * 0.19245008972987535;
    res[640] = k9_9_7_2 * 0.19245008972987535;
    res[641] = k9_9_7_3 * 0.19245008972987535;
    res[642] = k9_9_8_1 * 0.3333333333333334;
    res[643] = k9_9_8_2 * 0.3333333333333334;
    res[644] = k9_9_8_3 * 0.3333333333333334;
    res[645] = k9_9_9_1 * 0.19245008972987535;
    res[646] = k9_9_9_2 * 0.19245008972987535;
    res[647] = k9_9_9_3 * 0.19245008972987535;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[648]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_dddp(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[496];
    vrr_dddp<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 496; ++x) acc_out[x] = acc[x];
    }
    hrr_dddp(P, p, q, acc, res);
}

__device__ __forceinline__ void store_dddp(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_0_1;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_0_2;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_0, kl = kl_1_1;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_0, kl = kl_1_2;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_0, kl = kl_2_1;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_0, kl = kl_2_2;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_0_0, kl = kl_3_0;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_0_0, kl = kl_3_1;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_0_0, kl = kl_3_2;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_0_0, kl = kl_4_0;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_0_0, kl = kl_4_1;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_0_0, kl = kl_4_2;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_0_0, kl = kl_5_0;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_0_0, kl = kl_5_1;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_0_0, kl = kl_5_2;
      if ((!dab || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_0_1, kl = kl_0_1;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_0_1, kl = kl_0_2;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_0_1, kl = kl_1_0;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_0_1, kl = kl_1_1;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_0_1, kl = kl_1_2;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_0_1, kl = kl_2_0;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_0_1, kl = kl_2_1;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_0_1, kl = kl_2_2;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_0_1, kl = kl_3_0;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_0_1, kl = kl_3_1;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_0_1, kl = kl_3_2;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_0_1, kl = kl_4_0;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_0_1, kl = kl_4_1;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_0_1, kl = kl_4_2;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_0_1, kl = kl_5_0;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_0_1, kl = kl_5_1;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_0_1, kl = kl_5_2;
      if ((!dab || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_0_2, kl = kl_0_1;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_0_2, kl = kl_0_2;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_0_2, kl = kl_1_0;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_0_2, kl = kl_1_1;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_0_2, kl = kl_1_2;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_0_2, kl = kl_2_0;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_0_2, kl = kl_2_1;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_0_2, kl = kl_2_2;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_0_2, kl = kl_3_0;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_0_2, kl = kl_3_1;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_0_2, kl = kl_3_2;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_0_2, kl = kl_4_0;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_0_2, kl = kl_4_1;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_0_2, kl = kl_4_2;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_0_2, kl = kl_5_0;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_0_2, kl = kl_5_1;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_0_2, kl = kl_5_2;
      if ((!dab || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_0_3, kl = kl_0_0;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_0_3, kl = kl_0_1;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_0_3, kl = kl_0_2;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_0_3, kl = kl_1_0;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_0_3, kl = kl_1_1;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_0_3, kl = kl_1_2;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_0_3, kl = kl_2_0;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_0_3, kl = kl_2_1;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_0_3, kl = kl_2_2;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_0_3, kl = kl_3_0;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_0_3, kl = kl_3_1;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_0_3, kl = kl_3_2;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_0_3, kl = kl_4_0;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_0_3, kl = kl_4_1;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_0_3, kl = kl_4_2;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_0_3, kl = kl_5_0;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_0_3, kl = kl_5_1;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_0_3, kl = kl_5_2;
      if ((!dab || 0 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_0_4, kl = kl_0_0;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_0_4, kl = kl_0_1;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_0_4, kl = kl_0_2;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_0_4, kl = kl_1_0;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_0_4, kl = kl_1_1;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_0_4, kl = kl_1_2;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_0_4, kl = kl_2_0;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_0_4, kl = kl_2_1;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_0_4, kl = kl_2_2;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
    { const long long ij = ij_0_4, kl = kl_3_0;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[81]; }
    { const long long ij = ij_0_4, kl = kl_3_1;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[82]; }
    { const long long ij = ij_0_4, kl = kl_3_2;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[83]; }
    { const long long ij = ij_0_4, kl = kl_4_0;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[84]; }
    { const long long ij = ij_0_4, kl = kl_4_1;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[85]; }
    { const long long ij = ij_0_4, kl = kl_4_2;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[86]; }
    { const long long ij = ij_0_4, kl = kl_5_0;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[87]; }
    { const long long ij = ij_0_4, kl = kl_5_1;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[88]; }
    { const long long ij = ij_0_4, kl = kl_5_2;
      if ((!dab || 0 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[89]; }
    { const long long ij = ij_0_5, kl = kl_0_0;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[90]; }
    { const long long ij = ij_0_5, kl = kl_0_1;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[91]; }
    { const long long ij = ij_0_5, kl = kl_0_2;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[92]; }
    { const long long ij = ij_0_5, kl = kl_1_0;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[93]; }
    { const long long ij = ij_0_5, kl = kl_1_1;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[94]; }
    { const long long ij = ij_0_5, kl = kl_1_2;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[95]; }
    { const long long ij = ij_0_5, kl = kl_2_0;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[96]; }
    { const long long ij = ij_0_5, kl = kl_2_1;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[97]; }
    { const long long ij = ij_0_5, kl = kl_2_2;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[98]; }
    { const long long ij = ij_0_5, kl = kl_3_0;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[99]; }
    { const long long ij = ij_0_5, kl = kl_3_1;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[100]; }
    { const long long ij = ij_0_5, kl = kl_3_2;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[101]; }
    { const long long ij = ij_0_5, kl = kl_4_0;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[102]; }
    { const long long ij = ij_0_5, kl = kl_4_1;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[103]; }
    { const long long ij = ij_0_5, kl = kl_4_2;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[104]; }
    { const long long ij = ij_0_5, kl = kl_5_0;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[105]; }
    { const long long ij = ij_0_5, kl = kl_5_1;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[106]; }
    { const long long ij = ij_0_5, kl = kl_5_2;
      if ((!dab || 0 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[107]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[108]; }
    { const long long ij = ij_1_0, kl = kl_0_1;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[109]; }
    { const long long ij = ij_1_0, kl = kl_0_2;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[110]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[111]; }
    { const long long ij = ij_1_0, kl = kl_1_1;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[112]; }
    { const long long ij = ij_1_0, kl = kl_1_2;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[113]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[114]; }
    { const long long ij = ij_1_0, kl = kl_2_1;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[115]; }
    { const long long ij = ij_1_0, kl = kl_2_2;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[116]; }
    { const long long ij = ij_1_0, kl = kl_3_0;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[117]; }
    { const long long ij = ij_1_0, kl = kl_3_1;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[118]; }
    { const long long ij = ij_1_0, kl = kl_3_2;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[119]; }
    { const long long ij = ij_1_0, kl = kl_4_0;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[120]; }
    { const long long ij = ij_1_0, kl = kl_4_1;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[121]; }
    { const long long ij = ij_1_0, kl = kl_4_2;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[122]; }
    { const long long ij = ij_1_0, kl = kl_5_0;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[123]; }
    { const long long ij = ij_1_0, kl = kl_5_1;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[124]; }
    { const long long ij = ij_1_0, kl = kl_5_2;
      if ((!dab || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[125]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[126]; }
    { const long long ij = ij_1_1, kl = kl_0_1;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[127]; }
    { const long long ij = ij_1_1, kl = kl_0_2;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[128]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[129]; }
    { const long long ij = ij_1_1, kl = kl_1_1;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[130]; }
    { const long long ij = ij_1_1, kl = kl_1_2;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[131]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[132]; }
    { const long long ij = ij_1_1, kl = kl_2_1;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[133]; }
    { const long long ij = ij_1_1, kl = kl_2_2;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[134]; }
    { const long long ij = ij_1_1, kl = kl_3_0;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[135]; }
    { const long long ij = ij_1_1, kl = kl_3_1;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[136]; }
    { const long long ij = ij_1_1, kl = kl_3_2;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[137]; }
    { const long long ij = ij_1_1, kl = kl_4_0;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[138]; }
    { const long long ij = ij_1_1, kl = kl_4_1;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[139]; }
    { const long long ij = ij_1_1, kl = kl_4_2;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[140]; }
    { const long long ij = ij_1_1, kl = kl_5_0;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[141]; }
    { const long long ij = ij_1_1, kl = kl_5_1;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[142]; }
    { const long long ij = ij_1_1, kl = kl_5_2;
      if ((!dab || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[143]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[144]; }
    { const long long ij = ij_1_2, kl = kl_0_1;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[145]; }
    { const long long ij = ij_1_2, kl = kl_0_2;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[146]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[147]; }
    { const long long ij = ij_1_2, kl = kl_1_1;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[148]; }
    { const long long ij = ij_1_2, kl = kl_1_2;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[149]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[150]; }
    { const long long ij = ij_1_2, kl = kl_2_1;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[151]; }
    { const long long ij = ij_1_2, kl = kl_2_2;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[152]; }
    { const long long ij = ij_1_2, kl = kl_3_0;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[153]; }
    { const long long ij = ij_1_2, kl = kl_3_1;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[154]; }
    { const long long ij = ij_1_2, kl = kl_3_2;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[155]; }
    { const long long ij = ij_1_2, kl = kl_4_0;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[156]; }
    { const long long ij = ij_1_2, kl = kl_4_1;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[157]; }
    { const long long ij = ij_1_2, kl = kl_4_2;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[158]; }
    { const long long ij = ij_1_2, kl = kl_5_0;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[159]; }
    { const long long ij = ij_1_2, kl = kl_5_1;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[160]; }
    { const long long ij = ij_1_2, kl = kl_5_2;
      if ((!dab || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[161]; }
    { const long long ij = ij_1_3, kl = kl_0_0;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[162]; }
    { const long long ij = ij_1_3, kl = kl_0_1;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[163]; }
    { const long long ij = ij_1_3, kl = kl_0_2;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[164]; }
    { const long long ij = ij_1_3, kl = kl_1_0;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[165]; }
    { const long long ij = ij_1_3, kl = kl_1_1;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[166]; }
    { const long long ij = ij_1_3, kl = kl_1_2;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[167]; }
    { const long long ij = ij_1_3, kl = kl_2_0;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[168]; }
    { const long long ij = ij_1_3, kl = kl_2_1;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[169]; }
    { const long long ij = ij_1_3, kl = kl_2_2;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[170]; }
    { const long long ij = ij_1_3, kl = kl_3_0;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[171]; }
    { const long long ij = ij_1_3, kl = kl_3_1;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[172]; }
    { const long long ij = ij_1_3, kl = kl_3_2;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[173]; }
    { const long long ij = ij_1_3, kl = kl_4_0;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[174]; }
    { const long long ij = ij_1_3, kl = kl_4_1;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[175]; }
    { const long long ij = ij_1_3, kl = kl_4_2;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[176]; }
    { const long long ij = ij_1_3, kl = kl_5_0;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[177]; }
    { const long long ij = ij_1_3, kl = kl_5_1;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[178]; }
    { const long long ij = ij_1_3, kl = kl_5_2;
      if ((!dab || 1 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[179]; }
    { const long long ij = ij_1_4, kl = kl_0_0;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[180]; }
    { const long long ij = ij_1_4, kl = kl_0_1;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[181]; }
    { const long long ij = ij_1_4, kl = kl_0_2;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[182]; }
    { const long long ij = ij_1_4, kl = kl_1_0;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[183]; }
    { const long long ij = ij_1_4, kl = kl_1_1;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[184]; }
    { const long long ij = ij_1_4, kl = kl_1_2;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[185]; }
    { const long long ij = ij_1_4, kl = kl_2_0;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[186]; }
    { const long long ij = ij_1_4, kl = kl_2_1;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[187]; }
    { const long long ij = ij_1_4, kl = kl_2_2;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[188]; }
    { const long long ij = ij_1_4, kl = kl_3_0;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[189]; }
    { const long long ij = ij_1_4, kl = kl_3_1;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[190]; }
    { const long long ij = ij_1_4, kl = kl_3_2;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[191]; }
    { const long long ij = ij_1_4, kl = kl_4_0;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[192]; }
    { const long long ij = ij_1_4, kl = kl_4_1;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[193]; }
    { const long long ij = ij_1_4, kl = kl_4_2;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[194]; }
    { const long long ij = ij_1_4, kl = kl_5_0;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[195]; }
    { const long long ij = ij_1_4, kl = kl_5_1;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[196]; }
    { const long long ij = ij_1_4, kl = kl_5_2;
      if ((!dab || 1 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[197]; }
    { const long long ij = ij_1_5, kl = kl_0_0;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[198]; }
    { const long long ij = ij_1_5, kl = kl_0_1;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[199]; }
    { const long long ij = ij_1_5, kl = kl_0_2;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[200]; }
    { const long long ij = ij_1_5, kl = kl_1_0;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[201]; }
    { const long long ij = ij_1_5, kl = kl_1_1;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[202]; }
    { const long long ij = ij_1_5, kl = kl_1_2;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[203]; }
    { const long long ij = ij_1_5, kl = kl_2_0;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[204]; }
    { const long long ij = ij_1_5, kl = kl_2_1;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[205]; }
    { const long long ij = ij_1_5, kl = kl_2_2;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[206]; }
    { const long long ij = ij_1_5, kl = kl_3_0;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[207]; }
    { const long long ij = ij_1_5, kl = kl_3_1;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[208]; }
    { const long long ij = ij_1_5, kl = kl_3_2;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[209]; }
    { const long long ij = ij_1_5, kl = kl_4_0;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[210]; }
    { const long long ij = ij_1_5, kl = kl_4_1;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[211]; }
    { const long long ij = ij_1_5, kl = kl_4_2;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[212]; }
    { const long long ij = ij_1_5, kl = kl_5_0;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[213]; }
    { const long long ij = ij_1_5, kl = kl_5_1;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[214]; }
    { const long long ij = ij_1_5, kl = kl_5_2;
      if ((!dab || 1 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[215]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[216]; }
    { const long long ij = ij_2_0, kl = kl_0_1;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[217]; }
    { const long long ij = ij_2_0, kl = kl_0_2;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[218]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[219]; }
    { const long long ij = ij_2_0, kl = kl_1_1;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[220]; }
    { const long long ij = ij_2_0, kl = kl_1_2;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[221]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[222]; }
    { const long long ij = ij_2_0, kl = kl_2_1;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[223]; }
    { const long long ij = ij_2_0, kl = kl_2_2;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[224]; }
    { const long long ij = ij_2_0, kl = kl_3_0;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[225]; }
    { const long long ij = ij_2_0, kl = kl_3_1;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[226]; }
    { const long long ij = ij_2_0, kl = kl_3_2;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[227]; }
    { const long long ij = ij_2_0, kl = kl_4_0;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[228]; }
    { const long long ij = ij_2_0, kl = kl_4_1;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[229]; }
    { const long long ij = ij_2_0, kl = kl_4_2;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[230]; }
    { const long long ij = ij_2_0, kl = kl_5_0;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[231]; }
    { const long long ij = ij_2_0, kl = kl_5_1;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[232]; }
    { const long long ij = ij_2_0, kl = kl_5_2;
      if ((!dab || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[233]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[234]; }
    { const long long ij = ij_2_1, kl = kl_0_1;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[235]; }
    { const long long ij = ij_2_1, kl = kl_0_2;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[236]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[237]; }
    { const long long ij = ij_2_1, kl = kl_1_1;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[238]; }
    { const long long ij = ij_2_1, kl = kl_1_2;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[239]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[240]; }
    { const long long ij = ij_2_1, kl = kl_2_1;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[241]; }
    { const long long ij = ij_2_1, kl = kl_2_2;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[242]; }
    { const long long ij = ij_2_1, kl = kl_3_0;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[243]; }
    { const long long ij = ij_2_1, kl = kl_3_1;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[244]; }
    { const long long ij = ij_2_1, kl = kl_3_2;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[245]; }
    { const long long ij = ij_2_1, kl = kl_4_0;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[246]; }
    { const long long ij = ij_2_1, kl = kl_4_1;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[247]; }
    { const long long ij = ij_2_1, kl = kl_4_2;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[248]; }
    { const long long ij = ij_2_1, kl = kl_5_0;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[249]; }
    { const long long ij = ij_2_1, kl = kl_5_1;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[250]; }
    { const long long ij = ij_2_1, kl = kl_5_2;
      if ((!dab || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[251]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[252]; }
    { const long long ij = ij_2_2, kl = kl_0_1;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[253]; }
    { const long long ij = ij_2_2, kl = kl_0_2;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[254]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[255]; }
    { const long long ij = ij_2_2, kl = kl_1_1;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[256]; }
    { const long long ij = ij_2_2, kl = kl_1_2;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[257]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[258]; }
    { const long long ij = ij_2_2, kl = kl_2_1;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[259]; }
    { const long long ij = ij_2_2, kl = kl_2_2;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[260]; }
    { const long long ij = ij_2_2, kl = kl_3_0;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[261]; }
    { const long long ij = ij_2_2, kl = kl_3_1;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[262]; }
    { const long long ij = ij_2_2, kl = kl_3_2;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[263]; }
    { const long long ij = ij_2_2, kl = kl_4_0;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[264]; }
    { const long long ij = ij_2_2, kl = kl_4_1;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[265]; }
    { const long long ij = ij_2_2, kl = kl_4_2;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[266]; }
    { const long long ij = ij_2_2, kl = kl_5_0;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[267]; }
    { const long long ij = ij_2_2, kl = kl_5_1;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[268]; }
    { const long long ij = ij_2_2, kl = kl_5_2;
      if ((!dab || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[269]; }
    { const long long ij = ij_2_3, kl = kl_0_0;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[270]; }
    { const long long ij = ij_2_3, kl = kl_0_1;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[271]; }
    { const long long ij = ij_2_3, kl = kl_0_2;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[272]; }
    { const long long ij = ij_2_3, kl = kl_1_0;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[273]; }
    { const long long ij = ij_2_3, kl = kl_1_1;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[274]; }
    { const long long ij = ij_2_3, kl = kl_1_2;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[275]; }
    { const long long ij = ij_2_3, kl = kl_2_0;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[276]; }
    { const long long ij = ij_2_3, kl = kl_2_1;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[277]; }
    { const long long ij = ij_2_3, kl = kl_2_2;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[278]; }
    { const long long ij = ij_2_3, kl = kl_3_0;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[279]; }
    { const long long ij = ij_2_3, kl = kl_3_1;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[280]; }
    { const long long ij = ij_2_3, kl = kl_3_2;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[281]; }
    { const long long ij = ij_2_3, kl = kl_4_0;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[282]; }
    { const long long ij = ij_2_3, kl = kl_4_1;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[283]; }
    { const long long ij = ij_2_3, kl = kl_4_2;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[284]; }
    { const long long ij = ij_2_3, kl = kl_5_0;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[285]; }
    { const long long ij = ij_2_3, kl = kl_5_1;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[286]; }
    { const long long ij = ij_2_3, kl = kl_5_2;
      if ((!dab || 2 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[287]; }
    { const long long ij = ij_2_4, kl = kl_0_0;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[288]; }
    { const long long ij = ij_2_4, kl = kl_0_1;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[289]; }
    { const long long ij = ij_2_4, kl = kl_0_2;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[290]; }
    { const long long ij = ij_2_4, kl = kl_1_0;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[291]; }
    { const long long ij = ij_2_4, kl = kl_1_1;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[292]; }
    { const long long ij = ij_2_4, kl = kl_1_2;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[293]; }
    { const long long ij = ij_2_4, kl = kl_2_0;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[294]; }
    { const long long ij = ij_2_4, kl = kl_2_1;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[295]; }
    { const long long ij = ij_2_4, kl = kl_2_2;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[296]; }
    { const long long ij = ij_2_4, kl = kl_3_0;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[297]; }
    { const long long ij = ij_2_4, kl = kl_3_1;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[298]; }
    { const long long ij = ij_2_4, kl = kl_3_2;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[299]; }
    { const long long ij = ij_2_4, kl = kl_4_0;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[300]; }
    { const long long ij = ij_2_4, kl = kl_4_1;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[301]; }
    { const long long ij = ij_2_4, kl = kl_4_2;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[302]; }
    { const long long ij = ij_2_4, kl = kl_5_0;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[303]; }
    { const long long ij = ij_2_4, kl = kl_5_1;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[304]; }
    { const long long ij = ij_2_4, kl = kl_5_2;
      if ((!dab || 2 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[305]; }
    { const long long ij = ij_2_5, kl = kl_0_0;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[306]; }
    { const long long ij = ij_2_5, kl = kl_0_1;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[307]; }
    { const long long ij = ij_2_5, kl = kl_0_2;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[308]; }
    { const long long ij = ij_2_5, kl = kl_1_0;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[309]; }
    { const long long ij = ij_2_5, kl = kl_1_1;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[310]; }
    { const long long ij = ij_2_5, kl = kl_1_2;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[311]; }
    { const long long ij = ij_2_5, kl = kl_2_0;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[312]; }
    { const long long ij = ij_2_5, kl = kl_2_1;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[313]; }
    { const long long ij = ij_2_5, kl = kl_2_2;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[314]; }
    { const long long ij = ij_2_5, kl = kl_3_0;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[315]; }
    { const long long ij = ij_2_5, kl = kl_3_1;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[316]; }
    { const long long ij = ij_2_5, kl = kl_3_2;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[317]; }
    { const long long ij = ij_2_5, kl = kl_4_0;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[318]; }
    { const long long ij = ij_2_5, kl = kl_4_1;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[319]; }
    { const long long ij = ij_2_5, kl = kl_4_2;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[320]; }
    { const long long ij = ij_2_5, kl = kl_5_0;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[321]; }
    { const long long ij = ij_2_5, kl = kl_5_1;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[322]; }
    { const long long ij = ij_2_5, kl = kl_5_2;
      if ((!dab || 2 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[323]; }
    { const long long ij = ij_3_0, kl = kl_0_0;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[324]; }
    { const long long ij = ij_3_0, kl = kl_0_1;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[325]; }
    { const long long ij = ij_3_0, kl = kl_0_2;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[326]; }
    { const long long ij = ij_3_0, kl = kl_1_0;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[327]; }
    { const long long ij = ij_3_0, kl = kl_1_1;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[328]; }
    { const long long ij = ij_3_0, kl = kl_1_2;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[329]; }
    { const long long ij = ij_3_0, kl = kl_2_0;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[330]; }
    { const long long ij = ij_3_0, kl = kl_2_1;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[331]; }
    { const long long ij = ij_3_0, kl = kl_2_2;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[332]; }
    { const long long ij = ij_3_0, kl = kl_3_0;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[333]; }
    { const long long ij = ij_3_0, kl = kl_3_1;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[334]; }
    { const long long ij = ij_3_0, kl = kl_3_2;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[335]; }
    { const long long ij = ij_3_0, kl = kl_4_0;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[336]; }
    { const long long ij = ij_3_0, kl = kl_4_1;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[337]; }
    { const long long ij = ij_3_0, kl = kl_4_2;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[338]; }
    { const long long ij = ij_3_0, kl = kl_5_0;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[339]; }
    { const long long ij = ij_3_0, kl = kl_5_1;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[340]; }
    { const long long ij = ij_3_0, kl = kl_5_2;
      if ((!dab || 3 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[341]; }
    { const long long ij = ij_3_1, kl = kl_0_0;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[342]; }
    { const long long ij = ij_3_1, kl = kl_0_1;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[343]; }
    { const long long ij = ij_3_1, kl = kl_0_2;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[344]; }
    { const long long ij = ij_3_1, kl = kl_1_0;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[345]; }
    { const long long ij = ij_3_1, kl = kl_1_1;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[346]; }
    { const long long ij = ij_3_1, kl = kl_1_2;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[347]; }
    { const long long ij = ij_3_1, kl = kl_2_0;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[348]; }
    { const long long ij = ij_3_1, kl = kl_2_1;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[349]; }
    { const long long ij = ij_3_1, kl = kl_2_2;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[350]; }
    { const long long ij = ij_3_1, kl = kl_3_0;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[351]; }
    { const long long ij = ij_3_1, kl = kl_3_1;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[352]; }
    { const long long ij = ij_3_1, kl = kl_3_2;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[353]; }
    { const long long ij = ij_3_1, kl = kl_4_0;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[354]; }
    { const long long ij = ij_3_1, kl = kl_4_1;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[355]; }
    { const long long ij = ij_3_1, kl = kl_4_2;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[356]; }
    { const long long ij = ij_3_1, kl = kl_5_0;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[357]; }
    { const long long ij = ij_3_1, kl = kl_5_1;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[358]; }
    { const long long ij = ij_3_1, kl = kl_5_2;
      if ((!dab || 3 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[359]; }
    { const long long ij = ij_3_2, kl = kl_0_0;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[360]; }
    { const long long ij = ij_3_2, kl = kl_0_1;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[361]; }
    { const long long ij = ij_3_2, kl = kl_0_2;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[362]; }
    { const long long ij = ij_3_2, kl = kl_1_0;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[363]; }
    { const long long ij = ij_3_2, kl = kl_1_1;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[364]; }
    { const long long ij = ij_3_2, kl = kl_1_2;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[365]; }
    { const long long ij = ij_3_2, kl = kl_2_0;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[366]; }
    { const long long ij = ij_3_2, kl = kl_2_1;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[367]; }
    { const long long ij = ij_3_2, kl = kl_2_2;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[368]; }
    { const long long ij = ij_3_2, kl = kl_3_0;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[369]; }
    { const long long ij = ij_3_2, kl = kl_3_1;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[370]; }
    { const long long ij = ij_3_2, kl = kl_3_2;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[371]; }
    { const long long ij = ij_3_2, kl = kl_4_0;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[372]; }
    { const long long ij = ij_3_2, kl = kl_4_1;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[373]; }
    { const long long ij = ij_3_2, kl = kl_4_2;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[374]; }
    { const long long ij = ij_3_2, kl = kl_5_0;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[375]; }
    { const long long ij = ij_3_2, kl = kl_5_1;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[376]; }
    { const long long ij = ij_3_2, kl = kl_5_2;
      if ((!dab || 3 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[377]; }
    { const long long ij = ij_3_3, kl = kl_0_0;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[378]; }
    { const long long ij = ij_3_3, kl = kl_0_1;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[379]; }
    { const long long ij = ij_3_3, kl = kl_0_2;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[380]; }
    { const long long ij = ij_3_3, kl = kl_1_0;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[381]; }
    { const long long ij = ij_3_3, kl = kl_1_1;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[382]; }
    { const long long ij = ij_3_3, kl = kl_1_2;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[383]; }
    { const long long ij = ij_3_3, kl = kl_2_0;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[384]; }
    { const long long ij = ij_3_3, kl = kl_2_1;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[385]; }
    { const long long ij = ij_3_3, kl = kl_2_2;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[386]; }
    { const long long ij = ij_3_3, kl = kl_3_0;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[387]; }
    { const long long ij = ij_3_3, kl = kl_3_1;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[388]; }
    { const long long ij = ij_3_3, kl = kl_3_2;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[389]; }
    { const long long ij = ij_3_3, kl = kl_4_0;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[390]; }
    { const long long ij = ij_3_3, kl = kl_4_1;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[391]; }
    { const long long ij = ij_3_3, kl = kl_4_2;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[392]; }
    { const long long ij = ij_3_3, kl = kl_5_0;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[393]; }
    { const long long ij = ij_3_3, kl = kl_5_1;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[394]; }
    { const long long ij = ij_3_3, kl = kl_5_2;
      if ((!dab || 3 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[395]; }
    { const long long ij = ij_3_4, kl = kl_0_0;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[396]; }
    { const long long ij = ij_3_4, kl = kl_0_1;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[397]; }
    { const long long ij = ij_3_4, kl = kl_0_2;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[398]; }
    { const long long ij = ij_3_4, kl = kl_1_0;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[399]; }
    { const long long ij = ij_3_4, kl = kl_1_1;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[400]; }
    { const long long ij = ij_3_4, kl = kl_1_2;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[401]; }
    { const long long ij = ij_3_4, kl = kl_2_0;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[402]; }
    { const long long ij = ij_3_4, kl = kl_2_1;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[403]; }
    { const long long ij = ij_3_4, kl = kl_2_2;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[404]; }
    { const long long ij = ij_3_4, kl = kl_3_0;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[405]; }
    { const long long ij = ij_3_4, kl = kl_3_1;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[406]; }
    { const long long ij = ij_3_4, kl = kl_3_2;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[407]; }
    { const long long ij = ij_3_4, kl = kl_4_0;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[408]; }
    { const long long ij = ij_3_4, kl = kl_4_1;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[409]; }
    { const long long ij = ij_3_4, kl = kl_4_2;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[410]; }
    { const long long ij = ij_3_4, kl = kl_5_0;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[411]; }
    { const long long ij = ij_3_4, kl = kl_5_1;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[412]; }
    { const long long ij = ij_3_4, kl = kl_5_2;
      if ((!dab || 3 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[413]; }
    { const long long ij = ij_3_5, kl = kl_0_0;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[414]; }
    { const long long ij = ij_3_5, kl = kl_0_1;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[415]; }
    { const long long ij = ij_3_5, kl = kl_0_2;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[416]; }
    { const long long ij = ij_3_5, kl = kl_1_0;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[417]; }
    { const long long ij = ij_3_5, kl = kl_1_1;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[418]; }
    { const long long ij = ij_3_5, kl = kl_1_2;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[419]; }
    { const long long ij = ij_3_5, kl = kl_2_0;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[420]; }
    { const long long ij = ij_3_5, kl = kl_2_1;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[421]; }
    { const long long ij = ij_3_5, kl = kl_2_2;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[422]; }
    { const long long ij = ij_3_5, kl = kl_3_0;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[423]; }
    { const long long ij = ij_3_5, kl = kl_3_1;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[424]; }
    { const long long ij = ij_3_5, kl = kl_3_2;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[425]; }
    { const long long ij = ij_3_5, kl = kl_4_0;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[426]; }
    { const long long ij = ij_3_5, kl = kl_4_1;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[427]; }
    { const long long ij = ij_3_5, kl = kl_4_2;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[428]; }
    { const long long ij = ij_3_5, kl = kl_5_0;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[429]; }
    { const long long ij = ij_3_5, kl = kl_5_1;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[430]; }
    { const long long ij = ij_3_5, kl = kl_5_2;
      if ((!dab || 3 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[431]; }
    { const long long ij = ij_4_0, kl = kl_0_0;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[432]; }
    { const long long ij = ij_4_0, kl = kl_0_1;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[433]; }
    { const long long ij = ij_4_0, kl = kl_0_2;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[434]; }
    { const long long ij = ij_4_0, kl = kl_1_0;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[435]; }
    { const long long ij = ij_4_0, kl = kl_1_1;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[436]; }
    { const long long ij = ij_4_0, kl = kl_1_2;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[437]; }
    { const long long ij = ij_4_0, kl = kl_2_0;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[438]; }
    { const long long ij = ij_4_0, kl = kl_2_1;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[439]; }
    { const long long ij = ij_4_0, kl = kl_2_2;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[440]; }
    { const long long ij = ij_4_0, kl = kl_3_0;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[441]; }
    { const long long ij = ij_4_0, kl = kl_3_1;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[442]; }
    { const long long ij = ij_4_0, kl = kl_3_2;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[443]; }
    { const long long ij = ij_4_0, kl = kl_4_0;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[444]; }
    { const long long ij = ij_4_0, kl = kl_4_1;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[445]; }
    { const long long ij = ij_4_0, kl = kl_4_2;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[446]; }
    { const long long ij = ij_4_0, kl = kl_5_0;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[447]; }
    { const long long ij = ij_4_0, kl = kl_5_1;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[448]; }
    { const long long ij = ij_4_0, kl = kl_5_2;
      if ((!dab || 4 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[449]; }
    { const long long ij = ij_4_1, kl = kl_0_0;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[450]; }
    { const long long ij = ij_4_1, kl = kl_0_1;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[451]; }
    { const long long ij = ij_4_1, kl = kl_0_2;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[452]; }
    { const long long ij = ij_4_1, kl = kl_1_0;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[453]; }
    { const long long ij = ij_4_1, kl = kl_1_1;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[454]; }
    { const long long ij = ij_4_1, kl = kl_1_2;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[455]; }
    { const long long ij = ij_4_1, kl = kl_2_0;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[456]; }
    { const long long ij = ij_4_1, kl = kl_2_1;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[457]; }
    { const long long ij = ij_4_1, kl = kl_2_2;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[458]; }
    { const long long ij = ij_4_1, kl = kl_3_0;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[459]; }
    { const long long ij = ij_4_1, kl = kl_3_1;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[460]; }
    { const long long ij = ij_4_1, kl = kl_3_2;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[461]; }
    { const long long ij = ij_4_1, kl = kl_4_0;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[462]; }
    { const long long ij = ij_4_1, kl = kl_4_1;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[463]; }
    { const long long ij = ij_4_1, kl = kl_4_2;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[464]; }
    { const long long ij = ij_4_1, kl = kl_5_0;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[465]; }
    { const long long ij = ij_4_1, kl = kl_5_1;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[466]; }
    { const long long ij = ij_4_1, kl = kl_5_2;
      if ((!dab || 4 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[467]; }
    { const long long ij = ij_4_2, kl = kl_0_0;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[468]; }
    { const long long ij = ij_4_2, kl = kl_0_1;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[469]; }
    { const long long ij = ij_4_2, kl = kl_0_2;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[470]; }
    { const long long ij = ij_4_2, kl = kl_1_0;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[471]; }
    { const long long ij = ij_4_2, kl = kl_1_1;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[472]; }
    { const long long ij = ij_4_2, kl = kl_1_2;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[473]; }
    { const long long ij = ij_4_2, kl = kl_2_0;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[474]; }
    { const long long ij = ij_4_2, kl = kl_2_1;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[475]; }
    { const long long ij = ij_4_2, kl = kl_2_2;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[476]; }
    { const long long ij = ij_4_2, kl = kl_3_0;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[477]; }
    { const long long ij = ij_4_2, kl = kl_3_1;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[478]; }
    { const long long ij = ij_4_2, kl = kl_3_2;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[479]; }
    { const long long ij = ij_4_2, kl = kl_4_0;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[480]; }
    { const long long ij = ij_4_2, kl = kl_4_1;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[481]; }
    { const long long ij = ij_4_2, kl = kl_4_2;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[482]; }
    { const long long ij = ij_4_2, kl = kl_5_0;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[483]; }
    { const long long ij = ij_4_2, kl = kl_5_1;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[484]; }
    { const long long ij = ij_4_2, kl = kl_5_2;
      if ((!dab || 4 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[485]; }
    { const long long ij = ij_4_3, kl = kl_0_0;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[486]; }
    { const long long ij = ij_4_3, kl = kl_0_1;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[487]; }
    { const long long ij = ij_4_3, kl = kl_0_2;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[488]; }
    { const long long ij = ij_4_3, kl = kl_1_0;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[489]; }
    { const long long ij = ij_4_3, kl = kl_1_1;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[490]; }
    { const long long ij = ij_4_3, kl = kl_1_2;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[491]; }
    { const long long ij = ij_4_3, kl = kl_2_0;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[492]; }
    { const long long ij = ij_4_3, kl = kl_2_1;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[493]; }
    { const long long ij = ij_4_3, kl = kl_2_2;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[494]; }
    { const long long ij = ij_4_3, kl = kl_3_0;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[495]; }
    { const long long ij = ij_4_3, kl = kl_3_1;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[496]; }
    { const long long ij = ij_4_3, kl = kl_3_2;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[497]; }
    { const long long ij = ij_4_3, kl = kl_4_0;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[498]; }
    { const long long ij = ij_4_3, kl = kl_4_1;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[499]; }
    { const long long ij = ij_4_3, kl = kl_4_2;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[500]; }
    { const long long ij = ij_4_3, kl = kl_5_0;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[501]; }
    { const long long ij = ij_4_3, kl = kl_5_1;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[502]; }
    { const long long ij = ij_4_3, kl = kl_5_2;
      if ((!dab || 4 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[503]; }
    { const long long ij = ij_4_4, kl = kl_0_0;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[504]; }
    { const long long ij = ij_4_4, kl = kl_0_1;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[505]; }
    { const long long ij = ij_4_4, kl = kl_0_2;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[506]; }
    { const long long ij = ij_4_4, kl = kl_1_0;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[507]; }
    { const long long ij = ij_4_4, kl = kl_1_1;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[508]; }
    { const long long ij = ij_4_4, kl = kl_1_2;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[509]; }
    { const long long ij = ij_4_4, kl = kl_2_0;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[510]; }
    { const long long ij = ij_4_4, kl = kl_2_1;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[511]; }
    { const long long ij = ij_4_4, kl = kl_2_2;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[512]; }
    { const long long ij = ij_4_4, kl = kl_3_0;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[513]; }
    { const long long ij = ij_4_4, kl = kl_3_1;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[514]; }
    { const long long ij = ij_4_4, kl = kl_3_2;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[515]; }
    { const long long ij = ij_4_4, kl = kl_4_0;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[516]; }
    { const long long ij = ij_4_4, kl = kl_4_1;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[517]; }
    { const long long ij = ij_4_4, kl = kl_4_2;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[518]; }
    { const long long ij = ij_4_4, kl = kl_5_0;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[519]; }
    { const long long ij = ij_4_4, kl = kl_5_1;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[520]; }
    { const long long ij = ij_4_4, kl = kl_5_2;
      if ((!dab || 4 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[521]; }
    { const long long ij = ij_4_5, kl = kl_0_0;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[522]; }
    { const long long ij = ij_4_5, kl = kl_0_1;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[523]; }
    { const long long ij = ij_4_5, kl = kl_0_2;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[524]; }
    { const long long ij = ij_4_5, kl = kl_1_0;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[525]; }
    { const long long ij = ij_4_5, kl = kl_1_1;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[526]; }
    { const long long ij = ij_4_5, kl = kl_1_2;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[527]; }
    { const long long ij = ij_4_5, kl = kl_2_0;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[528]; }
    { const long long ij = ij_4_5, kl = kl_2_1;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[529]; }
    { const long long ij = ij_4_5, kl = kl_2_2;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[530]; }
    { const long long ij = ij_4_5, kl = kl_3_0;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[531]; }
    { const long long ij = ij_4_5, kl = kl_3_1;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[532]; }
    { const long long ij = ij_4_5, kl = kl_3_2;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[533]; }
    { const long long ij = ij_4_5, kl = kl_4_0;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[534]; }
    { const long long ij = ij_4_5, kl = kl_4_1;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[535]; }
    { const long long ij = ij_4_5, kl = kl_4_2;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[536]; }
    { const long long ij = ij_4_5, kl = kl_5_0;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[537]; }
    { const long long ij = ij_4_5, kl = kl_5_1;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[538]; }
    { const long long ij = ij_4_5, kl = kl_5_2;
      if ((!dab || 4 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[539]; }
    { const long long ij = ij_5_0, kl = kl_0_0;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[540]; }
    { const long long ij = ij_5_0, kl = kl_0_1;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[541]; }
    { const long long ij = ij_5_0, kl = kl_0_2;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[542]; }
    { const long long ij = ij_5_0, kl = kl_1_0;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[543]; }
    { const long long ij = ij_5_0, kl = kl_1_1;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[544]; }
    { const long long ij = ij_5_0, kl = kl_1_2;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[545]; }
    { const long long ij = ij_5_0, kl = kl_2_0;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[546]; }
    { const long long ij = ij_5_0, kl = kl_2_1;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[547]; }
    { const long long ij = ij_5_0, kl = kl_2_2;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[548]; }
    { const long long ij = ij_5_0, kl = kl_3_0;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[549]; }
    { const long long ij = ij_5_0, kl = kl_3_1;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[550]; }
    { const long long ij = ij_5_0, kl = kl_3_2;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[551]; }
    { const long long ij = ij_5_0, kl = kl_4_0;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[552]; }
    { const long long ij = ij_5_0, kl = kl_4_1;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[553]; }
    { const long long ij = ij_5_0, kl = kl_4_2;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[554]; }
    { const long long ij = ij_5_0, kl = kl_5_0;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[555]; }
    { const long long ij = ij_5_0, kl = kl_5_1;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[556]; }
    { const long long ij = ij_5_0, kl = kl_5_2;
      if ((!dab || 5 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[557]; }
    { const long long ij = ij_5_1, kl = kl_0_0;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[558]; }
    { const long long ij = ij_5_1, kl = kl_0_1;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[559]; }
    { const long long ij = ij_5_1, kl = kl_0_2;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[560]; }
    { const long long ij = ij_5_1, kl = kl_1_0;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[561]; }
    { const long long ij = ij_5_1, kl = kl_1_1;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[562]; }
    { const long long ij = ij_5_1, kl = kl_1_2;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[563]; }
    { const long long ij = ij_5_1, kl = kl_2_0;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[564]; }
    { const long long ij = ij_5_1, kl = kl_2_1;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[565]; }
    { const long long ij = ij_5_1, kl = kl_2_2;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[566]; }
    { const long long ij = ij_5_1, kl = kl_3_0;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[567]; }
    { const long long ij = ij_5_1, kl = kl_3_1;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[568]; }
    { const long long ij = ij_5_1, kl = kl_3_2;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[569]; }
    { const long long ij = ij_5_1, kl = kl_4_0;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[570]; }
    { const long long ij = ij_5_1, kl = kl_4_1;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[571]; }
    { const long long ij = ij_5_1, kl = kl_4_2;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[572]; }
    { const long long ij = ij_5_1, kl = kl_5_0;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[573]; }
    { const long long ij = ij_5_1, kl = kl_5_1;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[574]; }
    { const long long ij = ij_5_1, kl = kl_5_2;
      if ((!dab || 5 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[575]; }
    { const long long ij = ij_5_2, kl = kl_0_0;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[576]; }
    { const long long ij = ij_5_2, kl = kl_0_1;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[577]; }
    { const long long ij = ij_5_2, kl = kl_0_2;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[578]; }
    { const long long ij = ij_5_2, kl = kl_1_0;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[579]; }
    { const long long ij = ij_5_2, kl = kl_1_1;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[580]; }
    { const long long ij = ij_5_2, kl = kl_1_2;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[581]; }
    { const long long ij = ij_5_2, kl = kl_2_0;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[582]; }
    { const long long ij = ij_5_2, kl = kl_2_1;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[583]; }
    { const long long ij = ij_5_2, kl = kl_2_2;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[584]; }
    { const long long ij = ij_5_2, kl = kl_3_0;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[585]; }
    { const long long ij = ij_5_2, kl = kl_3_1;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[586]; }
    { const long long ij = ij_5_2, kl = kl_3_2;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[587]; }
    { const long long ij = ij_5_2, kl = kl_4_0;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[588]; }
    { const long long ij = ij_5_2, kl = kl_4_1;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[589]; }
    { const long long ij = ij_5_2, kl = kl_4_2;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[590]; }
    { const long long ij = ij_5_2, kl = kl_5_0;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[591]; }
    { const long long ij = ij_5_2, kl = kl_5_1;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[592]; }
    { const long long ij = ij_5_2, kl = kl_5_2;
      if ((!dab || 5 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[593]; }
    { const long long ij = ij_5_3, kl = kl_0_0;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[594]; }
    { const long long ij = ij_5_3, kl = kl_0_1;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[595]; }
    { const long long ij = ij_5_3, kl = kl_0_2;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[596]; }
    { const long long ij = ij_5_3, kl = kl_1_0;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[597]; }
    { const long long ij = ij_5_3, kl = kl_1_1;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[598]; }
    { const long long ij = ij_5_3, kl = kl_1_2;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[599]; }
    { const long long ij = ij_5_3, kl = kl_2_0;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[600]; }
    { const long long ij = ij_5_3, kl = kl_2_1;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[601]; }
    { const long long ij = ij_5_3, kl = kl_2_2;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[602]; }
    { const long long ij = ij_5_3, kl = kl_3_0;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[603]; }
    { const long long ij = ij_5_3, kl = kl_3_1;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[604]; }
    { const long long ij = ij_5_3, kl = kl_3_2;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[605]; }
    { const long long ij = ij_5_3, kl = kl_4_0;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[606]; }
    { const long long ij = ij_5_3, kl = kl_4_1;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[607]; }
    { const long long ij = ij_5_3, kl = kl_4_2;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[608]; }
    { const long long ij = ij_5_3, kl = kl_5_0;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[609]; }
    { const long long ij = ij_5_3, kl = kl_5_1;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[610]; }
    { const long long ij = ij_5_3, kl = kl_5_2;
      if ((!dab || 5 >= 3) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[611]; }
    { const long long ij = ij_5_4, kl = kl_0_0;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[612]; }
    { const long long ij = ij_5_4, kl = kl_0_1;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[613]; }
    { const long long ij = ij_5_4, kl = kl_0_2;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[614]; }
    { const long long ij = ij_5_4, kl = kl_1_0;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[615]; }
    { const long long ij = ij_5_4, kl = kl_1_1;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[616]; }
    { const long long ij = ij_5_4, kl = kl_1_2;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[617]; }
    { const long long ij = ij_5_4, kl = kl_2_0;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[618]; }
    { const long long ij = ij_5_4, kl = kl_2_1;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[619]; }
    { const long long ij = ij_5_4, kl = kl_2_2;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[620]; }
    { const long long ij = ij_5_4, kl = kl_3_0;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[621]; }
    { const long long ij = ij_5_4, kl = kl_3_1;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[622]; }
    { const long long ij = ij_5_4, kl = kl_3_2;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[623]; }
    { const long long ij = ij_5_4, kl = kl_4_0;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[624]; }
    { const long long ij = ij_5_4, kl = kl_4_1;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[625]; }
    { const long long ij = ij_5_4, kl = kl_4_2;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[626]; }
    { const long long ij = ij_5_4, kl = kl_5_0;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[627]; }
    { const long long ij = ij_5_4, kl = kl_5_1;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[628]; }
    { const long long ij = ij_5_4, kl = kl_5_2;
      if ((!dab || 5 >= 4) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[629]; }
    { const long long ij = ij_5_5, kl = kl_0_0;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[630]; }
    { const long long ij = ij_5_5, kl = kl_0_1;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[631]; }
    { const long long ij = ij_5_5, kl = kl_0_2;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[632]; }
    { const long long ij = ij_5_5, kl = kl_1_0;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[633]; }
    { const long long ij = ij_5_5, kl = kl_1_1;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[634]; }
    { const long long ij = ij_5_5, kl = kl_1_2;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[635]; }
    { const long long ij = ij_5_5, kl = kl_2_0;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[636]; }
    { const long long ij = ij_5_5, kl = kl_2_1;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[637]; }
    { const long long ij = ij_5_5, kl = kl_2_2;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[638]; }
    { const long long ij = ij_5_5, kl = kl_3_0;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[639]; }
    { const long long ij = ij_5_5, kl = kl_3_1;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[640]; }
    { const long long ij = ij_5_5, kl = kl_3_2;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[641]; }
    { const long long ij = ij_5_5, kl = kl_4_0;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[642]; }
    { const long long ij = ij_5_5, kl = kl_4_1;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[643]; }
    { const long long ij = ij_5_5, kl = kl_4_2;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[644]; }
    { const long long ij = ij_5_5, kl = kl_5_0;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[645]; }
    { const long long ij = ij_5_5, kl = kl_5_1;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[646]; }
    { const long long ij = ij_5_5, kl = kl_5_2;
      if ((!dab || 5 >= 5) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[647]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_dddp(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 648; ++x) {
        const int ia = x / 108, ibb = (x / 18) % 6, ic = (x / 3) % 6, id = x % 3;
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
__global__ void __launch_bounds__(128) eri_queue_dddp(const EriQueue Q) {
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
        double acc[496];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 496; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_dddp<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_dddp<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 496; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: each leader stores its quartet's whole block at its slot
            if (lead) {
                double res[648];
                hrr_dddp(Q.pairs, p, q, acc, res);
                double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                    (__ldg(&Q.chunk_slot[c]) + base + kq) * (long long)648;
#pragma unroll
                for (int x = 0; x < 648; ++x) dst[x] = res[x];
            }
        } else if (lead) {
            double res[648];
            hrr_dddp(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_dddp(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_dddp(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


void launch_eri_dddp(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    constexpr size_t smem = 0;
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_dddp<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_dddp<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_dddp<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_dddp<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_dddp(int mixed) {

    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dddp<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dddp<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

// Generated by gen_eri.py -- class (pp|pp).  Do not edit.
// VRR entries: 146, contracted block: 81, HRR lines: 162, outputs: 81.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[81], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_pppp(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 81; ++x) acc[x] = 0.0;
    for (int j = j0; j < j1; j += jstep) {
        const PrimPair ket = load_pp(P.pp, ik_.x + j);
        for (int i = i0; i < i1; i += istep) {
            const PrimPair bra = load_pp(P.pp, ib_.x + i);
            const double r = rsqrt(bra.zeta + ket.zeta);
            const double r2 = r * r;
            const double PQx = bra.px - ket.px, PQy = bra.py - ket.py, PQz = bra.pz - ket.pz;
            const double T = bra.zeta * ket.zeta * r2 * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = bra.kab * ket.kab * r;
            double F[5];
            boys_fm<4>(T, B, F);
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
            const VT v1_0_0 = PAx * v0_0_0 + WPx * v0_0_1;
            const VT v1_0_1 = PAx * v0_0_1 + WPx * v0_0_2;
            const VT v1_0_2 = PAx * v0_0_2 + WPx * v0_0_3;
            const VT v1_0_3 = PAx * v0_0_3 + WPx * v0_0_4;
            const VT v2_0_0 = PAy * v0_0_0 + WPy * v0_0_1;
            const VT v2_0_1 = PAy * v0_0_1 + WPy * v0_0_2;
            const VT v2_0_2 = PAy * v0_0_2 + WPy * v0_0_3;
            const VT v2_0_3 = PAy * v0_0_3 + WPy * v0_0_4;
            const VT v3_0_0 = PAz * v0_0_0 + WPz * v0_0_1;
            const VT v3_0_1 = PAz * v0_0_1 + WPz * v0_0_2;
            const VT v3_0_2 = PAz * v0_0_2 + WPz * v0_0_3;
            const VT v3_0_3 = PAz * v0_0_3 + WPz * v0_0_4;
            const VT v4_0_0 = PAx * v1_0_0 + WPx * v1_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v4_0_1 = PAx * v1_0_1 + WPx * v1_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v4_0_2 = PAx * v1_0_2 + WPx * v1_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v5_0_0 = PAx * v2_0_0 + WPx * v2_0_1;
            const VT v5_0_1 = PAx * v2_0_1 + WPx * v2_0_2;
            const VT v5_0_2 = PAx * v2_0_2 + WPx * v2_0_3;
            const VT v6_0_0 = PAx * v3_0_0 + WPx * v3_0_1;
            const VT v6_0_1 = PAx * v3_0_1 + WPx * v3_0_2;
            const VT v6_0_2 = PAx * v3_0_2 + WPx * v3_0_3;
            const VT v7_0_0 = PAy * v2_0_0 + WPy * v2_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v7_0_1 = PAy * v2_0_1 + WPy * v2_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v7_0_2 = PAy * v2_0_2 + WPy * v2_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v8_0_0 = PAy * v3_0_0 + WPy * v3_0_1;
            const VT v8_0_1 = PAy * v3_0_1 + WPy * v3_0_2;
            const VT v8_0_2 = PAy * v3_0_2 + WPy * v3_0_3;
            const VT v9_0_0 = PAz * v3_0_0 + WPz * v3_0_1 + (VT)1.0 * oo2z * (v0_0_0 - rho_z * v0_0_1);
            const VT v9_0_1 = PAz * v3_0_1 + WPz * v3_0_2 + (VT)1.0 * oo2z * (v0_0_1 - rho_z * v0_0_2);
            const VT v9_0_2 = PAz * v3_0_2 + WPz * v3_0_3 + (VT)1.0 * oo2z * (v0_0_2 - rho_z * v0_0_3);
            const VT v0_1_1 = QCx * v0_0_1 + WQx * v0_0_2;
            const VT v1_1_0 = QCx * v1_0_0 + WQx * v1_0_1 + (VT)1.0 * oo2ze * v0_0_1;
            const VT v1_1_1 = QCx * v1_0_1 + WQx * v1_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v2_1_0 = QCx * v2_0_0 + WQx * v2_0_1;
            const VT v2_1_1 = QCx * v2_0_1 + WQx * v2_0_2;
            const VT v3_1_0 = QCx * v3_0_0 + WQx * v3_0_1;
            const VT v3_1_1 = QCx * v3_0_1 + WQx * v3_0_2;
            const VT v4_1_0 = QCx * v4_0_0 + WQx * v4_0_1 + (VT)2.0 * oo2ze * v1_0_1;
            const VT v4_1_1 = QCx * v4_0_1 + WQx * v4_0_2 + (VT)2.0 * oo2ze * v1_0_2;
            const VT v5_1_0 = QCx * v5_0_0 + WQx * v5_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v5_1_1 = QCx * v5_0_1 + WQx * v5_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v6_1_0 = QCx * v6_0_0 + WQx * v6_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v6_1_1 = QCx * v6_0_1 + WQx * v6_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v7_1_0 = QCx * v7_0_0 + WQx * v7_0_1;
            const VT v7_1_1 = QCx * v7_0_1 + WQx * v7_0_2;
            const VT v8_1_0 = QCx * v8_0_0 + WQx * v8_0_1;
            const VT v8_1_1 = QCx * v8_0_1 + WQx * v8_0_2;
            const VT v9_1_0 = QCx * v9_0_0 + WQx * v9_0_1;
            const VT v9_1_1 = QCx * v9_0_1 + WQx * v9_0_2;
            const VT v0_2_1 = QCy * v0_0_1 + WQy * v0_0_2;
            const VT v1_2_0 = QCy * v1_0_0 + WQy * v1_0_1;
            const VT v1_2_1 = QCy * v1_0_1 + WQy * v1_0_2;
            const VT v2_2_0 = QCy * v2_0_0 + WQy * v2_0_1 + (VT)1.0 * oo2ze * v0_0_1;
            const VT v2_2_1 = QCy * v2_0_1 + WQy * v2_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v3_2_0 = QCy * v3_0_0 + WQy * v3_0_1;
            const VT v3_2_1 = QCy * v3_0_1 + WQy * v3_0_2;
            const VT v4_2_0 = QCy * v4_0_0 + WQy * v4_0_1;
            const VT v4_2_1 = QCy * v4_0_1 + WQy * v4_0_2;
            const VT v5_2_0 = QCy * v5_0_0 + WQy * v5_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v5_2_1 = QCy * v5_0_1 + WQy * v5_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v6_2_0 = QCy * v6_0_0 + WQy * v6_0_1;
            const VT v6_2_1 = QCy * v6_0_1 + WQy * v6_0_2;
            const VT v7_2_0 = QCy * v7_0_0 + WQy * v7_0_1 + (VT)2.0 * oo2ze * v2_0_1;
            const VT v7_2_1 = QCy * v7_0_1 + WQy * v7_0_2 + (VT)2.0 * oo2ze * v2_0_2;
            const VT v8_2_0 = QCy * v8_0_0 + WQy * v8_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v8_2_1 = QCy * v8_0_1 + WQy * v8_0_2 + (VT)1.0 * oo2ze * v3_0_2;
            const VT v9_2_0 = QCy * v9_0_0 + WQy * v9_0_1;
            const VT v9_2_1 = QCy * v9_0_1 + WQy * v9_0_2;
            const VT v0_3_1 = QCz * v0_0_1 + WQz * v0_0_2;
            const VT v1_3_0 = QCz * v1_0_0 + WQz * v1_0_1;
            const VT v1_3_1 = QCz * v1_0_1 + WQz * v1_0_2;
            const VT v2_3_0 = QCz * v2_0_0 + WQz * v2_0_1;
            const VT v2_3_1 = QCz * v2_0_1 + WQz * v2_0_2;
            const VT v3_3_0 = QCz * v3_0_0 + WQz * v3_0_1 + (VT)1.0 * oo2ze * v0_0_1;
            const VT v3_3_1 = QCz * v3_0_1 + WQz * v3_0_2 + (VT)1.0 * oo2ze * v0_0_2;
            const VT v4_3_0 = QCz * v4_0_0 + WQz * v4_0_1;
            const VT v4_3_1 = QCz * v4_0_1 + WQz * v4_0_2;
            const VT v5_3_0 = QCz * v5_0_0 + WQz * v5_0_1;
            const VT v5_3_1 = QCz * v5_0_1 + WQz * v5_0_2;
            const VT v6_3_0 = QCz * v6_0_0 + WQz * v6_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v6_3_1 = QCz * v6_0_1 + WQz * v6_0_2 + (VT)1.0 * oo2ze * v1_0_2;
            const VT v7_3_0 = QCz * v7_0_0 + WQz * v7_0_1;
            const VT v7_3_1 = QCz * v7_0_1 + WQz * v7_0_2;
            const VT v8_3_0 = QCz * v8_0_0 + WQz * v8_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v8_3_1 = QCz * v8_0_1 + WQz * v8_0_2 + (VT)1.0 * oo2ze * v2_0_2;
            const VT v9_3_0 = QCz * v9_0_0 + WQz * v9_0_1 + (VT)2.0 * oo2ze * v3_0_1;
            const VT v9_3_1 = QCz * v9_0_1 + WQz * v9_0_2 + (VT)2.0 * oo2ze * v3_0_2;
            const VT v1_4_0 = QCx * v1_1_0 + WQx * v1_1_1 + (VT)1.0 * oo2ze * v0_1_1 + (VT)1.0 * oo2e * (v1_0_0 - rho_e * v1_0_1);
            const VT v2_4_0 = QCx * v2_1_0 + WQx * v2_1_1 + (VT)1.0 * oo2e * (v2_0_0 - rho_e * v2_0_1);
            const VT v3_4_0 = QCx * v3_1_0 + WQx * v3_1_1 + (VT)1.0 * oo2e * (v3_0_0 - rho_e * v3_0_1);
            const VT v4_4_0 = QCx * v4_1_0 + WQx * v4_1_1 + (VT)2.0 * oo2ze * v1_1_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v5_4_0 = QCx * v5_1_0 + WQx * v5_1_1 + (VT)1.0 * oo2ze * v2_1_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v6_4_0 = QCx * v6_1_0 + WQx * v6_1_1 + (VT)1.0 * oo2ze * v3_1_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v7_4_0 = QCx * v7_1_0 + WQx * v7_1_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v8_4_0 = QCx * v8_1_0 + WQx * v8_1_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v9_4_0 = QCx * v9_1_0 + WQx * v9_1_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v1_5_0 = QCx * v1_2_0 + WQx * v1_2_1 + (VT)1.0 * oo2ze * v0_2_1;
            const VT v2_5_0 = QCx * v2_2_0 + WQx * v2_2_1;
            const VT v3_5_0 = QCx * v3_2_0 + WQx * v3_2_1;
            const VT v4_5_0 = QCx * v4_2_0 + WQx * v4_2_1 + (VT)2.0 * oo2ze * v1_2_1;
            const VT v5_5_0 = QCx * v5_2_0 + WQx * v5_2_1 + (VT)1.0 * oo2ze * v2_2_1;
            const VT v6_5_0 = QCx * v6_2_0 + WQx * v6_2_1 + (VT)1.0 * oo2ze * v3_2_1;
            const VT v7_5_0 = QCx * v7_2_0 + WQx * v7_2_1;
            const VT v8_5_0 = QCx * v8_2_0 + WQx * v8_2_1;
            const VT v9_5_0 = QCx * v9_2_0 + WQx * v9_2_1;
            const VT v1_6_0 = QCx * v1_3_0 + WQx * v1_3_1 + (VT)1.0 * oo2ze * v0_3_1;
            const VT v2_6_0 = QCx * v2_3_0 + WQx * v2_3_1;
            const VT v3_6_0 = QCx * v3_3_0 + WQx * v3_3_1;
            const VT v4_6_0 = QCx * v4_3_0 + WQx * v4_3_1 + (VT)2.0 * oo2ze * v1_3_1;
            const VT v5_6_0 = QCx * v5_3_0 + WQx * v5_3_1 + (VT)1.0 * oo2ze * v2_3_1;
            const VT v6_6_0 = QCx * v6_3_0 + WQx * v6_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v7_6_0 = QCx * v7_3_0 + WQx * v7_3_1;
            const VT v8_6_0 = QCx * v8_3_0 + WQx * v8_3_1;
            const VT v9_6_0 = QCx * v9_3_0 + WQx * v9_3_1;
            const VT v1_7_0 = QCy * v1_2_0 + WQy * v1_2_1 + (VT)1.0 * oo2e * (v1_0_0 - rho_e * v1_0_1);
            const VT v2_7_0 = QCy * v2_2_0 + WQy * v2_2_1 + (VT)1.0 * oo2ze * v0_2_1 + (VT)1.0 * oo2e * (v2_0_0 - rho_e * v2_0_1);
            const VT v3_7_0 = QCy * v3_2_0 + WQy * v3_2_1 + (VT)1.0 * oo2e * (v3_0_0 - rho_e * v3_0_1);
            const VT v4_7_0 = QCy * v4_2_0 + WQy * v4_2_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v5_7_0 = QCy * v5_2_0 + WQy * v5_2_1 + (VT)1.0 * oo2ze * v1_2_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v6_7_0 = QCy * v6_2_0 + WQy * v6_2_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v7_7_0 = QCy * v7_2_0 + WQy * v7_2_1 + (VT)2.0 * oo2ze * v2_2_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v8_7_0 = QCy * v8_2_0 + WQy * v8_2_1 + (VT)1.0 * oo2ze * v3_2_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v9_7_0 = QCy * v9_2_0 + WQy * v9_2_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            const VT v1_8_0 = QCy * v1_3_0 + WQy * v1_3_1;
            const VT v2_8_0 = QCy * v2_3_0 + WQy * v2_3_1 + (VT)1.0 * oo2ze * v0_3_1;
            const VT v3_8_0 = QCy * v3_3_0 + WQy * v3_3_1;
            const VT v4_8_0 = QCy * v4_3_0 + WQy * v4_3_1;
            const VT v5_8_0 = QCy * v5_3_0 + WQy * v5_3_1 + (VT)1.0 * oo2ze * v1_3_1;
            const VT v6_8_0 = QCy * v6_3_0 + WQy * v6_3_1;
            const VT v7_8_0 = QCy * v7_3_0 + WQy * v7_3_1 + (VT)2.0 * oo2ze * v2_3_1;
            const VT v8_8_0 = QCy * v8_3_0 + WQy * v8_3_1 + (VT)1.0 * oo2ze * v3_3_1;
            const VT v9_8_0 = QCy * v9_3_0 + WQy * v9_3_1;
            const VT v1_9_0 = QCz * v1_3_0 + WQz * v1_3_1 + (VT)1.0 * oo2e * (v1_0_0 - rho_e * v1_0_1);
            const VT v2_9_0 = QCz * v2_3_0 + WQz * v2_3_1 + (VT)1.0 * oo2e * (v2_0_0 - rho_e * v2_0_1);
            const VT v3_9_0 = QCz * v3_3_0 + WQz * v3_3_1 + (VT)1.0 * oo2ze * v0_3_1 + (VT)1.0 * oo2e * (v3_0_0 - rho_e * v3_0_1);
            const VT v4_9_0 = QCz * v4_3_0 + WQz * v4_3_1 + (VT)1.0 * oo2e * (v4_0_0 - rho_e * v4_0_1);
            const VT v5_9_0 = QCz * v5_3_0 + WQz * v5_3_1 + (VT)1.0 * oo2e * (v5_0_0 - rho_e * v5_0_1);
            const VT v6_9_0 = QCz * v6_3_0 + WQz * v6_3_1 + (VT)1.0 * oo2ze * v1_3_1 + (VT)1.0 * oo2e * (v6_0_0 - rho_e * v6_0_1);
            const VT v7_9_0 = QCz * v7_3_0 + WQz * v7_3_1 + (VT)1.0 * oo2e * (v7_0_0 - rho_e * v7_0_1);
            const VT v8_9_0 = QCz * v8_3_0 + WQz * v8_3_1 + (VT)1.0 * oo2ze * v2_3_1 + (VT)1.0 * oo2e * (v8_0_0 - rho_e * v8_0_1);
            const VT v9_9_0 = QCz * v9_3_0 + WQz * v9_3_1 + (VT)2.0 * oo2ze * v3_3_1 + (VT)1.0 * oo2e * (v9_0_0 - rho_e * v9_0_1);
            acc[0] += (double)v1_1_0;
            acc[1] += (double)v1_2_0;
            acc[2] += (double)v1_3_0;
            acc[3] += (double)v1_4_0;
            acc[4] += (double)v1_5_0;
            acc[5] += (double)v1_6_0;
            acc[6] += (double)v1_7_0;
            acc[7] += (double)v1_8_0;
            acc[8] += (double)v1_9_0;
            acc[9] += (double)v2_1_0;
            acc[10] += (double)v2_2_0;
            acc[11] += (double)v2_3_0;
            acc[12] += (double)v2_4_0;
            acc[13] += (double)v2_5_0;
            acc[14] += (double)v2_6_0;
            acc[15] += (double)v2_7_0;
            acc[16] += (double)v2_8_0;
            acc[17] += (double)v2_9_0;
            acc[18] += (double)v3_1_0;
            acc[19] += (double)v3_2_0;
            acc[20] += (double)v3_3_0;
            acc[21] += (double)v3_4_0;
            acc[22] += (double)v3_5_0;
            acc[23] += (double)v3_6_0;
            acc[24] += (double)v3_7_0;
            acc[25] += (double)v3_8_0;
            acc[26] += (double)v3_9_0;
            acc[27] += (double)v4_1_0;
            acc[28] += (double)v4_2_0;
            acc[29] += (double)v4_3_0;
            acc[30] += (double)v4_4_0;
            acc[31] += (double)v4_5_0;
            acc[32] += (double)v4_6_0;
            acc[33] += (double)v4_7_0;
            acc[34] += (double)v4_8_0;
            acc[35] += (double)v4_9_0;
            acc[36] += (double)v5_1_0;
            acc[37] += (double)v5_2_0;
            acc[38] += (double)v5_3_0;
            acc[39] += (double)v5_4_0;
            acc[40] += (double)v5_5_0;
            acc[41] += (double)v5_6_0;
            acc[42] += (double)v5_7_0;
            acc[43] += (double)v5_8_0;
            acc[44] += (double)v5_9_0;
            acc[45] += (double)v6_1_0;
            acc[46] += (double)v6_2_0;
            acc[47] += (double)v6_3_0;
            acc[48] += (double)v6_4_0;
            acc[49] += (double)v6_5_0;
            acc[50] += (double)v6_6_0;
            acc[51] += (double)v6_7_0;
            acc[52] += (double)v6_8_0;
            acc[53] += (double)v6_9_0;
            acc[54] += (double)v7_1_0;
            acc[55] += (double)v7_2_0;
            acc[56] += (double)v7_3_0;
            acc[57] += (double)v7_4_0;
            acc[58] += (double)v7_5_0;
            acc[59] += (double)v7_6_0;
            acc[60] += (double)v7_7_0;
            acc[61] += (double)v7_8_0;
            acc[62] += (double)v7_9_0;
            acc[63] += (double)v8_1_0;
            acc[64] += (double)v8_2_0;
            acc[65] += (double)v8_3_0;
            acc[66] += (double)v8_4_0;
            acc[67] += (double)v8_5_0;
            acc[68] += (double)v8_6_0;
            acc[69] += (double)v8_7_0;
            acc[70] += (double)v8_8_0;
            acc[71] += (double)v8_9_0;
            acc[72] += (double)v9_1_0;
            acc[73] += (double)v9_2_0;
            acc[74] += (double)v9_3_0;
            acc[75] += (double)v9_4_0;
            acc[76] += (double)v9_5_0;
            acc[77] += (double)v9_6_0;
            acc[78] += (double)v9_7_0;
            acc[79] += (double)v9_8_0;
            acc[80] += (double)v9_9_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[81] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_pppp(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h1_1_4 = acc[30] + ABx * acc[3];
    const double h1_1_1 = acc[27] + ABx * acc[0];
    const double k1_1_1_1 = h1_1_4 + CDx * h1_1_1;
    const double h1_1_5 = acc[31] + ABx * acc[4];
    const double k1_1_1_2 = h1_1_5 + CDy * h1_1_1;
    const double h1_1_6 = acc[32] + ABx * acc[5];
    const double k1_1_1_3 = h1_1_6 + CDz * h1_1_1;
    const double h1_1_2 = acc[28] + ABx * acc[1];
    const double k1_1_2_1 = h1_1_5 + CDx * h1_1_2;
    const double h1_1_7 = acc[33] + ABx * acc[6];
    const double k1_1_2_2 = h1_1_7 + CDy * h1_1_2;
    const double h1_1_8 = acc[34] + ABx * acc[7];
    const double k1_1_2_3 = h1_1_8 + CDz * h1_1_2;
    const double h1_1_3 = acc[29] + ABx * acc[2];
    const double k1_1_3_1 = h1_1_6 + CDx * h1_1_3;
    const double k1_1_3_2 = h1_1_8 + CDy * h1_1_3;
    const double h1_1_9 = acc[35] + ABx * acc[8];
    const double k1_1_3_3 = h1_1_9 + CDz * h1_1_3;
    const double h1_2_4 = acc[39] + ABy * acc[3];
    const double h1_2_1 = acc[36] + ABy * acc[0];
    const double k1_2_1_1 = h1_2_4 + CDx * h1_2_1;
    const double h1_2_5 = acc[40] + ABy * acc[4];
    const double k1_2_1_2 = h1_2_5 + CDy * h1_2_1;
    const double h1_2_6 = acc[41] + ABy * acc[5];
    const double k1_2_1_3 = h1_2_6 + CDz * h1_2_1;
    const double h1_2_2 = acc[37] + ABy * acc[1];
    const double k1_2_2_1 = h1_2_5 + CDx * h1_2_2;
    const double h1_2_7 = acc[42] + ABy * acc[6];
    const double k1_2_2_2 = h1_2_7 + CDy * h1_2_2;
    const double h1_2_8 = acc[43] + ABy * acc[7];
    const double k1_2_2_3 = h1_2_8 + CDz * h1_2_2;
    const double h1_2_3 = acc[38] + ABy * acc[2];
    const double k1_2_3_1 = h1_2_6 + CDx * h1_2_3;
    const double k1_2_3_2 = h1_2_8 + CDy * h1_2_3;
    const double h1_2_9 = acc[44] + ABy * acc[8];
    const double k1_2_3_3 = h1_2_9 + CDz * h1_2_3;
    const double h1_3_4 = acc[48] + ABz * acc[3];
    const double h1_3_1 = acc[45] + ABz * acc[0];
    const double k1_3_1_1 = h1_3_4 + CDx * h1_3_1;
    const double h1_3_5 = acc[49] + ABz * acc[4];
    const double k1_3_1_2 = h1_3_5 + CDy * h1_3_1;
    const double h1_3_6 = acc[50] + ABz * acc[5];
    const double k1_3_1_3 = h1_3_6 + CDz * h1_3_1;
    const double h1_3_2 = acc[46] + ABz * acc[1];
    const double k1_3_2_1 = h1_3_5 + CDx * h1_3_2;
    const double h1_3_7 = acc[51] + ABz * acc[6];
    const double k1_3_2_2 = h1_3_7 + CDy * h1_3_2;
    const double h1_3_8 = acc[52] + ABz * acc[7];
    const double k1_3_2_3 = h1_3_8 + CDz * h1_3_2;
    const double h1_3_3 = acc[47] + ABz * acc[2];
    const double k1_3_3_1 = h1_3_6 + CDx * h1_3_3;
    const double k1_3_3_2 = h1_3_8 + CDy * h1_3_3;
    const double h1_3_9 = acc[53] + ABz * acc[8];
    const double k1_3_3_3 = h1_3_9 + CDz * h1_3_3;
    const double h2_1_4 = acc[39] + ABx * acc[12];
    const double h2_1_1 = acc[36] + ABx * acc[9];
    const double k2_1_1_1 = h2_1_4 + CDx * h2_1_1;
    const double h2_1_5 = acc[40] + ABx * acc[13];
    const double k2_1_1_2 = h2_1_5 + CDy * h2_1_1;
    const double h2_1_6 = acc[41] + ABx * acc[14];
    const double k2_1_1_3 = h2_1_6 + CDz * h2_1_1;
    const double h2_1_2 = acc[37] + ABx * acc[10];
    const double k2_1_2_1 = h2_1_5 + CDx * h2_1_2;
    const double h2_1_7 = acc[42] + ABx * acc[15];
    const double k2_1_2_2 = h2_1_7 + CDy * h2_1_2;
    const double h2_1_8 = acc[43] + ABx * acc[16];
    const double k2_1_2_3 = h2_1_8 + CDz * h2_1_2;
    const double h2_1_3 = acc[38] + ABx * acc[11];
    const double k2_1_3_1 = h2_1_6 + CDx * h2_1_3;
    const double k2_1_3_2 = h2_1_8 + CDy * h2_1_3;
    const double h2_1_9 = acc[44] + ABx * acc[17];
    const double k2_1_3_3 = h2_1_9 + CDz * h2_1_3;
    const double h2_2_4 = acc[57] + ABy * acc[12];
    const double h2_2_1 = acc[54] + ABy * acc[9];
    const double k2_2_1_1 = h2_2_4 + CDx * h2_2_1;
    const double h2_2_5 = acc[58] + ABy * acc[13];
    const double k2_2_1_2 = h2_2_5 + CDy * h2_2_1;
    const double h2_2_6 = acc[59] + ABy * acc[14];
    const double k2_2_1_3 = h2_2_6 + CDz * h2_2_1;
    const double h2_2_2 = acc[55] + ABy * acc[10];
    const double k2_2_2_1 = h2_2_5 + CDx * h2_2_2;
    const double h2_2_7 = acc[60] + ABy * acc[15];
    const double k2_2_2_2 = h2_2_7 + CDy * h2_2_2;
    const double h2_2_8 = acc[61] + ABy * acc[16];
    const double k2_2_2_3 = h2_2_8 + CDz * h2_2_2;
    const double h2_2_3 = acc[56] + ABy * acc[11];
    const double k2_2_3_1 = h2_2_6 + CDx * h2_2_3;
    const double k2_2_3_2 = h2_2_8 + CDy * h2_2_3;
    const double h2_2_9 = acc[62] + ABy * acc[17];
    const double k2_2_3_3 = h2_2_9 + CDz * h2_2_3;
    const double h2_3_4 = acc[66] + ABz * acc[12];
    const double h2_3_1 = acc[63] + ABz * acc[9];
    const double k2_3_1_1 = h2_3_4 + CDx * h2_3_1;
    const double h2_3_5 = acc[67] + ABz * acc[13];
    const double k2_3_1_2 = h2_3_5 + CDy * h2_3_1;
    const double h2_3_6 = acc[68] + ABz * acc[14];
    const double k2_3_1_3 = h2_3_6 + CDz * h2_3_1;
    const double h2_3_2 = acc[64] + ABz * acc[10];
    const double k2_3_2_1 = h2_3_5 + CDx * h2_3_2;
    const double h2_3_7 = acc[69] + ABz * acc[15];
    const double k2_3_2_2 = h2_3_7 + CDy * h2_3_2;
    const double h2_3_8 = acc[70] + ABz * acc[16];
    const double k2_3_2_3 = h2_3_8 + CDz * h2_3_2;
    const double h2_3_3 = acc[65] + ABz * acc[11];
    const double k2_3_3_1 = h2_3_6 + CDx * h2_3_3;
    const double k2_3_3_2 = h2_3_8 + CDy * h2_3_3;
    const double h2_3_9 = acc[71] + ABz * acc[17];
    const double k2_3_3_3 = h2_3_9 + CDz * h2_3_3;
    const double h3_1_4 = acc[48] + ABx * acc[21];
    const double h3_1_1 = acc[45] + ABx * acc[18];
    const double k3_1_1_1 = h3_1_4 + CDx * h3_1_1;
    const double h3_1_5 = acc[49] + ABx * acc[22];
    const double k3_1_1_2 = h3_1_5 + CDy * h3_1_1;
    const double h3_1_6 = acc[50] + ABx * acc[23];
    const double k3_1_1_3 = h3_1_6 + CDz * h3_1_1;
    const double h3_1_2 = acc[46] + ABx * acc[19];
    const double k3_1_2_1 = h3_1_5 + CDx * h3_1_2;
    const double h3_1_7 = acc[51] + ABx * acc[24];
    const double k3_1_2_2 = h3_1_7 + CDy * h3_1_2;
    const double h3_1_8 = acc[52] + ABx * acc[25];
    const double k3_1_2_3 = h3_1_8 + CDz * h3_1_2;
    const double h3_1_3 = acc[47] + ABx * acc[20];
    const double k3_1_3_1 = h3_1_6 + CDx * h3_1_3;
    const double k3_1_3_2 = h3_1_8 + CDy * h3_1_3;
    const double h3_1_9 = acc[53] + ABx * acc[26];
    const double k3_1_3_3 = h3_1_9 + CDz * h3_1_3;
    const double h3_2_4 = acc[66] + ABy * acc[21];
    const double h3_2_1 = acc[63] + ABy * acc[18];
    const double k3_2_1_1 = h3_2_4 + CDx * h3_2_1;
    const double h3_2_5 = acc[67] + ABy * acc[22];
    const double k3_2_1_2 = h3_2_5 + CDy * h3_2_1;
    const double h3_2_6 = acc[68] + ABy * acc[23];
    const double k3_2_1_3 = h3_2_6 + CDz * h3_2_1;
    const double h3_2_2 = acc[64] + ABy * acc[19];
    const double k3_2_2_1 = h3_2_5 + CDx * h3_2_2;
    const double h3_2_7 = acc[69] + ABy * acc[24];
    const double k3_2_2_2 = h3_2_7 + CDy * h3_2_2;
    const double h3_2_8 = acc[70] + ABy * acc[25];
    const double k3_2_2_3 = h3_2_8 + CDz * h3_2_2;
    const double h3_2_3 = acc[65] + ABy * acc[20];
    const double k3_2_3_1 = h3_2_6 + CDx * h3_2_3;
    const double k3_2_3_2 = h3_2_8 + CDy * h3_2_3;
    const double h3_2_9 = acc[71] + ABy * acc[26];
    const double k3_2_3_3 = h3_2_9 + CDz * h3_2_3;
    const double h3_3_4 = acc[75] + ABz * acc[21];
    const double h3_3_1 = acc[72] + ABz * acc[18];
    const double k3_3_1_1 = h3_3_4 + CDx * h3_3_1;
    const double h3_3_5 = acc[76] + ABz * acc[22];
    const double k3_3_1_2 = h3_3_5 + CDy * h3_3_1;
    const double h3_3_6 = acc[77] + ABz * acc[23];
    const double k3_3_1_3 = h3_3_6 + CDz * h3_3_1;
    const double h3_3_2 = acc[73] + ABz * acc[19];
    const double k3_3_2_1 = h3_3_5 + CDx * h3_3_2;
    const double h3_3_7 = acc[78] + ABz * acc[24];
    const double k3_3_2_2 = h3_3_7 + CDy * h3_3_2;
    const double h3_3_8 = acc[79] + ABz * acc[25];
    const double k3_3_2_3 = h3_3_8 + CDz * h3_3_2;
    const double h3_3_3 = acc[74] + ABz * acc[20];
    const double k3_3_3_1 = h3_3_6 + CDx * h3_3_3;
    const double k3_3_3_2 = h3_3_8 + CDy * h3_3_3;
    const double h3_3_9 = acc[80] + ABz * acc[26];
    const double k3_3_3_3 = h3_3_9 + CDz * h3_3_3;
    res[0] = k1_1_1_1;
    res[1] = k1_1_1_2;
    res[2] = k1_1_1_3;
    res[3] = k1_1_2_1;
    res[4] = k1_1_2_2;
    res[5] = k1_1_2_3;
    res[6] = k1_1_3_1;
    res[7] = k1_1_3_2;
    res[8] = k1_1_3_3;
    res[9] = k1_2_1_1;
    res[10] = k1_2_1_2;
    res[11] = k1_2_1_3;
    res[12] = k1_2_2_1;
    res[13] = k1_2_2_2;
    res[14] = k1_2_2_3;
    res[15] = k1_2_3_1;
    res[16] = k1_2_3_2;
    res[17] = k1_2_3_3;
    res[18] = k1_3_1_1;
    res[19] = k1_3_1_2;
    res[20] = k1_3_1_3;
    res[21] = k1_3_2_1;
    res[22] = k1_3_2_2;
    res[23] = k1_3_2_3;
    res[24] = k1_3_3_1;
    res[25] = k1_3_3_2;
    res[26] = k1_3_3_3;
    res[27] = k2_1_1_1;
    res[28] = k2_1_1_2;
    res[29] = k2_1_1_3;
    res[30] = k2_1_2_1;
    res[31] = k2_1_2_2;
    res[32] = k2_1_2_3;
    res[33] = k2_1_3_1;
    res[34] = k2_1_3_2;
    res[35] = k2_1_3_3;
    res[36] = k2_2_1_1;
    res[37] = k2_2_1_2;
    res[38] = k2_2_1_3;
    res[39] = k2_2_2_1;
    res[40] = k2_2_2_2;
    res[41] = k2_2_2_3;
    res[42] = k2_2_3_1;
    res[43] = k2_2_3_2;
    res[44] = k2_2_3_3;
    res[45] = k2_3_1_1;
    res[46] = k2_3_1_2;
    res[47] = k2_3_1_3;
    res[48] = k2_3_2_1;
    res[49] = k2_3_2_2;
    res[50] = k2_3_2_3;
    res[51] = k2_3_3_1;
    res[52] = k2_3_3_2;
    res[53] = k2_3_3_3;
    res[54] = k3_1_1_1;
    res[55] = k3_1_1_2;
    res[56] = k3_1_1_3;
    res[57] = k3_1_2_1;
    res[58] = k3_1_2_2;
    res[59] = k3_1_2_3;
    res[60] = k3_1_3_1;
    res[61] = k3_1_3_2;
    res[62] = k3_1_3_3;
    res[63] = k3_2_1_1;
    res[64] = k3_2_1_2;
    res[65] = k3_2_1_3;
    res[66] = k3_2_2_1;
    res[67] = k3_2_2_2;
    res[68] = k3_2_2_3;
    res[69] = k3_2_3_1;
    res[70] = k3_2_3_2;
    res[71] = k3_2_3_3;
    res[72] = k3_3_1_1;
    res[73] = k3_3_1_2;
    res[74] = k3_3_1_3;
    res[75] = k3_3_2_1;
    res[76] = k3_3_2_2;
    res[77] = k3_3_2_3;
    res[78] = k3_3_3_1;
    res[79] = k3_3_3_2;
    res[80] = k3_3_3_3;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[81]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_pppp(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[81];
    vrr_pppp<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 81; ++x) acc_out[x] = acc[x];
    }
    hrr_pppp(P, p, q, acc, res);
}

__device__ __forceinline__ void store_pppp(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[0]; }
    { const long long ij = ij_0_0, kl = kl_0_1;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[1]; }
    { const long long ij = ij_0_0, kl = kl_0_2;
      if ((!dab || 0 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[2]; }
    { const long long ij = ij_0_0, kl = kl_1_0;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[3]; }
    { const long long ij = ij_0_0, kl = kl_1_1;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[4]; }
    { const long long ij = ij_0_0, kl = kl_1_2;
      if ((!dab || 0 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[5]; }
    { const long long ij = ij_0_0, kl = kl_2_0;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[6]; }
    { const long long ij = ij_0_0, kl = kl_2_1;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[7]; }
    { const long long ij = ij_0_0, kl = kl_2_2;
      if ((!dab || 0 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[8]; }
    { const long long ij = ij_0_1, kl = kl_0_0;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[9]; }
    { const long long ij = ij_0_1, kl = kl_0_1;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[10]; }
    { const long long ij = ij_0_1, kl = kl_0_2;
      if ((!dab || 0 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[11]; }
    { const long long ij = ij_0_1, kl = kl_1_0;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[12]; }
    { const long long ij = ij_0_1, kl = kl_1_1;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[13]; }
    { const long long ij = ij_0_1, kl = kl_1_2;
      if ((!dab || 0 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[14]; }
    { const long long ij = ij_0_1, kl = kl_2_0;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[15]; }
    { const long long ij = ij_0_1, kl = kl_2_1;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[16]; }
    { const long long ij = ij_0_1, kl = kl_2_2;
      if ((!dab || 0 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[17]; }
    { const long long ij = ij_0_2, kl = kl_0_0;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[18]; }
    { const long long ij = ij_0_2, kl = kl_0_1;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[19]; }
    { const long long ij = ij_0_2, kl = kl_0_2;
      if ((!dab || 0 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[20]; }
    { const long long ij = ij_0_2, kl = kl_1_0;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[21]; }
    { const long long ij = ij_0_2, kl = kl_1_1;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[22]; }
    { const long long ij = ij_0_2, kl = kl_1_2;
      if ((!dab || 0 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[23]; }
    { const long long ij = ij_0_2, kl = kl_2_0;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[24]; }
    { const long long ij = ij_0_2, kl = kl_2_1;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[25]; }
    { const long long ij = ij_0_2, kl = kl_2_2;
      if ((!dab || 0 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[26]; }
    { const long long ij = ij_1_0, kl = kl_0_0;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[27]; }
    { const long long ij = ij_1_0, kl = kl_0_1;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[28]; }
    { const long long ij = ij_1_0, kl = kl_0_2;
      if ((!dab || 1 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[29]; }
    { const long long ij = ij_1_0, kl = kl_1_0;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[30]; }
    { const long long ij = ij_1_0, kl = kl_1_1;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[31]; }
    { const long long ij = ij_1_0, kl = kl_1_2;
      if ((!dab || 1 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[32]; }
    { const long long ij = ij_1_0, kl = kl_2_0;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[33]; }
    { const long long ij = ij_1_0, kl = kl_2_1;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[34]; }
    { const long long ij = ij_1_0, kl = kl_2_2;
      if ((!dab || 1 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[35]; }
    { const long long ij = ij_1_1, kl = kl_0_0;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[36]; }
    { const long long ij = ij_1_1, kl = kl_0_1;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[37]; }
    { const long long ij = ij_1_1, kl = kl_0_2;
      if ((!dab || 1 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[38]; }
    { const long long ij = ij_1_1, kl = kl_1_0;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[39]; }
    { const long long ij = ij_1_1, kl = kl_1_1;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[40]; }
    { const long long ij = ij_1_1, kl = kl_1_2;
      if ((!dab || 1 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[41]; }
    { const long long ij = ij_1_1, kl = kl_2_0;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[42]; }
    { const long long ij = ij_1_1, kl = kl_2_1;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[43]; }
    { const long long ij = ij_1_1, kl = kl_2_2;
      if ((!dab || 1 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[44]; }
    { const long long ij = ij_1_2, kl = kl_0_0;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[45]; }
    { const long long ij = ij_1_2, kl = kl_0_1;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[46]; }
    { const long long ij = ij_1_2, kl = kl_0_2;
      if ((!dab || 1 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[47]; }
    { const long long ij = ij_1_2, kl = kl_1_0;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[48]; }
    { const long long ij = ij_1_2, kl = kl_1_1;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[49]; }
    { const long long ij = ij_1_2, kl = kl_1_2;
      if ((!dab || 1 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[50]; }
    { const long long ij = ij_1_2, kl = kl_2_0;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[51]; }
    { const long long ij = ij_1_2, kl = kl_2_1;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[52]; }
    { const long long ij = ij_1_2, kl = kl_2_2;
      if ((!dab || 1 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[53]; }
    { const long long ij = ij_2_0, kl = kl_0_0;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[54]; }
    { const long long ij = ij_2_0, kl = kl_0_1;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[55]; }
    { const long long ij = ij_2_0, kl = kl_0_2;
      if ((!dab || 2 >= 0) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[56]; }
    { const long long ij = ij_2_0, kl = kl_1_0;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[57]; }
    { const long long ij = ij_2_0, kl = kl_1_1;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[58]; }
    { const long long ij = ij_2_0, kl = kl_1_2;
      if ((!dab || 2 >= 0) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[59]; }
    { const long long ij = ij_2_0, kl = kl_2_0;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[60]; }
    { const long long ij = ij_2_0, kl = kl_2_1;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[61]; }
    { const long long ij = ij_2_0, kl = kl_2_2;
      if ((!dab || 2 >= 0) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[62]; }
    { const long long ij = ij_2_1, kl = kl_0_0;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[63]; }
    { const long long ij = ij_2_1, kl = kl_0_1;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[64]; }
    { const long long ij = ij_2_1, kl = kl_0_2;
      if ((!dab || 2 >= 1) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[65]; }
    { const long long ij = ij_2_1, kl = kl_1_0;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[66]; }
    { const long long ij = ij_2_1, kl = kl_1_1;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[67]; }
    { const long long ij = ij_2_1, kl = kl_1_2;
      if ((!dab || 2 >= 1) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[68]; }
    { const long long ij = ij_2_1, kl = kl_2_0;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[69]; }
    { const long long ij = ij_2_1, kl = kl_2_1;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[70]; }
    { const long long ij = ij_2_1, kl = kl_2_2;
      if ((!dab || 2 >= 1) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[71]; }
    { const long long ij = ij_2_2, kl = kl_0_0;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[72]; }
    { const long long ij = ij_2_2, kl = kl_0_1;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[73]; }
    { const long long ij = ij_2_2, kl = kl_0_2;
      if ((!dab || 2 >= 2) && (!dcd || 0 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[74]; }
    { const long long ij = ij_2_2, kl = kl_1_0;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[75]; }
    { const long long ij = ij_2_2, kl = kl_1_1;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[76]; }
    { const long long ij = ij_2_2, kl = kl_1_2;
      if ((!dab || 2 >= 2) && (!dcd || 1 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[77]; }
    { const long long ij = ij_2_2, kl = kl_2_0;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 0) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[78]; }
    { const long long ij = ij_2_2, kl = kl_2_1;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 1) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[79]; }
    { const long long ij = ij_2_2, kl = kl_2_2;
      if ((!dab || 2 >= 2) && (!dcd || 2 >= 2) && (!same || ij >= kl)) out[packed_index(ij, kl)] = res[80]; }
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_pppp(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 81; ++x) {
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
__global__ void __launch_bounds__(128) eri_queue_pppp(const EriQueue Q) {
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
        double acc[81];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 81; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_pppp<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_pppp<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 81; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 81 doubles (launch_eri_pppp)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 81);
            if (lead) hrr_pppp(Q.pairs, p, q, acc, sb + kq * 81);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)81;
            for (int t = lane; t < nlive * 81; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[81];
            hrr_pppp(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_pppp(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_pppp(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (82944 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_pppp() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_pppp<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 82944);
        cudaFuncSetAttribute(eri_queue_pppp<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 82944);
        done[dev] = true;
    }
}

void launch_eri_pppp(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 82944 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 82944 : 0;
    if (smem) eri_prepare_pppp();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_pppp<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_pppp<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_pppp<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_pppp<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_pppp(int mixed) {
    eri_prepare_pppp();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_pppp<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_pppp<0, 0>, 128, 0);
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
__global__ void __launch_bounds__(128) schwarz_kernel_pppp(PairTab P, BoysTab B, int p0, int np,
                                                          double2 *pbound, double *qout, int full) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int p = p0 + t;
    const int4 in = __ldg(&P.info[p]);
    double res[81];
    if (full) {
        quartet_pppp<double>(P, B, p, p, 0, in.y, 0, in.y, res);
        double m = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[10]));
    m = fmax(m, fabs(res[20]));
    m = fmax(m, fabs(res[30]));
    m = fmax(m, fabs(res[40]));
    m = fmax(m, fabs(res[50]));
    m = fmax(m, fabs(res[60]));
    m = fmax(m, fabs(res[70]));
    m = fmax(m, fabs(res[80]));
        qout[p] = sqrt(m);
        return;
    }
    double acc[81];
    for (int k = 0; k < in.y; ++k) {
        quartet_pppp<double>(P, B, p, p, k, k + 1, k, k + 1, res, acc);
        double m = 0.0, w = 0.0;
    m = fmax(m, fabs(res[0]));
    m = fmax(m, fabs(res[10]));
    m = fmax(m, fabs(res[20]));
    m = fmax(m, fabs(res[30]));
    m = fmax(m, fabs(res[40]));
    m = fmax(m, fabs(res[50]));
    m = fmax(m, fabs(res[60]));
    m = fmax(m, fabs(res[70]));
    m = fmax(m, fabs(res[80]));
        w = fmax(w, fabs(acc[0]));
        w = fmax(w, fabs(acc[10]));
        w = fmax(w, fabs(acc[20]));
        w = fmax(w, fabs(acc[30]));
        w = fmax(w, fabs(acc[40]));
        w = fmax(w, fabs(acc[50]));
        w = fmax(w, fabs(acc[60]));
        w = fmax(w, fabs(acc[70]));
        w = fmax(w, fabs(acc[80]));
        pbound[in.x + k] = make_double2(sqrt(m), sqrt(w));
    }
}

void launch_schwarz_pppp(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound,
                          double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    schwarz_kernel_pppp<<<(np + 127) / 128, 128, 0, s>>>(P, B, p0, np, pbound, qout, full);
}

}  // namespace molints

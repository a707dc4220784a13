// Generated by gen_eri.py -- class (dp|ps).  Do not edit.
// VRR entries: 103, contracted block: 48, HRR lines: 54, outputs: 54.
#include "../eri_common.cuh"

namespace molints {

// The contracted [e0|f0] block of bra pair p and ket pair q into acc[48], summed over
// the bra primitive pairs i0, i0 + istep, ... < i1 and the ket primitive pairs j0, j0 + jstep,
// ... < j1 of the two shell pairs.  VT is the VRR arithmetic type (double, or float for MIXED).
// The ket loop is outside: a warp shares its bra pair, so the inner bra loads are broadcasts
// and each lane's ket record is loaded once.  Steps above 1 split one quartet's primitive
// quartets over the lanes of a split group (their blocks are summed before the HRR).
template <typename VT>
__device__ __forceinline__ void vrr_dpps(const PairTab &P, const BoysTab &B, int p, int q,
                                          int i0, int i1, int istep, int j0, int j1, int jstep,
                                          double *__restrict__ acc) {
    const int4 ib_ = __ldg(&P.info[p]);
    const int4 ik_ = __ldg(&P.info[q]);
#pragma unroll
    for (int x = 0; x < 48; ++x) acc[x] = 0.0;
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
            const VT v10_0_0 = PAx * v4_0_0 + WPx * v4_0_1 + (VT)2.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v10_0_1 = PAx * v4_0_1 + WPx * v4_0_2 + (VT)2.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v11_0_0 = PAx * v5_0_0 + WPx * v5_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v11_0_1 = PAx * v5_0_1 + WPx * v5_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v12_0_0 = PAx * v6_0_0 + WPx * v6_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v12_0_1 = PAx * v6_0_1 + WPx * v6_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v13_0_0 = PAy * v5_0_0 + WPy * v5_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v13_0_1 = PAy * v5_0_1 + WPy * v5_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v14_0_0 = PAz * v6_0_0 + WPz * v6_0_1 + (VT)1.0 * oo2z * (v1_0_0 - rho_z * v1_0_1);
            const VT v14_0_1 = PAz * v6_0_1 + WPz * v6_0_2 + (VT)1.0 * oo2z * (v1_0_1 - rho_z * v1_0_2);
            const VT v15_0_0 = PAx * v8_0_0 + WPx * v8_0_1;
            const VT v15_0_1 = PAx * v8_0_1 + WPx * v8_0_2;
            const VT v16_0_0 = PAy * v7_0_0 + WPy * v7_0_1 + (VT)2.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v16_0_1 = PAy * v7_0_1 + WPy * v7_0_2 + (VT)2.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v17_0_0 = PAy * v8_0_0 + WPy * v8_0_1 + (VT)1.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v17_0_1 = PAy * v8_0_1 + WPy * v8_0_2 + (VT)1.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v18_0_0 = PAz * v8_0_0 + WPz * v8_0_1 + (VT)1.0 * oo2z * (v2_0_0 - rho_z * v2_0_1);
            const VT v18_0_1 = PAz * v8_0_1 + WPz * v8_0_2 + (VT)1.0 * oo2z * (v2_0_1 - rho_z * v2_0_2);
            const VT v19_0_0 = PAz * v9_0_0 + WPz * v9_0_1 + (VT)2.0 * oo2z * (v3_0_0 - rho_z * v3_0_1);
            const VT v19_0_1 = PAz * v9_0_1 + WPz * v9_0_2 + (VT)2.0 * oo2z * (v3_0_1 - rho_z * v3_0_2);
            const VT v4_1_0 = QCx * v4_0_0 + WQx * v4_0_1 + (VT)2.0 * oo2ze * v1_0_1;
            const VT v5_1_0 = QCx * v5_0_0 + WQx * v5_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v6_1_0 = QCx * v6_0_0 + WQx * v6_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v7_1_0 = QCx * v7_0_0 + WQx * v7_0_1;
            const VT v8_1_0 = QCx * v8_0_0 + WQx * v8_0_1;
            const VT v9_1_0 = QCx * v9_0_0 + WQx * v9_0_1;
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
            const VT v4_2_0 = QCy * v4_0_0 + WQy * v4_0_1;
            const VT v5_2_0 = QCy * v5_0_0 + WQy * v5_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v6_2_0 = QCy * v6_0_0 + WQy * v6_0_1;
            const VT v7_2_0 = QCy * v7_0_0 + WQy * v7_0_1 + (VT)2.0 * oo2ze * v2_0_1;
            const VT v8_2_0 = QCy * v8_0_0 + WQy * v8_0_1 + (VT)1.0 * oo2ze * v3_0_1;
            const VT v9_2_0 = QCy * v9_0_0 + WQy * v9_0_1;
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
            const VT v4_3_0 = QCz * v4_0_0 + WQz * v4_0_1;
            const VT v5_3_0 = QCz * v5_0_0 + WQz * v5_0_1;
            const VT v6_3_0 = QCz * v6_0_0 + WQz * v6_0_1 + (VT)1.0 * oo2ze * v1_0_1;
            const VT v7_3_0 = QCz * v7_0_0 + WQz * v7_0_1;
            const VT v8_3_0 = QCz * v8_0_0 + WQz * v8_0_1 + (VT)1.0 * oo2ze * v2_0_1;
            const VT v9_3_0 = QCz * v9_0_0 + WQz * v9_0_1 + (VT)2.0 * oo2ze * v3_0_1;
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
            acc[0] += (double)v4_1_0;
            acc[1] += (double)v4_2_0;
            acc[2] += (double)v4_3_0;
            acc[3] += (double)v5_1_0;
            acc[4] += (double)v5_2_0;
            acc[5] += (double)v5_3_0;
            acc[6] += (double)v6_1_0;
            acc[7] += (double)v6_2_0;
            acc[8] += (double)v6_3_0;
            acc[9] += (double)v7_1_0;
            acc[10] += (double)v7_2_0;
            acc[11] += (double)v7_3_0;
            acc[12] += (double)v8_1_0;
            acc[13] += (double)v8_2_0;
            acc[14] += (double)v8_3_0;
            acc[15] += (double)v9_1_0;
            acc[16] += (double)v9_2_0;
            acc[17] += (double)v9_3_0;
            acc[18] += (double)v10_1_0;
            acc[19] += (double)v10_2_0;
            acc[20] += (double)v10_3_0;
            acc[21] += (double)v11_1_0;
            acc[22] += (double)v11_2_0;
            acc[23] += (double)v11_3_0;
            acc[24] += (double)v12_1_0;
            acc[25] += (double)v12_2_0;
            acc[26] += (double)v12_3_0;
            acc[27] += (double)v13_1_0;
            acc[28] += (double)v13_2_0;
            acc[29] += (double)v13_3_0;
            acc[30] += (double)v14_1_0;
            acc[31] += (double)v14_2_0;
            acc[32] += (double)v14_3_0;
            acc[33] += (double)v15_1_0;
            acc[34] += (double)v15_2_0;
            acc[35] += (double)v15_3_0;
            acc[36] += (double)v16_1_0;
            acc[37] += (double)v16_2_0;
            acc[38] += (double)v16_3_0;
            acc[39] += (double)v17_1_0;
            acc[40] += (double)v17_2_0;
            acc[41] += (double)v17_3_0;
            acc[42] += (double)v18_1_0;
            acc[43] += (double)v18_2_0;
            acc[44] += (double)v18_3_0;
            acc[45] += (double)v19_1_0;
            acc[46] += (double)v19_2_0;
            acc[47] += (double)v19_3_0;
        }
    }
}

// Bra and ket HRR of the contracted block (src/HGP.jl:92-114), then the component norms:
// the normalised (ab|cd) of bra pair p and ket pair q into res[54] (ma, mb, mc, md
// row-major).
__device__ __forceinline__ void hrr_dpps(const PairTab &P, int p, int q, const double *__restrict__ acc,
                                          double *__restrict__ res) {
    const double4 gb = ldg4(&P.geo[p]);
    const double4 gk = ldg4(&P.geo[q]);
    const double ABx = gb.x, ABy = gb.y, ABz = gb.z;
    const double CDx = gk.x, CDy = gk.y, CDz = gk.z;
    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;
    const double h4_1_1 = acc[18] + ABx * acc[0];
    const double h4_1_2 = acc[19] + ABx * acc[1];
    const double h4_1_3 = acc[20] + ABx * acc[2];
    const double h4_2_1 = acc[21] + ABy * acc[0];
    const double h4_2_2 = acc[22] + ABy * acc[1];
    const double h4_2_3 = acc[23] + ABy * acc[2];
    const double h4_3_1 = acc[24] + ABz * acc[0];
    const double h4_3_2 = acc[25] + ABz * acc[1];
    const double h4_3_3 = acc[26] + ABz * acc[2];
    const double h5_1_1 = acc[21] + ABx * acc[3];
    const double h5_1_2 = acc[22] + ABx * acc[4];
    const double h5_1_3 = acc[23] + ABx * acc[5];
    const double h5_2_1 = acc[27] + ABy * acc[3];
    const double h5_2_2 = acc[28] + ABy * acc[4];
    const double h5_2_3 = acc[29] + ABy * acc[5];
    const double h5_3_1 = acc[33] + ABz * acc[3];
    const double h5_3_2 = acc[34] + ABz * acc[4];
    const double h5_3_3 = acc[35] + ABz * acc[5];
    const double h6_1_1 = acc[24] + ABx * acc[6];
    const double h6_1_2 = acc[25] + ABx * acc[7];
    const double h6_1_3 = acc[26] + ABx * acc[8];
    const double h6_2_1 = acc[33] + ABy * acc[6];
    const double h6_2_2 = acc[34] + ABy * acc[7];
    const double h6_2_3 = acc[35] + ABy * acc[8];
    const double h6_3_1 = acc[30] + ABz * acc[6];
    const double h6_3_2 = acc[31] + ABz * acc[7];
    const double h6_3_3 = acc[32] + ABz * acc[8];
    const double h7_1_1 = acc[27] + ABx * acc[9];
    const double h7_1_2 = acc[28] + ABx * acc[10];
    const double h7_1_3 = acc[29] + ABx * acc[11];
    const double h7_2_1 = acc[36] + ABy * acc[9];
    const double h7_2_2 = acc[37] + ABy * acc[10];
    const double h7_2_3 = acc[38] + ABy * acc[11];
    const double h7_3_1 = acc[39] + ABz * acc[9];
    const double h7_3_2 = acc[40] + ABz * acc[10];
    const double h7_3_3 = acc[41] + ABz * acc[11];
    const double h8_1_1 = acc[33] + ABx * acc[12];
    const double h8_1_2 = acc[34] + ABx * acc[13];
    const double h8_1_3 = acc[35] + ABx * acc[14];
    const double h8_2_1 = acc[39] + ABy * acc[12];
    const double h8_2_2 = acc[40] + ABy * acc[13];
    const double h8_2_3 = acc[41] + ABy * acc[14];
    const double h8_3_1 = acc[42] + ABz * acc[12];
    const double h8_3_2 = acc[43] + ABz * acc[13];
    const double h8_3_3 = acc[44] + ABz * acc[14];
    const double h9_1_1 = acc[30] + ABx * acc[15];
    const double h9_1_2 = acc[31] + ABx * acc[16];
    const double h9_1_3 = acc[32] + ABx * acc[17];
    const double h9_2_1 = acc[42] + ABy * acc[15];
    const double h9_2_2 = acc[43] + ABy * acc[16];
    const double h9_2_3 = acc[44] + ABy * acc[17];
    const double h9_3_1 = acc[45] + ABz * acc[15];
    const double h9_3_2 = acc[46] + ABz * acc[16];
    const double h9_3_3 = acc[47] + ABz * acc[17];
    res[0] = h4_1_1 * 0.5773502691896258;
    res[1] = h4_1_2 * 0.5773502691896258;
    res[2] = h4_1_3 * 0.5773502691896258;
    res[3] = h4_2_1 * 0.5773502691896258;
    res[4] = h4_2_2 * 0.5773502691896258;
    res[5] = h4_2_3 * 0.5773502691896258;
    res[6] = h4_3_1 * 0.5773502691896258;
    res[7] = h4_3_2 * 0.5773502691896258;
    res[8] = h4_3_3 * 0.5773502691896258;
    res[9] = h5_1_1;
    res[10] = h5_1_2;
    res[11] = h5_1_3;
    res[12] = h5_2_1;
    res[13] = h5_2_2;
    res[14] = h5_2_3;
    res[15] = h5_3_1;
    res[16] = h5_3_2;
    res[17] = h5_3_3;
    res[18] = h6_1_1;
    res[19] = h6_1_2;
    res[20] = h6_1_3;
    res[21] = h6_2_1;
    res[22] = h6_2_2;
    res[23] = h6_2_3;
    res[24] = h6_3_1;
    res[25] = h6_3_2;
    res[26] = h6_3_3;
    res[27] = h7_1_1 * 0.5773502691896258;
    res[28] = h7_1_2 * 0.5773502691896258;
    res[29] = h7_1_3 * 0.5773502691896258;
    res[30] = h7_2_1 * 0.5773502691896258;
    res[31] = h7_2_2 * 0.5773502691896258;
    res[32] = h7_2_3 * 0.5773502691896258;
    res[33] = h7_3_1 * 0.5773502691896258;
    res[34] = h7_3_2 * 0.5773502691896258;
    res[35] = h7_3_3 * 0.5773502691896258;
    res[36] = h8_1_1;
    res[37] = h8_1_2;
    res[38] = h8_1_3;
    res[39] = h8_2_1;
    res[40] = h8_2_2;
    res[41] = h8_2_3;
    res[42] = h8_3_1;
    res[43] = h8_3_2;
    res[44] = h8_3_3;
    res[45] = h9_1_1 * 0.5773502691896258;
    res[46] = h9_1_2 * 0.5773502691896258;
    res[47] = h9_1_3 * 0.5773502691896258;
    res[48] = h9_2_1 * 0.5773502691896258;
    res[49] = h9_2_2 * 0.5773502691896258;
    res[50] = h9_2_3 * 0.5773502691896258;
    res[51] = h9_3_1 * 0.5773502691896258;
    res[52] = h9_3_2 * 0.5773502691896258;
    res[53] = h9_3_3 * 0.5773502691896258;
}

// (ab|cd) over the bra primitive pairs [i0, i1) and ket primitive pairs [j0, j1) into
// res[54]; the contracted block also into acc_out when given (the bound kernels).
template <typename VT>
__device__ __forceinline__ void quartet_dpps(const PairTab &P, const BoysTab &B, int p, int q,
                                              int i0, int i1, int j0, int j1,
                                              double *__restrict__ res,
                                              double *__restrict__ acc_out = nullptr) {
    double acc[48];
    vrr_dpps<VT>(P, B, p, q, i0, i1, 1, j0, j1, 1, acc);
    if (acc_out) {
#pragma unroll
        for (int x = 0; x < 48; ++x) acc_out[x] = acc[x];
    }
    hrr_dpps(P, p, q, acc, res);
}

__device__ __forceinline__ void store_dpps(double *__restrict__ out, const int4 ib_, const int4 ik_,
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
}

// The quartet's unique integrals digested into J and K (molints_plan_jk) instead of stored.
__device__ __noinline__ void jk_dpps(const JKOut &jk, const int4 ib_, const int4 ik_, bool same,
                                      const double *__restrict__ res) {
    const bool dab = ib_.z == ib_.w, dcd = ik_.z == ik_.w;
    for (int x = 0; x < 54; ++x) {
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
__global__ void __launch_bounds__(128) eri_queue_dpps(const EriQueue Q) {
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
        double acc[48];
        double2 bp = make_double2(0.0, 0.0), bq = bp;
        if (live) {
            bp = __ldg(&Q.pairs.bnd[p]);
            bq = __ldg(&Q.pairs.bnd[q]);
        }
        if (!live || bp.x * bq.x < Q.screen_cut) {
#pragma unroll
            for (int x = 0; x < 48; ++x) acc[x] = 0.0;
        } else {
            const int nb = __ldg(&Q.pairs.info[p]).y, nk = __ldg(&Q.pairs.info[q]).y;
            if (MIXED && bp.y * bq.y < Q.fp32_cut)
                vrr_dpps<float>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
            else vrr_dpps<double>(Q.pairs, Q.boys, p, q, is, nb, 1 << (lg - lgj), js, nk, 1 << lgj, acc);
        }
        if (lg) {
            for (int off = W; off < 32; off <<= 1) {
#pragma unroll
                for (int x = 0; x < 48; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
            }
        }
        const bool lead = live && s == 0;
        if (!JK && Q.scratch) {
            // two-phase: the leaders' HRR writes the blocks of the chunk's quartets straight
            // into shared memory, where they lie as in the scratch (consecutive slots); the warp
            // then copies them out as one contiguous run
            extern __shared__ double stg[];  // 4 * 32 * 54 doubles (launch_eri_dpps)
            double *sb = stg + (threadIdx.x >> 5) * (32 * 54);
            if (lead) hrr_dpps(Q.pairs, p, q, acc, sb + kq * 54);
            __syncwarp();
            const int nlive = min(W, cnt - base);
            double *__restrict__ dst = Q.scratch + __ldg(&Q.region[ch.w * kRegionFields]) +
                (__ldg(&Q.chunk_slot[c]) + base) * (long long)54;
            for (int t = lane; t < nlive * 54; t += 32) dst[t] = sb[t];
            __syncwarp();
        } else if (lead) {
            double res[54];
            hrr_dpps(Q.pairs, p, q, acc, res);
            if constexpr (JK) {
                jk_dpps(Q.jk, __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]), p == q, res);
            } else {
                store_dpps(Q.out + __ldg(&Q.mol_out[ch.w]), __ldg(&Q.pairs.info[p]), __ldg(&Q.pairs.info[q]),
                            p == q, res);
            }
        }
        }
    }
}


// The dynamic shared memory of the two-phase staging (55296 bytes), allowed once per device
// (before any graph capture: the occupancy query of plan creation calls it first).
static void eri_prepare_dpps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(eri_queue_dpps<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 55296);
        cudaFuncSetAttribute(eri_queue_dpps<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 55296);
        done[dev] = true;
    }
}

void launch_eri_dpps(const EriQueue &Q, int mixed, int grid, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid <= 0) return;
    // two-phase plans stage the chunk's blocks in 55296 bytes of dynamic shared memory
    const size_t smem = Q.scratch && !Q.jk.J ? 55296 : 0;
    if (smem) eri_prepare_dpps();
    const bool jk = Q.jk.J != nullptr;
    if (mixed) { if (jk) eri_queue_dpps<1, 1><<<grid, 128, 0, s>>>(Q); else eri_queue_dpps<1, 0><<<grid, 128, smem, s>>>(Q); }
    else if (jk) eri_queue_dpps<0, 1><<<grid, 128, 0, s>>>(Q);
    else eri_queue_dpps<0, 0><<<grid, 128, smem, s>>>(Q);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_eri_dpps(int mixed) {
    eri_prepare_dpps();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dpps<1, 0>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, eri_queue_dpps<0, 0>, 128, 0);
    return n;
}

}  // namespace molints

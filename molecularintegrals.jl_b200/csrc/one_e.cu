// one_e.cu -- the one-electron matrices of a basis on the device: overlap S, kinetic energy T
// and nuclear attraction V (all_1e_ints, src/OneInts.jl:267-290), shells up to f.
//
// One thread per shell pair (a, b), a >= b by shell index, loops over the primitive pairs:
//   * overlap: 1-D Obara-Saika tables S_t(i, j) per axis (i <= la, j <= lb + 2),
//       S(i+1, j) = PA S(i, j) + (i S(i-1, j) + j S(i, j-1)) / 2g,
//       S(i, j+1) = PB S(i, j) + (i S(i-1, j) + j S(i, j-1)) / 2g,
//     times (pi/g)^(3/2) exp(-ab/g |AB|^2);
//   * kinetic energy from the overlaps of b raised and lowered by two,
//       T = b (2 lb + 3) S(a, b) - 2 b^2 sum_t S(a, b + 2_t) - 1/2 sum_t b_t (b_t - 1) S(a, b - 2_t)
//     (the expression kinetic() evaluates, src/OneInts.jl:124-135);
//   * nuclear attraction by Rys quadrature with the point charge as the second centre: for
//     each atom C, roots u_r and weights W_r of order floor((la+lb)/2)+1 at X = g |PC|^2, and
//       I(i+1, j) = (PA - u PC) I(i, j) + (1 - u)/2g (i I(i-1, j) + j I(i, j-1)),
//       I(i, j+1) = (PB - u PC) I(i, j) + (1 - u)/2g (i I(i-1, j) + j I(i, j-1)),
//     V += -Z_C 2pi/g exp(-ab/g |AB|^2) sum_r W_r I_x I_y I_z.
// Results are for normalised contracted functions (the ERI engine's coefficients and component
// norms) and are written to both the (a, b) and the (b, a) blocks of the n x n matrices.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/molints.h"
#include "eri_common.cuh"
#include "rys_common.cuh"

namespace molints {

int basis_ncoef(const molints_basis *b, std::vector<double> &ncoef, std::string &err);  // molints.cu
int ctx_device_of(const molints_ctx *ctx);
RysTab ctx_rys(const molints_ctx *ctx);

namespace {

constexpr int kL = 3;                 // shells up to f
constexpr int kNc = (kL + 1) * (kL + 2) / 2;

__device__ __forceinline__ void comp_of(int l, int m, int &x, int &y, int &z) {
    // component m of shell l in the reference order (x-power descending, then y; l=3 has xzz
    // before xyz, src/Basis.jl:269-279)
    int k = 0;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) {
            int kk = k;
            if (l == 3 && (k == 4 || k == 5)) kk = 9 - k;  // swap positions 4 and 5
            if (kk == m) { x = i; y = j; z = l - i - j; }
            ++k;
        }
}

__device__ __forceinline__ double comp_norm(int x, int y, int z) {
    auto df = [](int n) { double r = 1.0; for (int k = n; k > 1; k -= 2) r *= k; return r; };
    return rsqrt(df(2 * x - 1) * df(2 * y - 1) * df(2 * z - 1));
}

template <int NR>
__device__ __forceinline__ void nuclear_rys(const RysTab &R, double X, double *u, double *w) {
    for (int r = 0; r < NR; ++r) rys_root<NR>(R, X, r, u[r], w[r]);
}

__global__ void one_e_kernel(int nshell, const double *__restrict__ xyz, const int *__restrict__ L,
                             const int *__restrict__ nprim, const int *__restrict__ poff,
                             const int *__restrict__ fn, const double *__restrict__ expn,
                             const double *__restrict__ ncoef, int natom,
                             const double *__restrict__ axyz, const double *__restrict__ az,
                             RysTab R, int n, double *__restrict__ S, double *__restrict__ T,
                             double *__restrict__ V) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npair = (long long)nshell * (nshell + 1) / 2;
    if (t >= npair) return;
    int a = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)a * (a + 1) / 2 > t) --a;
    while ((long long)(a + 1) * (a + 2) / 2 <= t) ++a;
    const int b = (int)(t - (long long)a * (a + 1) / 2);
    const int la = L[a], lb = L[b];
    const int na = (la + 1) * (la + 2) / 2, nb = (lb + 1) * (lb + 2) / 2;
    const double A[3] = {xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]};
    const double B[3] = {xyz[3 * b], xyz[3 * b + 1], xyz[3 * b + 2]};
    const double AB2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
    double s[kNc * kNc], k[kNc * kNc], v[kNc * kNc];
    for (int x = 0; x < na * nb; ++x) s[x] = k[x] = v[x] = 0.0;
    int ca[kNc][3], cb[kNc][3];
    for (int m = 0; m < na; ++m) comp_of(la, m, ca[m][0], ca[m][1], ca[m][2]);
    for (int m = 0; m < nb; ++m) comp_of(lb, m, cb[m][0], cb[m][1], cb[m][2]);
    const int nr = (la + lb) / 2 + 1;
    for (int i = 0; i < nprim[a]; ++i)
        for (int j = 0; j < nprim[b]; ++j) {
            const double ea = expn[poff[a] + i], eb = expn[poff[b] + j];
            const double g = ea + eb, og = 1.0 / g;
            const double cc = ncoef[poff[a] + i] * ncoef[poff[b] + j];
            double P[3], PA[3], PB[3];
            for (int d = 0; d < 3; ++d) {
                P[d] = A[d] + eb * og * (B[d] - A[d]);
                PA[d] = P[d] - A[d];
                PB[d] = P[d] - B[d];
            }
            const double kab = exp(-ea * eb * og * AB2);
            // 1-D overlap tables, i <= la, j <= lb + 2
            double O[3][kL + 1][kL + 3];
            for (int d = 0; d < 3; ++d) {
                for (int ii = 0; ii <= la; ++ii)
                    for (int jj = 0; jj <= lb + 2; ++jj) {
                        double val;
                        if (ii == 0 && jj == 0) val = 1.0;
                        else if (ii > 0) {
                            val = PA[d] * O[d][ii - 1][jj];
                            if (ii > 1) val += (ii - 1) * 0.5 * og * O[d][ii - 2][jj];
                            if (jj > 0) val += jj * 0.5 * og * O[d][ii - 1][jj - 1];
                        } else {
                            val = PB[d] * O[d][0][jj - 1];
                            if (jj > 1) val += (jj - 1) * 0.5 * og * O[d][0][jj - 2];
                        }
                        O[d][ii][jj] = val;
                    }
            }
            const double so = cc * kab * og * sqrt(og) * 5.568327996831707845;  // pi^(3/2)
            for (int p = 0; p < na; ++p)
                for (int q = 0; q < nb; ++q) {
                    const int *x = ca[p], *y = cb[q];
                    const double s0 = O[0][x[0]][y[0]] * O[1][x[1]][y[1]] * O[2][x[2]][y[2]];
                    double up = O[0][x[0]][y[0] + 2] * O[1][x[1]][y[1]] * O[2][x[2]][y[2]] +
                                O[0][x[0]][y[0]] * O[1][x[1]][y[1] + 2] * O[2][x[2]][y[2]] +
                                O[0][x[0]][y[0]] * O[1][x[1]][y[1]] * O[2][x[2]][y[2] + 2];
                    double dn = 0.0;
                    if (y[0] > 1) dn += y[0] * (y[0] - 1) * O[0][x[0]][y[0] - 2] * O[1][x[1]][y[1]] * O[2][x[2]][y[2]];
                    if (y[1] > 1) dn += y[1] * (y[1] - 1) * O[0][x[0]][y[0]] * O[1][x[1]][y[1] - 2] * O[2][x[2]][y[2]];
                    if (y[2] > 1) dn += y[2] * (y[2] - 1) * O[0][x[0]][y[0]] * O[1][x[1]][y[1]] * O[2][x[2]][y[2] - 2];
                    s[p * nb + q] += so * s0;
                    k[p * nb + q] += so * (eb * (2 * lb + 3) * s0 - 2.0 * eb * eb * up - 0.5 * dn);
                }
            // nuclear attraction, Rys quadrature per atom
            const double pv = -cc * kab * 2.0 * 3.14159265358979323846 * og;
            for (int c = 0; c < natom; ++c) {
                const double PC[3] = {P[0] - axyz[3 * c], P[1] - axyz[3 * c + 1], P[2] - axyz[3 * c + 2]};
                const double X = g * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                double u[4], w[4];
                switch (nr) {
                    case 1: nuclear_rys<1>(R, X, u, w); break;
                    case 2: nuclear_rys<2>(R, X, u, w); break;
                    case 3: nuclear_rys<3>(R, X, u, w); break;
                    default: nuclear_rys<4>(R, X, u, w); break;
                }
                const double zc = az[c] * pv;
                for (int r = 0; r < nr; ++r) {
                    double I[3][kL + 1][kL + 1];
                    const double f = (1.0 - u[r]) * 0.5 * og;
                    for (int d = 0; d < 3; ++d) {
                        const double ca0 = PA[d] - u[r] * PC[d], cb0 = PB[d] - u[r] * PC[d];
                        for (int ii = 0; ii <= la; ++ii)
                            for (int jj = 0; jj <= lb; ++jj) {
                                double val;
                                if (ii == 0 && jj == 0) val = 1.0;
                                else if (ii > 0) {
                                    val = ca0 * I[d][ii - 1][jj];
                                    if (ii > 1) val += (ii - 1) * f * I[d][ii - 2][jj];
                                    if (jj > 0) val += jj * f * I[d][ii - 1][jj - 1];
                                } else {
                                    val = cb0 * I[d][0][jj - 1];
                                    if (jj > 1) val += (jj - 1) * f * I[d][0][jj - 2];
                                }
                                I[d][ii][jj] = val;
                            }
                    }
                    const double wz = w[r] * zc;
                    for (int p = 0; p < na; ++p)
                        for (int q = 0; q < nb; ++q) {
                            const int *x = ca[p], *y = cb[q];
                            v[p * nb + q] += wz * I[0][x[0]][y[0]] * I[1][x[1]][y[1]] * I[2][x[2]][y[2]];
                        }
                }
            }
        }
    for (int p = 0; p < na; ++p)
        for (int q = 0; q < nb; ++q) {
            const double g = comp_norm(ca[p][0], ca[p][1], ca[p][2]) * comp_norm(cb[q][0], cb[q][1], cb[q][2]);
            const long long i = fn[a] + p, j = fn[b] + q;
            S[i * n + j] = S[j * n + i] = g * s[p * nb + q];
            T[i * n + j] = T[j * n + i] = g * k[p * nb + q];
            V[i * n + j] = V[j * n + i] = g * v[p * nb + q];
        }
}

}  // namespace
}  // namespace molints

using namespace molints;

extern "C" int molints_one_e(molints_ctx *ctx, const molints_basis *b, int32_t natom,
                             const double *atom_xyz, const double *atom_charge, double *S_host,
                             double *T_host, double *V_host) {
    if (!ctx || !b || natom < 0 || (natom > 0 && (!atom_xyz || !atom_charge))) return MOLINTS_ERR_INVALID;
    const int64_t n = molints_nbf(b);
    if (n < 0) return MOLINTS_ERR_INVALID;
    if (n == 0) return MOLINTS_OK;
    if (!S_host || !T_host || !V_host) return MOLINTS_ERR_INVALID;
    const int ns = b->nshell;
    for (int s = 0; s < ns; ++s)
        if (b->L[s] > kL) return MOLINTS_ERR_UNSUPPORTED;
    std::vector<double> ncoef;
    std::string err;
    int rc = basis_ncoef(b, ncoef, err);
    if (rc) return rc;
    int nprim = 0;
    for (int s = 0; s < ns; ++s) nprim = std::max(nprim, b->prim_off[s] + b->nprim[s]);
    std::vector<int> fn(ns);
    for (int s = 0, f = 0; s < ns; ++s) { fn[s] = f; f += (b->L[s] + 1) * (b->L[s] + 2) / 2; }
    if (cudaSetDevice(ctx_device_of(ctx)) != cudaSuccess) return MOLINTS_ERR_CUDA;
    // one device block: shells, primitives, atoms, then the three matrices
    const size_t nd_sh = 3 * (size_t)ns, nd_pr = 2 * (size_t)nprim, nd_at = 4 * (size_t)natom;
    const size_t ni = 4 * (size_t)ns, nm = 3 * (size_t)n * n;
    double *d = nullptr;
    int *di = nullptr;
    if (cudaMalloc(&d, (nd_sh + nd_pr + nd_at + nm) * sizeof(double)) != cudaSuccess) return MOLINTS_ERR_CUDA;
    if (cudaMalloc(&di, ni * sizeof(int)) != cudaSuccess) { cudaFree(d); return MOLINTS_ERR_CUDA; }
    std::vector<double> hd(nd_sh + nd_pr + nd_at);
    std::vector<int> hi(ni);
    for (int s = 0; s < ns; ++s) {
        for (int c = 0; c < 3; ++c) hd[3 * s + c] = b->xyz[3 * s + c];
        hi[s] = b->L[s];
        hi[ns + s] = b->nprim[s];
        hi[2 * ns + s] = b->prim_off[s];
        hi[3 * ns + s] = fn[s];
    }
    for (int k = 0; k < nprim; ++k) {
        hd[nd_sh + k] = b->expn[k];
        hd[nd_sh + nprim + k] = ncoef[k];
    }
    for (int c = 0; c < natom; ++c) {
        for (int t = 0; t < 3; ++t) hd[nd_sh + nd_pr + 3 * c + t] = atom_xyz[3 * c + t];
        hd[nd_sh + nd_pr + 3 * natom + c] = atom_charge[c];
    }
    double *dS = d + nd_sh + nd_pr + nd_at, *dT = dS + n * n, *dV = dT + n * n;
    cudaError_t e = cudaMemcpy(d, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(di, hi.data(), ni * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const long long npair = (long long)ns * (ns + 1) / 2;
        one_e_kernel<<<(unsigned)((npair + 63) / 64), 64>>>(
            ns, d, di, di + ns, di + 2 * ns, di + 3 * ns, d + nd_sh, d + nd_sh + nprim, natom,
            d + nd_sh + nd_pr, d + nd_sh + nd_pr + 3 * natom, ctx_rys(ctx), (int)n, dS, dT, dV);
        e = cudaGetLastError();
    }
    const size_t mb = (size_t)n * n * sizeof(double);
    if (e == cudaSuccess) e = cudaMemcpy(S_host, dS, mb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(T_host, dT, mb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(V_host, dV, mb, cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaFree(di);
    return e == cudaSuccess ? MOLINTS_OK : MOLINTS_ERR_CUDA;
}

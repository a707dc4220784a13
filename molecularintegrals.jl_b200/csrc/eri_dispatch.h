// Generated by gen_eri.py.  Do not edit.
#pragma once
#include "eri_common.cuh"
namespace molints {
void launch_eri_ssss(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_schwarz_ssss(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_psss(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_psps(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_schwarz_psps(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_ppss(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_ppps(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_pppp(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_schwarz_pppp(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_dsss(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dsps(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dspp(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dsds(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_schwarz_dsds(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_dpss(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dpps(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dppp(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dpds(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dpdp(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_schwarz_dpdp(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_ddss(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_ddps(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_ddpp(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_ddds(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dddp(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_eri_dddd(const EriLaunch &L, int mixed, cudaStream_t s);
void launch_schwarz_dddd(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
typedef void (*EriLauncher)(const EriLaunch &, int, cudaStream_t);
typedef void (*SchwarzLauncher)(const PairTab &, const BoysTab &, int, int, double2 *, double *, int, cudaStream_t);
constexpr int kLmax = 2;
constexpr int kNumPairClasses = 6;
// pair class c = (kPairClassLa[c], kPairClassLb[c]), ordered by la+lb then la
constexpr int kPairClassLa[] = {0, 1, 1, 2, 2, 2};
constexpr int kPairClassLb[] = {0, 0, 1, 0, 1, 2};
// kEriLaunchers[x][y], x >= y (bra class x, ket class y)
static const EriLauncher kEriLaunchers[6][6] = {
    {launch_eri_ssss, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_psss, launch_eri_psps, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_ppss, launch_eri_ppps, launch_eri_pppp, nullptr, nullptr, nullptr},
    {launch_eri_dsss, launch_eri_dsps, launch_eri_dspp, launch_eri_dsds, nullptr, nullptr},
    {launch_eri_dpss, launch_eri_dpps, launch_eri_dppp, launch_eri_dpds, launch_eri_dpdp, nullptr},
    {launch_eri_ddss, launch_eri_ddps, launch_eri_ddpp, launch_eri_ddds, launch_eri_dddp, launch_eri_dddd},
};
static const char *const kEriNames[6][6] = {
    {"eri_ssss", nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_psss", "eri_psps", nullptr, nullptr, nullptr, nullptr},
    {"eri_ppss", "eri_ppps", "eri_pppp", nullptr, nullptr, nullptr},
    {"eri_dsss", "eri_dsps", "eri_dspp", "eri_dsds", nullptr, nullptr},
    {"eri_dpss", "eri_dpps", "eri_dppp", "eri_dpds", "eri_dpdp", nullptr},
    {"eri_ddss", "eri_ddps", "eri_ddpp", "eri_ddds", "eri_dddp", "eri_dddd"},
};
static const char *const kSchwarzNames[6] = {
    "schwarz_ss", "schwarz_ps", "schwarz_pp", "schwarz_ds", "schwarz_dp", "schwarz_dd"
};
static const SchwarzLauncher kSchwarzLaunchers[6] = {
    launch_schwarz_ssss, launch_schwarz_psps, launch_schwarz_pppp, launch_schwarz_dsds, launch_schwarz_dpdp, launch_schwarz_dddd
};
}  // namespace molints

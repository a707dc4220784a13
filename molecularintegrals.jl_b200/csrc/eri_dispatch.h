// Generated by gen_eri.py.  Do not edit.
#pragma once
#include "eri_common.cuh"
namespace molints {
void launch_eri_ssss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ssss(int mixed);
void launch_schwarz_ssss(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_psss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_psss(int mixed);
void launch_eri_psps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_psps(int mixed);
void launch_schwarz_psps(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_ppss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ppss(int mixed);
void launch_eri_ppps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ppps(int mixed);
void launch_eri_pppp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_pppp(int mixed);
void launch_schwarz_pppp(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_dsss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dsss(int mixed);
void launch_eri_dsps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dsps(int mixed);
void launch_eri_dspp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dspp(int mixed);
void launch_eri_dsds(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dsds(int mixed);
void launch_schwarz_dsds(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_dpss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dpss(int mixed);
void launch_eri_dpps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dpps(int mixed);
void launch_eri_dppp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dppp(int mixed);
void launch_eri_dpds(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dpds(int mixed);
void launch_eri_dpdp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dpdp(int mixed);
void launch_schwarz_dpdp(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_eri_ddss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ddss(int mixed);
void launch_eri_ddps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ddps(int mixed);
void launch_eri_ddpp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ddpp(int mixed);
void launch_eri_ddds(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ddds(int mixed);
void launch_eri_dddp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dddp(int mixed);
void launch_eri_dddd(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_dddd(int mixed);
void launch_schwarz_dddd(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
typedef void (*EriLauncher)(const EriQueue &, int, int, cudaStream_t);
typedef int (*EriOccupancy)(int);
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
static const EriOccupancy kEriOccupancy[6][6] = {
    {occupancy_eri_ssss, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_psss, occupancy_eri_psps, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_ppss, occupancy_eri_ppps, occupancy_eri_pppp, nullptr, nullptr, nullptr},
    {occupancy_eri_dsss, occupancy_eri_dsps, occupancy_eri_dspp, occupancy_eri_dsds, nullptr, nullptr},
    {occupancy_eri_dpss, occupancy_eri_dpps, occupancy_eri_dppp, occupancy_eri_dpds, occupancy_eri_dpdp, nullptr},
    {occupancy_eri_ddss, occupancy_eri_ddps, occupancy_eri_ddpp, occupancy_eri_ddds, occupancy_eri_dddp, occupancy_eri_dddd},
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

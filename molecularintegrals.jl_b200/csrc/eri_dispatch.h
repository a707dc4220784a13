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
void launch_eri_fsss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fsss(int mixed);
void launch_eri_fsps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fsps(int mixed);
void launch_eri_fspp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fspp(int mixed);
void launch_eri_fsds(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fsds(int mixed);
void launch_eri_fsdp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fsdp(int mixed);
void launch_eri_fsfs(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fsfs(int mixed);
void launch_schwarz_fsfs(const PairTab &P, const BoysTab &B, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
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
void launch_eri_fpss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fpss(int mixed);
void launch_eri_fpps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fpps(int mixed);
void launch_eri_fppp(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fppp(int mixed);
void launch_eri_fpds(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fpds(int mixed);
void launch_eri_fdss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fdss(int mixed);
void launch_eri_fdps(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_fdps(int mixed);
void launch_eri_ffss(const EriQueue &Q, int mixed, int grid, cudaStream_t s);
int occupancy_eri_ffss(int mixed);
void launch_rys_ssss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ssss(int mixed);
void launch_rys_bound_ssss(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_psss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_psss(int mixed);
void launch_rys_psps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_psps(int mixed);
void launch_rys_bound_psps(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_ppss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ppss(int mixed);
void launch_rys_ppps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ppps(int mixed);
void launch_rys_pppp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_pppp(int mixed);
void launch_rys_bound_pppp(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_dsss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dsss(int mixed);
void launch_rys_dsps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dsps(int mixed);
void launch_rys_dspp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dspp(int mixed);
void launch_rys_dsds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dsds(int mixed);
void launch_rys_bound_dsds(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_dpss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dpss(int mixed);
void launch_rys_dpps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dpps(int mixed);
void launch_rys_dppp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dppp(int mixed);
void launch_rys_dpds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dpds(int mixed);
void launch_rys_dpdp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dpdp(int mixed);
void launch_rys_bound_dpdp(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_fsss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fsss(int mixed);
void launch_rys_fsps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fsps(int mixed);
void launch_rys_fspp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fspp(int mixed);
void launch_rys_fsds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fsds(int mixed);
void launch_rys_fsdp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fsdp(int mixed);
void launch_rys_fsfs(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fsfs(int mixed);
void launch_rys_bound_fsfs(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_ddss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ddss(int mixed);
void launch_rys_ddps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ddps(int mixed);
void launch_rys_ddpp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ddpp(int mixed);
void launch_rys_ddds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ddds(int mixed);
void launch_rys_dddp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dddp(int mixed);
void launch_rys_ddfs(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ddfs(int mixed);
void launch_rys_dddd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dddd(int mixed);
void launch_rys_bound_dddd(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_fpss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpss(int mixed);
void launch_rys_fpps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpps(int mixed);
void launch_rys_fppp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fppp(int mixed);
void launch_rys_fpds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpds(int mixed);
void launch_rys_fpdp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpdp(int mixed);
void launch_rys_fpfs(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpfs(int mixed);
void launch_rys_fpdd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpdd(int mixed);
void launch_rys_fpfp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fpfp(int mixed);
void launch_rys_bound_fpfp(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_dfss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfss(int mixed);
void launch_rys_dfps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfps(int mixed);
void launch_rys_dfpp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfpp(int mixed);
void launch_rys_dfds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfds(int mixed);
void launch_rys_dfdp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfdp(int mixed);
void launch_rys_dffs(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dffs(int mixed);
void launch_rys_dfdd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfdd(int mixed);
void launch_rys_dffp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dffp(int mixed);
void launch_rys_dfdf(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_dfdf(int mixed);
void launch_rys_bound_dfdf(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_fdss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdss(int mixed);
void launch_rys_fdps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdps(int mixed);
void launch_rys_fdpp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdpp(int mixed);
void launch_rys_fdds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdds(int mixed);
void launch_rys_fddp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fddp(int mixed);
void launch_rys_fdfs(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdfs(int mixed);
void launch_rys_fddd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fddd(int mixed);
void launch_rys_fdfp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdfp(int mixed);
void launch_rys_fddf(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fddf(int mixed);
void launch_rys_fdfd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fdfd(int mixed);
void launch_rys_bound_fdfd(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
void launch_rys_ffss(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffss(int mixed);
void launch_rys_ffps(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffps(int mixed);
void launch_rys_ffpp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffpp(int mixed);
void launch_rys_ffds(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffds(int mixed);
void launch_rys_ffdp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffdp(int mixed);
void launch_rys_fffs(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fffs(int mixed);
void launch_rys_ffdd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffdd(int mixed);
void launch_rys_fffp(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fffp(int mixed);
void launch_rys_ffdf(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffdf(int mixed);
void launch_rys_fffd(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_fffd(int mixed);
void launch_rys_ffff(const EriQueue &Q, const RysTab &R, int mixed, int grid, cudaStream_t s);
int occupancy_rys_ffff(int mixed);
void launch_rys_bound_ffff(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound, double *qout, int full, cudaStream_t s);
typedef void (*EriLauncher)(const EriQueue &, int, int, cudaStream_t);
typedef int (*EriOccupancy)(int);
typedef void (*SchwarzLauncher)(const PairTab &, const BoysTab &, int, int, double2 *, double *, int, cudaStream_t);
typedef void (*RysLauncher)(const EriQueue &, const RysTab &, int, int, cudaStream_t);
typedef int (*RysOccupancy)(int);
typedef void (*RysBoundLauncher)(const PairTab &, const RysTab &, int, int, double2 *, double *, int, cudaStream_t);
constexpr int kLmax = 3;      // shells up to f (Rys)
constexpr int kLmaxHgp = 2;   // every class pair up to d has an HGP kernel
constexpr int kNumPairClasses = 11;
// pair class c = (kPairClassLa[c], kPairClassLb[c]), ordered by la+lb then la
constexpr int kPairClassLa[] = {0, 1, 1, 2, 2, 3, 2, 3, 2, 3, 3};
constexpr int kPairClassLb[] = {0, 0, 1, 0, 1, 0, 2, 1, 3, 2, 3};
// [x][y], x >= y (bra class x, ket class y); nullptr where no HGP kernel exists
static const EriLauncher kEriLaunchers[11][11] = {
    {launch_eri_ssss, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_psss, launch_eri_psps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_ppss, launch_eri_ppps, launch_eri_pppp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_dsss, launch_eri_dsps, launch_eri_dspp, launch_eri_dsds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_dpss, launch_eri_dpps, launch_eri_dppp, launch_eri_dpds, launch_eri_dpdp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_fsss, launch_eri_fsps, launch_eri_fspp, launch_eri_fsds, launch_eri_fsdp, launch_eri_fsfs, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_ddss, launch_eri_ddps, launch_eri_ddpp, launch_eri_ddds, launch_eri_dddp, nullptr, launch_eri_dddd, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_fpss, launch_eri_fpps, launch_eri_fppp, launch_eri_fpds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_fdss, launch_eri_fdps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_eri_ffss, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
};
static const EriOccupancy kEriOccupancy[11][11] = {
    {occupancy_eri_ssss, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_psss, occupancy_eri_psps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_ppss, occupancy_eri_ppps, occupancy_eri_pppp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_dsss, occupancy_eri_dsps, occupancy_eri_dspp, occupancy_eri_dsds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_dpss, occupancy_eri_dpps, occupancy_eri_dppp, occupancy_eri_dpds, occupancy_eri_dpdp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_fsss, occupancy_eri_fsps, occupancy_eri_fspp, occupancy_eri_fsds, occupancy_eri_fsdp, occupancy_eri_fsfs, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_ddss, occupancy_eri_ddps, occupancy_eri_ddpp, occupancy_eri_ddds, occupancy_eri_dddp, nullptr, occupancy_eri_dddd, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_fpss, occupancy_eri_fpps, occupancy_eri_fppp, occupancy_eri_fpds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_fdss, occupancy_eri_fdps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_eri_ffss, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
};
static const char *const kEriNames[11][11] = {
    {"eri_ssss", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_psss", "eri_psps", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_ppss", "eri_ppps", "eri_pppp", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_dsss", "eri_dsps", "eri_dspp", "eri_dsds", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_dpss", "eri_dpps", "eri_dppp", "eri_dpds", "eri_dpdp", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_fsss", "eri_fsps", "eri_fspp", "eri_fsds", "eri_fsdp", "eri_fsfs", nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_ddss", "eri_ddps", "eri_ddpp", "eri_ddds", "eri_dddp", nullptr, "eri_dddd", nullptr, nullptr, nullptr, nullptr},
    {"eri_fpss", "eri_fpps", "eri_fppp", "eri_fpds", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_fdss", "eri_fdps", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"eri_ffss", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
};
// relative cost of one primitive quartet of the HGP kernel, 1 + VRR entries / 4 (the
// (ss|ss) quartet ~ 1); sizes the lane split of heavy quartets; 0 where no HGP kernel
static const float kEriPrimCost[11][11] = {
    {1.25f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {2.25f, 5.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {4.75f, 14.0f, 37.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {4.75f, 11.75f, 30.0f, 30.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {9.75f, 26.75f, 70.0f, 70.0f, 158.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {9.75f, 22.25f, 54.25f, 54.25f, 122.5f, 122.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {18.5f, 50.5f, 131.25f, 131.25f, 294.75f, 0.0f, 583.5f, 0.0f, 0.0f, 0.0f, 0.0f},
    {18.5f, 46.0f, 115.5f, 115.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {32.5f, 81.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {53.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
};
// 1 where the class pair's kernel has an FP32 variant for MIXED quartets (HGP: at least
// 40 VRR entries; Rys: gen_rys's MIXED_MIN_NBLK / MIXED_MAX_ACC rule), else 0
static const unsigned char kEriHasFp32[11][11] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0},
    {0, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0},
    {0, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0},
    {1, 1, 1, 1, 1, 0, 1, 0, 0, 0, 0},
    {1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
};
static const unsigned char kRysHasFp32[11][11] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 1, 1, 0, 0, 0, 0, 0, 0, 0},
    {0, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0},
    {0, 0, 1, 1, 1, 1, 0, 0, 0, 0, 0},
    {0, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0},
    {0, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0},
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0},
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0},
    {1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0},
};
static const RysLauncher kRysLaunchers[11][11] = {
    {launch_rys_ssss, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_psss, launch_rys_psps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_ppss, launch_rys_ppps, launch_rys_pppp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_dsss, launch_rys_dsps, launch_rys_dspp, launch_rys_dsds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_dpss, launch_rys_dpps, launch_rys_dppp, launch_rys_dpds, launch_rys_dpdp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_fsss, launch_rys_fsps, launch_rys_fspp, launch_rys_fsds, launch_rys_fsdp, launch_rys_fsfs, nullptr, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_ddss, launch_rys_ddps, launch_rys_ddpp, launch_rys_ddds, launch_rys_dddp, launch_rys_ddfs, launch_rys_dddd, nullptr, nullptr, nullptr, nullptr},
    {launch_rys_fpss, launch_rys_fpps, launch_rys_fppp, launch_rys_fpds, launch_rys_fpdp, launch_rys_fpfs, launch_rys_fpdd, launch_rys_fpfp, nullptr, nullptr, nullptr},
    {launch_rys_dfss, launch_rys_dfps, launch_rys_dfpp, launch_rys_dfds, launch_rys_dfdp, launch_rys_dffs, launch_rys_dfdd, launch_rys_dffp, launch_rys_dfdf, nullptr, nullptr},
    {launch_rys_fdss, launch_rys_fdps, launch_rys_fdpp, launch_rys_fdds, launch_rys_fddp, launch_rys_fdfs, launch_rys_fddd, launch_rys_fdfp, launch_rys_fddf, launch_rys_fdfd, nullptr},
    {launch_rys_ffss, launch_rys_ffps, launch_rys_ffpp, launch_rys_ffds, launch_rys_ffdp, launch_rys_fffs, launch_rys_ffdd, launch_rys_fffp, launch_rys_ffdf, launch_rys_fffd, launch_rys_ffff},
};
static const RysOccupancy kRysOccupancy[11][11] = {
    {occupancy_rys_ssss, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_psss, occupancy_rys_psps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_ppss, occupancy_rys_ppps, occupancy_rys_pppp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_dsss, occupancy_rys_dsps, occupancy_rys_dspp, occupancy_rys_dsds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_dpss, occupancy_rys_dpps, occupancy_rys_dppp, occupancy_rys_dpds, occupancy_rys_dpdp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_fsss, occupancy_rys_fsps, occupancy_rys_fspp, occupancy_rys_fsds, occupancy_rys_fsdp, occupancy_rys_fsfs, nullptr, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_ddss, occupancy_rys_ddps, occupancy_rys_ddpp, occupancy_rys_ddds, occupancy_rys_dddp, occupancy_rys_ddfs, occupancy_rys_dddd, nullptr, nullptr, nullptr, nullptr},
    {occupancy_rys_fpss, occupancy_rys_fpps, occupancy_rys_fppp, occupancy_rys_fpds, occupancy_rys_fpdp, occupancy_rys_fpfs, occupancy_rys_fpdd, occupancy_rys_fpfp, nullptr, nullptr, nullptr},
    {occupancy_rys_dfss, occupancy_rys_dfps, occupancy_rys_dfpp, occupancy_rys_dfds, occupancy_rys_dfdp, occupancy_rys_dffs, occupancy_rys_dfdd, occupancy_rys_dffp, occupancy_rys_dfdf, nullptr, nullptr},
    {occupancy_rys_fdss, occupancy_rys_fdps, occupancy_rys_fdpp, occupancy_rys_fdds, occupancy_rys_fddp, occupancy_rys_fdfs, occupancy_rys_fddd, occupancy_rys_fdfp, occupancy_rys_fddf, occupancy_rys_fdfd, nullptr},
    {occupancy_rys_ffss, occupancy_rys_ffps, occupancy_rys_ffpp, occupancy_rys_ffds, occupancy_rys_ffdp, occupancy_rys_fffs, occupancy_rys_ffdd, occupancy_rys_fffp, occupancy_rys_ffdf, occupancy_rys_fffd, occupancy_rys_ffff},
};
static const char *const kRysNames[11][11] = {
    {"rys_ssss", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"rys_psss", "rys_psps", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"rys_ppss", "rys_ppps", "rys_pppp", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"rys_dsss", "rys_dsps", "rys_dspp", "rys_dsds", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"rys_dpss", "rys_dpps", "rys_dppp", "rys_dpds", "rys_dpdp", nullptr, nullptr, nullptr, nullptr, nullptr, nullptr},
    {"rys_fsss", "rys_fsps", "rys_fspp", "rys_fsds", "rys_fsdp", "rys_fsfs", nullptr, nullptr, nullptr, nullptr, nullptr},
    {"rys_ddss", "rys_ddps", "rys_ddpp", "rys_ddds", "rys_dddp", "rys_ddfs", "rys_dddd", nullptr, nullptr, nullptr, nullptr},
    {"rys_fpss", "rys_fpps", "rys_fppp", "rys_fpds", "rys_fpdp", "rys_fpfs", "rys_fpdd", "rys_fpfp", nullptr, nullptr, nullptr},
    {"rys_dfss", "rys_dfps", "rys_dfpp", "rys_dfds", "rys_dfdp", "rys_dffs", "rys_dfdd", "rys_dffp", "rys_dfdf", nullptr, nullptr},
    {"rys_fdss", "rys_fdps", "rys_fdpp", "rys_fdds", "rys_fddp", "rys_fdfs", "rys_fddd", "rys_fdfp", "rys_fddf", "rys_fdfd", nullptr},
    {"rys_ffss", "rys_ffps", "rys_ffpp", "rys_ffds", "rys_ffdp", "rys_fffs", "rys_ffdd", "rys_fffp", "rys_ffdf", "rys_fffd", "rys_ffff"},
};
static const char *const kSchwarzNames[11] = {
    "schwarz_ss", "schwarz_ps", "schwarz_pp", "schwarz_ds", "schwarz_dp", "schwarz_fs", "schwarz_dd", "schwarz_fp", "schwarz_df", "schwarz_fd", "schwarz_ff"
};
static const SchwarzLauncher kSchwarzLaunchers[11] = {
    launch_schwarz_ssss, launch_schwarz_psps, launch_schwarz_pppp, launch_schwarz_dsds, launch_schwarz_dpdp, launch_schwarz_fsfs, launch_schwarz_dddd, nullptr, nullptr, nullptr, nullptr
};
static const RysBoundLauncher kRysBoundLaunchers[11] = {
    launch_rys_bound_ssss, launch_rys_bound_psps, launch_rys_bound_pppp, launch_rys_bound_dsds, launch_rys_bound_dpdp, launch_rys_bound_fsfs, launch_rys_bound_dddd, launch_rys_bound_fpfp, launch_rys_bound_dfdf, launch_rys_bound_fdfd, launch_rys_bound_ffff
};
}  // namespace molints

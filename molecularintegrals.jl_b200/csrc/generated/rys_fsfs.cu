// Generated by gen_rys.py -- Rys class (fs|fs).  Do not edit.
// roots 4, block 10 x 10, outputs 10 x 10, group 32 threads,
// 8 primitive quartets per batch, 1 slot(s), 4 accumulators per thread, 50432 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fsfs {
    static constexpr int LA = 3, LB = 0, LC = 3, LD = 0;
    static constexpr int E = 3, F = 3, NR = 4;
    static constexpr int NA = 10, NC = 10, NBLK = 100;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 10, NCD = 10;
    static constexpr int G = 32, NPB = 8, NSLOT = 1, ACC = 4;
    static constexpr int S = 16;
    static constexpr int SMEM_GROUP = 1576;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fsfs[100] = {
    15, 270, 65550, 525, 131085, 65805, 780, 66060, 131340, 196620, 1035, 1290,
    66570, 1545, 132105, 66825, 1800, 67080, 132360, 197640, 262155, 262410, 327690, 262665,
    393225, 327945, 262920, 328200, 393480, 458760, 2055, 2310, 67590, 2565, 133125, 67845,
    2820, 68100, 133380, 198660, 524295, 524550, 589830, 524805, 655365, 590085, 525060, 590340,
    655620, 720900, 263175, 263430, 328710, 263685, 394245, 328965, 263940, 329220, 394500, 459780,
    3075, 3330, 68610, 3585, 134145, 68865, 3840, 69120, 134400, 199680, 264195, 264450,
    329730, 264705, 395265, 329985, 264960, 330240, 395520, 460800, 525315, 525570, 590850, 525825,
    656385, 591105, 526080, 591360, 656640, 721920, 786435, 786690, 851970, 786945, 917505, 852225,
    787200, 852480, 917760, 983040,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fsfs[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kBraTerm_fsfs[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const uint16_t kKetOff_fsfs[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kKetTerm_fsfs[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const double kNormAB_fsfs[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};
__device__ const double kNormCD_fsfs[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};


__device__ __forceinline__ RysClassTabs tabs_fsfs() {
    return RysClassTabs{kBlk_fsfs, kBraOff_fsfs, kBraTerm_fsfs, kKetOff_fsfs, kKetTerm_fsfs,
                        kNormAB_fsfs, kNormCD_fsfs, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fsfs(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fsfs, MIXED>(Q, R, tabs_fsfs());
}

__global__ void __launch_bounds__(128) rys_bound_kernel_fsfs(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {
    rys_bound_body<C_fsfs>(P, R, tabs_fsfs(), p0, np, pbound, qout, full);
}

static void rys_prepare_fsfs() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fsfs<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 50432);
        cudaFuncSetAttribute(rys_queue_fsfs<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 50432);
        cudaFuncSetAttribute(rys_bound_kernel_fsfs, cudaFuncAttributeMaxDynamicSharedMemorySize, 50432);
        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fsfs(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fsfs();
    constexpr int ng = 128 / C_fsfs::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fsfs<1><<<grid, 128, 50432, s>>>(Q, R);
    else rys_queue_fsfs<0><<<grid, 128, 50432, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fsfs(int mixed) {
    rys_prepare_fsfs();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fsfs<1>, 128, 50432);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fsfs<0>, 128, 50432);
    return n;
}

void launch_rys_bound_fsfs(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    rys_prepare_fsfs();
    constexpr int ng = 128 / C_fsfs::G;
    rys_bound_kernel_fsfs<<<(np + ng - 1) / ng, 128, 50432, s>>>(P, R, p0, np, pbound, qout, full);
}

}  // namespace molints

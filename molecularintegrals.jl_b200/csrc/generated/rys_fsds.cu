// Generated by gen_rys.py -- Rys class (fs|ds).  Do not edit.
// roots 3, block 10 x 6, outputs 10 x 6, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 2 accumulators per thread, 35840 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fsds {
    static constexpr int LA = 3, LB = 0, LC = 2, LD = 0;
    static constexpr int E = 3, F = 2, NR = 3;
    static constexpr int NA = 10, NC = 6, NBLK = 60;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 10, NCD = 6;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 2;
    static constexpr int S = 12;
    static constexpr int SMEM_GROUP = 1120;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fsds[60] = {
    11, 266, 65546, 521, 65801, 131081, 776, 1031, 66311, 1286, 66566, 131846,
    196616, 196871, 262151, 197126, 262406, 327686, 1541, 1796, 67076, 2051, 67331, 132611,
    393221, 393476, 458756, 393731, 459011, 524291, 197381, 197636, 262916, 197891, 263171, 328451,
    2306, 2561, 67841, 2816, 68096, 133376, 198146, 198401, 263681, 198656, 263936, 329216,
    393986, 394241, 459521, 394496, 459776, 525056, 589826, 590081, 655361, 590336, 655616, 720896,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fsds[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kBraTerm_fsds[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const uint16_t kKetOff_fsds[7] = {
    0, 1, 2, 3, 4, 5, 6,
};
__device__ const uint32_t kKetTerm_fsds[6] = {
    65536, 65537, 65538, 65539, 65540, 65541,
};
__device__ const double kNormAB_fsds[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};
__device__ const double kNormCD_fsds[6] = {
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258,
};


__device__ __forceinline__ RysClassTabs tabs_fsds() {
    return RysClassTabs{kBlk_fsds, kBraOff_fsds, kBraTerm_fsds, kKetOff_fsds, kKetTerm_fsds,
                        kNormAB_fsds, kNormCD_fsds, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fsds(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fsds, MIXED>(Q, R, tabs_fsds());
}

static void rys_prepare_fsds() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fsds<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 35840);
        cudaFuncSetAttribute(rys_queue_fsds<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 35840);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fsds(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fsds();
    constexpr int ng = 128 / C_fsds::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fsds<1><<<grid, 128, 35840, s>>>(Q, R);
    else rys_queue_fsds<0><<<grid, 128, 35840, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fsds(int mixed) {
    rys_prepare_fsds();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fsds<1>, 128, 35840);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fsds<0>, 128, 35840);
    return n;
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (fs|pp).  Do not edit.
// roots 3, block 10 x 9, outputs 10 x 9, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 35840 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fspp {
    static constexpr int LA = 3, LB = 0, LC = 1, LD = 1;
    static constexpr int E = 3, F = 2, NR = 3;
    static constexpr int NA = 10, NC = 9, NBLK = 90;
    static constexpr int NB = 1, ND = 3;
    static constexpr int NAB = 10, NCD = 9;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 3;
    static constexpr int S = 12;
    static constexpr int SMEM_GROUP = 1120;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fspp[90] = {
    10, 265, 65545, 11, 266, 65546, 521, 65801, 131081, 775, 1030, 66310,
    776, 1031, 66311, 1286, 66566, 131846, 196615, 196870, 262150, 196616, 196871, 262151,
    197126, 262406, 327686, 1540, 1795, 67075, 1541, 1796, 67076, 2051, 67331, 132611,
    393220, 393475, 458755, 393221, 393476, 458756, 393731, 459011, 524291, 197380, 197635, 262915,
    197381, 197636, 262916, 197891, 263171, 328451, 2305, 2560, 67840, 2306, 2561, 67841,
    2816, 68096, 133376, 198145, 198400, 263680, 198146, 198401, 263681, 198656, 263936, 329216,
    393985, 394240, 459520, 393986, 394241, 459521, 394496, 459776, 525056, 589825, 590080, 655360,
    589826, 590081, 655361, 590336, 655616, 720896,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fspp[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kBraTerm_fspp[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const uint16_t kKetOff_fspp[10] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18,
};
__device__ const uint32_t kKetTerm_fspp[18] = {
    65792, 65539, 66048, 65540, 66304, 65541, 65793, 65540, 66049, 65542, 66305, 65543,
    65794, 65541, 66050, 65543, 66306, 65544,
};
__device__ const double kNormAB_fspp[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};
__device__ const double kNormCD_fspp[9] = {
    1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fspp() {
    return RysClassTabs{kBlk_fspp, kBraOff_fspp, kBraTerm_fspp, kKetOff_fspp, kKetTerm_fspp,
                        kNormAB_fspp, kNormCD_fspp, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fspp(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fspp, MIXED>(Q, R, tabs_fspp());
}

static void rys_prepare_fspp() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fspp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 35840);
        cudaFuncSetAttribute(rys_queue_fspp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 35840);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fspp(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fspp();
    constexpr int ng = 128 / C_fspp::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fspp<1><<<grid, 128, 35840, s>>>(Q, R);
    else rys_queue_fspp<0><<<grid, 128, 35840, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fspp(int mixed) {
    rys_prepare_fspp();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fspp<1>, 128, 35840);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fspp<0>, 128, 35840);
    return n;
}

}  // namespace molints

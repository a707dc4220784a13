// Generated by gen_rys.py -- Rys class (fs|ps).  Do not edit.
// roots 3, block 10 x 3, outputs 10 x 3, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 1 accumulators per thread, 24320 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fsps {
    static constexpr int LA = 3, LB = 0, LC = 1, LD = 0;
    static constexpr int E = 3, F = 1, NR = 3;
    static constexpr int NA = 10, NC = 3, NBLK = 30;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 10, NCD = 3;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 1;
    static constexpr int S = 8;
    static constexpr int SMEM_GROUP = 760;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fsps[30] = {
    7, 262, 65542, 517, 772, 66052, 131077, 131332, 196612, 1027, 1282, 66562,
    262147, 262402, 327682, 131587, 131842, 197122, 1537, 1792, 67072, 132097, 132352, 197632,
    262657, 262912, 328192, 393217, 393472, 458752,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fsps[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kBraTerm_fsps[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const uint16_t kKetOff_fsps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_fsps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_fsps[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};
__device__ const double kNormCD_fsps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fsps() {
    return RysClassTabs{kBlk_fsps, kBraOff_fsps, kBraTerm_fsps, kKetOff_fsps, kKetTerm_fsps,
                        kNormAB_fsps, kNormCD_fsps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fsps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fsps, MIXED>(Q, R, tabs_fsps());
}

static void rys_prepare_fsps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fsps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 24320);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fsps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fsps();
    constexpr int ng = 128 / C_fsps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_fsps<0><<<grid, 128, 24320, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fsps(int mixed) {
    rys_prepare_fsps();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fsps<0>, 128, 24320);
    return n;
}

}  // namespace molints

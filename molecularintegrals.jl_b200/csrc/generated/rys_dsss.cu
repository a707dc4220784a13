// Generated by gen_rys.py -- Rys class (ds|ss).  Do not edit.
// roots 2, block 6 x 1, outputs 6 x 1, group 32 threads,
// 16 primitive quartets per batch, 5 slot(s), 1 accumulators per thread, 10496 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_dsss {
    static constexpr int LA = 2, LB = 0, LC = 0, LD = 0;
    static constexpr int E = 2, F = 0, NR = 2;
    static constexpr int NA = 6, NC = 1, NBLK = 6;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 6, NCD = 1;
    static constexpr int G = 32, NPB = 16, NSLOT = 5, ACC = 1;
    static constexpr int S = 3;
    static constexpr int SMEM_GROUP = 328;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_dsss[6] = {
    2, 257, 65537, 512, 65792, 131072,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_dsss[7] = {
    0, 1, 2, 3, 4, 5, 6,
};
__device__ const uint32_t kBraTerm_dsss[6] = {
    65536, 65537, 65538, 65539, 65540, 65541,
};
__device__ const uint16_t kKetOff_dsss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_dsss[1] = {
    65536,
};
__device__ const double kNormAB_dsss[6] = {
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258,
};
__device__ const double kNormCD_dsss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_dsss() {
    return RysClassTabs{kBlk_dsss, kBraOff_dsss, kBraTerm_dsss, kKetOff_dsss, kKetTerm_dsss,
                        kNormAB_dsss, kNormCD_dsss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_dsss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_dsss, MIXED>(Q, R, tabs_dsss());
}

static void rys_prepare_dsss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_dsss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 10496);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_dsss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_dsss();
    constexpr int ng = 128 / C_dsss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_dsss<0><<<grid, 128, 10496, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_dsss(int mixed) {
    rys_prepare_dsss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dsss<0>, 128, 10496);
    return n;
}

}  // namespace molints

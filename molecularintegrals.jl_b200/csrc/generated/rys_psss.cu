// Generated by gen_rys.py -- Rys class (ps|ss).  Do not edit.
// roots 1, block 3 x 1, outputs 3 x 1, group 32 threads,
// 32 primitive quartets per batch, 10 slot(s), 1 accumulators per thread, 7424 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_psss {
    static constexpr int LA = 1, LB = 0, LC = 0, LD = 0;
    static constexpr int E = 1, F = 0, NR = 1;
    static constexpr int NA = 3, NC = 1, NBLK = 3;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 3, NCD = 1;
    static constexpr int G = 32, NPB = 32, NSLOT = 10, ACC = 1;
    static constexpr int S = 2;
    static constexpr int SMEM_GROUP = 232;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_psss[3] = {
    1, 256, 65536,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_psss[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kBraTerm_psss[3] = {
    65536, 65537, 65538,
};
__device__ const uint16_t kKetOff_psss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_psss[1] = {
    65536,
};
__device__ const double kNormAB_psss[3] = {
    1.0, 1.0, 1.0,
};
__device__ const double kNormCD_psss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_psss() {
    return RysClassTabs{kBlk_psss, kBraOff_psss, kBraTerm_psss, kKetOff_psss, kKetTerm_psss,
                        kNormAB_psss, kNormCD_psss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_psss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_psss, MIXED>(Q, R, tabs_psss());
}

static void rys_prepare_psss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_psss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 7424);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_psss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_psss();
    constexpr int ng = 128 / C_psss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_psss<0><<<grid, 128, 7424, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_psss(int mixed) {
    rys_prepare_psss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_psss<0>, 128, 7424);
    return n;
}

}  // namespace molints

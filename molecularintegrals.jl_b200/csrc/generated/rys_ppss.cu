// Generated by gen_rys.py -- Rys class (pp|ss).  Do not edit.
// roots 2, block 9 x 1, outputs 9 x 1, group 32 threads,
// 16 primitive quartets per batch, 3 slot(s), 1 accumulators per thread, 10496 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_ppss {
    static constexpr int LA = 1, LB = 1, LC = 0, LD = 0;
    static constexpr int E = 2, F = 0, NR = 2;
    static constexpr int NA = 9, NC = 1, NBLK = 9;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 9, NCD = 1;
    static constexpr int G = 32, NPB = 16, NSLOT = 3, ACC = 1;
    static constexpr int S = 3;
    static constexpr int SMEM_GROUP = 328;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_ppss[9] = {
    1, 256, 65536, 2, 257, 65537, 512, 65792, 131072,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_ppss[10] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18,
};
__device__ const uint32_t kBraTerm_ppss[18] = {
    65792, 65539, 66048, 65540, 66304, 65541, 65793, 65540, 66049, 65542, 66305, 65543,
    65794, 65541, 66050, 65543, 66306, 65544,
};
__device__ const uint16_t kKetOff_ppss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_ppss[1] = {
    65536,
};
__device__ const double kNormAB_ppss[9] = {
    1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0,
};
__device__ const double kNormCD_ppss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_ppss() {
    return RysClassTabs{kBlk_ppss, kBraOff_ppss, kBraTerm_ppss, kKetOff_ppss, kKetTerm_ppss,
                        kNormAB_ppss, kNormCD_ppss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_ppss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_ppss, MIXED>(Q, R, tabs_ppss());
}

static void rys_prepare_ppss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_ppss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 10496);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_ppss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_ppss();
    constexpr int ng = 128 / C_ppss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_ppss<0><<<grid, 128, 10496, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_ppss(int mixed) {
    rys_prepare_ppss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ppss<0>, 128, 10496);
    return n;
}

}  // namespace molints

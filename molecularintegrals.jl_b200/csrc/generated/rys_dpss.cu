// Generated by gen_rys.py -- Rys class (dp|ss).  Do not edit.
// roots 2, block 16 x 1, outputs 18 x 1, group 32 threads,
// 16 primitive quartets per batch, 2 slot(s), 1 accumulators per thread, 13568 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_dpss {
    static constexpr int LA = 2, LB = 1, LC = 0, LD = 0;
    static constexpr int E = 3, F = 0, NR = 2;
    static constexpr int NA = 16, NC = 1, NBLK = 16;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 18, NCD = 1;
    static constexpr int G = 32, NPB = 16, NSLOT = 2, ACC = 1;
    static constexpr int S = 4;
    static constexpr int SMEM_GROUP = 424;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_dpss[16] = {
    2, 257, 65537, 512, 65792, 131072, 3, 258, 65538, 513, 131073, 65793,
    768, 66048, 131328, 196608,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_dpss[19] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36,
};
__device__ const uint32_t kBraTerm_dpss[36] = {
    65792, 65542, 66048, 65543, 66304, 65544, 65793, 65543, 66049, 65545, 66305, 65547,
    65794, 65544, 66050, 65547, 66306, 65546, 65795, 65545, 66051, 65548, 66307, 65549,
    65796, 65547, 66052, 65549, 66308, 65550, 65797, 65546, 66053, 65550, 66309, 65551,
};
__device__ const uint16_t kKetOff_dpss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_dpss[1] = {
    65536,
};
__device__ const double kNormAB_dpss[18] = {
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    1.0, 1.0, 1.0, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258,
};
__device__ const double kNormCD_dpss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_dpss() {
    return RysClassTabs{kBlk_dpss, kBraOff_dpss, kBraTerm_dpss, kKetOff_dpss, kKetTerm_dpss,
                        kNormAB_dpss, kNormCD_dpss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_dpss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_dpss, MIXED>(Q, R, tabs_dpss());
}

static void rys_prepare_dpss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_dpss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 13568);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_dpss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_dpss();
    constexpr int ng = 128 / C_dpss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_dpss<0><<<grid, 128, 13568, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_dpss(int mixed) {
    rys_prepare_dpss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dpss<0>, 128, 13568);
    return n;
}

}  // namespace molints

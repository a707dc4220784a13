// Generated by gen_rys.py -- Rys class (fs|ss).  Do not edit.
// roots 2, block 10 x 1, outputs 10 x 1, group 32 threads,
// 16 primitive quartets per batch, 3 slot(s), 1 accumulators per thread, 13568 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fsss {
    static constexpr int LA = 3, LB = 0, LC = 0, LD = 0;
    static constexpr int E = 3, F = 0, NR = 2;
    static constexpr int NA = 10, NC = 1, NBLK = 10;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 10, NCD = 1;
    static constexpr int G = 32, NPB = 16, NSLOT = 3, ACC = 1;
    static constexpr int S = 4;
    static constexpr int SMEM_GROUP = 424;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fsss[10] = {
    3, 258, 65538, 513, 131073, 65793, 768, 66048, 131328, 196608,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fsss[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kBraTerm_fsss[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const uint16_t kKetOff_fsss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_fsss[1] = {
    65536,
};
__device__ const double kNormAB_fsss[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};
__device__ const double kNormCD_fsss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fsss() {
    return RysClassTabs{kBlk_fsss, kBraOff_fsss, kBraTerm_fsss, kKetOff_fsss, kKetTerm_fsss,
                        kNormAB_fsss, kNormCD_fsss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fsss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fsss, MIXED>(Q, R, tabs_fsss());
}

static void rys_prepare_fsss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fsss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 13568);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fsss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fsss();
    constexpr int ng = 128 / C_fsss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_fsss<0><<<grid, 128, 13568, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fsss(int mixed) {
    rys_prepare_fsss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fsss<0>, 128, 13568);
    return n;
}

}  // namespace molints

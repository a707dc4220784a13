// Generated by gen_rys.py -- Rys class (ss|ss).  Do not edit.
// roots 1, block 1 x 1, outputs 1 x 1, group 32 threads,
// 32 primitive quartets per batch, 32 slot(s), 1 accumulators per thread, 4352 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_ssss {
    static constexpr int LA = 0, LB = 0, LC = 0, LD = 0;
    static constexpr int E = 0, F = 0, NR = 1;
    static constexpr int NA = 1, NC = 1, NBLK = 1;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 1, NCD = 1;
    static constexpr int G = 32, NPB = 32, NSLOT = 32, ACC = 1;
    static constexpr int S = 1;
    static constexpr int SMEM_GROUP = 136;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_ssss[1] = {
    0,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_ssss[2] = {
    0, 1,
};
__device__ const uint32_t kBraTerm_ssss[1] = {
    65536,
};
__device__ const uint16_t kKetOff_ssss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_ssss[1] = {
    65536,
};
__device__ const double kNormAB_ssss[1] = {
    1.0,
};
__device__ const double kNormCD_ssss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_ssss() {
    return RysClassTabs{kBlk_ssss, kBraOff_ssss, kBraTerm_ssss, kKetOff_ssss, kKetTerm_ssss,
                        kNormAB_ssss, kNormCD_ssss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_ssss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_ssss, MIXED>(Q, R, tabs_ssss());
}

__global__ void __launch_bounds__(128) rys_bound_kernel_ssss(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {
    rys_bound_body<C_ssss>(P, R, tabs_ssss(), p0, np, pbound, qout, full);
}

static void rys_prepare_ssss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_ssss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4352);

        cudaFuncSetAttribute(rys_bound_kernel_ssss, cudaFuncAttributeMaxDynamicSharedMemorySize, 4352);
        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_ssss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_ssss();
    constexpr int ng = 128 / C_ssss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_ssss<0><<<grid, 128, 4352, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_ssss(int mixed) {
    rys_prepare_ssss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ssss<0>, 128, 4352);
    return n;
}

void launch_rys_bound_ssss(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    rys_prepare_ssss();
    constexpr int ng = 128 / C_ssss::G;
    rys_bound_kernel_ssss<<<(np + ng - 1) / ng, 128, 4352, s>>>(P, R, p0, np, pbound, qout, full);
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (ps|ps).  Do not edit.
// roots 2, block 3 x 3, outputs 3 x 3, group 32 threads,
// 16 primitive quartets per batch, 3 slot(s), 1 accumulators per thread, 13568 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_psps {
    static constexpr int LA = 1, LB = 0, LC = 1, LD = 0;
    static constexpr int E = 1, F = 1, NR = 2;
    static constexpr int NA = 3, NC = 3, NBLK = 9;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 3, NCD = 3;
    static constexpr int G = 32, NPB = 16, NSLOT = 3, ACC = 1;
    static constexpr int S = 4;
    static constexpr int SMEM_GROUP = 424;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_psps[9] = {
    3, 258, 65538, 513, 768, 66048, 131073, 131328, 196608,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_psps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kBraTerm_psps[3] = {
    65536, 65537, 65538,
};
__device__ const uint16_t kKetOff_psps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_psps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_psps[3] = {
    1.0, 1.0, 1.0,
};
__device__ const double kNormCD_psps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_psps() {
    return RysClassTabs{kBlk_psps, kBraOff_psps, kBraTerm_psps, kKetOff_psps, kKetTerm_psps,
                        kNormAB_psps, kNormCD_psps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_psps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_psps, MIXED>(Q, R, tabs_psps());
}

__global__ void __launch_bounds__(128) rys_bound_kernel_psps(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {
    rys_bound_body<C_psps>(P, R, tabs_psps(), p0, np, pbound, qout, full);
}

static void rys_prepare_psps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_psps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 13568);

        cudaFuncSetAttribute(rys_bound_kernel_psps, cudaFuncAttributeMaxDynamicSharedMemorySize, 13568);
        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_psps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_psps();
    constexpr int ng = 128 / C_psps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_psps<0><<<grid, 128, 13568, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_psps(int mixed) {
    rys_prepare_psps();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_psps<0>, 128, 13568);
    return n;
}

void launch_rys_bound_psps(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    rys_prepare_psps();
    constexpr int ng = 128 / C_psps::G;
    rys_bound_kernel_psps<<<(np + ng - 1) / ng, 128, 13568, s>>>(P, R, p0, np, pbound, qout, full);
}

}  // namespace molints

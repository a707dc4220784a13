// Generated by gen_rys.py -- Rys class (ds|ds).  Do not edit.
// roots 3, block 6 x 6, outputs 6 x 6, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 2 accumulators per thread, 27200 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_dsds {
    static constexpr int LA = 2, LB = 0, LC = 2, LD = 0;
    static constexpr int E = 2, F = 2, NR = 3;
    static constexpr int NA = 6, NC = 6, NBLK = 36;
    static constexpr int NB = 1, ND = 1;
    static constexpr int NAB = 6, NCD = 6;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 2;
    static constexpr int S = 9;
    static constexpr int SMEM_GROUP = 850;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_dsds[36] = {
    8, 263, 65543, 518, 65798, 131078, 773, 1028, 66308, 1283, 66563, 131843,
    196613, 196868, 262148, 197123, 262403, 327683, 1538, 1793, 67073, 2048, 67328, 132608,
    197378, 197633, 262913, 197888, 263168, 328448, 393218, 393473, 458753, 393728, 459008, 524288,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_dsds[7] = {
    0, 1, 2, 3, 4, 5, 6,
};
__device__ const uint32_t kBraTerm_dsds[6] = {
    65536, 65537, 65538, 65539, 65540, 65541,
};
__device__ const uint16_t kKetOff_dsds[7] = {
    0, 1, 2, 3, 4, 5, 6,
};
__device__ const uint32_t kKetTerm_dsds[6] = {
    65536, 65537, 65538, 65539, 65540, 65541,
};
__device__ const double kNormAB_dsds[6] = {
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258,
};
__device__ const double kNormCD_dsds[6] = {
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258,
};


__device__ __forceinline__ RysClassTabs tabs_dsds() {
    return RysClassTabs{kBlk_dsds, kBraOff_dsds, kBraTerm_dsds, kKetOff_dsds, kKetTerm_dsds,
                        kNormAB_dsds, kNormCD_dsds, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_dsds(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_dsds, MIXED>(Q, R, tabs_dsds());
}

__global__ void __launch_bounds__(128) rys_bound_kernel_dsds(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {
    rys_bound_body<C_dsds>(P, R, tabs_dsds(), p0, np, pbound, qout, full);
}

static void rys_prepare_dsds() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_dsds<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 27200);
        cudaFuncSetAttribute(rys_queue_dsds<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 27200);
        cudaFuncSetAttribute(rys_bound_kernel_dsds, cudaFuncAttributeMaxDynamicSharedMemorySize, 27200);
        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_dsds(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_dsds();
    constexpr int ng = 128 / C_dsds::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_dsds<1><<<grid, 128, 27200, s>>>(Q, R);
    else rys_queue_dsds<0><<<grid, 128, 27200, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_dsds(int mixed) {
    rys_prepare_dsds();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dsds<1>, 128, 27200);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dsds<0>, 128, 27200);
    return n;
}

void launch_rys_bound_dsds(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    rys_prepare_dsds();
    constexpr int ng = 128 / C_dsds::G;
    rys_bound_kernel_dsds<<<(np + ng - 1) / ng, 128, 27200, s>>>(P, R, p0, np, pbound, qout, full);
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (pp|pp).  Do not edit.
// roots 3, block 9 x 9, outputs 9 x 9, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 27200 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_pppp {
    static constexpr int LA = 1, LB = 1, LC = 1, LD = 1;
    static constexpr int E = 2, F = 2, NR = 3;
    static constexpr int NA = 9, NC = 9, NBLK = 81;
    static constexpr int NB = 3, ND = 3;
    static constexpr int NAB = 9, NCD = 9;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 3;
    static constexpr int S = 9;
    static constexpr int SMEM_GROUP = 850;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_pppp[81] = {
    4, 259, 65539, 5, 260, 65540, 515, 65795, 131075, 769, 1024, 66304,
    770, 1025, 66305, 1280, 66560, 131840, 196609, 196864, 262144, 196610, 196865, 262145,
    197120, 262400, 327680, 7, 262, 65542, 8, 263, 65543, 518, 65798, 131078,
    772, 1027, 66307, 773, 1028, 66308, 1283, 66563, 131843, 196612, 196867, 262147,
    196613, 196868, 262148, 197123, 262403, 327683, 1537, 1792, 67072, 1538, 1793, 67073,
    2048, 67328, 132608, 197377, 197632, 262912, 197378, 197633, 262913, 197888, 263168, 328448,
    393217, 393472, 458752, 393218, 393473, 458753, 393728, 459008, 524288,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_pppp[10] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18,
};
__device__ const uint32_t kBraTerm_pppp[18] = {
    65792, 65539, 66048, 65540, 66304, 65541, 65793, 65540, 66049, 65542, 66305, 65543,
    65794, 65541, 66050, 65543, 66306, 65544,
};
__device__ const uint16_t kKetOff_pppp[10] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18,
};
__device__ const uint32_t kKetTerm_pppp[18] = {
    65792, 65539, 66048, 65540, 66304, 65541, 65793, 65540, 66049, 65542, 66305, 65543,
    65794, 65541, 66050, 65543, 66306, 65544,
};
__device__ const double kNormAB_pppp[9] = {
    1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0,
};
__device__ const double kNormCD_pppp[9] = {
    1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_pppp() {
    return RysClassTabs{kBlk_pppp, kBraOff_pppp, kBraTerm_pppp, kKetOff_pppp, kKetTerm_pppp,
                        kNormAB_pppp, kNormCD_pppp, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_pppp(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_pppp, MIXED>(Q, R, tabs_pppp());
}

__global__ void __launch_bounds__(128) rys_bound_kernel_pppp(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {
    rys_bound_body<C_pppp>(P, R, tabs_pppp(), p0, np, pbound, qout, full);
}

static void rys_prepare_pppp() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_pppp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 27200);
        cudaFuncSetAttribute(rys_queue_pppp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 27200);
        cudaFuncSetAttribute(rys_bound_kernel_pppp, cudaFuncAttributeMaxDynamicSharedMemorySize, 27200);
        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_pppp(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_pppp();
    constexpr int ng = 128 / C_pppp::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_pppp<1><<<grid, 128, 27200, s>>>(Q, R);
    else rys_queue_pppp<0><<<grid, 128, 27200, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_pppp(int mixed) {
    rys_prepare_pppp();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_pppp<1>, 128, 27200);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_pppp<0>, 128, 27200);
    return n;
}

void launch_rys_bound_pppp(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    rys_prepare_pppp();
    constexpr int ng = 128 / C_pppp::G;
    rys_bound_kernel_pppp<<<(np + ng - 1) / ng, 128, 27200, s>>>(P, R, p0, np, pbound, qout, full);
}

}  // namespace molints

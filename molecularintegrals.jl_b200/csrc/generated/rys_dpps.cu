// Generated by gen_rys.py -- Rys class (dp|ps).  Do not edit.
// roots 3, block 16 x 3, outputs 18 x 3, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 2 accumulators per thread, 24320 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_dpps {
    static constexpr int LA = 2, LB = 1, LC = 1, LD = 0;
    static constexpr int E = 3, F = 1, NR = 3;
    static constexpr int NA = 16, NC = 3, NBLK = 48;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 18, NCD = 3;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 2;
    static constexpr int S = 8;
    static constexpr int SMEM_GROUP = 760;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_dpps[48] = {
    5, 260, 65540, 515, 770, 66050, 131075, 131330, 196610, 1025, 1280, 66560,
    131585, 131840, 197120, 262145, 262400, 327680, 7, 262, 65542, 517, 772, 66052,
    131077, 131332, 196612, 1027, 1282, 66562, 262147, 262402, 327682, 131587, 131842, 197122,
    1537, 1792, 67072, 132097, 132352, 197632, 262657, 262912, 328192, 393217, 393472, 458752,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_dpps[19] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36,
};
__device__ const uint32_t kBraTerm_dpps[36] = {
    65792, 65542, 66048, 65543, 66304, 65544, 65793, 65543, 66049, 65545, 66305, 65547,
    65794, 65544, 66050, 65547, 66306, 65546, 65795, 65545, 66051, 65548, 66307, 65549,
    65796, 65547, 66052, 65549, 66308, 65550, 65797, 65546, 66053, 65550, 66309, 65551,
};
__device__ const uint16_t kKetOff_dpps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_dpps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_dpps[18] = {
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    1.0, 1.0, 1.0, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258,
};
__device__ const double kNormCD_dpps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_dpps() {
    return RysClassTabs{kBlk_dpps, kBraOff_dpps, kBraTerm_dpps, kKetOff_dpps, kKetTerm_dpps,
                        kNormAB_dpps, kNormCD_dpps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_dpps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_dpps, MIXED>(Q, R, tabs_dpps());
}

static void rys_prepare_dpps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_dpps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 24320);
        cudaFuncSetAttribute(rys_queue_dpps<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 24320);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_dpps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_dpps();
    constexpr int ng = 128 / C_dpps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_dpps<1><<<grid, 128, 24320, s>>>(Q, R);
    else rys_queue_dpps<0><<<grid, 128, 24320, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_dpps(int mixed) {
    rys_prepare_dpps();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dpps<1>, 128, 24320);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dpps<0>, 128, 24320);
    return n;
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (fp|ps).  Do not edit.
// roots 3, block 25 x 3, outputs 30 x 3, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 30080 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fpps {
    static constexpr int LA = 3, LB = 1, LC = 1, LD = 0;
    static constexpr int E = 4, F = 1, NR = 3;
    static constexpr int NA = 25, NC = 3, NBLK = 75;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 30, NCD = 3;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 3;
    static constexpr int S = 10;
    static constexpr int SMEM_GROUP = 940;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fpps[75] = {
    7, 262, 65542, 517, 772, 66052, 131077, 131332, 196612, 1027, 1282, 66562,
    262147, 262402, 327682, 131587, 131842, 197122, 1537, 1792, 67072, 132097, 132352, 197632,
    262657, 262912, 328192, 393217, 393472, 458752, 9, 264, 65544, 519, 774, 66054,
    131079, 131334, 196614, 1029, 1284, 66564, 131589, 131844, 197124, 262149, 262404, 327684,
    1539, 1794, 67074, 132099, 132354, 197634, 262659, 262914, 328194, 393219, 393474, 458754,
    2049, 2304, 67584, 132609, 132864, 198144, 263169, 263424, 328704, 393729, 393984, 459264,
    524289, 524544, 589824,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fpps[31] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36, 38, 40, 42, 44, 46,
    48, 50, 52, 54, 56, 58, 60,
};
__device__ const uint32_t kBraTerm_fpps[60] = {
    65792, 65546, 66048, 65547, 66304, 65548, 65793, 65547, 66049, 65549, 66305, 65550,
    65794, 65548, 66050, 65550, 66306, 65551, 65795, 65549, 66051, 65552, 66307, 65553,
    65796, 65551, 66052, 65554, 66308, 65555, 65797, 65550, 66053, 65553, 66309, 65554,
    65798, 65552, 66054, 65556, 66310, 65557, 65799, 65553, 66055, 65557, 66311, 65558,
    65800, 65554, 66056, 65558, 66312, 65559, 65801, 65555, 66057, 65559, 66313, 65560,
};
__device__ const uint16_t kKetOff_fpps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_fpps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_fpps[30] = {
    0.2581988897471611, 0.2581988897471611, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 0.2581988897471611, 0.2581988897471611,
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.2581988897471611,
    0.2581988897471611, 0.2581988897471611,
};
__device__ const double kNormCD_fpps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fpps() {
    return RysClassTabs{kBlk_fpps, kBraOff_fpps, kBraTerm_fpps, kKetOff_fpps, kKetTerm_fpps,
                        kNormAB_fpps, kNormCD_fpps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fpps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fpps, MIXED>(Q, R, tabs_fpps());
}

static void rys_prepare_fpps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fpps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 30080);
        cudaFuncSetAttribute(rys_queue_fpps<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 30080);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fpps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fpps();
    constexpr int ng = 128 / C_fpps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fpps<1><<<grid, 128, 30080, s>>>(Q, R);
    else rys_queue_fpps<0><<<grid, 128, 30080, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fpps(int mixed) {
    rys_prepare_fpps();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpps<1>, 128, 30080);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpps<0>, 128, 30080);
    return n;
}

}  // namespace molints

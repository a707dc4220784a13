// Generated by gen_rys.py -- Rys class (dd|ps).  Do not edit.
// roots 3, block 31 x 3, outputs 36 x 3, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 30080 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_ddps {
    static constexpr int LA = 2, LB = 2, LC = 1, LD = 0;
    static constexpr int E = 4, F = 1, NR = 3;
    static constexpr int NA = 31, NC = 3, NBLK = 93;
    static constexpr int NB = 6, ND = 1;
    static constexpr int NAB = 36, NCD = 3;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 3;
    static constexpr int S = 10;
    static constexpr int SMEM_GROUP = 940;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_ddps[93] = {
    5, 260, 65540, 515, 770, 66050, 131075, 131330, 196610, 1025, 1280, 66560,
    131585, 131840, 197120, 262145, 262400, 327680, 7, 262, 65542, 517, 772, 66052,
    131077, 131332, 196612, 1027, 1282, 66562, 262147, 262402, 327682, 131587, 131842, 197122,
    1537, 1792, 67072, 132097, 132352, 197632, 262657, 262912, 328192, 393217, 393472, 458752,
    9, 264, 65544, 519, 774, 66054, 131079, 131334, 196614, 1029, 1284, 66564,
    131589, 131844, 197124, 262149, 262404, 327684, 1539, 1794, 67074, 132099, 132354, 197634,
    262659, 262914, 328194, 393219, 393474, 458754, 2049, 2304, 67584, 132609, 132864, 198144,
    263169, 263424, 328704, 393729, 393984, 459264, 524289, 524544, 589824,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_ddps[37] = {
    0, 3, 7, 11, 14, 18, 21, 24, 28, 32, 35, 39,
    42, 45, 49, 53, 56, 60, 63, 66, 70, 74, 77, 81,
    84, 87, 91, 95, 98, 102, 105, 108, 112, 116, 119, 123,
    126,
};
__device__ const uint32_t kBraTerm_ddps[126] = {
    66560, 131334, 65552, 66816, 65799, 66054, 65553, 67072, 65800, 66310, 65554, 67328,
    131591, 65555, 67584, 66056, 66311, 65556, 67840, 131848, 65557, 66561, 131335, 65553,
    66817, 65801, 66055, 65555, 67073, 65803, 66311, 65556, 67329, 131593, 65558, 67585,
    66059, 66313, 65559, 67841, 131851, 65560, 66562, 131336, 65554, 66818, 65803, 66056,
    65556, 67074, 65802, 66312, 65557, 67330, 131595, 65559, 67586, 66058, 66315, 65560,
    67842, 131850, 65561, 66563, 131337, 65555, 66819, 65804, 66057, 65558, 67075, 65805,
    66313, 65559, 67331, 131596, 65562, 67587, 66061, 66316, 65563, 67843, 131853, 65564,
    66564, 131339, 65556, 66820, 65805, 66059, 65559, 67076, 65806, 66315, 65560, 67332,
    131597, 65563, 67588, 66062, 66317, 65564, 67844, 131854, 65565, 66565, 131338, 65557,
    66821, 65806, 66058, 65560, 67077, 65807, 66314, 65561, 67333, 131598, 65564, 67589,
    66063, 66318, 65565, 67845, 131855, 65566,
};
__device__ const uint16_t kKetOff_ddps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_ddps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_ddps[36] = {
    0.3333333333333334, 0.5773502691896258, 0.5773502691896258, 0.3333333333333334,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 1.0,
    1.0, 0.5773502691896258, 1.0, 0.5773502691896258,
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258, 0.3333333333333334, 0.5773502691896258,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 0.3333333333333334,
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258, 0.3333333333333334, 0.5773502691896258,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 0.3333333333333334,
};
__device__ const double kNormCD_ddps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_ddps() {
    return RysClassTabs{kBlk_ddps, kBraOff_ddps, kBraTerm_ddps, kKetOff_ddps, kKetTerm_ddps,
                        kNormAB_ddps, kNormCD_ddps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_ddps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_ddps, MIXED>(Q, R, tabs_ddps());
}

static void rys_prepare_ddps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_ddps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 30080);
        cudaFuncSetAttribute(rys_queue_ddps<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 30080);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_ddps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_ddps();
    constexpr int ng = 128 / C_ddps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_ddps<1><<<grid, 128, 30080, s>>>(Q, R);
    else rys_queue_ddps<0><<<grid, 128, 30080, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_ddps(int mixed) {
    rys_prepare_ddps();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ddps<1>, 128, 30080);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ddps<0>, 128, 30080);
    return n;
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (fd|ps).  Do not edit.
// roots 4, block 46 x 3, outputs 60 x 3, group 64 threads,
// 16 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 37504 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fdps {
    static constexpr int LA = 3, LB = 2, LC = 1, LD = 0;
    static constexpr int E = 5, F = 1, NR = 4;
    static constexpr int NA = 46, NC = 3, NBLK = 138;
    static constexpr int NB = 6, ND = 1;
    static constexpr int NAB = 60, NCD = 3;
    static constexpr int G = 64, NPB = 16, NSLOT = 1, ACC = 3;
    static constexpr int S = 12;
    static constexpr int SMEM_GROUP = 2344;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fdps[138] = {
    7, 262, 65542, 517, 772, 66052, 131077, 131332, 196612, 1027, 1282, 66562,
    262147, 262402, 327682, 131587, 131842, 197122, 1537, 1792, 67072, 132097, 132352, 197632,
    262657, 262912, 328192, 393217, 393472, 458752, 9, 264, 65544, 519, 774, 66054,
    131079, 131334, 196614, 1029, 1284, 66564, 131589, 131844, 197124, 262149, 262404, 327684,
    1539, 1794, 67074, 132099, 132354, 197634, 262659, 262914, 328194, 393219, 393474, 458754,
    2049, 2304, 67584, 132609, 132864, 198144, 263169, 263424, 328704, 393729, 393984, 459264,
    524289, 524544, 589824, 11, 266, 65546, 521, 776, 66056, 131081, 131336, 196616,
    1031, 1286, 66566, 131591, 131846, 197126, 262151, 262406, 327686, 1541, 1796, 67076,
    132101, 132356, 197636, 262661, 262916, 328196, 393221, 393476, 458756, 2051, 2306, 67586,
    132611, 132866, 198146, 263171, 263426, 328706, 393731, 393986, 459266, 524291, 524546, 589826,
    2561, 2816, 68096, 133121, 133376, 198656, 263681, 263936, 329216, 394241, 394496, 459776,
    524801, 525056, 590336, 655361, 655616, 720896,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fdps[61] = {
    0, 3, 7, 11, 14, 18, 21, 24, 28, 32, 35, 39,
    42, 45, 49, 53, 56, 60, 63, 66, 70, 74, 77, 81,
    84, 87, 91, 95, 98, 102, 105, 108, 112, 116, 119, 123,
    126, 129, 133, 137, 140, 144, 147, 150, 154, 158, 161, 165,
    168, 171, 175, 179, 182, 186, 189, 192, 196, 200, 203, 207,
    210,
};
__device__ const uint32_t kBraTerm_fdps[210] = {
    66560, 131338, 65561, 66816, 65803, 66058, 65562, 67072, 65804, 66314, 65563, 67328,
    131595, 65564, 67584, 66060, 66315, 65565, 67840, 131852, 65566, 66561, 131339, 65562,
    66817, 65805, 66059, 65564, 67073, 65806, 66315, 65565, 67329, 131597, 65567, 67585,
    66062, 66317, 65568, 67841, 131854, 65569, 66562, 131340, 65563, 66818, 65806, 66060,
    65565, 67074, 65807, 66316, 65566, 67330, 131598, 65568, 67586, 66063, 66318, 65569,
    67842, 131855, 65570, 66563, 131341, 65564, 66819, 65808, 66061, 65567, 67075, 65809,
    66317, 65568, 67331, 131600, 65571, 67587, 66065, 66320, 65572, 67843, 131857, 65573,
    66564, 131343, 65566, 66820, 65810, 66063, 65569, 67076, 65811, 66319, 65570, 67332,
    131602, 65573, 67588, 66067, 66322, 65574, 67844, 131859, 65575, 66565, 131342, 65565,
    66821, 65809, 66062, 65568, 67077, 65810, 66318, 65569, 67333, 131601, 65572, 67589,
    66066, 66321, 65573, 67845, 131858, 65574, 66566, 131344, 65567, 66822, 65812, 66064,
    65571, 67078, 65813, 66320, 65572, 67334, 131604, 65576, 67590, 66069, 66324, 65577,
    67846, 131861, 65578, 66567, 131345, 65568, 66823, 65813, 66065, 65572, 67079, 65814,
    66321, 65573, 67335, 131605, 65577, 67591, 66070, 66325, 65578, 67847, 131862, 65579,
    66568, 131346, 65569, 66824, 65814, 66066, 65573, 67080, 65815, 66322, 65574, 67336,
    131606, 65578, 67592, 66071, 66326, 65579, 67848, 131863, 65580, 66569, 131347, 65570,
    66825, 65815, 66067, 65574, 67081, 65816, 66323, 65575, 67337, 131607, 65579, 67593,
    66072, 66327, 65580, 67849, 131864, 65581,
};
__device__ const uint16_t kKetOff_fdps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_fdps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_fdps[60] = {
    0.14907119849998599, 0.2581988897471611, 0.2581988897471611, 0.14907119849998599,
    0.2581988897471611, 0.14907119849998599, 0.3333333333333334, 0.5773502691896258,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 0.3333333333333334,
    0.3333333333333334, 0.5773502691896258, 0.5773502691896258, 0.3333333333333334,
    0.5773502691896258, 0.3333333333333334, 0.3333333333333334, 0.5773502691896258,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 0.3333333333333334,
    0.3333333333333334, 0.5773502691896258, 0.5773502691896258, 0.3333333333333334,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 1.0,
    1.0, 0.5773502691896258, 1.0, 0.5773502691896258,
    0.14907119849998599, 0.2581988897471611, 0.2581988897471611, 0.14907119849998599,
    0.2581988897471611, 0.14907119849998599, 0.3333333333333334, 0.5773502691896258,
    0.5773502691896258, 0.3333333333333334, 0.5773502691896258, 0.3333333333333334,
    0.3333333333333334, 0.5773502691896258, 0.5773502691896258, 0.3333333333333334,
    0.5773502691896258, 0.3333333333333334, 0.14907119849998599, 0.2581988897471611,
    0.2581988897471611, 0.14907119849998599, 0.2581988897471611, 0.14907119849998599,
};
__device__ const double kNormCD_fdps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fdps() {
    return RysClassTabs{kBlk_fdps, kBraOff_fdps, kBraTerm_fdps, kKetOff_fdps, kKetTerm_fdps,
                        kNormAB_fdps, kNormCD_fdps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fdps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fdps, MIXED>(Q, R, tabs_fdps());
}

static void rys_prepare_fdps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fdps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 37504);
        cudaFuncSetAttribute(rys_queue_fdps<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 37504);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fdps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fdps();
    constexpr int ng = 128 / C_fdps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fdps<1><<<grid, 128, 37504, s>>>(Q, R);
    else rys_queue_fdps<0><<<grid, 128, 37504, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fdps(int mixed) {
    rys_prepare_fdps();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fdps<1>, 128, 37504);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fdps<0>, 128, 37504);
    return n;
}

}  // namespace molints

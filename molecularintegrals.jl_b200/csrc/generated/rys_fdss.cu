// Generated by gen_rys.py -- Rys class (fd|ss).  Do not edit.
// roots 3, block 46 x 1, outputs 60 x 1, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 2 accumulators per thread, 18560 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fdss {
    static constexpr int LA = 3, LB = 2, LC = 0, LD = 0;
    static constexpr int E = 5, F = 0, NR = 3;
    static constexpr int NA = 46, NC = 1, NBLK = 46;
    static constexpr int NB = 6, ND = 1;
    static constexpr int NAB = 60, NCD = 1;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 2;
    static constexpr int S = 6;
    static constexpr int SMEM_GROUP = 580;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fdss[46] = {
    3, 258, 65538, 513, 131073, 65793, 768, 66048, 131328, 196608, 4, 259,
    65539, 514, 65794, 131074, 769, 66049, 131329, 196609, 1024, 66304, 131584, 196864,
    262144, 5, 260, 65540, 515, 65795, 131075, 770, 66050, 131330, 196610, 1025,
    66305, 131585, 196865, 262145, 1280, 66560, 131840, 197120, 262400, 327680,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fdss[61] = {
    0, 3, 7, 11, 14, 18, 21, 24, 28, 32, 35, 39,
    42, 45, 49, 53, 56, 60, 63, 66, 70, 74, 77, 81,
    84, 87, 91, 95, 98, 102, 105, 108, 112, 116, 119, 123,
    126, 129, 133, 137, 140, 144, 147, 150, 154, 158, 161, 165,
    168, 171, 175, 179, 182, 186, 189, 192, 196, 200, 203, 207,
    210,
};
__device__ const uint32_t kBraTerm_fdss[210] = {
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
__device__ const uint16_t kKetOff_fdss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_fdss[1] = {
    65536,
};
__device__ const double kNormAB_fdss[60] = {
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
__device__ const double kNormCD_fdss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fdss() {
    return RysClassTabs{kBlk_fdss, kBraOff_fdss, kBraTerm_fdss, kKetOff_fdss, kKetTerm_fdss,
                        kNormAB_fdss, kNormCD_fdss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fdss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fdss, MIXED>(Q, R, tabs_fdss());
}

static void rys_prepare_fdss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fdss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 18560);
        cudaFuncSetAttribute(rys_queue_fdss<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 18560);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fdss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fdss();
    constexpr int ng = 128 / C_fdss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fdss<1><<<grid, 128, 18560, s>>>(Q, R);
    else rys_queue_fdss<0><<<grid, 128, 18560, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fdss(int mixed) {
    rys_prepare_fdss();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fdss<1>, 128, 18560);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fdss<0>, 128, 18560);
    return n;
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (dd|ss).  Do not edit.
// roots 3, block 31 x 1, outputs 36 x 1, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 1 accumulators per thread, 15680 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_ddss {
    static constexpr int LA = 2, LB = 2, LC = 0, LD = 0;
    static constexpr int E = 4, F = 0, NR = 3;
    static constexpr int NA = 31, NC = 1, NBLK = 31;
    static constexpr int NB = 6, ND = 1;
    static constexpr int NAB = 36, NCD = 1;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 1;
    static constexpr int S = 5;
    static constexpr int SMEM_GROUP = 490;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_ddss[31] = {
    2, 257, 65537, 512, 65792, 131072, 3, 258, 65538, 513, 131073, 65793,
    768, 66048, 131328, 196608, 4, 259, 65539, 514, 65794, 131074, 769, 66049,
    131329, 196609, 1024, 66304, 131584, 196864, 262144,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_ddss[37] = {
    0, 3, 7, 11, 14, 18, 21, 24, 28, 32, 35, 39,
    42, 45, 49, 53, 56, 60, 63, 66, 70, 74, 77, 81,
    84, 87, 91, 95, 98, 102, 105, 108, 112, 116, 119, 123,
    126,
};
__device__ const uint32_t kBraTerm_ddss[126] = {
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
__device__ const uint16_t kKetOff_ddss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_ddss[1] = {
    65536,
};
__device__ const double kNormAB_ddss[36] = {
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
__device__ const double kNormCD_ddss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_ddss() {
    return RysClassTabs{kBlk_ddss, kBraOff_ddss, kBraTerm_ddss, kKetOff_ddss, kKetTerm_ddss,
                        kNormAB_ddss, kNormCD_ddss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_ddss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_ddss, MIXED>(Q, R, tabs_ddss());
}

static void rys_prepare_ddss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_ddss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 15680);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_ddss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_ddss();
    constexpr int ng = 128 / C_ddss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_ddss<0><<<grid, 128, 15680, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_ddss(int mixed) {
    rys_prepare_ddss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ddss<0>, 128, 15680);
    return n;
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (dd|ds).  Do not edit.
// roots 4, block 31 x 6, outputs 36 x 6, group 64 threads,
// 16 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 46720 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_ddds {
    static constexpr int LA = 2, LB = 2, LC = 2, LD = 0;
    static constexpr int E = 4, F = 2, NR = 4;
    static constexpr int NA = 31, NC = 6, NBLK = 186;
    static constexpr int NB = 6, ND = 1;
    static constexpr int NAB = 36, NCD = 6;
    static constexpr int G = 64, NPB = 16, NSLOT = 1, ACC = 3;
    static constexpr int S = 15;
    static constexpr int SMEM_GROUP = 2920;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_ddds[186] = {
    8, 263, 65543, 518, 65798, 131078, 773, 1028, 66308, 1283, 66563, 131843,
    196613, 196868, 262148, 197123, 262403, 327683, 1538, 1793, 67073, 2048, 67328, 132608,
    197378, 197633, 262913, 197888, 263168, 328448, 393218, 393473, 458753, 393728, 459008, 524288,
    11, 266, 65546, 521, 65801, 131081, 776, 1031, 66311, 1286, 66566, 131846,
    196616, 196871, 262151, 197126, 262406, 327686, 1541, 1796, 67076, 2051, 67331, 132611,
    393221, 393476, 458756, 393731, 459011, 524291, 197381, 197636, 262916, 197891, 263171, 328451,
    2306, 2561, 67841, 2816, 68096, 133376, 198146, 198401, 263681, 198656, 263936, 329216,
    393986, 394241, 459521, 394496, 459776, 525056, 589826, 590081, 655361, 590336, 655616, 720896,
    14, 269, 65549, 524, 65804, 131084, 779, 1034, 66314, 1289, 66569, 131849,
    196619, 196874, 262154, 197129, 262409, 327689, 1544, 1799, 67079, 2054, 67334, 132614,
    197384, 197639, 262919, 197894, 263174, 328454, 393224, 393479, 458759, 393734, 459014, 524294,
    2309, 2564, 67844, 2819, 68099, 133379, 198149, 198404, 263684, 198659, 263939, 329219,
    393989, 394244, 459524, 394499, 459779, 525059, 589829, 590084, 655364, 590339, 655619, 720899,
    3074, 3329, 68609, 3584, 68864, 134144, 198914, 199169, 264449, 199424, 264704, 329984,
    394754, 395009, 460289, 395264, 460544, 525824, 590594, 590849, 656129, 591104, 656384, 721664,
    786434, 786689, 851969, 786944, 852224, 917504,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_ddds[37] = {
    0, 3, 7, 11, 14, 18, 21, 24, 28, 32, 35, 39,
    42, 45, 49, 53, 56, 60, 63, 66, 70, 74, 77, 81,
    84, 87, 91, 95, 98, 102, 105, 108, 112, 116, 119, 123,
    126,
};
__device__ const uint32_t kBraTerm_ddds[126] = {
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
__device__ const uint16_t kKetOff_ddds[7] = {
    0, 1, 2, 3, 4, 5, 6,
};
__device__ const uint32_t kKetTerm_ddds[6] = {
    65536, 65537, 65538, 65539, 65540, 65541,
};
__device__ const double kNormAB_ddds[36] = {
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
__device__ const double kNormCD_ddds[6] = {
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258,
};


__device__ __forceinline__ RysClassTabs tabs_ddds() {
    return RysClassTabs{kBlk_ddds, kBraOff_ddds, kBraTerm_ddds, kKetOff_ddds, kKetTerm_ddds,
                        kNormAB_ddds, kNormCD_ddds, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_ddds(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_ddds, MIXED>(Q, R, tabs_ddds());
}

static void rys_prepare_ddds() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_ddds<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 46720);
        cudaFuncSetAttribute(rys_queue_ddds<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 46720);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_ddds(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_ddds();
    constexpr int ng = 128 / C_ddds::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_ddds<1><<<grid, 128, 46720, s>>>(Q, R);
    else rys_queue_ddds<0><<<grid, 128, 46720, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_ddds(int mixed) {
    rys_prepare_ddds();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ddds<1>, 128, 46720);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ddds<0>, 128, 46720);
    return n;
}

}  // namespace molints

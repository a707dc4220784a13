// Generated by gen_rys.py -- Rys class (fp|ds).  Do not edit.
// roots 4, block 25 x 6, outputs 30 x 6, group 64 threads,
// 16 primitive quartets per batch, 1 slot(s), 3 accumulators per thread, 46720 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fpds {
    static constexpr int LA = 3, LB = 1, LC = 2, LD = 0;
    static constexpr int E = 4, F = 2, NR = 4;
    static constexpr int NA = 25, NC = 6, NBLK = 150;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 30, NCD = 6;
    static constexpr int G = 64, NPB = 16, NSLOT = 1, ACC = 3;
    static constexpr int S = 15;
    static constexpr int SMEM_GROUP = 2920;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fpds[150] = {
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
__device__ const uint16_t kBraOff_fpds[31] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36, 38, 40, 42, 44, 46,
    48, 50, 52, 54, 56, 58, 60,
};
__device__ const uint32_t kBraTerm_fpds[60] = {
    65792, 65546, 66048, 65547, 66304, 65548, 65793, 65547, 66049, 65549, 66305, 65550,
    65794, 65548, 66050, 65550, 66306, 65551, 65795, 65549, 66051, 65552, 66307, 65553,
    65796, 65551, 66052, 65554, 66308, 65555, 65797, 65550, 66053, 65553, 66309, 65554,
    65798, 65552, 66054, 65556, 66310, 65557, 65799, 65553, 66055, 65557, 66311, 65558,
    65800, 65554, 66056, 65558, 66312, 65559, 65801, 65555, 66057, 65559, 66313, 65560,
};
__device__ const uint16_t kKetOff_fpds[7] = {
    0, 1, 2, 3, 4, 5, 6,
};
__device__ const uint32_t kKetTerm_fpds[6] = {
    65536, 65537, 65538, 65539, 65540, 65541,
};
__device__ const double kNormAB_fpds[30] = {
    0.2581988897471611, 0.2581988897471611, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 0.2581988897471611, 0.2581988897471611,
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.2581988897471611,
    0.2581988897471611, 0.2581988897471611,
};
__device__ const double kNormCD_fpds[6] = {
    0.5773502691896258, 1.0, 1.0, 0.5773502691896258,
    1.0, 0.5773502691896258,
};


__device__ __forceinline__ RysClassTabs tabs_fpds() {
    return RysClassTabs{kBlk_fpds, kBraOff_fpds, kBraTerm_fpds, kKetOff_fpds, kKetTerm_fpds,
                        kNormAB_fpds, kNormCD_fpds, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fpds(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fpds, MIXED>(Q, R, tabs_fpds());
}

static void rys_prepare_fpds() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fpds<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 46720);
        cudaFuncSetAttribute(rys_queue_fpds<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 46720);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fpds(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fpds();
    constexpr int ng = 128 / C_fpds::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fpds<1><<<grid, 128, 46720, s>>>(Q, R);
    else rys_queue_fpds<0><<<grid, 128, 46720, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fpds(int mixed) {
    rys_prepare_fpds();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpds<1>, 128, 46720);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpds<0>, 128, 46720);
    return n;
}

}  // namespace molints

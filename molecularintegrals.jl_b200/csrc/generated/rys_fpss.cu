// Generated by gen_rys.py -- Rys class (fp|ss).  Do not edit.
// roots 3, block 25 x 1, outputs 30 x 1, group 32 threads,
// 10 primitive quartets per batch, 1 slot(s), 1 accumulators per thread, 15680 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fpss {
    static constexpr int LA = 3, LB = 1, LC = 0, LD = 0;
    static constexpr int E = 4, F = 0, NR = 3;
    static constexpr int NA = 25, NC = 1, NBLK = 25;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 30, NCD = 1;
    static constexpr int G = 32, NPB = 10, NSLOT = 1, ACC = 1;
    static constexpr int S = 5;
    static constexpr int SMEM_GROUP = 490;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fpss[25] = {
    3, 258, 65538, 513, 131073, 65793, 768, 66048, 131328, 196608, 4, 259,
    65539, 514, 65794, 131074, 769, 66049, 131329, 196609, 1024, 66304, 131584, 196864,
    262144,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fpss[31] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36, 38, 40, 42, 44, 46,
    48, 50, 52, 54, 56, 58, 60,
};
__device__ const uint32_t kBraTerm_fpss[60] = {
    65792, 65546, 66048, 65547, 66304, 65548, 65793, 65547, 66049, 65549, 66305, 65550,
    65794, 65548, 66050, 65550, 66306, 65551, 65795, 65549, 66051, 65552, 66307, 65553,
    65796, 65551, 66052, 65554, 66308, 65555, 65797, 65550, 66053, 65553, 66309, 65554,
    65798, 65552, 66054, 65556, 66310, 65557, 65799, 65553, 66055, 65557, 66311, 65558,
    65800, 65554, 66056, 65558, 66312, 65559, 65801, 65555, 66057, 65559, 66313, 65560,
};
__device__ const uint16_t kKetOff_fpss[2] = {
    0, 1,
};
__device__ const uint32_t kKetTerm_fpss[1] = {
    65536,
};
__device__ const double kNormAB_fpss[30] = {
    0.2581988897471611, 0.2581988897471611, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 0.2581988897471611, 0.2581988897471611,
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.2581988897471611,
    0.2581988897471611, 0.2581988897471611,
};
__device__ const double kNormCD_fpss[1] = {
    1.0,
};


__device__ __forceinline__ RysClassTabs tabs_fpss() {
    return RysClassTabs{kBlk_fpss, kBraOff_fpss, kBraTerm_fpss, kKetOff_fpss, kKetTerm_fpss,
                        kNormAB_fpss, kNormCD_fpss, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fpss(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fpss, MIXED>(Q, R, tabs_fpss());
}

static void rys_prepare_fpss() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fpss<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 15680);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fpss(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fpss();
    constexpr int ng = 128 / C_fpss::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_fpss<0><<<grid, 128, 15680, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fpss(int mixed) {
    rys_prepare_fpss();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpss<0>, 128, 15680);
    return n;
}

}  // namespace molints

// Generated by gen_rys.py -- Rys class (pp|ps).  Do not edit.
// roots 2, block 9 x 3, outputs 9 x 3, group 32 threads,
// 16 primitive quartets per batch, 1 slot(s), 1 accumulators per thread, 19712 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_ppps {
    static constexpr int LA = 1, LB = 1, LC = 1, LD = 0;
    static constexpr int E = 2, F = 1, NR = 2;
    static constexpr int NA = 9, NC = 3, NBLK = 27;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 9, NCD = 3;
    static constexpr int G = 32, NPB = 16, NSLOT = 1, ACC = 1;
    static constexpr int S = 6;
    static constexpr int SMEM_GROUP = 616;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_ppps[27] = {
    3, 258, 65538, 513, 768, 66048, 131073, 131328, 196608, 5, 260, 65540,
    515, 770, 66050, 131075, 131330, 196610, 1025, 1280, 66560, 131585, 131840, 197120,
    262145, 262400, 327680,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_ppps[10] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18,
};
__device__ const uint32_t kBraTerm_ppps[18] = {
    65792, 65539, 66048, 65540, 66304, 65541, 65793, 65540, 66049, 65542, 66305, 65543,
    65794, 65541, 66050, 65543, 66306, 65544,
};
__device__ const uint16_t kKetOff_ppps[4] = {
    0, 1, 2, 3,
};
__device__ const uint32_t kKetTerm_ppps[3] = {
    65536, 65537, 65538,
};
__device__ const double kNormAB_ppps[9] = {
    1.0, 1.0, 1.0, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0,
};
__device__ const double kNormCD_ppps[3] = {
    1.0, 1.0, 1.0,
};


__device__ __forceinline__ RysClassTabs tabs_ppps() {
    return RysClassTabs{kBlk_ppps, kBraOff_ppps, kBraTerm_ppps, kKetOff_ppps, kKetTerm_ppps,
                        kNormAB_ppps, kNormCD_ppps, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_ppps(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_ppps, MIXED>(Q, R, tabs_ppps());
}

static void rys_prepare_ppps() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_ppps<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 19712);


        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_ppps(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_ppps();
    constexpr int ng = 128 / C_ppps::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    (void)mixed;  // no FP32 variant for this class
    rys_queue_ppps<0><<<grid, 128, 19712, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_ppps(int mixed) {
    rys_prepare_ppps();
    int n = 0;
    (void)mixed;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_ppps<0>, 128, 19712);
    return n;
}

}  // namespace molints

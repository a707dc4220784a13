// Generated by gen_rys.py -- Rys class (fp|fs).  Do not edit.
// roots 4, block 25 x 10, outputs 30 x 10, group 64 threads,
// 16 primitive quartets per batch, 1 slot(s), 4 accumulators per thread, 62080 B shared per block.
#include "../rys_common.cuh"

namespace molints {

struct C_fpfs {
    static constexpr int LA = 3, LB = 1, LC = 3, LD = 0;
    static constexpr int E = 4, F = 3, NR = 4;
    static constexpr int NA = 25, NC = 10, NBLK = 250;
    static constexpr int NB = 3, ND = 1;
    static constexpr int NAB = 30, NCD = 10;
    static constexpr int G = 64, NPB = 16, NSLOT = 1, ACC = 4;
    static constexpr int S = 20;
    static constexpr int SMEM_GROUP = 3880;
    static constexpr bool COL = false;
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *, const T *, const T *, A *) {}
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_fpfs[250] = {
    15, 270, 65550, 525, 131085, 65805, 780, 66060, 131340, 196620, 1035, 1290,
    66570, 1545, 132105, 66825, 1800, 67080, 132360, 197640, 262155, 262410, 327690, 262665,
    393225, 327945, 262920, 328200, 393480, 458760, 2055, 2310, 67590, 2565, 133125, 67845,
    2820, 68100, 133380, 198660, 524295, 524550, 589830, 524805, 655365, 590085, 525060, 590340,
    655620, 720900, 263175, 263430, 328710, 263685, 394245, 328965, 263940, 329220, 394500, 459780,
    3075, 3330, 68610, 3585, 134145, 68865, 3840, 69120, 134400, 199680, 264195, 264450,
    329730, 264705, 395265, 329985, 264960, 330240, 395520, 460800, 525315, 525570, 590850, 525825,
    656385, 591105, 526080, 591360, 656640, 721920, 786435, 786690, 851970, 786945, 917505, 852225,
    787200, 852480, 917760, 983040, 19, 274, 65554, 529, 131089, 65809, 784, 66064,
    131344, 196624, 1039, 1294, 66574, 1549, 132109, 66829, 1804, 67084, 132364, 197644,
    262159, 262414, 327694, 262669, 393229, 327949, 262924, 328204, 393484, 458764, 2059, 2314,
    67594, 2569, 133129, 67849, 2824, 68104, 133384, 198664, 263179, 263434, 328714, 263689,
    394249, 328969, 263944, 329224, 394504, 459784, 524299, 524554, 589834, 524809, 655369, 590089,
    525064, 590344, 655624, 720904, 3079, 3334, 68614, 3589, 134149, 68869, 3844, 69124,
    134404, 199684, 264199, 264454, 329734, 264709, 395269, 329989, 264964, 330244, 395524, 460804,
    525319, 525574, 590854, 525829, 656389, 591109, 526084, 591364, 656644, 721924, 786439, 786694,
    851974, 786949, 917509, 852229, 787204, 852484, 917764, 983044, 4099, 4354, 69634, 4609,
    135169, 69889, 4864, 70144, 135424, 200704, 265219, 265474, 330754, 265729, 396289, 331009,
    265984, 331264, 396544, 461824, 526339, 526594, 591874, 526849, 657409, 592129, 527104, 592384,
    657664, 722944, 787459, 787714, 852994, 787969, 918529, 853249, 788224, 853504, 918784, 984064,
    1048579, 1048834, 1114114, 1049089, 1179649, 1114369, 1049344, 1114624, 1179904, 1245184,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_fpfs[31] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36, 38, 40, 42, 44, 46,
    48, 50, 52, 54, 56, 58, 60,
};
__device__ const uint32_t kBraTerm_fpfs[60] = {
    65792, 65546, 66048, 65547, 66304, 65548, 65793, 65547, 66049, 65549, 66305, 65550,
    65794, 65548, 66050, 65550, 66306, 65551, 65795, 65549, 66051, 65552, 66307, 65553,
    65796, 65551, 66052, 65554, 66308, 65555, 65797, 65550, 66053, 65553, 66309, 65554,
    65798, 65552, 66054, 65556, 66310, 65557, 65799, 65553, 66055, 65557, 66311, 65558,
    65800, 65554, 66056, 65558, 66312, 65559, 65801, 65555, 66057, 65559, 66313, 65560,
};
__device__ const uint16_t kKetOff_fpfs[11] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10,
};
__device__ const uint32_t kKetTerm_fpfs[10] = {
    65536, 65537, 65538, 65539, 65540, 65541, 65542, 65543, 65544, 65545,
};
__device__ const double kNormAB_fpfs[30] = {
    0.2581988897471611, 0.2581988897471611, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 0.2581988897471611, 0.2581988897471611,
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 0.2581988897471611,
    0.2581988897471611, 0.2581988897471611,
};
__device__ const double kNormCD_fpfs[10] = {
    0.2581988897471611, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    0.5773502691896258, 1.0, 0.2581988897471611, 0.5773502691896258,
    0.5773502691896258, 0.2581988897471611,
};


__device__ __forceinline__ RysClassTabs tabs_fpfs() {
    return RysClassTabs{kBlk_fpfs, kBraOff_fpfs, kBraTerm_fpfs, kKetOff_fpfs, kKetTerm_fpfs,
                        kNormAB_fpfs, kNormCD_fpfs, nullptr};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_fpfs(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_fpfs, MIXED>(Q, R, tabs_fpfs());
}

static void rys_prepare_fpfs() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_fpfs<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 62080);
        cudaFuncSetAttribute(rys_queue_fpfs<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 62080);

        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_fpfs(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_fpfs();
    constexpr int ng = 128 / C_fpfs::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_fpfs<1><<<grid, 128, 62080, s>>>(Q, R);
    else rys_queue_fpfs<0><<<grid, 128, 62080, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_fpfs(int mixed) {
    rys_prepare_fpfs();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpfs<1>, 128, 62080);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_fpfs<0>, 128, 62080);
    return n;
}

}  // namespace molints

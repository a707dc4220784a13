// Generated by gen_rys.py -- Rys class (dp|dp).  Do not edit.
// roots 4, block 16 x 16, outputs 18 x 18, group 32 threads,
// 8 primitive quartets per batch, 1 slot(s), 1 accumulators per thread, 50432 B shared per block, column mode.
#include "../rys_common.cuh"

namespace molints {

struct C_dpdp {
    static constexpr int LA = 2, LB = 1, LC = 2, LD = 1;
    static constexpr int E = 3, F = 3, NR = 4;
    static constexpr int NA = 16, NC = 16, NBLK = 256;
    static constexpr int NB = 3, ND = 3;
    static constexpr int NAB = 18, NCD = 18;
    static constexpr int G = 32, NPB = 8, NSLOT = 1, ACC = 1;
    static constexpr int S = 16;
    static constexpr int SMEM_GROUP = 1576;
    static constexpr bool COL = true;
    // stage 2, column mode: acc[row] += x[ax] y[ay] z[az] for the column's table columns
    template <typename T, typename A>
    __device__ __forceinline__ static void col_update(const T *x, const T *y, const T *z, A *acc) {
        acc[0] = fma(x[2] * y[0], z[0], acc[0]);
        acc[1] = fma(x[1] * y[1], z[0], acc[1]);
        acc[2] = fma(x[1] * y[0], z[1], acc[2]);
        acc[3] = fma(x[0] * y[2], z[0], acc[3]);
        acc[4] = fma(x[0] * y[1], z[1], acc[4]);
        acc[5] = fma(x[0] * y[0], z[2], acc[5]);
        acc[6] = fma(x[3] * y[0], z[0], acc[6]);
        acc[7] = fma(x[2] * y[1], z[0], acc[7]);
        acc[8] = fma(x[2] * y[0], z[1], acc[8]);
        acc[9] = fma(x[1] * y[2], z[0], acc[9]);
        acc[10] = fma(x[1] * y[0], z[2], acc[10]);
        acc[11] = fma(x[1] * y[1], z[1], acc[11]);
        acc[12] = fma(x[0] * y[3], z[0], acc[12]);
        acc[13] = fma(x[0] * y[2], z[1], acc[13]);
        acc[14] = fma(x[0] * y[1], z[2], acc[14]);
        acc[15] = fma(x[0] * y[0], z[3], acc[15]);
    }
    static constexpr int NCOLS = 16;
};

// block entry (row, col) -> 2-D table offsets x | y << 8 | z << 16
__device__ const uint32_t kBlk_dpdp[256] = {
    10, 265, 65545, 520, 65800, 131080, 11, 266, 65546, 521, 131081, 65801,
    776, 66056, 131336, 196616, 1030, 1285, 66565, 1540, 66820, 132100, 1031, 1286,
    66566, 1541, 132101, 66821, 1796, 67076, 132356, 197636, 262150, 262405, 327685, 262660,
    327940, 393220, 262151, 262406, 327686, 262661, 393221, 327941, 262916, 328196, 393476, 458756,
    2050, 2305, 67585, 2560, 67840, 133120, 2051, 2306, 67586, 2561, 133121, 67841,
    2816, 68096, 133376, 198656, 263170, 263425, 328705, 263680, 328960, 394240, 263171, 263426,
    328706, 263681, 394241, 328961, 263936, 329216, 394496, 459776, 524290, 524545, 589825, 524800,
    590080, 655360, 524291, 524546, 589826, 524801, 655361, 590081, 525056, 590336, 655616, 720896,
    14, 269, 65549, 524, 65804, 131084, 15, 270, 65550, 525, 131085, 65805,
    780, 66060, 131340, 196620, 1034, 1289, 66569, 1544, 66824, 132104, 1035, 1290,
    66570, 1545, 132105, 66825, 1800, 67080, 132360, 197640, 262154, 262409, 327689, 262664,
    327944, 393224, 262155, 262410, 327690, 262665, 393225, 327945, 262920, 328200, 393480, 458760,
    2054, 2309, 67589, 2564, 67844, 133124, 2055, 2310, 67590, 2565, 133125, 67845,
    2820, 68100, 133380, 198660, 524294, 524549, 589829, 524804, 590084, 655364, 524295, 524550,
    589830, 524805, 655365, 590085, 525060, 590340, 655620, 720900, 263174, 263429, 328709, 263684,
    328964, 394244, 263175, 263430, 328710, 263685, 394245, 328965, 263940, 329220, 394500, 459780,
    3074, 3329, 68609, 3584, 68864, 134144, 3075, 3330, 68610, 3585, 134145, 68865,
    3840, 69120, 134400, 199680, 264194, 264449, 329729, 264704, 329984, 395264, 264195, 264450,
    329730, 264705, 395265, 329985, 264960, 330240, 395520, 460800, 525314, 525569, 590849, 525824,
    591104, 656384, 525315, 525570, 590850, 525825, 656385, 591105, 526080, 591360, 656640, 721920,
    786434, 786689, 851969, 786944, 852224, 917504, 786435, 786690, 851970, 786945, 917505, 852225,
    787200, 852480, 917760, 983040,
};
// HRR terms: block index | monomial << 8 | binomial << 16, per output pair
__device__ const uint16_t kBraOff_dpdp[19] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36,
};
__device__ const uint32_t kBraTerm_dpdp[36] = {
    65792, 65542, 66048, 65543, 66304, 65544, 65793, 65543, 66049, 65545, 66305, 65547,
    65794, 65544, 66050, 65547, 66306, 65546, 65795, 65545, 66051, 65548, 66307, 65549,
    65796, 65547, 66052, 65549, 66308, 65550, 65797, 65546, 66053, 65550, 66309, 65551,
};
__device__ const uint16_t kKetOff_dpdp[19] = {
    0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22,
    24, 26, 28, 30, 32, 34, 36,
};
__device__ const uint32_t kKetTerm_dpdp[36] = {
    65792, 65542, 66048, 65543, 66304, 65544, 65793, 65543, 66049, 65545, 66305, 65547,
    65794, 65544, 66050, 65547, 66306, 65546, 65795, 65545, 66051, 65548, 66307, 65549,
    65796, 65547, 66052, 65549, 66308, 65550, 65797, 65546, 66053, 65550, 66309, 65551,
};
__device__ const double kNormAB_dpdp[18] = {
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    1.0, 1.0, 1.0, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258,
};
__device__ const double kNormCD_dpdp[18] = {
    0.5773502691896258, 0.5773502691896258, 0.5773502691896258, 1.0,
    1.0, 1.0, 1.0, 1.0,
    1.0, 0.5773502691896258, 0.5773502691896258, 0.5773502691896258,
    1.0, 1.0, 1.0, 0.5773502691896258,
    0.5773502691896258, 0.5773502691896258,
};


// column components cx | cy << 4 | cz << 8
__device__ const uint16_t kCol_dpdp[16] = { 2, 17, 257, 32, 272, 512, 3, 18, 258, 33, 513, 273, 48, 288, 528, 768 };

__device__ __forceinline__ RysClassTabs tabs_dpdp() {
    return RysClassTabs{kBlk_dpdp, kBraOff_dpdp, kBraTerm_dpdp, kKetOff_dpdp, kKetTerm_dpdp,
                        kNormAB_dpdp, kNormCD_dpdp, kCol_dpdp};
}

template <int MIXED>
__global__ void __launch_bounds__(128) rys_queue_dpdp(const EriQueue Q, const RysTab R) {
    rys_queue_body<C_dpdp, MIXED>(Q, R, tabs_dpdp());
}

__global__ void __launch_bounds__(128) rys_bound_kernel_dpdp(PairTab P, RysTab R, int p0, int np,
                                                              double2 *pbound, double *qout, int full) {
    rys_bound_body<C_dpdp>(P, R, tabs_dpdp(), p0, np, pbound, qout, full);
}

static void rys_prepare_dpdp() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(rys_queue_dpdp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 50432);
        cudaFuncSetAttribute(rys_queue_dpdp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 50432);
        cudaFuncSetAttribute(rys_bound_kernel_dpdp, cudaFuncAttributeMaxDynamicSharedMemorySize, 50432);
        done[dev] = true;
    }
}

// grid_max: resident blocks on the device; the grid is cut to the chunks' groups.
void launch_rys_dpdp(const EriQueue &Q, const RysTab &R, int mixed, int grid_max, cudaStream_t s) {
    if (Q.nchunks <= 0 || grid_max <= 0) return;
    rys_prepare_dpdp();
    constexpr int ng = 128 / C_dpdp::G;
    const int grid = (int)std::min<long long>(grid_max, ((long long)Q.nchunks + ng - 1) / ng);
    if (mixed) rys_queue_dpdp<1><<<grid, 128, 50432, s>>>(Q, R);
    else rys_queue_dpdp<0><<<grid, 128, 50432, s>>>(Q, R);
}

// Resident blocks of 128 threads per SM for the queue kernel (sizes the persistent grid).
int occupancy_rys_dpdp(int mixed) {
    rys_prepare_dpdp();
    int n = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dpdp<1>, 128, 50432);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_queue_dpdp<0>, 128, 50432);
    return n;
}

void launch_rys_bound_dpdp(const PairTab &P, const RysTab &R, int p0, int np, double2 *pbound,
                            double *qout, int full, cudaStream_t s) {
    if (np <= 0) return;
    rys_prepare_dpdp();
    constexpr int ng = 128 / C_dpdp::G;
    rys_bound_kernel_dpdp<<<(np + ng - 1) / ng, 128, 50432, s>>>(P, R, p0, np, pbound, qout, full);
}

}  // namespace molints

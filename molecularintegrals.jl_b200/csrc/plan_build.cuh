// Device half of plan creation: primitive-pair screening, the pair re-sort by kept count, the
// final pair tables and the per-class-pair work queues, built from the stage-1 pair tables and
// the bound pass's per-primitive-pair bounds without a round trip through the host.
//
// The reference builds its work list on the host, one shell quartet at a time
// (eri_fetcher, src/Basis.jl:201-262); here the list is chunks of one bra pair and a run of
// ket pairs, emitted in parallel (one thread per bra pair of each class pair) and ordered by
// class pair and decreasing cost with a stable radix sort.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "eri_dispatch.h"

namespace molints {

constexpr int kNumClassPairs = kNumPairClasses * (kNumPairClasses + 1) / 2;  // (x, y <= x)
constexpr int kCostBuckets = 64;

// Lane split of an HGP work-queue chunk whose bra pair has nb and ket pair nk kept primitive
// pairs, in a class whose primitive quartet costs `cost` (kEriPrimCost; (ss|ss) ~ 1).  A lane
// evaluates its quartet's primitive quartets one after another; a heavy quartet (six-primitive
// core shells: 36 x 36) on one lane outlasts the rest of the launch.  Its primitive quartets
// are therefore split over S = 2^lg lanes (S <= 32) -- ket primitives over Sj = 2^lgj of them
// first (Sj <= nk), then bra primitives over S / Sj -- until a lane's share costs at most
// lane_cost.  Returns lg | lgj << 4, the chunk's split field.  A pure function of
// (nb, nk, class, lane_cost): the same quartet gets the same split, and so the same rounding,
// in every plan of a context.
__host__ __device__ inline int hgp_split(int nb, int nk, double cost, double lane_cost) {
    int lg = 0, lgj = 0;
    while (lg < 5) {
        const int gi = lg - lgj;
        const double share = cost * (double)((nk + (1 << lgj) - 1) >> lgj) * (double)((nb + (1 << gi) - 1) >> gi);
        if (share <= lane_cost) break;
        if ((nk >> lgj) >= 2) ++lgj;
        else if ((nb >> gi) < 2) break;
        ++lg;
    }
    return lg | (lgj << 4);
}

// Cost bucket of a chunk, heaviest first: 0 for the largest binary exponents.  An O(1) key
// whose order is all the load balance needs.
__host__ __device__ inline int cost_bucket(double c) {
    if (!(c > 0.0)) return kCostBuckets - 1 - 9;  // e2 = 1, as for a cost in [1, 2)
    int e2 = 0;
    frexp(c, &e2);  // c = f 2^e2, f in [0.5, 1)
    const int b = kCostBuckets - 1 - (e2 + 8);
    return b < 0 ? 0 : (b > kCostBuckets - 1 ? kCostBuckets - 1 : b);
}

// Bucket of a pair's Schwarz factor Qabs for the screening order: a factor of 256 in Qabs per
// bucket.  With Qabs = f 2^e (f in [0.5, 1), so Qabs < 2^e), the bucket is
// (e + kQabsBias) / 8 clamped to [1, 255], and 0 for Qabs = 0.  Plans that screen quartets
// order each (class, molecule) run of pairs by bucket, descending, so that a bra's unscreened
// kets come first; within a bucket the kept count descends, which keeps a chunk's lanes alike
// and its lane split constant.  Wider buckets leave more screened quartets inside the runs,
// narrower ones cut more chunks where the split changes (measured on B200 over the eight
// largest groups of the 256-molecule batch, MIXED: factors 4 / 16 / 256 / 65536 / 2^32 per
// bucket, 60.8 / 55.9 / 54.2 / 54.7 / 56.3 ms per execute).
constexpr int kQabsBias = 1280;
__host__ __device__ inline int qabs_bucket(double q) {
    if (!(q > 0.0)) return 0;
    int e2 = 0;
    frexp(q, &e2);
    const int b = (e2 + kQabsBias) >> 3;
    return b < 1 ? 1 : (b > 255 ? 255 : b);
}

// Upper bound of the Qabs values in a bucket (infinite for the top one).
__host__ __device__ inline double qabs_bucket_hi(int b) {
    if (b <= 0) return 0.0;
    if (b >= 255) return HUGE_VAL;
    return ldexp(1.0, 8 * b + 7 - kQabsBias);  // e <= 8b + 7 - kQabsBias
}

// Plans that screen quartets: the end of bra pb's ket run [kbeg, kend) after its last ket q
// with Qabs_pb Qabs_q >= cut (kbeg if there is none); bnd[k].x = Qabs of pair k.  The run is in
// Qabs-bucket order, descending, so the kets screened by their bucket's upper bound alone form a
// suffix, found by bisection; the last unscreened ket lies just before it.  The quartets past
// the end are screened: their zeros come from the gather or from the cleared output.
__host__ __device__ inline int unscreened_end(const double2 *bnd, double cut, int pb, int kbeg, int kend) {
    const double qp = bnd[pb].x;
    int lo = kbeg, hi = kend;  // first q with qabs_bucket_hi(q) * qp < cut, in [kbeg, kend]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (qabs_bucket_hi(qabs_bucket(bnd[mid].x)) * qp < cut) hi = mid; else lo = mid + 1;
    }
    int e = lo;
    while (e > kbeg && qp * bnd[e - 1].x < cut) --e;
    return e;
}

// What the queue kernels need per class pair (x, y <= x), in the host's class-pair order
// (x outer, y inner): a plain struct passed by value.
struct QueueSetup {
    int item_base[kNumClassPairs + 1];  // thread t of class pair ci: item_base[ci] <= t < [ci + 1]
    int cx[kNumClassPairs], cy[kNumClassPairs];
    int width[kNumClassPairs];          // ket pairs of an unsplit chunk
    int hgp[kNumClassPairs];            // HGP kernel (lane split) or Rys
    double pcost[kNumClassPairs];       // primitive-quartet cost of the HGP kernel
    double w[kNumClassPairs];           // cost weight 1 + (la + lb + lc + ld)^2
    int cls_start[kNumPairClasses + 1];
    int nmol;
    int widen;                          // HGP chunk widths are (32 >> lg) * widen
    double lane_cost;
    int sharded, shard_s0, shard_s1;    // shard plans: owned highest-shell range [s0, s1)
    int ps0[kNumPairClasses], ps1[kNumPairClasses];  // first pair of each class with ms >= s0 / s1
    int two_phase;
    // Quartet screening (Qabs_p Qabs_q < screen_cut written as 0): the pair runs are in
    // Qabs-bucket order (screen_sort) and each bra's ket run ends after its last unscreened
    // ket (screen_trunc); the zeros of the quartets no chunk holds come from the gather
    // (two-phase plans) or from clearing the output before the class kernels (direct plans).
    int screen_sort, screen_trunc;
    double screen_cut;
};

// Device arrays of one device plan build (all owned by the caller).
struct PlanBuildArgs {
    int npair;
    int nall;                      // stage-1 primitive pairs
    double prim_cutoff;
    int screen_sort;               // order runs by Qabs bucket (descending), then kept count
    // stage 1 (pair order by class, molecule[, ms], all-primitive count)
    const int2 *ab1;               // global shells (A, B)
    const int4 *info1;             // {first primitive pair, count, first function of A, of B}
    const int *src1;               // primitive pair -> (ia << 8) | ib
    const int4 *rec1;              // {molecule, reference pair index, class | swapped << 8, ms}
    const int *seg1;               // first stage-1 pair of the pair's (class, molecule[, ms]) run
    const double2 *pbound;         // per primitive pair: (b_k, w_k) of the bound pass
    const double *xyz;             // shell centres
    const int *sh_L;
    unsigned long long *qmax;      // per molecule, zeroed: max over pairs of sum b_k (bits)
    // re-sort scratch
    int *npp1;                     // kept count per stage-1 pair
    double2 *bnd1;                 // (Qabs, R) per stage-1 pair
    unsigned long long *key1, *key2;
    int *idx1, *idx2;              // idx2 = stage-1 position of final pair k
    long long *npp_prefix;         // npair + 1: kept primitive pairs of final pairs [0, k)
    int *npp;                      // npair + 1: kept count per final pair (last entry 0)
    int *ms;                       // highest shell index per final pair (shard plans)
    // final tables
    int2 *pair_ab;
    int4 *info;
    double2 *bnd;
    int *pp_src;
    double *pbk;
    int *g_pair;                   // two-phase: per molecule shell pair, or null
    const long long *g_mol;        // two-phase: per molecule {.., first pair entry, ..}
};

// Stage-1 primitive-pair list: pair k's K_A x K_B entries (ia << 8) | ib, A's primitive
// outer, at info1[k].x.
cudaError_t plan_stage1_src(int npair, const int2 *ab1, const int4 *info1, const int *sh_K, int *src1,
                            cudaStream_t s);

// Screening, re-sort and final pair tables.  temp: CUB scratch of at least
// plan_build_temp_bytes(npair) bytes.
cudaError_t plan_build_pairs(const PlanBuildArgs &A, void *temp, size_t temp_bytes, cudaStream_t s);
size_t plan_build_temp_bytes(int npair);

// Work queues, pass 1: chunks and cost per item (bra pair of a class pair), their prefix sum,
// and per class pair the first chunk and the total cost.  summary: kNumClassPairs + 1 chunk
// offsets (the last one the queue length), then kNumClassPairs costs, on the device.
struct QueueArgs {
    int n_items;
    const int *npp;                // per final pair
    const int *mol;                // per pair (stage-1 and final order agree on it)
    const int *cm_start;           // per (class, molecule): first pair; [cls * (nmol + 1) + m]
    const int *ms;                 // shard plans
    const long long *npp_prefix;
    const long long *region;       // two-phase: per (x, y, molecule) 4 fields, else null
    const double2 *bnd;            // per final pair (Qabs, R): the screening order's cut
    long long *cnt;                // n_items + 1
    double *cost;                  // n_items
    long long *off;                // n_items + 1
    long long *summary;            // kNumClassPairs + 1
    double *class_cost;            // kNumClassPairs
};
cudaError_t queue_count(const QueueSetup &S, const QueueArgs &A, void *temp, size_t temp_bytes,
                        cudaStream_t s);
size_t queue_count_temp_bytes(int n_items);

// Work queues, pass 2: emit every chunk at its item's offset, then order the queue by class
// pair and cost bucket (stable), writing chunks[] and, for two-phase plans, chunk_slot[].
struct QueueEmitArgs {
    int4 *raw;                     // nq
    unsigned short *key1, *key2;   // nq
    int *idx1, *idx2;              // nq
    long long *raw_slot;           // nq (two-phase) or null
    int4 *chunks;                  // nq
    long long *chunk_slot;         // nq (two-phase) or null
    long long nq;
};
cudaError_t queue_emit(const QueueSetup &S, const QueueArgs &A, const QueueEmitArgs &E, void *temp,
                       size_t temp_bytes, cudaStream_t s);
size_t queue_emit_temp_bytes(long long nq);

}  // namespace molints

// Device half of plan creation (plan_build.cuh): screening, the pair re-sort, the final pair
// tables and the work queues.
#include "plan_build.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace molints {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__global__ void pair_src_kernel(int npair, const int2 *__restrict__ ab1, const int4 *__restrict__ info1,
                                const int *__restrict__ sh_K, int *__restrict__ src1) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npair) return;
    const int4 in = info1[k];
    const int kb = sh_K[ab1[k].y];
    for (int x = 0, ia = 0, ib = 0; x < in.y; ++x) {
        src1[in.x + x] = (ia << 8) | ib;
        if (++ib == kb) { ib = 0; ++ia; }
    }
}

// max over a molecule's pairs of Qabs = sum_k b_k (every primitive pair), summed in list order
// as the screening needs it.  The sums are >= 0, so their bit patterns order like the values.
__global__ void pair_qmax_kernel(PlanBuildArgs A) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.npair) return;
    const int4 in = A.info1[k];
    double q = 0.0;
    for (int x = 0; x < in.y; ++x) q += A.pbound[in.x + x].x;
    atomicMax(&A.qmax[A.rec1[k].x], (unsigned long long)__double_as_longlong(q));
}

// Per stage-1 pair: primitive pairs kept (b_k * max Qabs of the molecule >= prim_cutoff; each
// dropped term of any integral is below prim_cutoff by the Schwarz inequality), the pair's
// bounds Qabs = sum of kept b_k and R = (1 + |AB|)^lb sum of kept w_k, and its sort key:
// (class, molecule[, ms]) run first, then kept count descending (plans that screen quartets:
// Qabs bucket descending, then kept count descending).
__global__ void pair_screen_kernel(PlanBuildArgs A) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.npair) return;
    const int4 in = A.info1[k];
    const int4 r = A.rec1[k];
    const double qm = __longlong_as_double((long long)A.qmax[r.x]);
    double qa = 0.0, wa = 0.0;
    int kept = 0;
    for (int x = 0; x < in.y; ++x) {
        const double2 b = A.pbound[in.x + x];
        if (A.prim_cutoff > 0.0 && b.x * qm < A.prim_cutoff) continue;
        ++kept;
        qa += b.x;
        wa += b.y;
    }
    const int2 ab = A.ab1[k];
    const double dx = A.xyz[3 * ab.x] - A.xyz[3 * ab.y], dy = A.xyz[3 * ab.x + 1] - A.xyz[3 * ab.y + 1],
                 dz = A.xyz[3 * ab.x + 2] - A.xyz[3 * ab.y + 2];
    const double dab1 = 1.0 + sqrt(dx * dx + dy * dy + dz * dz);
    double f = 1.0;
    for (int l = 0; l < A.sh_L[ab.y]; ++l) f *= dab1;
    A.npp1[k] = kept;
    A.bnd1[k] = make_double2(qa, wa * f);
    const unsigned long long within =
        A.screen_sort ? ((unsigned long long)(255 - qabs_bucket(qa)) << 12) | (unsigned long long)(0xFFF - min(kept, 0xFFF))
                      : (unsigned long long)(0xFFFFF - kept);
    A.key1[k] = ((unsigned long long)A.seg1[k] << 20) | within;
    A.idx1[k] = k;
}

__global__ void pair_npp_kernel(PlanBuildArgs A) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > A.npair) return;
    A.npp[k] = k < A.npair ? A.npp1[A.idx2[k]] : 0;
}

// Final pair k (the stage-1 pair idx2[k]): its tables, with the kept primitive pairs packed
// at npp_prefix[k], in stage-1 order.
__global__ void pair_tables_kernel(PlanBuildArgs A) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.npair) return;
    const int k1 = A.idx2[k];
    const int4 in = A.info1[k1];
    const int4 r = A.rec1[k1];
    const int off = (int)A.npp_prefix[k];
    const double qm = __longlong_as_double((long long)A.qmax[r.x]);
    int j = off;
    for (int x = 0; x < in.y; ++x) {
        const double2 b = A.pbound[in.x + x];
        if (A.prim_cutoff > 0.0 && b.x * qm < A.prim_cutoff) continue;
        A.pp_src[j] = A.src1[in.x + x];
        A.pbk[j] = b.x;
        ++j;
    }
    A.pair_ab[k] = A.ab1[k1];
    A.info[k] = make_int4(off, j - off, in.z, in.w);
    A.bnd[k] = A.bnd1[k1];
    A.ms[k] = r.w;
    if (A.g_pair) {
        // the gather's entry of the molecule's shell pair: list position, class, A == J
        A.g_pair[A.g_mol[4 * r.x + 1] + r.y] = (k << 5) | ((r.z & 255) << 1) | (r.z >> 8);
    }
}

// ---- work queues

// The chunks of one item: bra pair pb of class pair ci against its ket run, in ket order.
// Chunks hold one bra pair and up to `width` ket pairs of the same molecule.  HGP chunks whose
// quartets are split over lanes (hgp_split) hold (32 >> lg) * widen ket pairs and end where the
// split changes: the kets of a molecule's class run are in descending kept count, so the split
// only falls along the run and a chunk that starts unsplit stays unsplit (shard plans, ordered
// by highest shell first, and plans that screen quartets, ordered by Qabs bucket first, test
// every ket).
template <class Emit>
__device__ void walk_item(const QueueSetup &S, const QueueArgs &A, int ci, int pb, Emit &&emit) {
    const int x = S.cx[ci], y = S.cy[ci];
    const int m = A.mol[pb];
    const int k0 = A.cm_start[y * (S.nmol + 1) + m], k1 = A.cm_start[y * (S.nmol + 1) + m + 1];
    int kbeg = k0, kend = x == y ? pb + 1 : k1;
    if (S.sharded) {
        // quartet owner: the higher of the two pairs' highest shells
        const int mp = A.ms[pb];
        if (mp >= S.shard_s1) return;
        if (x == y) {
            if (mp < S.shard_s0) return;  // q <= pb in list order: the owner is mp
        } else if (mp >= S.shard_s0) {
            kend = S.ps1[y];
        } else {
            kbeg = S.ps0[y];
            kend = S.ps1[y];
        }
    }
    if (S.screen_trunc && kend > kbeg) kend = unscreened_end(A.bnd, S.screen_cut, pb, kbeg, kend);
    const int nb = A.npp[pb];
    const double wp = S.w[ci] * nb, pcost = S.pcost[ci];
    // this bra's remaining kets may still need a split (in Qabs order the kept counts do not
    // descend along the run: every chunk is tested)
    bool heavy = S.hgp[ci] != 0;
    for (int q0 = kbeg; q0 < kend;) {
        int n = min(S.width[ci], kend - q0), lg = 0;
        if (heavy) {
            lg = hgp_split(nb, A.npp[q0], pcost, S.lane_cost);
            n = min((32 >> (lg & 7)) * S.widen, kend - q0);
            if (lg || S.sharded || S.screen_sort)
                for (int k = 1; k < n; ++k)
                    if (hgp_split(nb, A.npp[q0 + k], pcost, S.lane_cost) != lg) { n = k; break; }
            heavy = lg != 0 || S.sharded || S.screen_sort;
        }
        const double cost = wp * (double)(A.npp_prefix[q0 + n] - A.npp_prefix[q0]);
        emit(q0, n, lg, m, cost);
        q0 += n;
    }
}

__device__ __forceinline__ int item_class_pair(const QueueSetup &S, int t) {
    int lo = 0, hi = kNumClassPairs;  // last ci with item_base[ci] <= t
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (S.item_base[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void queue_count_kernel(const QueueSetup S, QueueArgs A) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > A.n_items) return;
    if (t == A.n_items) { A.cnt[t] = 0; return; }
    const int ci = item_class_pair(S, t);
    const int pb = S.cls_start[S.cx[ci]] + (t - S.item_base[ci]);
    long long c = 0;
    double total = 0.0;
    walk_item(S, A, ci, pb, [&](int, int, int, int, double cost) { ++c; total += cost; });
    A.cnt[t] = c;
    A.cost[t] = total;
}

// Per class pair: its first chunk (and the queue length last) and its total cost, summed in
// item order by one block per class pair.
__global__ void queue_summary_kernel(const QueueSetup S, QueueArgs A) {
    const int ci = blockIdx.x;
    if (threadIdx.x == 0) {
        A.summary[ci] = A.off[S.item_base[ci]];
        if (ci == kNumClassPairs - 1) A.summary[kNumClassPairs] = A.off[A.n_items];
    }
    __shared__ double part[kThreads];
    double s = 0.0;
    for (int t = S.item_base[ci] + threadIdx.x; t < S.item_base[ci + 1]; t += blockDim.x) s += A.cost[t];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) A.class_cost[ci] = part[0];
}

__global__ void queue_emit_kernel(const QueueSetup S, QueueArgs A, QueueEmitArgs E) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.n_items) return;
    const int ci = item_class_pair(S, t);
    const int x = S.cx[ci], y = S.cy[ci];
    const int pb = S.cls_start[x] + (t - S.item_base[ci]);
    long long d = A.off[t];
    walk_item(S, A, ci, pb, [&](int q0, int n, int lg, int m, double cost) {
        E.raw[d] = make_int4(pb, q0, n | (lg << 16), m);
        E.key1[d] = (unsigned short)((ci << 6) | cost_bucket(cost));
        E.idx1[d] = (int)d;
        if (E.raw_slot) {
            // two-phase: the scratch slot of the chunk's first quartet in its (x, y, molecule)
            // region, bra-major (the triangle q <= p for equal classes)
            const long long *rg = &A.region[(((long long)x * kNumPairClasses + y) * S.nmol + m) * 4];
            const long long db = pb - rg[1], dk = q0 - rg[2];
            E.raw_slot[d] = x == y ? db * (db + 1) / 2 + dk : db * rg[3] + dk;
        }
        ++d;
    });
}

__global__ void queue_place_kernel(QueueEmitArgs E) {
    const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= E.nq) return;
    const int i = E.idx2[d];
    E.chunks[d] = E.raw[i];
    if (E.chunk_slot) E.chunk_slot[d] = E.raw_slot[i];
}

}  // namespace

cudaError_t plan_stage1_src(int npair, const int2 *ab1, const int4 *info1, const int *sh_K, int *src1,
                            cudaStream_t s) {
    if (npair <= 0) return cudaSuccess;
    pair_src_kernel<<<blocks_for(npair), kThreads, 0, s>>>(npair, ab1, info1, sh_K, src1);
    return cudaGetLastError();
}

size_t plan_build_temp_bytes(int npair) {
    size_t a = 0, b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                    (int *)nullptr, (int *)nullptr, npair, 0, 52);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (int *)nullptr, (long long *)nullptr, npair + 1);
    return a > b ? a : b;
}

cudaError_t plan_build_pairs(const PlanBuildArgs &A, void *temp, size_t temp_bytes, cudaStream_t s) {
    if (A.npair <= 0) return cudaSuccess;
    pair_qmax_kernel<<<blocks_for(A.npair), kThreads, 0, s>>>(A);
    pair_screen_kernel<<<blocks_for(A.npair), kThreads, 0, s>>>(A);
    size_t tb = temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, tb, A.key1, A.key2, A.idx1, A.idx2, A.npair, 0, 52, s);
    if (e != cudaSuccess) return e;
    pair_npp_kernel<<<blocks_for(A.npair + 1), kThreads, 0, s>>>(A);
    // kept primitive pairs before each final pair (their sum is below 2^31: stage-1 offsets
    // are int)
    tb = temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(temp, tb, A.npp, A.npp_prefix, A.npair + 1, s);
    if (e != cudaSuccess) return e;
    pair_tables_kernel<<<blocks_for(A.npair), kThreads, 0, s>>>(A);
    return cudaGetLastError();
}

size_t queue_count_temp_bytes(int n_items) {
    size_t a = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, a, (long long *)nullptr, (long long *)nullptr, n_items + 1);
    return a;
}

cudaError_t queue_count(const QueueSetup &S, const QueueArgs &A, void *temp, size_t temp_bytes,
                        cudaStream_t s) {
    queue_count_kernel<<<blocks_for(A.n_items + 1), kThreads, 0, s>>>(S, A);
    size_t tb = temp_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(temp, tb, A.cnt, A.off, A.n_items + 1, s);
    if (e != cudaSuccess) return e;
    queue_summary_kernel<<<kNumClassPairs, kThreads, 0, s>>>(S, A);
    return cudaGetLastError();
}

size_t queue_emit_temp_bytes(long long nq) {
    size_t a = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned short *)nullptr, (unsigned short *)nullptr,
                                    (int *)nullptr, (int *)nullptr, (int)nq, 0, 13);
    return a;
}

cudaError_t queue_emit(const QueueSetup &S, const QueueArgs &A, const QueueEmitArgs &E, void *temp,
                       size_t temp_bytes, cudaStream_t s) {
    if (E.nq <= 0) return cudaSuccess;
    if (A.n_items > 0) queue_emit_kernel<<<blocks_for(A.n_items), kThreads, 0, s>>>(S, A, E);
    size_t tb = temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, tb, E.key1, E.key2, E.idx1, E.idx2, (int)E.nq, 0, 13, s);
    if (e != cudaSuccess) return e;
    queue_place_kernel<<<blocks_for(E.nq), kThreads, 0, s>>>(E);
    return cudaGetLastError();
}

}  // namespace molints

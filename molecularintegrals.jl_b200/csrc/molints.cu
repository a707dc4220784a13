// molints.cu -- host side of libmolints_cuda.so: contexts, plans and the C ABI of
// include/molints.h, plus the device pair builder and the Boys-table kernels.
//
// Execution of a plan (all on the context's stream, no host synchronisation):
//   1. build_pairs_kernel: one thread per canonical shell pair writes its primitive-pair
//      records (zeta, P, P-A, exp(-ab/zeta |A-B|^2) prefactor) and A-B;
//   2. schwarz kernels, one per pair class: Q_p = sqrt(max |(ab|ab)|);
//   3. one generated kernel per class pair (bra class >= ket class) over all its unique
//      shell quartets, writing the packed iindex vector.
// The drivers this replaces are all_twoe_ints_chrr (src/HGP.jl:22-34) and all_twoe_ints
// (src/ERI.jl:104-112) of MolecularIntegrals.jl.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/molints.h"
#include "eri_common.cuh"
#include "class_table.h"
#include "eri_dispatch.h"
#include "plan_build.cuh"

using namespace molints;

struct molints_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t cap_stream = nullptr;  // CUDA-graph capture (the legacy stream cannot capture)
    std::vector<molints_plan *> plans;  // live plans, orphaned when the context goes first
    cudaStream_t stream = nullptr;
    int64_t budget = 0;        // bytes, 0 = unbounded
    int64_t held = 0;          // bytes currently allocated by this context and its plans
    // Stream-ordered pool for every device buffer of the context and its plans: freed blocks
    // stay cached (release threshold = max), so plan creation and destruction neither call
    // cudaMalloc/cudaFree nor synchronise the device.
    cudaMemPool_t pool = nullptr;
    double *boys_tab = nullptr;
    double *boys_scaled = nullptr;  // per-M tables F_{M+k}(T_n)/k!, k < 8, and e^-T_n
    double *out_cache = nullptr;  // device buffer for host-output calls
    int64_t out_cache_len = 0;
    // Two-phase output scratch, shared by the context's plans (it is needed only while an
    // execute runs): grown to the largest plan's need and kept.  scratch_gen counts the
    // reallocations (a captured graph holds the address); scratch_ev orders the executes that
    // use it, whatever stream each is launched on.
    double *scratch = nullptr;
    int64_t scratch_len = 0;
    int scratch_gen = 0;
    cudaEvent_t scratch_ev = nullptr;
    bool scratch_ev_live = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // class-pair kernels run concurrently on side streams forked from `stream`
    static constexpr int kSide = 6;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr, join[kSide] = {};
    int num_sms = 0;
    // blocks/SM of the queue kernels, 0 = not queried: [x][y][HGP FP64, HGP MIXED, Rys FP64,
    // Rys MIXED]
    int occupancy[kNumPairClasses][kNumPairClasses][4] = {};
    RysTab rys{};  // device addresses of the Rys root/weight tables on this device
    int32_t class_method[kNumPairClasses][kNumPairClasses] = {};  // AUTO choices (0 = HGP)
    // the table molints_set_class_methods(NULL) restores: the tuned table of class_table.h on
    // the device it was measured on, all zero (HGP everywhere) elsewhere
    int32_t default_method[kNumPairClasses][kNumPairClasses] = {};
    char *stage = nullptr;     // pinned host buffer of plan uploads (shells, stage-1 pair tables)
    size_t stage_bytes = 0;
    // work-queue schedule of the plans it creates (molints_set_schedule)
    molints_schedule sched{};
    molints_schedule default_sched{};  // what molints_set_schedule(NULL) restores
    std::string err;
};

struct molints_plan {
    molints_ctx *ctx = nullptr;
    molints_options opts{};
    int nmol = 0;
    int nshell = 0;
    int64_t nbf0 = 0;                  // functions of molecule 0 (J/K dimension)
    int64_t npacked = 0;               // all molecules
    std::vector<int64_t> mol_out_h;    // offset of each molecule's packed vector
    std::vector<int> mol_nshell;
    int npair = 0;
    int64_t nprim_pair_all = 0, nprim_pair_kept = 0;
    int class_start[kNumPairClasses + 1] = {0};
    // work queues: chunks of class pair (x, y) are chunk[q_off[x][y] .. + q_len[x][y])
    int q_off[kNumPairClasses][kNumPairClasses] = {};
    int q_len[kNumPairClasses][kNumPairClasses] = {};
    double class_cost[kNumPairClasses][kNumPairClasses] = {};  // kept primitive quartets
    int method[kNumPairClasses][kNumPairClasses] = {};  // MOLINTS_METHOD_HGP or _RYS
    int fp32[kNumPairClasses][kNumPairClasses] = {};    // MIXED and this class's FP32 variant used
    // host copies (final, screened order): pair_mol from plan creation (the re-sort by kept
    // count stays within each molecule's run), the rest fetched on first use (plan_host_tables)
    std::vector<int> pair_mol;         // canonical pair -> molecule
    bool host_tables = false;
    std::vector<int> pair_ref;         // canonical pair -> reference pair index i(i+1)/2+j
    std::vector<int> npp_h;            // kept primitive pairs per shell pair
    std::vector<double2> bnd_h;        // (Qabs, R) per shell pair
    // device buffers
    double *sh_xyz = nullptr, *expn = nullptr, *ncoef = nullptr;
    int *sh_poff = nullptr;
    int2 *pair_ab = nullptr;
    int4 *info = nullptr;
    int *pp_src = nullptr;             // primitive pair k -> (ia << 8) | ib within its shells
    double *pbk = nullptr;             // primitive pair k -> its Schwarz bound b_k (kept order)
    double4 *geo = nullptr;
    PrimPair *pp = nullptr;
    double2 *bnd = nullptr;
    int4 *chunks = nullptr;
    int *counters = nullptr;           // one per class pair, zeroed by every execute
    long long *mol_out = nullptr;
    double *qcon = nullptr;  // contracted Schwarz bounds, filled on demand by plan_schwarz
    // two-phase output (molints_output): the class kernels store whole quartet blocks into a
    // class-major scratch, a gather pass writes the packed vector in order from it
    int two_phase = 0;
    int gather_blocks = 0;             // the context's schedule at creation: gather blocks per SM
    int screen_trunc = 0;              // ket runs end at the last unscreened ket (quartet screening)
    int64_t scratch_need = 0;          // doubles of the context's scratch an execute uses: per
                                       // (class pair, molecule) a region of quartet blocks
    long long *chunk_slot = nullptr;   // per chunk: scratch offset of its first quartet's block
    int2 *g_fn = nullptr;              // per function (all molecules): {shell in molecule, component}
    int *g_pair = nullptr;             // per molecule shell pair I >= J: pos << 5 | class << 1 | A == J
    long long *g_region = nullptr;     // per (x, y, molecule): {scratch offset, first bra, first ket, kets}
    long long *g_mol = nullptr;        // per molecule: {first function, first pair entry, packed offset,
                                       // first function-pair entry of g_col}
    int2 *g_col = nullptr;             // per function pair of every molecule: gather_cols_kernel
    double *g_colq = nullptr;          // beside g_col when quartets are screened: Qabs of its pair
    double *g_qmax = nullptr;          // per molecule when quartets are screened: a bound of every
                                       // pair's Qabs (the largest sum of b_k over all its
                                       // primitive pairs)
    int4 *g_units = nullptr;           // gather units: shell pairs, heaviest first (gather_packed_kernel)
    int64_t n_units = 0;
    int64_t bytes = 0;
    int n_launches = 0;
    int n_fp32_launches = 0;           // class-pair launches of the last execute that ran FP32
    // shell quartets with a g shell (l = 4): computed by the generic kernel (eri_generic.cu)
    int64_t n_gq = 0;
    int4 *gq = nullptr;                // global shells (I, J, K, L), reference order
    int *gq_mol = nullptr;
    int *sh_L = nullptr, *sh_K = nullptr, *sh_fn = nullptr;  // shells' L and primitive count (all
                                                             // plans), first function (g plans)
    double plan_ms[4] = {0, 0, 0, 0};  // plan creation phases (molints_stats.plan_ms)
    // CUDA graph of one execute (molints_plan_set_graph), valid for graph_out
    int use_graph = 0;
    cudaGraphExec_t gexec = nullptr;
    double *graph_out = nullptr;
    int graph_gen = -1;                // the context's scratch_gen at capture
    // per-launch profiling (molints_plan_set_profiling)
    int profiling = 0;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<const char *> prof_name;
};

// ------------------------------------------------------------------ helpers
namespace {

int fail(molints_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(molints_ctx *ctx, cudaError_t e, const char *what) {
    return fail(ctx, MOLINTS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define MI_CUDA(ctx, call)                                            \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);    \
    } while (0)

int ncart(int l) { return (l + 1) * (l + 2) / 2; }

double dfact2(int n) {
    double r = 1;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

// Exact F_m(T) by the series e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)), long double.
double boys_series(int m, double T) {
    if (T == 0.0) return 1.0 / (2 * m + 1);
    long double t = T, sum = 0.0L, term = 1.0L / (2 * m + 1);
    for (int k = 0; k < 100000; ++k) {
        sum += term;
        if (k > T && term < sum * 1e-22L) break;
        term *= 2.0L * t / (2 * m + 2 * k + 3);
    }
    return (double)(expl(-t) * sum);
}

int pair_class_of(int la, int lb) {
    for (int c = 0; c < kNumPairClasses; ++c)
        if (kPairClassLa[c] == la && kPairClassLb[c] == lb) return c;
    return -1;
}

// Stable LSD radix order of keys[0..n) over their low `bits` bits (8-bit digits): the
// permutation position -> index, equal keys in index order.  O(n bits / 8).
std::vector<uint32_t> radix_order(const std::vector<uint64_t> &keys, int bits) {
    const size_t n = keys.size();
    std::vector<uint64_t> k(keys), k2(n);
    std::vector<uint32_t> v(n), v2(n);
    for (size_t i = 0; i < n; ++i) v[i] = (uint32_t)i;
    for (int sh = 0; sh < bits; sh += 8) {
        size_t at[257] = {};
        for (size_t i = 0; i < n; ++i) ++at[((k[i] >> sh) & 255) + 1];
        if (at[1] == n) continue;  // every key has this digit 0
        for (int d = 0; d < 256; ++d) at[d + 1] += at[d];
        for (size_t i = 0; i < n; ++i) {
            const size_t j = at[(k[i] >> sh) & 255]++;
            k2[j] = k[i];
            v2[j] = v[i];
        }
        k.swap(k2);
        v.swap(v2);
    }
    return v;
}

// Bits needed to hold values 0..v.
int bits_for(uint64_t v) {
    int b = 0;
    while (v >> b) ++b;
    return b;
}

// Sub-buffers of one allocation: take<T>(n) returns the byte offset of n elements of T, each
// sub-buffer 256-byte aligned (at least one element, so no two share an address).
struct Carve {
    size_t at = 0;
    template <typename T> size_t take(long long count) {
        const size_t o = at;
        at += ((size_t)std::max<long long>(count, 1) * sizeof(T) + 255) & ~(size_t)255;
        return o;
    }
};

template <typename T>
int dev_alloc(molints_ctx *ctx, T **p, size_t count, int64_t *tally) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (ctx->budget > 0 && ctx->held + (int64_t)bytes > ctx->budget)
        return fail(ctx, MOLINTS_ERR_BUDGET, "HBM budget exceeded");
    cudaError_t e = cudaMallocFromPoolAsync((void **)p, bytes, ctx->pool, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMallocFromPoolAsync");
    ctx->held += (int64_t)bytes;
    if (tally) *tally += (int64_t)bytes;
    return MOLINTS_OK;
}

void dev_free(molints_ctx *ctx, void *p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}

// The context's two-phase scratch grown to at least `need` doubles (the old buffer is freed in
// stream order, after the executes that used it).
int ctx_scratch(molints_ctx *ctx, int64_t need) {
    need = std::max<int64_t>(need, 1);
    if (ctx->scratch_len >= need) return MOLINTS_OK;
    if (ctx->scratch) {
        if (ctx->scratch_ev_live) cudaStreamWaitEvent(ctx->stream, ctx->scratch_ev, 0);
        dev_free(ctx, ctx->scratch);
        ctx->held -= ctx->scratch_len * (int64_t)sizeof(double);
        ctx->scratch = nullptr;
        ctx->scratch_len = 0;
    }
    int rc = dev_alloc(ctx, &ctx->scratch, (size_t)need, nullptr);
    if (rc) {
        ctx->scratch = nullptr;
        return rc;
    }
    ctx->scratch_len = need;
    ++ctx->scratch_gen;
    return MOLINTS_OK;
}

// The pinned upload buffer of the context, grown to at least `bytes` (a pinned source makes
// the plan uploads asynchronous DMA at full link speed).  Plan creation synchronises on its
// summary read-back after its last upload, so the buffer is free whenever a creation starts.
int ctx_stage(molints_ctx *ctx, size_t bytes) {
    if (ctx->stage_bytes >= bytes) return MOLINTS_OK;
    if (ctx->stage) cudaFreeHost(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    const size_t want = std::max<size_t>(bytes + bytes / 4, (size_t)1 << 20);
    cudaError_t e = cudaHostAlloc((void **)&ctx->stage, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        ctx->stage = nullptr;
        return cuda_fail(ctx, e, "cudaHostAlloc (plan upload buffer)");
    }
    ctx->stage_bytes = want;
    return MOLINTS_OK;
}

}  // namespace

// ------------------------------------------------------------------ device kernels
namespace molints {

// The normalised contraction coefficients of every shell, in place: raw coef x the primitive
// norm (2a/pi)^(3/4) (4a)^(L/2) x the contracted norm 1/sqrt(S), S = sum_ij c_i c_j
// (2 sqrt(a_i a_j) / (a_i + a_j))^(L + 3/2) the self-overlap of the shell's function (PGBF/CGBF
// normalize!, src/Basis.jl:42-83; the component factor 1/sqrt((2I-1)!!(2J-1)!!(2K-1)!!) is
// applied by the ERI kernels).  One thread per shell; a shell whose S is not positive sets
// *bad (the plan is refused).
__global__ void normalise_shells_kernel(int ns, const int *__restrict__ L, const int *__restrict__ K,
                                        const int *__restrict__ poff, const double *__restrict__ expn,
                                        double *__restrict__ coef, int *__restrict__ bad) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ns) return;
    const int Ls = L[g], Ks = K[g], p0 = poff[g];
    double S = 0.0;
    for (int i = 0; i < Ks; ++i)
        for (int j = 0; j < Ks; ++j) {
            const double x = expn[p0 + i], y = expn[p0 + j];
            S += coef[p0 + i] * coef[p0 + j] * pow(2.0 * sqrt(x * y) / (x + y), Ls + 1.5);
        }
    if (!(S > 0.0)) {
        atomicExch(bad, 1);
        return;
    }
    const double cn = 1.0 / sqrt(S);
    for (int i = 0; i < Ks; ++i) {
        const double a = expn[p0 + i];
        coef[p0 + i] *= cn * pow(2.0 * a / 3.14159265358979323846, 0.75) * pow(4.0 * a, 0.5 * Ls);
    }
}

__global__ void build_pairs_kernel(int npair, const int2 *__restrict__ pair_ab,
                                   const int4 *__restrict__ info, const int *__restrict__ pp_src,
                                   const double *__restrict__ xyz, const int *__restrict__ poff,
                                   const double *__restrict__ expn,
                                   const double *__restrict__ ncoef, double c0,
                                   const double *__restrict__ pb,
                                   PrimPair *__restrict__ pp, double4 *__restrict__ geo) {
    // one warp per shell pair, its lanes over the pair's primitive pairs (up to 7 x 7)
    const int p = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (p >= npair) return;
    const int2 ab = pair_ab[p];
    const int4 in = info[p];
    const double Ax = xyz[3 * ab.x], Ay = xyz[3 * ab.x + 1], Az = xyz[3 * ab.x + 2];
    const double Bx = xyz[3 * ab.y], By = xyz[3 * ab.y + 1], Bz = xyz[3 * ab.y + 2];
    const double ABx = Ax - Bx, ABy = Ay - By, ABz = Az - Bz;
    const double rab2 = ABx * ABx + ABy * ABy + ABz * ABz;
    const int pa0 = poff[ab.x], pb0 = poff[ab.y];
    for (int k = in.x + lane; k < in.x + in.y; k += 32) {
        const int src = pp_src[k];
        const double a = expn[pa0 + (src >> 8)], ca = ncoef[pa0 + (src >> 8)];
        const double b = expn[pb0 + (src & 255)], cb = ncoef[pb0 + (src & 255)];
        const double zeta = a + b, ooz = 1.0 / zeta;
        PrimPair r;
        r.zeta = zeta;
        r.kab = c0 * ca * cb * exp(-a * b * ooz * rab2) * ooz;
        r.oo2z = 0.5 * ooz;
        // P = A + (b/zeta)(B - A): P - A is exactly 0 when A == B, and P - Q exactly 0 when
        // all four centres coincide, so symmetry-zero one-centre integrals come out as 0.
        const double boz = b * ooz;
        r.pax = boz * (Bx - Ax);
        r.pay = boz * (By - Ay);
        r.paz = boz * (Bz - Az);
        r.px = Ax + r.pax;
        r.py = Ay + r.pay;
        r.pz = Az + r.paz;
        r.b = pb ? pb[k] : 0.0;
        pp[k] = r;
    }
    if (lane == 0) geo[p] = make_double4(ABx, ABy, ABz, 0.0);
}

// Blocks of 128 threads for build_pairs_kernel over npair shell pairs (a warp each).
inline int build_pairs_blocks(int npair) { return (int)(((long long)npair + 3) / 4); }

// Cartesian components of each pair class's two shells, for the gather pass.
__constant__ int c_pair_na[kNumPairClasses] = {
#define MI_NC(c) (kPairClassLa[c] + 1) * (kPairClassLa[c] + 2) / 2
    MI_NC(0), MI_NC(1), MI_NC(2), MI_NC(3), MI_NC(4), MI_NC(5), MI_NC(6), MI_NC(7), MI_NC(8), MI_NC(9), MI_NC(10)};
#undef MI_NC
__constant__ int c_pair_nb[kNumPairClasses] = {
#define MI_NC(c) (kPairClassLb[c] + 1) * (kPairClassLb[c] + 2) / 2
    MI_NC(0), MI_NC(1), MI_NC(2), MI_NC(3), MI_NC(4), MI_NC(5), MI_NC(6), MI_NC(7), MI_NC(8), MI_NC(9), MI_NC(10)};
#undef MI_NC
static_assert(kNumPairClasses == 11, "c_pair_na / c_pair_nb list every pair class");

// n with n(n+1)/2 <= t < (n+1)(n+2)/2, from an FP32 square root and an exact integer fix-up
// (t < 2^31 is off by at most a few units in n).
__device__ __forceinline__ long long untri_f(long long t) {
    long long n = (long long)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while ((n + 1) * (n + 2) / 2 <= t) ++n;
    while (n > 0 && n * (n + 1) / 2 > t) --n;
    return n;
}

constexpr int kGatherThreads = 256;

// Per function pair (i >= j) of every molecule of a two-phase plan, what the gather needs to
// place its entries, built once per plan on the device: x = list position << 4 | pair class of
// the shell pair holding (i, j), y = component of the function in that pair's A << 16 |
// component in its B; colq (plans that screen quartets) the pair's Qabs.  Entry (m, ij) is at
// col[mol[4m+3] + ij]; thread r takes entry r, of the molecule m with
// mol[4m+3] <= r < mol[4(m+1)+3] (the molecules' entries follow one another).
__global__ void gather_cols_kernel(int2 *__restrict__ col, double *__restrict__ colq,
                                   const double2 *__restrict__ bnd, const int2 *__restrict__ fn,
                                   const int *__restrict__ pairs, const long long *__restrict__ mol,
                                   int nmol, long long nrows) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    int m = 0, hi = nmol;  // last m with mol[4m+3] <= r
    while (hi - m > 1) {
        const int mid = (m + hi) >> 1;
        if (__ldg(&mol[4 * mid + 3]) <= r) m = mid; else hi = mid;
    }
    const long long ij = r - __ldg(&mol[4 * m + 3]);
    const long long fb = __ldg(&mol[4 * m]), pb = __ldg(&mol[4 * m + 1]);
    const long long i = untri_f(ij), j = ij - i * (i + 1) / 2;
    const int2 fi = __ldg(&fn[fb + i]), fj = __ldg(&fn[fb + j]);
    const int P = __ldg(&pairs[pb + (long long)fi.x * (fi.x + 1) / 2 + fj.x]);
    const int ca = (P & 1) ? fj.y : fi.y, cb = (P & 1) ? fi.y : fj.y;
    col[__ldg(&mol[4 * m + 3]) + ij] = make_int2(((P >> 5) << 4) | ((P >> 1) & 15), (ca << 16) | cb);
    if (colq) colq[__ldg(&mol[4 * m + 3]) + ij] = __ldg(&bnd[P >> 5]).x;
}

// Second phase of the two-phase output: the packed vector written from the scratch blocks, one
// shell pair P at a time.  A block of threads takes the next pair from units[] (heaviest first,
// through an atomic counter) and writes all of P's rows (function pairs ij of P) column by
// column: each thread takes a column kl, reads its descriptor once, and stores that column of
// every row of P with kl <= ij.  The stores of one row are coalesced; the scratch entries of a
// quartet (P, Q) for all of P's rows lie in one block, read by the same threads in the
// same pass, so each scratch sector is fetched once.  Each entry comes from the block and
// component the direct path would have stored it from: the quartet's bra is the pair of the
// higher class, or of the later list position within a class (P for the diagonal quartet
// P == Q); a pair's components are taken in its A, B orientation, with the larger component
// first within a same-shell pair, as the direct store conditions pick.  With quartet
// screening, the entries of a screened quartet are written as 0 without reading the scratch:
// plans that screen end each bra's ket run after its last unscreened ket, so no chunk computes
// the rest.
constexpr int kGatherMaxRows = 100;  // components of an (ff) pair

// The columns of one shell pair P for the gather: NC columns per thread and pass (kl,
// kl + kGatherThreads, ...), their descriptor loads first, then the scratch loads of NR rows of
// each column (NC * NR in flight), then their stores.  RMAX > 0: P has at most RMAX rows, known
// at compile time (RMAX <= NR: one row step per pass, no loop).  (Measured on B200: NC = 2,
// NR = 4 with the small pairs' copies specialised beats more columns or rows per pass and
// prefetching the next pass's descriptors, which cost occupancy.)
template <int NC, int NR, int RMAX>
__device__ __forceinline__ void gather_pair_columns(
    double *__restrict__ obase, const double *__restrict__ scratch, const int2 *__restrict__ col,
    const double *__restrict__ colq, long long cbase, const long long (*reg)[kNumPairClasses][5],
    const long long *s_ij, const long long *s_tri, const int *s_rc, int R, int posP, int clsP,
    double qP, double screen_cut) {
    if (RMAX == 1) R = 1;
    const long long ijmax = s_ij[R - 1];  // rows are in increasing ij
    const int nP = c_pair_na[clsP] * c_pair_nb[clsP];
    for (long long kl0 = threadIdx.x; kl0 <= ijmax; kl0 += NC * kGatherThreads) {
        const double *src[NC];
        long long kl[NC];
        int r0[NC], rs[NC];
        bool zero[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            kl[c] = kl0 + c * kGatherThreads;
            const bool on = kl[c] <= ijmax;
            const int2 qe = on ? __ldg(&col[cbase + kl[c]]) : make_int2(clsP, 0);
            // a screened quartet (the class kernels' test, Qabs_P Qabs_Q < screen_cut) is 0;
            // its block is not read (no chunk may have computed it)
            zero[c] = on && screen_cut > 0.0 && qP * __ldg(&colq[cbase + kl[c]]) < screen_cut;
            src[c] = scratch;
            rs[c] = 0;
            if (!zero[c]) {
                // the column's scratch block and component (skipped for screened columns, most
                // of a screened plan's)
                const int posQ = on ? qe.x >> 4 : posP, clsQ = qe.x & 15;
                const int qa = qe.y >> 16, qb = qe.y & 0xffff;
                const bool braP = clsP > clsQ || (clsP == clsQ && posP >= posQ);
                const long long *rg = reg[braP ? 0 : 1][clsQ];
                const int bpos = braP ? posP : posQ, kpos = braP ? posQ : posP;
                const long long db = bpos - rg[1], dk = kpos - rg[2];
                const long long slot = (clsP == clsQ) ? db * (db + 1) / 2 + dk : db * rg[3] + dk;
                // component x = row part * rstride + column part
                const int nq = c_pair_na[clsQ] * c_pair_nb[clsQ], qc = qa * c_pair_nb[clsQ] + qb;
                rs[c] = braP ? nq : 1;
                src[c] = scratch + rg[0] + slot * rg[4] + (braP ? qc : qc * nP);
            }
            // rows with ij >= kl: a suffix of the increasing row list (none past ijmax)
            int r = 0;
            while (r < R && s_ij[r] < kl[c]) ++r;
            r0[c] = on ? r : R;
        }
        int rmin = r0[0];
#pragma unroll
        for (int c = 1; c < NC; ++c) rmin = min(rmin, r0[c]);
        for (int r = rmin; r < R; r += NR) {
            double v[NC][NR];
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int t = 0; t < NR; ++t)
                    v[c][t] = (r + t < R && r + t >= r0[c] && !zero[c]) ? __ldg(src[c] + s_rc[r + t] * rs[c]) : 0.0;
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int t = 0; t < NR; ++t)
                    if (r + t < R && r + t >= r0[c]) obase[s_tri[r + t] + kl[c]] = v[c][t];
            if (RMAX > 0 && RMAX <= NR) break;
        }
    }
}

__global__ void __launch_bounds__(kGatherThreads) gather_packed_kernel(
    double *__restrict__ out, const double *__restrict__ scratch, const int2 *__restrict__ col,
    const double *__restrict__ colq, const long long *__restrict__ region, const long long *__restrict__ mol,
    const int4 *__restrict__ units, long long nunits, int *__restrict__ counter, int nmol,
    const double2 *__restrict__ bnd, const double *__restrict__ qmax, double screen_cut) {
    // [P as bra, P as ket][class of the other pair]: {scratch offset, first bra, first ket,
    // kets, block size}
    __shared__ long long reg[2][kNumPairClasses][5];
    __shared__ long long s_ij[kGatherMaxRows], s_tri[kGatherMaxRows];
    __shared__ int s_rc[kGatherMaxRows];
    __shared__ long long s_unit;
    for (;;) {
        __syncthreads();  // the previous unit's readers are done with the shared tables
        if (threadIdx.x == 0) s_unit = atomicAdd(counter, 1);
        __syncthreads();
        const long long u = s_unit;
        if (u >= nunits) return;
        const int4 un = __ldg(&units[u]);
        const int m = un.x, fi0 = un.y, fj0 = un.z;
        const int nI = un.w & 255, nJ = (un.w >> 8) & 255, same = (un.w >> 16) & 1;
        const long long cbase = __ldg(&mol[4 * m + 3]);
        double *__restrict__ obase = out + __ldg(&mol[4 * m + 2]);
        // P's rows: ij, the row's first packed index tri(ij), and the row's component index in
        // P's A, B orientation
        const int2 pe = __ldg(&col[cbase + (long long)fi0 * (fi0 + 1) / 2 + fj0]);
        const int posP = pe.x >> 4, clsP = pe.x & 15;
        const int nbP = c_pair_nb[clsP];
        const double qP = screen_cut > 0.0 ? __ldg(&bnd[posP]).x : 0.0;
        int R = 0;
        for (int a = 0; a < nI; ++a) R += same ? a + 1 : nJ;
        for (int r = threadIdx.x; r < R; r += kGatherThreads) {
            int a = 0, b = r;
            if (same) { while (b > a) { b -= a + 1; ++a; } }
            else { a = r / nJ; b = r - a * nJ; }
            const long long i = fi0 + a, j = fj0 + b, ij = i * (i + 1) / 2 + j;
            const int2 re = __ldg(&col[cbase + ij]);
            s_ij[r] = ij;
            s_tri[r] = ij * (ij + 1) / 2;
            s_rc[r] = (re.y >> 16) * nbP + (re.y & 0xffff);
        }
        if (threadIdx.x < 2 * kNumPairClasses) {
            const int o = threadIdx.x / kNumPairClasses, t = threadIdx.x % kNumPairClasses;
            const int x = o == 0 ? clsP : t, y = o == 0 ? t : clsP;
            if (x >= y) {
                const long long *rg = region + kRegionFields * (((long long)x * kNumPairClasses + y) * nmol + m);
                for (int f = 0; f < kRegionFields; ++f) reg[o][t][f] = __ldg(&rg[f]);
                reg[o][t][4] = (long long)c_pair_na[x] * c_pair_nb[x] * c_pair_na[y] * c_pair_nb[y];
            }
        }
        __syncthreads();
        if (screen_cut > 0.0 && qP * __ldg(&qmax[m]) < screen_cut) {
            // every quartet of P is screened (Qabs_P times the molecule's largest Qabs is below
            // the cutoff): its rows are zeros, written as contiguous runs with no descriptor or
            // scratch loads
            for (int r = 0; r < R; ++r) {
                const long long t0 = s_tri[r], n = s_ij[r] + 1;
                for (long long k = threadIdx.x; k < n; k += kGatherThreads) obase[t0 + k] = 0.0;
            }
            continue;
        }
        // pairs of one or a few rows (ss, sp) are most of the units: their copies have no row loop
        if (R == 1)
            gather_pair_columns<2, 1, 1>(obase, scratch, col, colq, cbase, reg, s_ij, s_tri, s_rc, R, posP, clsP,
                                         qP, screen_cut);
        else if (R <= 4)
            gather_pair_columns<2, 4, 4>(obase, scratch, col, colq, cbase, reg, s_ij, s_tri, s_rc, R, posP, clsP,
                                         qP, screen_cut);
        else
            gather_pair_columns<2, 4, 0>(obase, scratch, col, colq, cbase, reg, s_ij, s_tri, s_rc, R, posP, clsP,
                                         qP, screen_cut);
    }
}

// Copy the lower triangles of J and K (the digestion accumulates only those) to the upper.
__global__ void mirror_lower_kernel(double *__restrict__ J, double *__restrict__ K, int n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int r = (int)(t / n), c = (int)(t - (long long)r * n);
    if (r < c) {
        J[(long long)r * n + c] = J[(long long)c * n + r];
        K[(long long)r * n + c] = K[(long long)c * n + r];
    }
}

__global__ void boys_eval_kernel(BoysTab bt, int mmax, const double *__restrict__ T, long long n,
                                 double *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double F[23];
    const double t = T[i];
    switch (mmax - 1) {
#define MI_CASE(M) case M: boys_fm<M>(t, bt, F); break;
        MI_CASE(0) MI_CASE(1) MI_CASE(2) MI_CASE(3) MI_CASE(4) MI_CASE(5) MI_CASE(6)
        MI_CASE(7) MI_CASE(8) MI_CASE(9) MI_CASE(10) MI_CASE(11) MI_CASE(12)
        MI_CASE(13) MI_CASE(14) MI_CASE(15)
#undef MI_CASE
        default: return;
    }
    for (int m = 0; m < mmax; ++m) out[i * mmax + m] = F[m];
}

}  // namespace molints

// ------------------------------------------------------------------ g shells (eri_generic.cu)
namespace molints {
struct GenQuartets {
    const int4 *quartet;
    const int *mol;
    long long n;
    const double *xyz;
    const int *L, *nprim, *poff, *fn_off;
    const double *expn, *ncoef;
    const long long *mol_out;
    double *out;
    RysTab rys;
};
void launch_eri_generic(const GenQuartets &G, int grid, cudaStream_t s);
}  // namespace molints

// ------------------------------------------------------------------ helpers for noalloc.cu
namespace molints {

// Launch the primitive-pair builder (used by the allocation-free entry point).
void launch_build_pairs(int npair, const int2 *pair_ab, const int4 *info, const int *pp_src,
                        const double *xyz, const int *poff, const double *expn,
                        const double *ncoef, PrimPair *pp, double4 *geo, cudaStream_t s) {
    if (npair <= 0) return;
    build_pairs_kernel<<<build_pairs_blocks(npair), 128, 0, s>>>(npair, pair_ab, info, pp_src, xyz, poff,
                                                          expn, ncoef, std::sqrt(2.0) * std::pow(M_PI, 1.25),
                                                          nullptr, pp, geo);
}

// The scaled Boys tables of the kernels for M = 0..nM-1: row n of table M holds
// F_{M+k}(T_n)/k! (k < 8), e^-T_n and a pad, T_n = n/16, n = 0..640.
void fill_boys_scaled(double *sc, int nM) {
    for (int M = 0; M < nM; ++M)
        for (int n = 0; n < kBoysRows; ++n) {
            const double T = n * kBoysStep;
            double *row = sc + ((size_t)M * kBoysRows + n) * kBoysScaledCols;
            double fact = 1.0;
            for (int k = 0; k < kBoysTaylor; ++k) {
                if (k > 0) fact *= k;
                row[k] = boys_series(M + k, T) / fact;
            }
            row[kBoysTaylor] = std::exp(-T);
            row[kBoysTaylor + 1] = 0.0;
        }
}

}  // namespace molints

namespace molints {
int ctx_device_of(const molints_ctx *ctx) { return ctx->device; }
RysTab ctx_rys(const molints_ctx *ctx) { return ctx->rys; }

// Normalised contraction coefficients of a basis (indexed like its primitives): raw coef x
// (2a/pi)^(3/4) (4a)^(L/2) x the CGBF norm (PGBF/CGBF normalize!, src/Basis.jl:42-83).
int basis_ncoef(const molints_basis *b, std::vector<double> &ncoef, std::string &err) {
    int nprim = 0;
    for (int s = 0; s < b->nshell; ++s) {
        if (b->nprim[s] < 1 || b->prim_off[s] < 0) { err = "shell without primitives"; return MOLINTS_ERR_INVALID; }
        nprim = std::max(nprim, b->prim_off[s] + b->nprim[s]);
    }
    for (int k = 0; k < nprim; ++k)
        if (!(b->expn[k] > 0.0) || !std::isfinite(b->expn[k]) || !std::isfinite(b->coef[k])) {
            err = "exponents must be finite and > 0";
            return MOLINTS_ERR_INVALID;
        }
    ncoef.assign(std::max(nprim, 1), 0.0);
    for (int s = 0; s < b->nshell; ++s) {
        const int p0 = b->prim_off[s], K = b->nprim[s], Ls = b->L[s];
        double S = 0;
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) {
                const double x = b->expn[p0 + i], y = b->expn[p0 + j];
                S += b->coef[p0 + i] * b->coef[p0 + j] * std::pow(2 * std::sqrt(x * y) / (x + y), Ls + 1.5);
            }
        if (!(S > 0.0)) { err = "zero contracted function"; return MOLINTS_ERR_INVALID; }
        const double cn = 1.0 / std::sqrt(S);
        for (int i = 0; i < K; ++i) {
            const double a = b->expn[p0 + i];
            ncoef[p0 + i] = b->coef[p0 + i] * cn * std::pow(2 * a / M_PI, 0.75) * std::pow(4 * a, 0.5 * Ls);
        }
    }
    return MOLINTS_OK;
}
// The AUTO method table of src, given to dst (the serving slots inherit their owner's table).
void ctx_copy_methods(molints_ctx *dst, const molints_ctx *src) {
    std::memcpy(dst->class_method, src->class_method, sizeof(dst->class_method));
    dst->sched = src->sched;
}

// The schedule of contexts on devices without a tuned one.
constexpr molints_schedule kBuiltinSchedule = {80.0, 1, 4096, 8, 5};
constexpr int kGatherBlocksDefault = 5;

bool schedule_ok(const molints_schedule &s) {
    return s.lane_cost > 0.0 && s.lane_cost <= 1e6 && s.hgp_widen >= 1 && s.hgp_widen <= 64 &&
           s.rys_chunks >= 1 && s.rys_max_width >= 1 && s.rys_max_width <= 64 && s.gather_blocks >= 0 &&
           s.gather_blocks <= 16;
}
}  // namespace molints

// ------------------------------------------------------------------ C ABI
extern "C" {

int molints_abi_version(void) { return MOLINTS_ABI_VERSION; }

void molints_default_options(molints_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->method = MOLINTS_METHOD_AUTO;
    o->precision = MOLINTS_FP64;
    o->boys = MOLINTS_BOYS_REFERENCE;
    o->fp32_cutoff = 0.0;
    o->screen_cutoff = 0.0;
    o->prim_cutoff = 1e-18;
}

int64_t molints_npacked(int64_t n) { return n < 0 ? -1 : n * (n + 1) * (n * n + n + 2) / 8; }

int64_t molints_nbf(const molints_basis *b) {
    if (!b || b->nshell < 0 || (b->nshell > 0 && (!b->L || !b->xyz || !b->nprim || !b->prim_off)))
        return MOLINTS_ERR_INVALID;
    int64_t n = 0;
    for (int s = 0; s < b->nshell; ++s) {
        if (b->L[s] < 0) return MOLINTS_ERR_INVALID;
        n += ncart(b->L[s]);
    }
    return n;
}

int molints_create(molints_ctx **out, int device, int64_t budget, uint32_t flags) {
    if (!out) return MOLINTS_ERR_INVALID;
    *out = nullptr;
    if (flags != 0) return MOLINTS_ERR_INVALID;
    molints_ctx *ctx = new (std::nothrow) molints_ctx();
    if (!ctx) return MOLINTS_ERR_NOMEM;
    ctx->device = device;
    ctx->budget = budget;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete ctx; return MOLINTS_ERR_CUDA; }
    bool ok = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&ctx->ev0) == cudaSuccess && cudaEventCreate(&ctx->ev1) == cudaSuccess &&
              cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < molints_ctx::kSide; ++i)
        ok = cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&ctx->join[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&ctx->scratch_ev, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        molints_destroy(ctx);
        return MOLINTS_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    if (rys_tables(&ctx->rys) != 0) {
        molints_destroy(ctx);
        return MOLINTS_ERR_CUDA;
    }
    if (cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        ctx->num_sms = 1;
    {
        cudaDeviceProp prop;
        ctx->default_sched = kBuiltinSchedule;
        if (cudaGetDeviceProperties(&prop, device) == cudaSuccess &&
            std::strncmp(prop.name, kTunedDevice, std::strlen(kTunedDevice)) == 0) {
            std::memcpy(ctx->default_method, kTunedClassMethods, sizeof(ctx->default_method));
            ctx->default_sched = {kTunedSchedule[0], (int32_t)kTunedSchedule[1], (int32_t)kTunedSchedule[2],
                                  (int32_t)kTunedSchedule[3], (int32_t)kTunedSchedule[4]};
        }
        std::memcpy(ctx->class_method, ctx->default_method, sizeof(ctx->class_method));
        ctx->sched = ctx->default_sched;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&ctx->pool, &props) != cudaSuccess) {
        ctx->pool = nullptr;
        molints_destroy(ctx);
        return MOLINTS_ERR_CUDA;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    // Boys table: F_0..F_22 and e^-T at T_n = n/16, n = 0..640.
    std::vector<double> tab((size_t)kBoysRows * kBoysCols);
    for (int n = 0; n < kBoysRows; ++n) {
        const double T = n * kBoysStep;
        for (int m = 0; m < kBoysCols - 1; ++m) tab[(size_t)n * kBoysCols + m] = boys_series(m, T);
        tab[(size_t)n * kBoysCols + kBoysCols - 1] = std::exp(-T);
    }
    // Per-M tables for the kernels: row n of table M holds F_{M+k}(T_n)/k! (k = 0..7) and
    // e^-T_n, padded to 10 doubles, so the Taylor sum is a Horner chain of 7 FMAs.
    std::vector<double> sc((size_t)kBoysMaxM1 * kBoysRows * kBoysScaledCols, 0.0);
    fill_boys_scaled(sc.data(), kBoysMaxM1);
    int rc = dev_alloc(ctx, &ctx->boys_tab, tab.size(), nullptr);
    if (!rc) rc = dev_alloc(ctx, &ctx->boys_scaled, sc.size(), nullptr);
    if (rc) { molints_destroy(ctx); return rc; }
    if (cudaMemcpyAsync(ctx->boys_tab, tab.data(), tab.size() * sizeof(double),
                        cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(ctx->boys_scaled, sc.data(), sc.size() * sizeof(double),
                        cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        molints_destroy(ctx);
        return MOLINTS_ERR_CUDA;
    }
    *out = ctx;
    return MOLINTS_OK;
}

static void plan_release_device(molints_plan *p);

int molints_destroy(molints_ctx *ctx) {
    if (!ctx) return MOLINTS_OK;
    molints_serve_stop(ctx);
    cudaSetDevice(ctx->device);
    // Plans the caller has not destroyed lose their device state now; destroying one later
    // only frees its host record.
    for (molints_plan *p : ctx->plans) plan_release_device(p);
    ctx->plans.clear();
    if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->stream = ctx->own_stream;
    if (ctx->own_stream) {
        dev_free(ctx, ctx->boys_tab);
        dev_free(ctx, ctx->boys_scaled);
        dev_free(ctx, ctx->out_cache);
        dev_free(ctx, ctx->scratch);
        cudaStreamSynchronize(ctx->own_stream);
    }
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    for (int i = 0; i < molints_ctx::kSide; ++i) {
        if (ctx->side[i]) cudaStreamSynchronize(ctx->side[i]);
        if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
        if (ctx->join[i]) cudaEventDestroy(ctx->join[i]);
    }
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    if (ctx->scratch_ev) cudaEventDestroy(ctx->scratch_ev);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    delete ctx;
    return MOLINTS_OK;
}

const char *molints_last_error(const molints_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int molints_set_class_methods(molints_ctx *ctx, const int32_t *methods, int32_t n) {
    if (!ctx) return MOLINTS_ERR_INVALID;
    if (!methods) {
        std::memcpy(ctx->class_method, ctx->default_method, sizeof(ctx->class_method));
        return MOLINTS_OK;
    }
    if (n != kNumPairClasses * kNumPairClasses)
        return fail(ctx, MOLINTS_ERR_INVALID, "set_class_methods: n must be MOLINTS_NUM_PAIR_CLASSES^2");
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            const int32_t m = methods[x * kNumPairClasses + y] & ~MOLINTS_CLASS_NO_FP32;
            if (m != MOLINTS_METHOD_AUTO && m != MOLINTS_METHOD_HGP && m != MOLINTS_METHOD_RYS)
                return fail(ctx, MOLINTS_ERR_INVALID, "set_class_methods: unknown method");
        }
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) ctx->class_method[x][y] = methods[x * kNumPairClasses + y];
    return MOLINTS_OK;
}

int molints_get_class_methods(const molints_ctx *ctx, int32_t *methods, int32_t n) {
    if (!ctx || !methods || n != kNumPairClasses * kNumPairClasses) return MOLINTS_ERR_INVALID;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y < kNumPairClasses; ++y) methods[x * kNumPairClasses + y] = y <= x ? ctx->class_method[x][y] : 0;
    return MOLINTS_OK;
}

int molints_set_schedule(molints_ctx *ctx, const molints_schedule *s) {
    if (!ctx) return MOLINTS_ERR_INVALID;
    if (!s) {
        ctx->sched = ctx->default_sched;
        return MOLINTS_OK;
    }
    if (!schedule_ok(*s))
        return fail(ctx, MOLINTS_ERR_INVALID,
                    "set_schedule: lane_cost in (0, 1e6], hgp_widen and rys_max_width in [1, 64], rys_chunks >= 1, "
                    "gather_blocks in [0, 16]");
    ctx->sched = *s;
    if (ctx->sched.gather_blocks == 0) ctx->sched.gather_blocks = kGatherBlocksDefault;
    return MOLINTS_OK;
}

int molints_get_schedule(const molints_ctx *ctx, molints_schedule *s) {
    if (!ctx || !s) return MOLINTS_ERR_INVALID;
    *s = ctx->sched;
    return MOLINTS_OK;
}

int molints_set_stream(molints_ctx *ctx, void *stream) {
    if (!ctx) return MOLINTS_ERR_INVALID;
    // NULL selects the context's own stream; the legacy default stream is cudaStreamLegacy.
    cudaStream_t next = stream ? (cudaStream_t)stream : ctx->own_stream;
    if (next != ctx->stream) {
        // what the context left in flight on the old stream (a plan creation returns with its
        // last kernels queued) comes before anything it launches on the new one
        MI_CUDA(ctx, cudaSetDevice(ctx->device));
        MI_CUDA(ctx, cudaEventRecord(ctx->fork, ctx->stream));
        MI_CUDA(ctx, cudaStreamWaitEvent(next, ctx->fork, 0));
    }
    ctx->stream = next;
    return MOLINTS_OK;
}

static BoysTab boys_of(const molints_ctx *ctx, int mode) {
    BoysTab bt;
    bt.tab = ctx->boys_tab;
    bt.scaled = ctx->boys_scaled;
    bt.t_switch = (mode == MOLINTS_BOYS_EXACT) ? kBoysTableMax : kBoysReferenceSwitch;
    return bt;
}

int molints_boys_eval(molints_ctx *ctx, int32_t mode, int32_t mmax, const double *T, int64_t n,
                      double *out) {
    if (!ctx || !T || !out || n < 0 || mmax < 1 || mmax > 16 ||
        (mode != MOLINTS_BOYS_REFERENCE && mode != MOLINTS_BOYS_EXACT))
        return fail(ctx, MOLINTS_ERR_INVALID, "molints_boys_eval: bad argument");
    for (int64_t i = 0; i < n; ++i)
        if (!(T[i] >= 0.0) || !std::isfinite(T[i]))
            return fail(ctx, MOLINTS_ERR_INVALID, "molints_boys_eval: T must be finite and >= 0");
    if (n == 0) return MOLINTS_OK;
    MI_CUDA(ctx, cudaSetDevice(ctx->device));
    double *dT = nullptr, *dout = nullptr;
    int rc = dev_alloc(ctx, &dT, (size_t)n, nullptr);
    if (rc) return rc;
    rc = dev_alloc(ctx, &dout, (size_t)n * mmax, nullptr);
    if (rc) { dev_free(ctx, dT); ctx->held -= n * 8; return rc; }
    cudaError_t e = cudaMemcpyAsync(dT, T, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        boys_eval_kernel<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(boys_of(ctx, mode), mmax,
                                                                               dT, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dout, n * mmax * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, dT);
    dev_free(ctx, dout);
    ctx->held -= (int64_t)(n + n * mmax) * 8;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "molints_boys_eval");
    return MOLINTS_OK;
}

// The plan's CUDA objects and device buffers (stream-ordered frees after its queued work);
// the plan is left orphaned (ctx == nullptr).
static void plan_release_device(molints_plan *p) {
    if (!p || !p->ctx) return;
    if (p->gexec) cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
    for (cudaEvent_t e : p->prof_ev) cudaEventDestroy(e);
    p->prof_ev.clear();
    void *bufs[] = {p->sh_xyz, p->expn, p->ncoef, p->sh_poff, p->pair_ab, p->info, p->pp_src, p->pbk,
                    p->geo, p->pp, p->bnd, p->chunks, p->counters, p->mol_out, p->qcon,
                    p->chunk_slot, p->g_fn, p->g_pair, p->g_region, p->g_mol, p->g_col, p->g_colq,
                    p->g_qmax, p->g_units, p->gq, p->gq_mol, p->sh_L, p->sh_K, p->sh_fn};
    for (void *b : bufs) dev_free(p->ctx, b);
    p->ctx->held -= p->bytes;
    p->ctx = nullptr;
}

static void plan_free(molints_plan *p) {
    if (!p) return;
    if (p->ctx) {
        std::vector<molints_plan *> &v = p->ctx->plans;
        v.erase(std::remove(v.begin(), v.end(), p), v.end());
    }
    plan_release_device(p);
    delete p;
}

int molints_plan_destroy(molints_plan *p) {
    if (!p) return MOLINTS_OK;
    if (p->ctx) cudaSetDevice(p->ctx->device);
    plan_free(p);
    return MOLINTS_OK;
}

// Validate one basis; returns its nprim_tot (>= 0) or a negative status with ctx->err set.
static int check_basis(molints_ctx *ctx, const molints_basis *b, int64_t *nbf_out) {
    const int64_t nbf = molints_nbf(b);
    if (nbf < 0) return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: malformed basis");
    if (nbf > 46000) return fail(ctx, MOLINTS_ERR_UNSUPPORTED, "plan_create: basis too large");
    const int ns = b->nshell;
    if (ns > 0 && (!b->expn || !b->coef)) return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: null primitives");
    int nprim_tot = 0;
    for (int s = 0; s < ns; ++s) {
        if (b->L[s] > MOLINTS_LMAX)
            return fail(ctx, MOLINTS_ERR_UNSUPPORTED,
                        "plan_create: shell angular momentum above " + std::to_string(MOLINTS_LMAX));
        if (b->nprim[s] < 1 || b->prim_off[s] < 0)
            return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: shell without primitives");
        if (b->nprim[s] > 255)
            return fail(ctx, MOLINTS_ERR_UNSUPPORTED, "plan_create: more than 255 primitives in a shell");
        nprim_tot = std::max(nprim_tot, b->prim_off[s] + b->nprim[s]);
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(b->xyz[3 * s + k])) return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: non-finite centre");
    }
    for (int k = 0; k < nprim_tot; ++k)
        if (!(b->expn[k] > 0.0) || !std::isfinite(b->expn[k]) || !std::isfinite(b->coef[k]))
            return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: exponents must be finite and > 0");
    *nbf_out = nbf;
    return nprim_tot;
}

// Shard `shard` of `nshards` of one basis: the shells M in [*s_lo, *s_hi) whose shell quartets
// (those whose highest shell index is M) it computes, and its packed slice [*lo, *hi).  Every
// entry of a quartet has its largest function index in the quartet's highest shell, and the
// entries whose largest function index lies in [f, f') are the contiguous packed range
// [tri(tri(f)), tri(tri(f'))).  Shells are split by an estimate of the quartet cost
// (K_p K_q (1 + L_p)^2 (1 + L_q)^2 per pair product, L_p = la + lb).
static void shard_bounds(const molints_basis *b, int shard, int nshards, int *s_lo, int *s_hi,
                         int64_t *lo, int64_t *hi) {
    const int ns = b->nshell;
    std::vector<double> cost(ns, 0.0);
    double below = 0.0, total = 0.0;
    for (int M = 0; M < ns; ++M) {
        double w = 0.0, w2 = 0.0;
        for (int j = 0; j <= M; ++j) {
            const double c = (double)b->nprim[M] * b->nprim[j] * (1 + b->L[M] + b->L[j]) * (1 + b->L[M] + b->L[j]);
            w += c;
            w2 += c * c;
        }
        cost[M] = w * below + 0.5 * (w * w + w2);
        below += w;
        total += cost[M];
    }
    std::vector<int> S(nshards + 1, ns);
    S[0] = 0;
    double acc = 0.0;
    int r = 1;
    for (int M = 0; M < ns && r < nshards; ++M) {
        acc += cost[M];
        while (r < nshards && acc >= total * r / nshards) S[r++] = M + 1;
    }
    for (int k = 1; k <= nshards; ++k) S[k] = std::max(S[k], S[k - 1]);
    *s_lo = S[shard];
    *s_hi = S[shard + 1];
    auto first_fn = [&](int sh) {
        int64_t f = 0;
        for (int t = 0; t < sh; ++t) f += ncart(b->L[t]);
        return f;
    };
    auto tri = [](int64_t n) { return n * (n + 1) / 2; };
    *lo = tri(tri(first_fn(*s_lo)));
    *hi = tri(tri(first_fn(*s_hi)));
}

// Plan creation synchronises the context's stream once, to read back the device build's
// summary (work-queue sizes), and returns with the work-queue emission in flight on that
// stream: work queued on it afterwards is ordered after it (molints_set_stream orders a new
// stream after the old one).
static int plan_create_impl(molints_ctx *ctx, int32_t nmol, const molints_basis *bases,
                            const molints_options *opts_in, int shard, int nshards,
                            molints_plan **out);

int molints_plan_create_batch(molints_ctx *ctx, int32_t nmol, const molints_basis *bases,
                              const molints_options *opts_in, molints_plan **out) {
    return plan_create_impl(ctx, nmol, bases, opts_in, 0, 1, out);
}

int molints_shard_range(const molints_basis *b, int32_t shard, int32_t nshards, int64_t *lo,
                        int64_t *hi) {
    if (!b || !lo || !hi || nshards < 1 || shard < 0 || shard >= nshards || molints_nbf(b) < 0)
        return MOLINTS_ERR_INVALID;
    int s0, s1;
    shard_bounds(b, shard, nshards, &s0, &s1, lo, hi);
    return MOLINTS_OK;
}

int molints_plan_create_shard(molints_ctx *ctx, const molints_basis *b, const molints_options *opts,
                              int32_t shard, int32_t nshards, molints_plan **out) {
    if (!b || nshards < 1 || shard < 0 || shard >= nshards)
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create_shard: bad argument");
    return plan_create_impl(ctx, 1, b, opts, shard, nshards, out);
}

static int plan_create_impl(molints_ctx *ctx, int32_t nmol, const molints_basis *bases,
                            const molints_options *opts_in, int shard, int nshards,
                            molints_plan **out) {
    if (!ctx || !out || nmol < 0 || (nmol > 0 && !bases))
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: null argument");
    *out = nullptr;
    molints_options opts;
    if (opts_in) opts = *opts_in; else molints_default_options(&opts);
    if (opts.precision != MOLINTS_FP64 && opts.precision != MOLINTS_MIXED)
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: unknown precision");
    if (opts.boys != MOLINTS_BOYS_REFERENCE && opts.boys != MOLINTS_BOYS_EXACT)
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: unknown Boys mode");
    if (opts.method != MOLINTS_METHOD_AUTO && opts.method != MOLINTS_METHOD_HGP &&
        opts.method != MOLINTS_METHOD_RYS)
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: unknown method");
    if (!(opts.fp32_cutoff >= 0.0) || !(opts.screen_cutoff >= 0.0) || !(opts.prim_cutoff >= 0.0))
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: cutoffs must be >= 0");
    if (opts.output != MOLINTS_OUTPUT_AUTO && opts.output != MOLINTS_OUTPUT_DIRECT &&
        opts.output != MOLINTS_OUTPUT_TWO_PHASE)
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: unknown output mode");
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t0) {
        return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    };
    clk::time_point t_phase = clk::now();

    // ---- molecules: validation, output offsets, global shell and primitive arrays
    std::vector<int> shell_off(nmol + 1, 0), prim_base(nmol + 1, 0);
    std::vector<int64_t> mol_nbf(nmol), mol_out(nmol + 1, 0);
    for (int m = 0; m < nmol; ++m) {
        int64_t nbf = 0;
        const int np = check_basis(ctx, &bases[m], &nbf);
        if (np < 0) return np;
        mol_nbf[m] = nbf;
        shell_off[m + 1] = shell_off[m] + bases[m].nshell;
        prim_base[m + 1] = prim_base[m] + np;
        mol_out[m + 1] = mol_out[m] + molints_npacked(nbf);
    }
    const int ns = shell_off[nmol], nprim = prim_base[nmol];
    molints_plan *p = new (std::nothrow) molints_plan();
    if (!p) return MOLINTS_ERR_NOMEM;
    p->ctx = ctx;
    p->opts = opts;
    p->nmol = nmol;
    p->nshell = ns;
    p->npacked = mol_out[nmol];
    p->mol_out_h.assign(mol_out.begin(), mol_out.end() - (nmol > 0 ? 1 : 0));
    int shard_s0 = 0, shard_s1 = 0;
    int64_t shard_lo = 0, shard_hi = 0;
    if (nshards > 1) {
        if (nmol != 1) { delete p; return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: shards need one molecule"); }
        shard_bounds(&bases[0], shard, nshards, &shard_s0, &shard_s1, &shard_lo, &shard_hi);
        p->npacked = shard_hi - shard_lo;
        p->mol_out_h[0] = -shard_lo;  // kernels write out[iindex - lo]
    }
    p->mol_nshell.resize(nmol);
    p->nbf0 = nmol > 0 ? mol_nbf[0] : 0;
    // two-phase output (whole-molecule plans only): AUTO takes it for outputs of at least
    // MOLINTS_TWO_PHASE_MIN integrals (256 MB, twice L2), where the direct stores' sector
    // read-modify-writes cost more than the gather pass; below, the output stays in L2
    p->two_phase = nshards == 1 && nmol > 0 &&
                   (opts.output == MOLINTS_OUTPUT_TWO_PHASE ||
                    (opts.output == MOLINTS_OUTPUT_AUTO && p->npacked >= MOLINTS_TWO_PHASE_MIN));
    // method per class pair: Rys where no HGP kernel exists (an f shell), else the request
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            const int32_t entry = ctx->class_method[x][y];
            int m = opts.method;
            if (m == MOLINTS_METHOD_AUTO) m = entry & ~MOLINTS_CLASS_NO_FP32;
            if (m == MOLINTS_METHOD_AUTO) m = MOLINTS_METHOD_HGP;
            if (!kEriLaunchers[x][y]) m = MOLINTS_METHOD_RYS;
            p->method[x][y] = m;
            // MIXED plans run this class's FP32 variant where the chosen kernel has one, unless
            // the table measured that kernel's FP32 variant no faster (the flag speaks for the
            // table's own method only)
            const bool has32 = m == MOLINTS_METHOD_RYS ? kRysHasFp32[x][y] : kEriHasFp32[x][y];
            const int tm = entry & ~MOLINTS_CLASS_NO_FP32;
            const bool slower32 = (entry & MOLINTS_CLASS_NO_FP32) && (tm == m || tm == MOLINTS_METHOD_AUTO);
            p->fp32[x][y] = opts.precision == MOLINTS_MIXED && has32 && !slower32;
        }

    // Shells of all molecules in one list, primitives in one array (raw coefficients: the
    // device normalises them, normalise_shells_kernel).
    std::vector<double> xyz(3 * (size_t)std::max(ns, 1)), expn(std::max(nprim, 1)), ncoef(std::max(nprim, 1));
    std::vector<int> L(std::max(ns, 1)), K(std::max(ns, 1)), poff(std::max(ns, 1)), fn_off(std::max(ns, 1));
    for (int m = 0; m < nmol; ++m) {
        const molints_basis *b = &bases[m];
        p->mol_nshell[m] = b->nshell;
        int f = 0;
        for (int s = 0; s < b->nshell; ++s) {
            const int g = shell_off[m] + s, p0 = b->prim_off[s], Ks = b->nprim[s], Ls = b->L[s];
            for (int k = 0; k < 3; ++k) xyz[3 * g + k] = b->xyz[3 * s + k];
            L[g] = Ls; K[g] = Ks; poff[g] = prim_base[m] + p0; fn_off[g] = f;
            f += ncart(Ls);
            for (int i = 0; i < Ks; ++i) {
                expn[poff[g] + i] = b->expn[p0 + i];
                ncoef[poff[g] + i] = b->coef[p0 + i];  // raw here; normalised on the device
            }
        }
    }

    // ---- canonical shell pairs of every molecule, ordered by class, molecule, then
    // descending primitive-pair count.  Orientation (A first): the larger L; for equal L, and
    // for an f-d pair, the tighter shell (larger sqrt(min * max exponent)), so that the HRR
    // moves angular momentum away from the tight shell: with a diffuse A and a tight B the
    // pair centre P sits near B and the HRR cancels large terms (up to 1e-6 Eh lost for
    // (ff|ff) with random contractions, measured against the long-double oracle).
    std::vector<double> tight(std::max(ns, 1));
    for (int g = 0; g < ns; ++g) {
        double lo = expn[poff[g]], hi = lo;
        for (int i = 1; i < K[g]; ++i) {
            lo = std::min(lo, expn[poff[g] + i]);
            hi = std::max(hi, expn[poff[g] + i]);
        }
        tight[g] = std::sqrt(lo * hi);
    }
    auto a_first = [&](int x, int y) {  // x should be A of the pair (x, y)
        if (L[x] == L[y] || (L[x] >= 2 && L[y] >= 2 && L[x] + L[y] == 5)) return tight[x] >= tight[y];
        return L[x] > L[y];
    };
    // ms: the pair's higher shell index in its molecule (shard plans order by it so that each
    // bra pair's owned ket pairs are one contiguous run)
    struct PairRec { int cls, mol, npp, a, b, ref, ms; };
    std::vector<PairRec> pr;
    // Shell pairs with a g shell stay out of the class-pair machinery: every shell quartet that
    // holds one goes to the generic kernel, listed here in reference order (I >= J, K >= L,
    // pair IJ >= pair KL).
    std::vector<int4> gq_h;
    std::vector<int> gq_mol_h;
    for (int m = 0; m < nmol; ++m) {
        const int n = bases[m].nshell, s0 = shell_off[m];
        bool has_g = false;
        for (int i = 0; i < n; ++i) has_g = has_g || L[s0 + i] > kLmax;
        if (has_g && nshards > 1) {
            plan_free(p);
            return fail(ctx, MOLINTS_ERR_UNSUPPORTED, "plan_create_shard: g shells are not sharded");
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j <= i; ++j) {
                int a = s0 + i, bb = s0 + j;
                const bool g_ij = L[a] > kLmax || L[bb] > kLmax;
                if (g_ij || has_g) {
                    for (int k = 0; k <= i; ++k)
                        for (int l = 0; l <= (k == i ? j : k); ++l)
                            if (g_ij || L[s0 + k] > kLmax || L[s0 + l] > kLmax) {
                                gq_h.push_back(make_int4(a, bb, s0 + k, s0 + l));
                                gq_mol_h.push_back(m);
                            }
                }
                if (g_ij) continue;
                if (!a_first(a, bb)) std::swap(a, bb);
                pr.push_back({pair_class_of(L[a], L[bb]), m, K[a] * K[bb], a, bb, i * (i + 1) / 2 + j, i});
            }
    }
    p->n_gq = (int64_t)gq_h.size();
    if (p->n_gq > 0) p->two_phase = 0;  // the gather would overwrite the generic kernel's entries
    const bool sharded = nshards > 1;
    {
        // list order: class, molecule, (shard plans) highest shell, then primitive pairs
        // descending; enumeration order among equals.  One stable radix pass per key byte.
        int maxnpp = 0, maxms = 0;
        for (const PairRec &r : pr) {
            maxnpp = std::max(maxnpp, r.npp);
            maxms = std::max(maxms, r.ms);
        }
        const int bn = bits_for((uint64_t)maxnpp), bs = sharded ? bits_for((uint64_t)maxms) : 0;
        const int bm = bits_for((uint64_t)std::max(nmol - 1, 0)), bc = bits_for(kNumPairClasses - 1);
        std::vector<uint64_t> key(pr.size());
        for (size_t k = 0; k < pr.size(); ++k) {
            const PairRec &r = pr[k];
            key[k] = ((((uint64_t)r.cls << bm | (uint64_t)r.mol) << bs | (uint64_t)(sharded ? r.ms : 0)) << bn) |
                     (uint64_t)(maxnpp - r.npp);
        }
        const std::vector<uint32_t> ord = radix_order(key, bc + bm + bs + bn);  // <= 4 + 31 + 31 + 16 bits
        std::vector<PairRec> sorted(pr.size());
        for (size_t k = 0; k < pr.size(); ++k) sorted[k] = pr[ord[k]];
        pr.swap(sorted);
    }
    const int npair = (int)pr.size();
    p->npair = npair;

    // ---- stage-1 pair tables (every primitive pair, list order) and the host-side structure
    // of the list: class runs, and per (class, molecule) the molecule's run in the class (the
    // pairs of a class are in molecule order)
    std::vector<int> cls_start(kNumPairClasses + 1, 0);
    int64_t nall = 0;
    for (int k = 0; k < npair; ++k) nall += (int64_t)K[pr[k].a] * K[pr[k].b];
    if (nall >= INT32_MAX) { plan_free(p); return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: too many primitive pairs"); }
    p->nprim_pair_all = nall;
    p->pair_mol.resize(npair);
    for (int k = 0; k < npair; ++k) {
        p->pair_mol[k] = pr[k].mol;
        cls_start[pr[k].cls + 1] = k + 1;
    }
    for (int c = 1; c <= kNumPairClasses; ++c) cls_start[c] = std::max(cls_start[c], cls_start[c - 1]);
    for (int c = 0; c <= kNumPairClasses; ++c) p->class_start[c] = cls_start[c];
    const int cm_stride = nmol + 1;
    std::vector<int> cm_start((size_t)kNumPairClasses * cm_stride);
    for (int c = 0; c < kNumPairClasses; ++c) {
        int k = cls_start[c];
        for (int m = 0; m < nmol; ++m) {
            cm_start[(size_t)c * cm_stride + m] = k;
            while (k < cls_start[c + 1] && pr[k].mol == m) ++k;
        }
        cm_start[(size_t)c * cm_stride + nmol] = cls_start[c + 1];
    }
    auto range_of = [&](int cls, int m, int &b0, int &b1) {
        b0 = cm_start[(size_t)cls * cm_stride + m];
        b1 = cm_start[(size_t)cls * cm_stride + m + 1];
    };

    // ---- work-queue shape per class pair: chunks of one bra pair and <= 32 ket pairs of the
    // same molecule, widened in steps of 32 for large batches so that the queues stay near
    // kMaxChunks entries
    constexpr double kMaxChunks = 4.0e6;
    double nchunk32 = 0.0;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y)
            for (int m = 0; m < nmol; ++m) {
                int b0, b1, k0, k1;
                range_of(x, m, b0, b1);
                range_of(y, m, k0, k1);
                const double nb = b1 - b0, nk = k1 - k0;
                nchunk32 += (x == y) ? nb * (nb + 1) / 64.0 + nb : nb * (nk / 32.0 + 1.0);
            }
    const int widen = std::max(1, (int)std::ceil(nchunk32 / kMaxChunks));
    const int hgp_widen = std::max(widen, (int)ctx->sched.hgp_widen);
    // A Rys group computes a chunk's quartets one after another.  Its chunks are as long as
    // keeps about rys_chunks chunks in the class queue (1..rys_max_width ket pairs): the large
    // classes have few quartets (e.g. 231 (ff|ff) quartets for six f shells) and need one group
    // per quartet, while the many small quartets of the low classes amortise the queue atomic.
    const double rys_chunks = ctx->sched.rys_chunks;
    const int rys_max_width = ctx->sched.rys_max_width;
    auto rys_width = [&](int x, int y) {
        double nq = 0.0;
        for (int m = 0; m < nmol; ++m) {
            int b0, b1, k0, k1;
            range_of(x, m, b0, b1);
            range_of(y, m, k0, k1);
            const double nb = b1 - b0, nk = k1 - k0;
            nq += (x == y) ? nb * (nb + 1) / 2 : nb * nk;
        }
        return std::max(1, std::min(rys_max_width, (int)(nq / rys_chunks)));
    };
    QueueSetup S{};
    {
        int ci = 0, items = 0;
        for (int x = 0; x < kNumPairClasses; ++x)
            for (int y = 0; y <= x; ++y, ++ci) {
                const bool hgp = p->method[x][y] != MOLINTS_METHOD_RYS;
                const int lsum = kPairClassLa[x] + kPairClassLb[x] + kPairClassLa[y] + kPairClassLb[y];
                S.item_base[ci] = items;
                S.cx[ci] = x;
                S.cy[ci] = y;
                S.hgp[ci] = hgp;
                S.width[ci] = hgp ? 32 * hgp_widen : rys_width(x, y) * widen;
                S.pcost[ci] = (double)kEriPrimCost[x][y];
                S.w[ci] = 1.0 + lsum * lsum;
                items += cls_start[x + 1] - cls_start[x];
            }
        S.item_base[kNumClassPairs] = items;
        for (int c = 0; c <= kNumPairClasses; ++c) S.cls_start[c] = cls_start[c];
        S.nmol = nmol;
        S.widen = hgp_widen;
        S.lane_cost = ctx->sched.lane_cost;
        p->gather_blocks = ctx->sched.gather_blocks;
        S.sharded = sharded;
        S.shard_s0 = shard_s0;
        S.shard_s1 = shard_s1;
        for (int c = 0; c < kNumPairClasses; ++c) {
            // shard plans (one molecule): a class's pairs are in highest-shell order
            auto first_ms_at_least = [&](int v) {
                return (int)(std::partition_point(pr.begin() + cls_start[c], pr.begin() + cls_start[c + 1],
                                                  [v](const PairRec &r) { return r.ms < v; }) -
                             pr.begin());
            };
            S.ps0[c] = sharded ? first_ms_at_least(shard_s0) : 0;
            S.ps1[c] = sharded ? first_ms_at_least(shard_s1) : 0;
        }
    }
    const int n_items = S.item_base[kNumClassPairs];

    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) { plan_free(p); return cuda_fail(ctx, e, "cudaSetDevice"); }

    // ---- two-phase scratch: per (class pair, molecule) a region of quartet blocks in slot order,
    // bra-major (the triangle q <= p for equal classes); region_h[((x nc + y) nmol + m) 4 ..] =
    // {offset in doubles, first bra pair, first ket pair, ket pairs}.  Quartet slot t's block
    // starts at offset + t * block.
    if (npair >= (1 << 26)) p->two_phase = 0;  // the gather's pair entries hold the position in 26 bits
    auto ncomp_of = [](int x, int y) {
        return (int64_t)ncart(kPairClassLa[x]) * ncart(kPairClassLb[x]) * ncart(kPairClassLa[y]) * ncart(kPairClassLb[y]);
    };
    std::vector<long long> region_h;
    int64_t scratch_len = 0;
    if (p->two_phase) {
        region_h.assign((size_t)kNumPairClasses * kNumPairClasses * nmol * kRegionFields, 0);
        for (int x = 0; x < kNumPairClasses; ++x)
            for (int y = 0; y <= x; ++y)
                for (int m = 0; m < nmol; ++m) {
                    int b0, b1, k0, k1;
                    range_of(x, m, b0, b1);
                    range_of(y, m, k0, k1);
                    const int64_t nb = b1 - b0, nk = k1 - k0;
                    long long *rg = &region_h[(((size_t)x * kNumPairClasses + y) * nmol + m) * kRegionFields];
                    rg[0] = scratch_len;
                    rg[1] = b0;
                    rg[2] = k0;
                    rg[3] = nk;
                    scratch_len += (x == y ? nb * (nb + 1) / 2 : nb * nk) * ncomp_of(x, y);
                }
        // The scratch (about npacked doubles) is taken now.  If it does not fit the budget or
        // the device, AUTO falls back to the direct stores, which need no scratch; only an
        // explicit MOLINTS_OUTPUT_TWO_PHASE fails.
        int src = ctx_scratch(ctx, scratch_len);
        if (src && opts.output == MOLINTS_OUTPUT_AUTO) {
            cudaGetLastError();  // an out-of-memory status is not sticky; clear it
            p->two_phase = 0;
            region_h.clear();
            scratch_len = 0;
            ctx->err.clear();
        } else if (src) {
            plan_free(p);
            return src;
        }
        p->scratch_need = scratch_len;
    }
    const bool tp = p->two_phase != 0;
    S.two_phase = tp;
    S.screen_sort = !sharded && opts.screen_cutoff > 0.0;
    S.screen_trunc = S.screen_sort;
    p->screen_trunc = S.screen_trunc;
    S.screen_cut = opts.screen_cutoff;

    // ---- pinned upload buffer: the summary read back after the device build, the plan's
    // shells, the stage-1 block (laid out as in the device temporaries, one copy), the molecule
    // offsets and the gather tables
    int64_t nfn_all = 0, npe_all = 0, nrows_all = 0;
    for (int m = 0; m < nmol; ++m) {
        nfn_all += mol_nbf[m];
        npe_all += (int64_t)bases[m].nshell * (bases[m].nshell + 1) / 2;
        nrows_all += mol_nbf[m] * (mol_nbf[m] + 1) / 2;
    }
    // device temporaries of the build; the stage-1 block comes first
    Carve tv;
    const size_t t_ab1 = tv.take<int2>(npair), t_info1 = tv.take<int4>(npair), t_rec1 = tv.take<int4>(npair);
    const size_t t_seg1 = tv.take<int>(npair), t_mol1 = tv.take<int>(npair);
    const size_t t_cm = tv.take<int>(cm_start.size());
    const size_t up_bytes = tv.at;
    const size_t t_src1 = tv.take<int>(nall);
    const size_t t_pbound = tv.take<double2>(nall), t_qmax = tv.take<unsigned long long>(nmol);
    const size_t t_npp1 = tv.take<int>(npair), t_bnd1 = tv.take<double2>(npair);
    const size_t t_key1 = tv.take<unsigned long long>(npair), t_key2 = tv.take<unsigned long long>(npair);
    const size_t t_idx1 = tv.take<int>(npair), t_idx2 = tv.take<int>(npair);
    const size_t t_prefix = tv.take<long long>((size_t)npair + 1), t_npp = tv.take<int>((size_t)npair + 1);
    const size_t t_ms = tv.take<int>(npair);
    const size_t t_cnt = tv.take<long long>((size_t)n_items + 1), t_cost = tv.take<double>(n_items);
    const size_t t_off = tv.take<long long>((size_t)n_items + 1);
    const size_t t_sum = tv.take<long long>(kNumClassPairs + 1), t_ccost = tv.take<double>(kNumClassPairs);
    const size_t cub_bytes = std::max(plan_build_temp_bytes(npair), queue_count_temp_bytes(n_items));
    const size_t t_cub = tv.take<char>(cub_bytes);
    Carve sv;
    // read back: class-pair chunk offsets, class-pair costs, kept primitive pairs, bad-shell flag
    const size_t o_sum = sv.take<long long>(kNumClassPairs + 1), o_ccost = sv.take<double>(kNumClassPairs);
    const size_t o_nkept = sv.take<long long>(1), o_bad = sv.take<int>(1);
    const size_t o_up = sv.take<char>(up_bytes);
    const size_t o_xyz = sv.take<double>(3 * (size_t)ns), o_expn = sv.take<double>(nprim);
    const size_t o_coef = sv.take<double>(nprim), o_poff = sv.take<int>(ns), o_L = sv.take<int>(ns);
    const size_t o_K = sv.take<int>(ns), o_mol = sv.take<long long>(nmol);
    const size_t o_greg = sv.take<long long>(tp ? region_h.size() : 0), o_gfn = sv.take<int2>(tp ? nfn_all : 0);
    const size_t o_gmol = sv.take<long long>(tp ? (size_t)nmol * 4 : 0);
    const size_t o_gunits = sv.take<int4>(tp ? npe_all : 0);
    int rc = ctx_stage(ctx, sv.at);
    if (rc) { plan_free(p); return rc; }
    char *stage = ctx->stage;
    {
        char *up = stage + o_up;
        int2 *ab1 = reinterpret_cast<int2 *>(up + t_ab1);
        int4 *info1 = reinterpret_cast<int4 *>(up + t_info1), *rec1 = reinterpret_cast<int4 *>(up + t_rec1);
        int *seg1 = reinterpret_cast<int *>(up + t_seg1), *mol1 = reinterpret_cast<int *>(up + t_mol1);
        int off = 0;  // the primitive pairs themselves are listed on the device (plan_stage1_src)
        for (int k = 0; k < npair; ++k) {
            const PairRec &r = pr[k];
            const int m = r.mol;
            ab1[k] = make_int2(r.a, r.b);
            info1[k] = make_int4(off, r.npp, fn_off[r.a], fn_off[r.b]);
            off += r.npp;
            const int swapped = (r.a - shell_off[m]) != r.ms;  // A is the lower shell J
            rec1[k] = make_int4(m, r.ref, r.cls | (swapped << 8), r.ms);
            // the pair's run of equal (class, molecule[, ms]): the re-sort by kept count stays in it
            const bool same = k > 0 && pr[k - 1].cls == r.cls && pr[k - 1].mol == m && (!sharded || pr[k - 1].ms == r.ms);
            seg1[k] = same ? seg1[k - 1] : k;
            mol1[k] = m;
        }
        std::memcpy(up + t_cm, cm_start.data(), cm_start.size() * sizeof(int));
    }
    std::memcpy(stage + o_xyz, xyz.data(), 3 * (size_t)ns * sizeof(double));
    std::memcpy(stage + o_expn, expn.data(), (size_t)nprim * sizeof(double));
    std::memcpy(stage + o_coef, ncoef.data(), (size_t)nprim * sizeof(double));
    std::memcpy(stage + o_poff, poff.data(), (size_t)ns * sizeof(int));
    std::memcpy(stage + o_L, L.data(), (size_t)ns * sizeof(int));
    std::memcpy(stage + o_K, K.data(), (size_t)ns * sizeof(int));
    {
        long long *mol_out_ll = reinterpret_cast<long long *>(stage + o_mol);
        mol_out_ll[0] = 0;
        for (int m = 0; m < nmol; ++m) mol_out_ll[m] = (long long)p->mol_out_h[m];
    }
    if (tp) {
        std::memcpy(stage + o_greg, region_h.data(), region_h.size() * sizeof(long long));
        int2 *gfn = reinterpret_cast<int2 *>(stage + o_gfn);
        long long *gmol = reinterpret_cast<long long *>(stage + o_gmol);
        long long cbase = 0, pbase = 0;
        for (int m = 0, fb = 0; m < nmol; ++m) {
            for (int sl = 0; sl < bases[m].nshell; ++sl) {
                const int g = shell_off[m] + sl;
                for (int c = 0; c < ncart(L[g]); ++c) gfn[fb + fn_off[g] + c] = make_int2(sl, c);
            }
            gmol[4 * m] = fb;
            gmol[4 * m + 1] = pbase;
            gmol[4 * m + 2] = (long long)p->mol_out_h[m];
            gmol[4 * m + 3] = cbase;
            pbase += (int64_t)bases[m].nshell * (bases[m].nshell + 1) / 2;
            cbase += mol_nbf[m] * (mol_nbf[m] + 1) / 2;
            fb += (int)mol_nbf[m];
        }
        // gather units: every shell pair I >= J of every molecule, heaviest first (rows x the
        // last row's columns), so that the big pairs do not finish last
        int4 *gu = reinterpret_cast<int4 *>(stage + o_gunits);
        std::vector<std::pair<double, int64_t>> wk;
        wk.reserve((size_t)npe_all);
        std::vector<int4> u_h;
        u_h.reserve((size_t)npe_all);
        for (int m = 0; m < nmol; ++m)
            for (int I = 0; I < bases[m].nshell; ++I)
                for (int J = 0; J <= I; ++J) {
                    const int gI = shell_off[m] + I, gJ = shell_off[m] + J;
                    const int nI = ncart(L[gI]), nJ = ncart(L[gJ]);
                    const int64_t li = fn_off[gI] + nI - 1, lj = I == J ? li : fn_off[gJ] + nJ - 1;
                    const double rows = I == J ? nI * (nI + 1) / 2.0 : (double)nI * nJ;
                    wk.push_back({rows * (double)(li * (li + 1) / 2 + lj + 1), (int64_t)u_h.size()});
                    u_h.push_back(make_int4(m, fn_off[gI], fn_off[gJ], nI | (nJ << 8) | ((I == J) << 16)));
                }
        // by weight descending at float precision (24 bits: exponent and 15 mantissa bits), list
        // order among equals
        std::vector<uint64_t> wkey(wk.size());
        for (size_t k = 0; k < wk.size(); ++k) {
            const float f = (float)wk[k].first;
            uint32_t fb;
            std::memcpy(&fb, &f, sizeof fb);
            wkey[k] = (uint64_t)((1u << 24) - 1 - (fb >> 7));
        }
        const std::vector<uint32_t> word = radix_order(wkey, 24);
        for (size_t k = 0; k < wk.size(); ++k) gu[k] = u_h[wk[word[k]].second];
        p->n_units = (int64_t)wk.size();
    }
    p->plan_ms[0] = ms_since(t_phase);
    t_phase = clk::now();

    // ---- device: plan buffers, uploads, normalisation, bound pass, then the device build
    const int nc2 = kNumPairClasses * kNumPairClasses;
    rc = rc ? rc : dev_alloc(ctx, &p->sh_xyz, (size_t)3 * ns, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->expn, (size_t)nprim, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->ncoef, (size_t)nprim, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->sh_poff, (size_t)ns, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->sh_L, (size_t)ns, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->sh_K, (size_t)ns, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->pair_ab, (size_t)npair, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->info, (size_t)npair, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->geo, (size_t)npair, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->bnd, (size_t)npair, &p->bytes);
    // kept primitive pairs: at most nall (the count is known on the device only)
    rc = rc ? rc : dev_alloc(ctx, &p->pp_src, (size_t)nall, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->pbk, (size_t)nall, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->pp, (size_t)nall, &p->bytes);
    rc = rc ? rc : dev_alloc(ctx, &p->counters, (size_t)nc2 + 1, &p->bytes);  // + the gather's
    rc = rc ? rc : dev_alloc(ctx, &p->mol_out, (size_t)std::max(nmol, 1), &p->bytes);
    if (tp) {
        rc = rc ? rc : dev_alloc(ctx, &p->g_fn, (size_t)std::max<int64_t>(nfn_all, 1), &p->bytes);
        rc = rc ? rc : dev_alloc(ctx, &p->g_pair, (size_t)std::max<int64_t>(npe_all, 1), &p->bytes);
        rc = rc ? rc : dev_alloc(ctx, &p->g_region, region_h.size(), &p->bytes);
        rc = rc ? rc : dev_alloc(ctx, &p->g_mol, (size_t)nmol * 4, &p->bytes);
        rc = rc ? rc : dev_alloc(ctx, &p->g_col, (size_t)std::max<int64_t>(nrows_all, 1), &p->bytes);
        if (opts.screen_cutoff > 0.0) {
            rc = rc ? rc : dev_alloc(ctx, &p->g_colq, (size_t)std::max<int64_t>(nrows_all, 1), &p->bytes);
            rc = rc ? rc : dev_alloc(ctx, &p->g_qmax, (size_t)std::max(nmol, 1), &p->bytes);
        }
        rc = rc ? rc : dev_alloc(ctx, &p->g_units, (size_t)std::max<int64_t>(npe_all, 1), &p->bytes);
    }
    int64_t temp_tally = 0;
    char *tmp = nullptr;
    rc = rc ? rc : dev_alloc(ctx, &tmp, tv.at, &temp_tally);
    auto release_temp = [&]() {
        if (tmp) dev_free(ctx, tmp);
        ctx->held -= temp_tally;
        tmp = nullptr;
        temp_tally = 0;
    };
    if (rc) { release_temp(); plan_free(p); return rc; }
    cudaStream_t s = ctx->stream;
    auto h2d = [&](void *dst, size_t off, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, stage + off, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
    };
    if ((e = h2d(tmp, o_up, up_bytes)) ||
        (e = h2d(p->sh_xyz, o_xyz, 3 * (size_t)ns * sizeof(double))) ||
        (e = h2d(p->expn, o_expn, (size_t)nprim * sizeof(double))) ||
        (e = h2d(p->ncoef, o_coef, (size_t)nprim * sizeof(double))) ||
        (e = h2d(p->sh_poff, o_poff, (size_t)ns * sizeof(int))) ||
        (e = h2d(p->sh_L, o_L, (size_t)ns * sizeof(int))) ||
        (e = h2d(p->sh_K, o_K, (size_t)ns * sizeof(int))) ||
        (e = h2d(p->mol_out, o_mol, (size_t)nmol * sizeof(long long))) ||
        (tp && ((e = h2d(p->g_region, o_greg, region_h.size() * sizeof(long long))) ||
                (e = h2d(p->g_fn, o_gfn, (size_t)nfn_all * sizeof(int2))) ||
                (e = h2d(p->g_mol, o_gmol, (size_t)nmol * 4 * sizeof(long long))) ||
                (e = h2d(p->g_units, o_gunits, (size_t)npe_all * sizeof(int4))))) ||
        (e = cudaMemsetAsync(p->counters + nc2, 0, sizeof(int), s)) ||
        (e = cudaMemsetAsync(tmp + t_qmax, 0, (size_t)std::max(nmol, 1) * sizeof(unsigned long long), s)) ||
        (e = cudaMemsetAsync(tmp + t_sum, 0, (kNumClassPairs + 1) * sizeof(long long), s)) ||
        (e = cudaMemsetAsync(tmp + t_ccost, 0, kNumClassPairs * sizeof(double), s)) ||
        (e = cudaMemsetAsync(tmp + t_prefix, 0, sizeof(long long), s))) {
        release_temp(); plan_free(p);
        return cuda_fail(ctx, e, "plan_create upload");
    }
    // the raw coefficients become normalised ones in place; a shell with no positive
    // self-overlap flags counters[nc2] (read back with the summary)
    if (ns > 0)
        normalise_shells_kernel<<<(ns + 127) / 128, 128, 0, s>>>(ns, p->sh_L, p->sh_K, p->sh_poff, p->expn,
                                                                 p->ncoef, p->counters + nc2);
    PlanBuildArgs A{};
    A.npair = npair;
    A.nall = (int)nall;
    A.prim_cutoff = opts.prim_cutoff;
    A.screen_sort = S.screen_sort;
    A.ab1 = reinterpret_cast<const int2 *>(tmp + t_ab1);
    A.info1 = reinterpret_cast<const int4 *>(tmp + t_info1);
    A.src1 = reinterpret_cast<const int *>(tmp + t_src1);
    A.rec1 = reinterpret_cast<const int4 *>(tmp + t_rec1);
    A.seg1 = reinterpret_cast<const int *>(tmp + t_seg1);
    A.pbound = reinterpret_cast<const double2 *>(tmp + t_pbound);
    A.xyz = p->sh_xyz;
    A.sh_L = p->sh_L;
    A.qmax = reinterpret_cast<unsigned long long *>(tmp + t_qmax);
    A.npp1 = reinterpret_cast<int *>(tmp + t_npp1);
    A.bnd1 = reinterpret_cast<double2 *>(tmp + t_bnd1);
    A.key1 = reinterpret_cast<unsigned long long *>(tmp + t_key1);
    A.key2 = reinterpret_cast<unsigned long long *>(tmp + t_key2);
    A.idx1 = reinterpret_cast<int *>(tmp + t_idx1);
    A.idx2 = reinterpret_cast<int *>(tmp + t_idx2);
    A.npp_prefix = reinterpret_cast<long long *>(tmp + t_prefix);
    A.npp = reinterpret_cast<int *>(tmp + t_npp);
    A.ms = reinterpret_cast<int *>(tmp + t_ms);
    A.pair_ab = p->pair_ab;
    A.info = p->info;
    A.bnd = p->bnd;
    A.pp_src = p->pp_src;
    A.pbk = p->pbk;
    A.g_pair = tp ? p->g_pair : nullptr;
    A.g_mol = tp ? p->g_mol : nullptr;
    QueueArgs QA{};
    QA.n_items = n_items;
    QA.npp = A.npp;
    QA.mol = reinterpret_cast<const int *>(tmp + t_mol1);
    QA.cm_start = reinterpret_cast<const int *>(tmp + t_cm);
    QA.ms = A.ms;
    QA.npp_prefix = A.npp_prefix;
    QA.region = tp ? p->g_region : nullptr;
    QA.bnd = p->bnd;
    QA.cnt = reinterpret_cast<long long *>(tmp + t_cnt);
    QA.cost = reinterpret_cast<double *>(tmp + t_cost);
    QA.off = reinterpret_cast<long long *>(tmp + t_off);
    QA.summary = reinterpret_cast<long long *>(tmp + t_sum);
    QA.class_cost = reinterpret_cast<double *>(tmp + t_ccost);
    if (npair > 0) {
        const double c0 = std::sqrt(2.0) * std::pow(M_PI, 1.25);
        if ((e = plan_stage1_src(npair, A.ab1, A.info1, p->sh_K, const_cast<int *>(A.src1), s))) {
            release_temp(); plan_free(p);
            return cuda_fail(ctx, e, "plan_create pair list");
        }
        build_pairs_kernel<<<build_pairs_blocks(npair), 128, 0, s>>>(npair, A.ab1, A.info1, A.src1, p->sh_xyz,
                                                                     p->sh_poff, p->expn, p->ncoef, c0, nullptr,
                                                                     p->pp, p->geo);
        PairTab P1{A.info1, p->geo, p->pp, p->bnd};
        BoysTab Bt = boys_of(ctx, opts.boys);
        double2 *pbound = reinterpret_cast<double2 *>(tmp + t_pbound);
        for (int c = 0; c < kNumPairClasses; ++c) {
            const int n = cls_start[c + 1] - cls_start[c];
            if (kSchwarzLaunchers[c]) kSchwarzLaunchers[c](P1, Bt, cls_start[c], n, pbound, nullptr, 0, s);
            else kRysBoundLaunchers[c](P1, ctx->rys, cls_start[c], n, pbound, nullptr, 0, s);
        }
        if ((e = cudaGetLastError()) || (e = plan_build_pairs(A, tmp + t_cub, cub_bytes, s)) ||
            (e = queue_count(S, QA, tmp + t_cub, cub_bytes, s))) {
            release_temp(); plan_free(p);
            return cuda_fail(ctx, e, "plan_create device build");
        }
    }
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(stage + o_sum, tmp + t_sum, (kNumClassPairs + 1) * sizeof(long long),
                             cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(stage + o_ccost, tmp + t_ccost, kNumClassPairs * sizeof(double),
                             cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(stage + o_nkept, A.npp_prefix + npair, sizeof(long long), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(stage + o_bad, p->counters + nc2, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s))) {
        release_temp(); plan_free(p);
        return cuda_fail(ctx, e, "plan_create bound pass");
    }
    if (*reinterpret_cast<const int *>(stage + o_bad)) {
        release_temp(); plan_free(p);
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: zero contracted function");
    }
    const long long *qsum = reinterpret_cast<const long long *>(stage + o_sum);
    const double *qcost = reinterpret_cast<const double *>(stage + o_ccost);
    p->nprim_pair_kept = *reinterpret_cast<const long long *>(stage + o_nkept);
    const long long nq = qsum[kNumClassPairs];
    if (nq > INT32_MAX) {
        release_temp(); plan_free(p);
        return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: work queue too long");
    }
    for (int ci = 0; ci < kNumClassPairs; ++ci) {
        const int x = S.cx[ci], y = S.cy[ci];
        p->q_off[x][y] = (int)qsum[ci];
        p->q_len[x][y] = (int)(qsum[ci + 1] - qsum[ci]);
        p->class_cost[x][y] = qcost[ci];
    }
    p->plan_ms[1] = ms_since(t_phase);
    t_phase = clk::now();

    // ---- the chunks, emitted in (class pair, bra, ket) order and placed by a stable sort on
    // (class pair, cost bucket): class pairs in order, heaviest bucket first
    rc = dev_alloc(ctx, &p->chunks, (size_t)std::max<long long>(nq, 1), &p->bytes);
    if (!rc && tp) rc = dev_alloc(ctx, &p->chunk_slot, (size_t)std::max<long long>(nq, 1), &p->bytes);
    Carve ev;
    const size_t e_raw = ev.take<int4>(nq), e_key1 = ev.take<unsigned short>(nq), e_key2 = ev.take<unsigned short>(nq);
    const size_t e_idx1 = ev.take<int>(nq), e_idx2 = ev.take<int>(nq), e_slot = ev.take<long long>(tp ? nq : 0);
    const size_t emit_cub = queue_emit_temp_bytes(nq);
    const size_t e_cub = ev.take<char>(emit_cub);
    char *etmp = nullptr;
    if (!rc && nq > 0) rc = dev_alloc(ctx, &etmp, ev.at, &temp_tally);
    if (rc) { release_temp(); plan_free(p); return rc; }
    if (nq > 0) {
        QueueEmitArgs E{};
        E.raw = reinterpret_cast<int4 *>(etmp + e_raw);
        E.key1 = reinterpret_cast<unsigned short *>(etmp + e_key1);
        E.key2 = reinterpret_cast<unsigned short *>(etmp + e_key2);
        E.idx1 = reinterpret_cast<int *>(etmp + e_idx1);
        E.idx2 = reinterpret_cast<int *>(etmp + e_idx2);
        E.raw_slot = tp ? reinterpret_cast<long long *>(etmp + e_slot) : nullptr;
        E.chunks = p->chunks;
        E.chunk_slot = tp ? p->chunk_slot : nullptr;
        E.nq = nq;
        e = queue_emit(S, QA, E, etmp + e_cub, emit_cub, s);
        dev_free(ctx, etmp);
        if (e != cudaSuccess) { release_temp(); plan_free(p); return cuda_fail(ctx, e, "plan_create work queues"); }
    }
    if (tp && nrows_all > 0) {
        gather_cols_kernel<<<(unsigned)((nrows_all + 255) / 256), 256, 0, s>>>(p->g_col, p->g_colq, p->bnd,
                                                                            p->g_fn, p->g_pair,
                                                                            p->g_mol, nmol, nrows_all);
        e = cudaGetLastError();
        if (!e && p->g_qmax)  // the molecules' Qabs bounds (doubles as bits) outlive the build
            e = cudaMemcpyAsync(p->g_qmax, tmp + t_qmax, (size_t)nmol * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (e) { release_temp(); plan_free(p); return cuda_fail(ctx, e, "plan_create gather columns"); }
    }
    release_temp();
    p->plan_ms[2] = ms_since(t_phase);
    t_phase = clk::now();
    if ((e = cudaGetLastError())) {
        plan_free(p);
        return cuda_fail(ctx, e, "plan_create work queues");
    }
    if (p->n_gq > 0) {
        // the generic kernel's shell data and quartet list (pageable sources: each copy is
        // staged before the call returns)
        rc = dev_alloc(ctx, &p->gq, (size_t)p->n_gq, &p->bytes);
        if (!rc) rc = dev_alloc(ctx, &p->gq_mol, (size_t)p->n_gq, &p->bytes);
        if (!rc) rc = dev_alloc(ctx, &p->sh_fn, (size_t)ns, &p->bytes);
        if (rc) { plan_free(p); return rc; }
        if ((e = cudaMemcpyAsync(p->gq, gq_h.data(), gq_h.size() * sizeof(int4), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(p->gq_mol, gq_mol_h.data(), gq_mol_h.size() * sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(p->sh_fn, fn_off.data(), (size_t)ns * sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaStreamSynchronize(s))) {
            plan_free(p);
            return cuda_fail(ctx, e, "plan_create upload (g shells)");
        }
    }
    p->plan_ms[3] = ms_since(t_phase);
    ctx->plans.push_back(p);
    *out = p;
    return MOLINTS_OK;
}

int molints_plan_create(molints_ctx *ctx, const molints_basis *b, const molints_options *opts,
                        molints_plan **out) {
    if (!b) return fail(ctx, MOLINTS_ERR_INVALID, "plan_create: null argument");
    return molints_plan_create_batch(ctx, 1, b, opts, out);
}

int64_t molints_plan_npacked(const molints_plan *p) { return p ? p->npacked : MOLINTS_ERR_INVALID; }

// Queue the device path of one execute on the context's stream (side streams forked from it
// and joined back).  timing: record the context's ev0/ev1 around it (not inside a graph).
static int plan_enqueue(molints_plan *p, double *out_device, bool timing, JKOut jk = JKOut{}) {
    molints_ctx *ctx = p->ctx;
    cudaStream_t s = ctx->stream;
    int launches = 0;
    // event pair around each launch when profiling (launch k uses events 2k, 2k+1)
    auto mark = [&](int k, const char *name, int end, cudaStream_t st) -> int {
        if (!p->profiling) return 0;
        while ((int)p->prof_ev.size() < 2 * k + 2) {
            cudaEvent_t e;
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return cuda_fail(ctx, err, "cudaEventCreate");
            p->prof_ev.push_back(e);
        }
        if ((int)p->prof_name.size() < k + 1) p->prof_name.resize(k + 1);
        p->prof_name[k] = name;
        cudaError_t err = cudaEventRecord(p->prof_ev[2 * k + end], st);
        return err == cudaSuccess ? 0 : cuda_fail(ctx, err, "cudaEventRecord");
    };
    if (timing) MI_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
    MI_CUDA(ctx, cudaMemsetAsync(p->counters, 0, sizeof(int) * (kNumPairClasses * kNumPairClasses + 1), s));
    // direct plans that screen quartets: the screened quartets past each bra's last unscreened
    // ket are in no chunk, so their zeros come from clearing the whole output first (a
    // streaming write instead of scattered 8-byte stores).  Two-phase plans' gather writes them
    // (measured on B200: clearing first and leaving them out of the gather cost more than the
    // gather's zero stores, which are coalesced)
    if (p->screen_trunc && !p->two_phase && !jk.J && p->npacked > 0)
        MI_CUDA(ctx, cudaMemsetAsync(out_device, 0, (size_t)p->npacked * sizeof(double), s));
    if (p->npair > 0) {
        if (int rc = mark(launches, "build_pairs", 0, s)) return rc;
        build_pairs_kernel<<<build_pairs_blocks(p->npair), 128, 0, s>>>(
            p->npair, p->pair_ab, p->info, p->pp_src, p->sh_xyz, p->sh_poff, p->expn, p->ncoef,
            std::sqrt(2.0) * std::pow(M_PI, 1.25), p->pbk, p->pp, p->geo);
        if (int rc = mark(launches, "build_pairs", 1, s)) return rc;
        ++launches;
    }
    PairTab P{p->info, p->geo, p->pp, p->bnd};
    BoysTab B = boys_of(ctx, p->opts.boys);
    // Class-pair queues, largest estimated work first, spread over the side streams so that
    // small classes fill the SMs next to large ones.
    struct Job { double cost; int x, y; };
    std::vector<Job> jobs;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y)
            if (p->q_len[x][y] > 0) jobs.push_back({p->class_cost[x][y], x, y});
    std::stable_sort(jobs.begin(), jobs.end(), [](const Job &a, const Job &b) { return a.cost > b.cost; });
    // Profiling runs every launch on the caller's stream, so each event pair times one kernel.
    const int nside = p->profiling ? 0 : std::min<int>(molints_ctx::kSide, (int)jobs.size());
    int fp32_launches = 0;
    if (nside > 0) MI_CUDA(ctx, cudaEventRecord(ctx->fork, s));
    for (int i = 0; i < nside; ++i) MI_CUDA(ctx, cudaStreamWaitEvent(ctx->side[i], ctx->fork, 0));
    for (size_t k = 0; k < jobs.size(); ++k) {
        const int x = jobs[k].x, y = jobs[k].y;
        cudaStream_t st = nside ? ctx->side[k % nside] : s;
        const bool rys = p->method[x][y] == MOLINTS_METHOD_RYS;
        const int mixed = p->fp32[x][y];
        int &occ = ctx->occupancy[x][y][(rys ? 2 : 0) + mixed];
        if (occ == 0) occ = std::max(1, rys ? kRysOccupancy[x][y](mixed) : kEriOccupancy[x][y](mixed));
        EriQueue Q{};
        Q.pairs = P;
        Q.boys = B;
        Q.jk = jk;
        Q.out = out_device;
        Q.mol_out = p->mol_out;
        Q.chunks = p->chunks + p->q_off[x][y];
        Q.nchunks = p->q_len[x][y];
        Q.counter = p->counters + x * kNumPairClasses + y;
        Q.screen_cut = p->opts.screen_cutoff;
        Q.fp32_cut = p->opts.fp32_cutoff;
        if (p->two_phase && !jk.J) {
            Q.scratch = ctx->scratch;
            Q.chunk_slot = p->chunk_slot + p->q_off[x][y];
            Q.region = p->g_region + ((size_t)x * kNumPairClasses + y) * p->nmol * kRegionFields;
        }
        // HGP: one warp per chunk, four per block; Rys: the launcher divides by its groups/block
        const int grid = rys ? occ * ctx->num_sms
                             : (int)std::min<long long>((long long)occ * ctx->num_sms, (Q.nchunks + 3) / 4);
        const char *name = rys ? kRysNames[x][y] : kEriNames[x][y];
        if (int rc = mark(launches, name, 0, st)) return rc;
        if (rys) kRysLaunchers[x][y](Q, ctx->rys, mixed, grid, st);
        else kEriLaunchers[x][y](Q, mixed, grid, st);
        fp32_launches += mixed;
        if (int rc = mark(launches, name, 1, st)) return rc;
        ++launches;
    }
    for (int i = 0; i < nside; ++i) {
        MI_CUDA(ctx, cudaEventRecord(ctx->join[i], ctx->side[i]));
        MI_CUDA(ctx, cudaStreamWaitEvent(s, ctx->join[i], 0));
    }
    if (p->n_gq > 0) {
        // shell quartets with a g shell (never two-phase plans; no J/K digestion)
        GenQuartets G{p->gq, p->gq_mol, p->n_gq, p->sh_xyz, p->sh_L, p->sh_K, p->sh_poff, p->sh_fn,
                      p->expn, p->ncoef, p->mol_out, out_device, ctx->rys};
        if (int rc = mark(launches, "eri_generic", 0, s)) return rc;
        launch_eri_generic(G, (int)std::min<int64_t>(p->n_gq, (int64_t)ctx->num_sms * 8), s);
        if (int rc = mark(launches, "eri_generic", 1, s)) return rc;
        ++launches;
    }
    if (p->two_phase && !jk.J && p->npacked > 0) {
        // second phase: the packed vector in order from the scratch blocks
        if (int rc = mark(launches, "gather_packed", 0, s)) return rc;
        // a persistent grid of gather_blocks blocks per SM; blocks beyond what the kernel's
        // registers let reside (five at 44 registers) start as others finish, and find the
        // unit list done
        const int gb = p->gather_blocks > 0 ? p->gather_blocks : kGatherBlocksDefault;
        const int grid = (int)std::min<long long>((long long)ctx->num_sms * gb, p->n_units);
        gather_packed_kernel<<<grid, kGatherThreads, 0, s>>>(out_device, ctx->scratch, p->g_col, p->g_colq, p->g_region,
                                                             p->g_mol, p->g_units, p->n_units,
                                                             p->counters + kNumPairClasses * kNumPairClasses,
                                                             p->nmol, p->bnd, p->g_qmax, p->opts.screen_cutoff);
        if (int rc = mark(launches, "gather_packed", 1, s)) return rc;
        ++launches;
    }
    MI_CUDA(ctx, cudaGetLastError());
    if (timing) MI_CUDA(ctx, cudaEventRecord(ctx->ev1, s));
    p->n_launches = launches;
    p->n_fp32_launches = fp32_launches;
    return MOLINTS_OK;
}

// Resident blocks per SM of every queue kernel the plan launches (queried once per context,
// before any graph capture).
static void plan_occupancy(molints_plan *p) {
    molints_ctx *ctx = p->ctx;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            if (p->q_len[x][y] == 0) continue;
            const int mixed = p->fp32[x][y];
            const bool rys = p->method[x][y] == MOLINTS_METHOD_RYS;
            int &occ = ctx->occupancy[x][y][(rys ? 2 : 0) + mixed];
            if (occ == 0) occ = std::max(1, rys ? kRysOccupancy[x][y](mixed) : kEriOccupancy[x][y](mixed));
        }
}

static int plan_execute_impl(molints_plan *p, double *out_device);

int molints_plan_execute(molints_plan *p, double *out_device) {
    if (!p || (!out_device && p->npacked > 0))
        return fail(p ? p->ctx : nullptr, MOLINTS_ERR_INVALID, "plan_execute: null argument");
    if (!p->ctx) return MOLINTS_ERR_INVALID;  // its context was destroyed first
    molints_ctx *ctx = p->ctx;
    MI_CUDA(ctx, cudaSetDevice(ctx->device));
    // executes that use the context's shared scratch run one after another
    const bool uses_scratch = p->two_phase && p->npacked > 0;
    if (uses_scratch && ctx->scratch_ev_live) MI_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->scratch_ev, 0));
    int rc = plan_execute_impl(p, out_device);
    if (!rc && uses_scratch) {
        MI_CUDA(ctx, cudaEventRecord(ctx->scratch_ev, ctx->stream));
        ctx->scratch_ev_live = true;
    }
    return rc;
}

static int plan_execute_impl(molints_plan *p, double *out_device) {
    molints_ctx *ctx = p->ctx;
    if (!p->use_graph || p->profiling) return plan_enqueue(p, out_device, true);
    // CUDA graph: captured once per output pointer (and scratch buffer), then launched whole
    cudaStream_t s = ctx->stream;
    if (!p->gexec || p->graph_out != out_device || (p->two_phase && p->graph_gen != ctx->scratch_gen)) {
        if (p->gexec) {
            cudaGraphExecDestroy(p->gexec);
            p->gexec = nullptr;
        }
        plan_occupancy(p);
        // captured on the context's capture stream, launched on its current stream
        MI_CUDA(ctx, cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
        ctx->stream = ctx->cap_stream;
        const int rc = plan_enqueue(p, out_device, false);
        ctx->stream = s;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->cap_stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&p->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            p->gexec = nullptr;
            return cuda_fail(ctx, e, "cudaGraphInstantiate");
        }
        p->graph_out = out_device;
        p->graph_gen = ctx->scratch_gen;
    }
    MI_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
    MI_CUDA(ctx, cudaGraphLaunch(p->gexec, s));
    MI_CUDA(ctx, cudaEventRecord(ctx->ev1, s));
    return MOLINTS_OK;
}

int molints_plan_jk(molints_plan *p, const double *D_device, double *J_device, double *K_device) {
    if (!p || !D_device || !J_device || !K_device)
        return fail(p ? p->ctx : nullptr, MOLINTS_ERR_INVALID, "plan_jk: null argument");
    if (!p->ctx) return MOLINTS_ERR_INVALID;  // its context was destroyed first
    molints_ctx *ctx = p->ctx;
    if (p->nmol != 1) return fail(ctx, MOLINTS_ERR_INVALID, "plan_jk: one molecule per plan");
    if (p->n_gq > 0) return fail(ctx, MOLINTS_ERR_UNSUPPORTED, "plan_jk: g shells are not digested");
    MI_CUDA(ctx, cudaSetDevice(ctx->device));
    const int64_t n = p->nbf0;
    const size_t bytes = (size_t)n * n * sizeof(double);
    MI_CUDA(ctx, cudaMemsetAsync(J_device, 0, bytes, ctx->stream));
    MI_CUDA(ctx, cudaMemsetAsync(K_device, 0, bytes, ctx->stream));
    JKOut jk;
    jk.D = D_device;
    jk.J = J_device;
    jk.K = K_device;
    jk.n = (int)n;
    const int rc = plan_enqueue(p, nullptr, true, jk);
    if (rc) return rc;
    if (n > 1) {
        const long long nn = (long long)n * n;
        mirror_lower_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, ctx->stream>>>(J_device, K_device, (int)n);
        MI_CUDA(ctx, cudaGetLastError());
    }
    return MOLINTS_OK;
}

int molints_jk(molints_ctx *ctx, const molints_basis *b, const molints_options *opts,
               const double *D_host, double *J_host, double *K_host) {
    if (!ctx || !b || !D_host || !J_host || !K_host) return fail(ctx, MOLINTS_ERR_INVALID, "jk: null argument");
    const int64_t n = molints_nbf(b);
    if (n < 0) return fail(ctx, MOLINTS_ERR_INVALID, "jk: malformed basis");
    molints_plan *p = nullptr;
    int rc = molints_plan_create(ctx, b, opts, &p);
    if (rc) return rc;
    if (n == 0) { molints_plan_destroy(p); return MOLINTS_OK; }
    double *d = nullptr;
    int64_t held = 0;
    rc = dev_alloc(ctx, &d, (size_t)3 * n * n, &held);
    if (!rc) {
        const size_t bytes = (size_t)n * n * sizeof(double);
        cudaError_t e = cudaMemcpyAsync(d, D_host, bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) rc = molints_plan_jk(p, d, d + n * n, d + 2 * n * n);
        else rc = cuda_fail(ctx, e, "jk upload");
        if (!rc && (e = cudaMemcpyAsync(J_host, d + n * n, bytes, cudaMemcpyDeviceToHost, ctx->stream)) == cudaSuccess)
            e = cudaMemcpyAsync(K_host, d + 2 * n * n, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "jk");
        dev_free(ctx, d);
        ctx->held -= held;
    }
    molints_plan_destroy(p);
    return rc;
}

int molints_plan_set_graph(molints_plan *p, int enable) {
    if (!p) return MOLINTS_ERR_INVALID;
    p->use_graph = enable ? 1 : 0;
    if (!enable && p->gexec) {
        cudaSetDevice(p->ctx->device);
        cudaGraphExecDestroy(p->gexec);
        p->gexec = nullptr;
    }
    return MOLINTS_OK;
}

// The host copies of the final pair tables that the statistics and the Schwarz read-out use.
// Plan creation builds the tables on the device only; they are fetched on first use.
static int plan_host_tables(const molints_plan *cp) {
    molints_plan *p = const_cast<molints_plan *>(cp);
    if (p->host_tables) return MOLINTS_OK;
    molints_ctx *ctx = p->ctx;
    const int n = p->npair;
    std::vector<int2> ab(n);
    std::vector<int4> info(n);
    p->bnd_h.resize(n);
    MI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n > 0) {
        MI_CUDA(ctx, cudaMemcpyAsync(ab.data(), p->pair_ab, n * sizeof(int2), cudaMemcpyDeviceToHost, ctx->stream));
        MI_CUDA(ctx, cudaMemcpyAsync(info.data(), p->info, n * sizeof(int4), cudaMemcpyDeviceToHost, ctx->stream));
        MI_CUDA(ctx, cudaMemcpyAsync(p->bnd_h.data(), p->bnd, n * sizeof(double2), cudaMemcpyDeviceToHost,
                                     ctx->stream));
        MI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    std::vector<int> first(std::max(p->nmol, 1), 0);  // first global shell of each molecule
    for (int m = 1; m < p->nmol; ++m) first[m] = first[m - 1] + p->mol_nshell[m - 1];
    p->pair_ref.resize(n);
    p->npp_h.resize(n);
    for (int k = 0; k < n; ++k) {
        const int f = first[p->pair_mol[k]];
        const int i = std::max(ab[k].x, ab[k].y) - f, j = std::min(ab[k].x, ab[k].y) - f;
        p->pair_ref[k] = i * (i + 1) / 2 + j;
        p->npp_h[k] = info[k].y;
    }
    p->host_tables = true;
    return MOLINTS_OK;
}

int molints_plan_stats(const molints_plan *p, molints_stats *st) {
    if (!p || !st) return MOLINTS_ERR_INVALID;
    if (!p->ctx) return MOLINTS_ERR_INVALID;  // its context was destroyed first
    molints_ctx *ctx = p->ctx;
    if (int rc = plan_host_tables(p)) return rc;
    std::memset(st, 0, sizeof(*st));
    st->n_eri = p->npacked;
    st->n_kernel_launches = p->n_launches;
    st->n_prim_pairs = p->nprim_pair_all;
    st->n_prim_pairs_kept = p->nprim_pair_kept;
    for (int k = 0; k < 4; ++k) st->plan_ms[k] = p->plan_ms[k];
    st->n_fp32_launches = p->n_fp32_launches;
    st->n_shell_quartets += p->n_gq;
    // per (molecule, pair class): the pairs, gathered from the class-major list
    const int nc = kNumPairClasses;
    std::vector<std::vector<int>> by(std::max(p->nmol, 1) * nc);
    for (int c = 0; c < nc; ++c)
        for (int k = p->class_start[c]; k < p->class_start[c + 1]; ++k) by[p->pair_mol[k] * nc + c].push_back(k);
    const bool mixed = p->opts.precision == MOLINTS_MIXED && p->opts.fp32_cutoff > 0.0;
    const double cut = p->opts.fp32_cutoff, scut = p->opts.screen_cutoff;
    for (int m = 0; m < p->nmol; ++m) {
        int64_t np = 0, sum = 0, sum2 = 0;
        for (int c = 0; c < nc; ++c)
            for (int k : by[m * nc + c]) { ++np; sum += p->npp_h[k]; sum2 += (int64_t)p->npp_h[k] * p->npp_h[k]; }
        st->n_shell_quartets += np * (np + 1) / 2;
        st->n_prim_quartets += (sum * sum + sum2) / 2;
        for (int x = 0; x < nc; ++x)
            for (int y = 0; y <= x; ++y) {
                const std::vector<int> &A = by[m * nc + x], &Bv = by[m * nc + y];
                if (A.empty() || Bv.empty()) continue;
                // only quartets of class pairs whose plan launches an FP32 kernel count as FP32
                const bool f32 = mixed && p->fp32[x][y];
                if (scut > 0.0) {
                    // both conditions: the direct count over the class pair's quartets
                    for (size_t a = 0; a < A.size(); ++a)
                        for (size_t c = 0; c < (x == y ? a + 1 : Bv.size()); ++c) {
                            const double2 ba = p->bnd_h[A[a]], bc = p->bnd_h[Bv[c]];
                            if (ba.x * bc.x < scut) ++st->n_screened;
                            else if (f32 && ba.y * bc.y < cut) ++st->n_fp32_quartets;
                        }
                } else if (f32) {
                    // quartets (a, c) with R_a R_c < cut from the sorted R of the ket class; for
                    // x == y the unordered pairs {a, c}: (ordered + diagonal) / 2
                    std::vector<double> yk(Bv.size());
                    for (size_t c = 0; c < Bv.size(); ++c) yk[c] = p->bnd_h[Bv[c]].y;
                    std::sort(yk.begin(), yk.end());
                    int64_t ordered = 0, diag = 0;
                    for (int k : A) {
                        const double ya = p->bnd_h[k].y;
                        if (ya <= 0.0) ordered += (int64_t)yk.size();
                        else ordered += std::lower_bound(yk.begin(), yk.end(), cut / ya) - yk.begin();
                        if (x == y && ya * ya < cut) ++diag;
                    }
                    st->n_fp32_quartets += x == y ? (ordered + diag) / 2 : ordered;
                }
            }
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return MOLINTS_ERR_CUDA;
    if (p->n_launches > 0 && cudaEventSynchronize(ctx->ev1) == cudaSuccess) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) st->device_ms = ms;
    }
    return MOLINTS_OK;
}

int molints_plan_class_work(const molints_plan *p, int64_t *quartets, double *prim_quartets, int32_t n) {
    if (!p || !quartets || !prim_quartets || n != kNumPairClasses * kNumPairClasses) return MOLINTS_ERR_INVALID;
    if (!p->ctx) return MOLINTS_ERR_INVALID;  // its context was destroyed first
    if (int rc = plan_host_tables(p)) return rc;
    const int nc = kNumPairClasses;
    for (int k = 0; k < n; ++k) { quartets[k] = 0; prim_quartets[k] = 0.0; }
    // per (molecule, pair class): pair count, sum and sum of squares of kept primitive pairs
    std::vector<double> cnt((size_t)std::max(p->nmol, 1) * nc, 0.0), sum(cnt.size(), 0.0), sq(cnt.size(), 0.0);
    for (int c = 0; c < nc; ++c)
        for (int k = p->class_start[c]; k < p->class_start[c + 1]; ++k) {
            const size_t i = (size_t)p->pair_mol[k] * nc + c;
            cnt[i] += 1.0;
            sum[i] += p->npp_h[k];
            sq[i] += (double)p->npp_h[k] * p->npp_h[k];
        }
    for (int m = 0; m < p->nmol; ++m)
        for (int x = 0; x < nc; ++x)
            for (int y = 0; y <= x; ++y) {
                const size_t a = (size_t)m * nc + x, b = (size_t)m * nc + y;
                if (x == y) {
                    quartets[x * nc + y] += (int64_t)(cnt[a] * (cnt[a] + 1) / 2);
                    prim_quartets[x * nc + y] += (sum[a] * sum[a] + sq[a]) / 2;
                } else {
                    quartets[x * nc + y] += (int64_t)(cnt[a] * cnt[b]);
                    prim_quartets[x * nc + y] += sum[a] * sum[b];
                }
            }
    return MOLINTS_OK;
}

int molints_plan_set_profiling(molints_plan *p, int enable) {
    if (!p) return MOLINTS_ERR_INVALID;
    p->profiling = enable ? 1 : 0;
    return MOLINTS_OK;
}

int molints_plan_launch_times(molints_plan *p, const char **names, float *ms, int cap) {
    if (!p || cap < 0 || (cap > 0 && (!names || !ms))) return MOLINTS_ERR_INVALID;
    if (!p->ctx) return MOLINTS_ERR_INVALID;  // its context was destroyed first
    molints_ctx *ctx = p->ctx;
    if (!p->profiling) return fail(ctx, MOLINTS_ERR_INVALID, "launch_times: profiling is off");
    MI_CUDA(ctx, cudaSetDevice(ctx->device));
    MI_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    const int n = p->n_launches;
    for (int k = 0; k < n && k < cap; ++k) {
        names[k] = p->prof_name[k];
        MI_CUDA(ctx, cudaEventElapsedTime(&ms[k], p->prof_ev[2 * k], p->prof_ev[2 * k + 1]));
    }
    return n;
}

int molints_plan_schwarz(molints_plan *p, double *out) {
    if (!p || !out) return MOLINTS_ERR_INVALID;
    if (!p->ctx) return MOLINTS_ERR_INVALID;  // its context was destroyed first
    molints_ctx *ctx = p->ctx;
    MI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (p->n_gq > 0) return fail(ctx, MOLINTS_ERR_UNSUPPORTED, "plan_schwarz: g shells have no bounds");
    if (p->npair == 0) return MOLINTS_OK;
    if (!p->qcon) {
        int rc = dev_alloc(ctx, &p->qcon, (size_t)p->npair, &p->bytes);
        if (rc) return rc;
    }
    PairTab P{p->info, p->geo, p->pp, p->bnd};
    BoysTab B = boys_of(ctx, p->opts.boys);
    for (int c = 0; c < kNumPairClasses; ++c) {
        const int n = p->class_start[c + 1] - p->class_start[c];
        if (n <= 0) continue;
        if (kSchwarzLaunchers[c]) kSchwarzLaunchers[c](P, B, p->class_start[c], n, nullptr, p->qcon, 1, ctx->stream);
        else kRysBoundLaunchers[c](P, ctx->rys, p->class_start[c], n, nullptr, p->qcon, 1, ctx->stream);
    }
    MI_CUDA(ctx, cudaGetLastError());
    std::vector<double> q(p->npair);
    MI_CUDA(ctx, cudaMemcpyAsync(q.data(), p->qcon, p->npair * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (int rc = plan_host_tables(p)) return rc;
    std::vector<int64_t> base(std::max(p->nmol, 1), 0);
    for (int m = 1; m < p->nmol; ++m)
        base[m] = base[m - 1] + (int64_t)p->mol_nshell[m - 1] * (p->mol_nshell[m - 1] + 1) / 2;
    for (int k = 0; k < p->npair; ++k) out[base[p->pair_mol[k]] + p->pair_ref[k]] = q[k];
    return MOLINTS_OK;
}

int molints_eri_packed(molints_ctx *ctx, const molints_basis *b, const molints_options *opts,
                       double *out, int out_is_device, molints_stats *stats) {
    if (!ctx || !b) return fail(ctx, MOLINTS_ERR_INVALID, "eri_packed: null argument");
    const int64_t nbf = molints_nbf(b);
    if (nbf < 0) return fail(ctx, MOLINTS_ERR_INVALID, "eri_packed: malformed basis");
    if (!out && molints_npacked(nbf) > 0) return fail(ctx, MOLINTS_ERR_INVALID, "eri_packed: null output");
    molints_plan *p = nullptr;
    int rc = plan_create_impl(ctx, 1, b, opts, 0, 1, &p);
    if (rc) return rc;
    if (p->npacked == 0) {
        if (stats) rc = molints_plan_stats(p, stats);
        molints_plan_destroy(p);
        return rc;
    }
    double *dout = out;
    if (!out_is_device) {
        if (ctx->out_cache_len < p->npacked) {
            if (ctx->out_cache) {
                dev_free(ctx, ctx->out_cache);
                ctx->held -= ctx->out_cache_len * 8;
                ctx->out_cache = nullptr;
                ctx->out_cache_len = 0;
            }
            rc = dev_alloc(ctx, &ctx->out_cache, (size_t)p->npacked, nullptr);
            if (rc) { molints_plan_destroy(p); return rc; }
            ctx->out_cache_len = p->npacked;
        }
        dout = ctx->out_cache;
    }
    rc = molints_plan_execute(p, dout);
    if (!rc && !out_is_device && p->npacked > 0) {
        cudaError_t e = cudaMemcpyAsync(out, dout, p->npacked * sizeof(double), cudaMemcpyDeviceToHost,
                                        ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "eri_packed D2H");
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "eri_packed sync");
    }
    if (!rc && stats) rc = molints_plan_stats(p, stats);
    molints_plan_destroy(p);
    return rc;
}

}  // extern "C"

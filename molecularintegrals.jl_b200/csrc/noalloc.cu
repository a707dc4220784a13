// noalloc.cu -- molints_eri_packed_noalloc: the ERI path without any device allocation.
//
// Some callers cannot allocate device memory where they need integrals.  A host program whose
// own allocator has reserved (nearly) all of the GPU's memory -- a framework's caching
// allocator, or the memory manager of a simulation code that owns the device -- leaves no room
// for another cudaMalloc and does not want one.  A time-critical loop cannot accept the device
// synchronisation a cudaMalloc or cudaFree may cause.  Such callers pass the basis (host
// arrays) and their own device output vector; everything else the path needs -- the Boys table
// and the per-call pair tables and work queues -- lives in one file-scope device array of
// kScratchBytes (8 MiB), which every GPU that loads this library holds until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the array's device
// address with cudaGetSymbolAddress and copies the Boys table into it (a synchronous copy), so
// that first call should come before any stream capture.  Later calls reuse the address and
// the table.
//
// The call only enqueues work on the caller's stream.  Every call shares the array and
// overwrites its pair tables and work-queue counters (the counters are cleared by each call's
// upload), so calls whose GPU work overlaps (different streams, or host threads with no
// ordering between their streams) race on it; order them on one stream.  Host threads are
// serialised while a call prepares and enqueues its work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/molints.h"
#include "eri_common.cuh"
#include "eri_dispatch.h"

namespace molints {
void launch_build_pairs(int npair, const int2 *pair_ab, const int4 *info, const int *pp_src,
                        const double *xyz, const int *poff, const double *expn,
                        const double *ncoef, PrimPair *pp, double4 *geo, cudaStream_t s);
void fill_boys_scaled(double *sc, int nM);
}  // namespace molints

using namespace molints;

namespace {

constexpr size_t kScratchBytes = (size_t)8 << 20;  // the stated maximum: 8 MiB
constexpr size_t kAlign = 256;
constexpr int kTableM = 4 * kLmaxHgp + 1;  // Boys orders the HGP class kernels use
constexpr size_t kTableBytes =
    ((size_t)kTableM * kBoysRows * kBoysScaledCols * sizeof(double) + kAlign - 1) / kAlign * kAlign;
constexpr int kMaxDevices = 64;

// Device scratch.  In host code this name is only a stand-in for the symbol, never an
// address: kernels get the pointer cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host mirror of the per-call part of the scratch (filled, then copied in one transfer),
// plus room for the pair sort keys.  Static, so a call allocates no host memory either.
alignas(256) static unsigned char g_host[kScratchBytes];
static int g_order[kScratchBytes / 64];
static std::mutex g_mutex;
static void *g_dev_ptr[kMaxDevices];
static bool g_dev_ready[kMaxDevices];

int noalloc_fail(char *err, size_t err_len, int code, const char *msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
    return code;
}

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

int ncart(int l) { return (l + 1) * (l + 2) / 2; }

int pair_class(int la, int lb) {
    for (int c = 0; c < kNumPairClasses; ++c)
        if (kPairClassLa[c] == la && kPairClassLb[c] == lb) return c;
    return -1;
}

}  // namespace

extern "C" int molints_eri_packed_noalloc(const molints_basis *b, const molints_options *opts,
                                          double *out_device, void *stream, char *err,
                                          size_t err_len) {
    if (err && err_len) err[0] = '\0';
    if (!b) return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "null basis");
    const int64_t nbf = molints_nbf(b);
    if (nbf < 0) return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "malformed basis");
    if (molints_npacked(nbf) > 0 && !out_device)
        return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "null output");
    int boys_mode = MOLINTS_BOYS_REFERENCE;
    if (opts) {
        if (opts->precision != MOLINTS_FP64 || opts->screen_cutoff != 0.0 ||
            (opts->method != MOLINTS_METHOD_AUTO && opts->method != MOLINTS_METHOD_HGP))
            return noalloc_fail(err, err_len, MOLINTS_ERR_UNSUPPORTED,
                                "noalloc entry point: FP64 without screening only");
        if (opts->boys != MOLINTS_BOYS_REFERENCE && opts->boys != MOLINTS_BOYS_EXACT)
            return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "unknown Boys mode");
        boys_mode = opts->boys;
    }
    const int ns = b->nshell;
    if (ns > 0 && (!b->expn || !b->coef)) return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "null primitives");
    int nprim_tot = 0;
    for (int s = 0; s < ns; ++s) {
        if (b->L[s] > kLmaxHgp) return noalloc_fail(err, err_len, MOLINTS_ERR_UNSUPPORTED, "shell above d");
        if (b->nprim[s] < 1 || b->nprim[s] > 255 || b->prim_off[s] < 0)
            return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "shell primitive count out of range");
        nprim_tot = std::max(nprim_tot, b->prim_off[s] + b->nprim[s]);
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(b->xyz[3 * s + k])) return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "non-finite centre");
    }
    for (int k = 0; k < nprim_tot; ++k)
        if (!(b->expn[k] > 0.0) || !std::isfinite(b->expn[k]) || !std::isfinite(b->coef[k]))
            return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "exponents must be finite and > 0");
    if (nbf == 0) return MOLINTS_OK;

    // Sizes of the per-call tables; reject what does not fit the static scratch.
    const int64_t npair = (int64_t)ns * (ns + 1) / 2;
    int64_t nall = 0;
    int64_t ncls[kNumPairClasses] = {0};
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j <= i; ++j) {
            nall += (int64_t)b->nprim[i] * b->nprim[j];
            ncls[pair_class(std::max(b->L[i], b->L[j]), std::min(b->L[i], b->L[j]))] += 1;
        }
    // work-queue chunks: one bra pair and up to 32 ket pairs each
    int64_t nchunk = 0;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            if (x == y)
                for (int64_t i = 0; i < ncls[x]; ++i) nchunk += (i + 1 + 31) / 32;
            else
                nchunk += ncls[x] * ((ncls[y] + 31) / 32);
        }
    const int nc2 = kNumPairClasses * kNumPairClasses;
    size_t off = 0;
    const size_t o_xyz = off;   off = align_up(off + 3 * (size_t)ns * sizeof(double));
    const size_t o_expn = off;  off = align_up(off + (size_t)nprim_tot * sizeof(double));
    const size_t o_ncoef = off; off = align_up(off + (size_t)nprim_tot * sizeof(double));
    const size_t o_poff = off;  off = align_up(off + (size_t)ns * sizeof(int));
    const size_t o_ab = off;    off = align_up(off + (size_t)npair * sizeof(int2));
    const size_t o_info = off;  off = align_up(off + (size_t)npair * sizeof(int4));
    const size_t o_src = off;   off = align_up(off + (size_t)nall * sizeof(int));
    const size_t o_bnd = off;   off = align_up(off + (size_t)npair * sizeof(double2));
    const size_t o_chunk = off; off = align_up(off + (size_t)nchunk * sizeof(int4));
    const size_t o_cnt = off;   off = align_up(off + (size_t)nc2 * sizeof(int));
    const size_t o_mol = off;   off = align_up(off + sizeof(long long));
    const size_t upload = off;  // everything above is copied from the host mirror
    const size_t o_geo = off;   off = align_up(off + (size_t)npair * sizeof(double4));
    const size_t o_pp = off;    off = align_up(off + (size_t)nall * sizeof(PrimPair));
    if (kTableBytes + off > kScratchBytes || npair > (int64_t)(sizeof(g_order) / sizeof(int))) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "basis needs %zu bytes of scratch; the noalloc entry point holds at most %zu",
                      kTableBytes + off, kScratchBytes);
        return noalloc_fail(err, err_len, MOLINTS_ERR_UNSUPPORTED, msg);
    }

    std::lock_guard<std::mutex> lock(g_mutex);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(err, err_len, MOLINTS_ERR_CUDA, "cudaGetDevice failed");
    if (!g_dev_ready[dev]) {
        // once per device, with the device current: the array's device address and the table
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess || !ptr) return noalloc_fail(err, err_len, MOLINTS_ERR_CUDA, "cudaGetSymbolAddress failed");
        fill_boys_scaled(reinterpret_cast<double *>(g_host), kTableM);
        e = cudaMemcpy(ptr, g_host, (size_t)kTableM * kBoysRows * kBoysScaledCols * sizeof(double),
                       cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return noalloc_fail(err, err_len, MOLINTS_ERR_CUDA, "Boys table copy failed");
        g_dev_ptr[dev] = ptr;
        g_dev_ready[dev] = true;
    }
    unsigned char *base = static_cast<unsigned char *>(g_dev_ptr[dev]);
    unsigned char *data = base + kTableBytes;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // Host side of the plan, as molints_plan_create does it with every primitive pair kept:
    // normalised coefficients, canonical pairs ordered by class then descending K_A K_B.
    double *xyz = reinterpret_cast<double *>(g_host + o_xyz);
    double *expn = reinterpret_cast<double *>(g_host + o_expn);
    double *ncoef = reinterpret_cast<double *>(g_host + o_ncoef);
    int *poff = reinterpret_cast<int *>(g_host + o_poff);
    int2 *ab = reinterpret_cast<int2 *>(g_host + o_ab);
    int4 *info = reinterpret_cast<int4 *>(g_host + o_info);
    int *src = reinterpret_cast<int *>(g_host + o_src);
    double2 *bnd = reinterpret_cast<double2 *>(g_host + o_bnd);
    std::memcpy(xyz, b->xyz, 3 * (size_t)ns * sizeof(double));
    std::memcpy(expn, b->expn, (size_t)nprim_tot * sizeof(double));
    std::memcpy(poff, b->prim_off, (size_t)ns * sizeof(int));
    std::memset(ncoef, 0, (size_t)nprim_tot * sizeof(double));
    for (int sh = 0; sh < ns; ++sh) {
        const int L = b->L[sh], p0 = b->prim_off[sh], K = b->nprim[sh];
        double S = 0;
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) {
                const double x = b->expn[p0 + i], y = b->expn[p0 + j];
                S += b->coef[p0 + i] * b->coef[p0 + j] * std::pow(2 * std::sqrt(x * y) / (x + y), L + 1.5);
            }
        if (!(S > 0.0)) return noalloc_fail(err, err_len, MOLINTS_ERR_INVALID, "zero contracted function");
        const double cn = 1.0 / std::sqrt(S);
        for (int i = 0; i < K; ++i) {
            const double a = b->expn[p0 + i];
            ncoef[p0 + i] = b->coef[p0 + i] * cn * std::pow(2 * a / M_PI, 0.75) * std::pow(4 * a, 0.5 * L);
        }
    }
    auto tightness = [&](int sh) {
        const int p0 = b->prim_off[sh];
        double lo = b->expn[p0], hi = lo;
        for (int i = 1; i < b->nprim[sh]; ++i) {
            lo = std::min(lo, b->expn[p0 + i]);
            hi = std::max(hi, b->expn[p0 + i]);
        }
        return std::sqrt(lo * hi);
    };
    // pair k (reference order i >= j) -> canonical (a, b), class, K; sort keys in g_order
    auto canon = [&](int k, int &a, int &bb, int &cls, int &npp) {
        int i = (int)((std::sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
        while ((int64_t)i * (i + 1) / 2 > k) --i;
        while ((int64_t)(i + 1) * (i + 2) / 2 <= k) ++i;
        const int j = k - i * (i + 1) / 2;
        a = i;
        bb = j;
        // larger L first; for equal L the tighter shell (larger sqrt(min * max exponent)), so
        // that the HRR moves angular momentum away from it
        if (b->L[a] < b->L[bb] || (b->L[a] == b->L[bb] && tightness(a) < tightness(bb))) std::swap(a, bb);
        cls = pair_class(b->L[a], b->L[bb]);
        npp = b->nprim[a] * b->nprim[bb];
    };
    for (int k = 0; k < npair; ++k) g_order[k] = k;
    std::sort(g_order, g_order + npair, [&](int x, int y) {
        int ax, bx, cx, kx, ay, by, cy, ky;
        canon(x, ax, bx, cx, kx);
        canon(y, ay, by, cy, ky);
        if (cx != cy) return cx < cy;
        if (kx != ky) return kx > ky;
        return x < y;
    });
    int class_start[kNumPairClasses + 1] = {0};
    // first function of each shell, by prefix sums over L (no array needed: shells are few)
    auto fn_of = [&](int sh) {
        int f = 0;
        for (int t = 0; t < sh; ++t) f += ncart(b->L[t]);
        return f;
    };
    int nsrc = 0;
    for (int k = 0; k < npair; ++k) {
        int a, bb, cls, npp;
        canon(g_order[k], a, bb, cls, npp);
        ab[k] = make_int2(a, bb);
        info[k] = make_int4(nsrc, npp, fn_of(a), fn_of(bb));
        for (int ia = 0; ia < b->nprim[a]; ++ia)
            for (int ib = 0; ib < b->nprim[bb]; ++ib) src[nsrc++] = (ia << 8) | ib;
        bnd[k] = make_double2(0.0, 0.0);
        class_start[cls + 1] = k + 1;
    }
    for (int c = 1; c <= kNumPairClasses; ++c) class_start[c] = std::max(class_start[c], class_start[c - 1]);
    // chunk queues in natural order; the counters and the molecule offset start at zero
    int4 *chunk = reinterpret_cast<int4 *>(g_host + o_chunk);
    int q_off[kNumPairClasses][kNumPairClasses] = {}, q_len[kNumPairClasses][kNumPairClasses] = {};
    int nq = 0;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            q_off[x][y] = nq;
            for (int pb = class_start[x]; pb < class_start[x + 1]; ++pb) {
                const int kend = (x == y) ? pb + 1 : class_start[y + 1];
                for (int q0 = class_start[y]; q0 < kend; q0 += 32)
                    chunk[nq++] = make_int4(pb, q0, std::min(32, kend - q0), 0);
            }
            q_len[x][y] = nq - q_off[x][y];
        }
    std::memset(g_host + o_cnt, 0, (size_t)nc2 * sizeof(int));
    std::memset(g_host + o_mol, 0, sizeof(long long));
    int nsm = 1;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) nsm = 1;

    // One copy of the prepared tables into the scratch, then the device path on `stream`.
    // g_host is pageable: cudaMemcpyAsync returns once it has been staged, so the next call
    // may refill it while this call's work is still queued.
    e = cudaMemcpyAsync(data, g_host, upload, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return noalloc_fail(err, err_len, MOLINTS_ERR_CUDA, "table upload failed");
    const int2 *d_ab = reinterpret_cast<const int2 *>(data + o_ab);
    const int4 *d_info = reinterpret_cast<const int4 *>(data + o_info);
    PrimPair *d_pp = reinterpret_cast<PrimPair *>(data + o_pp);
    double4 *d_geo = reinterpret_cast<double4 *>(data + o_geo);
    launch_build_pairs((int)npair, d_ab, d_info, reinterpret_cast<const int *>(data + o_src),
                       reinterpret_cast<const double *>(data + o_xyz), reinterpret_cast<const int *>(data + o_poff),
                       reinterpret_cast<const double *>(data + o_expn), reinterpret_cast<const double *>(data + o_ncoef),
                       d_pp, d_geo, s);
    PairTab P{d_info, d_geo, d_pp, reinterpret_cast<const double2 *>(data + o_bnd)};
    BoysTab B;
    B.tab = nullptr;  // the class kernels read only the scaled tables
    B.scaled = reinterpret_cast<const double *>(base);
    B.t_switch = boys_mode == MOLINTS_BOYS_EXACT ? kBoysTableMax : kBoysReferenceSwitch;
    for (int x = 0; x < kNumPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            if (q_len[x][y] == 0) continue;
            EriQueue Q{};
            Q.pairs = P;
            Q.boys = B;
            Q.out = out_device;
            Q.mol_out = reinterpret_cast<const long long *>(data + o_mol);
            Q.chunks = reinterpret_cast<const int4 *>(data + o_chunk) + q_off[x][y];
            Q.nchunks = q_len[x][y];
            Q.counter = reinterpret_cast<int *>(data + o_cnt) + x * kNumPairClasses + y;
            Q.screen_cut = 0.0;
            Q.fp32_cut = 0.0;
            const int occ = std::max(1, kEriOccupancy[x][y](0));
            const int grid = (int)std::min<long long>((long long)occ * nsm, (Q.nchunks + 3) / 4);
            kEriLaunchers[x][y](Q, 0, grid, s);
        }
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(err, err_len, MOLINTS_ERR_CUDA, cudaGetErrorString(e));
    return MOLINTS_OK;
}

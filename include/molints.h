/*
 * molints.h -- C ABI of libmolints_cuda.so, a B200 (sm_100a) engine for the two-electron
 * repulsion integrals (ERIs) of contracted cartesian Gaussian basis sets.
 *
 * It replaces the ERI drivers of MolecularIntegrals.jl (paths relative to that project):
 *   all_twoe_ints(bfs, ERI=coulomb)   src/ERI.jl:104-112
 *   all_twoe_ints_chrr(bfs::Basis)    src/HGP.jl:22-34
 *   all_twoe_ints_rys(bfs)            src/Rys.jl:16-24
 * All three return the unique integrals (ij|kl), i>=j, k>=l, ij>=kl, of normalised
 * functions in one packed vector indexed by iindex (src/Utils.jl:14-19); this library
 * writes exactly that vector (0-based: element iindex(i,j,k,l)-1).
 *
 * Conventions: every function returns an int status (MOLINTS_OK = 0, negative on error);
 * no C++ exception crosses the ABI; molints_last_error() describes the last failure of a
 * context.  A context belongs to one host thread at a time.  Pointers are plain host
 * pointers unless a name or comment says "device".
 */
#ifndef MOLINTS_H
#define MOLINTS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MOLINTS_ABI_VERSION 1

enum molints_status {
    MOLINTS_OK = 0,
    MOLINTS_ERR_INVALID = -1,      /* bad argument or malformed basis */
    MOLINTS_ERR_UNSUPPORTED = -2,  /* angular momentum or size beyond the engine's limits */
    MOLINTS_ERR_BUDGET = -3,       /* the request does not fit the context's HBM budget */
    MOLINTS_ERR_CUDA = -4,         /* a CUDA runtime call failed */
    MOLINTS_ERR_TIMEOUT = -5,      /* a bounded device or host wait gave up */
    MOLINTS_ERR_NOMEM = -6         /* host allocation failed */
};

/* AUTO: per class pair, the context's method table (molints_set_class_methods; on a B200 the
 * shipped tuned table by default), else HGP where an HGP kernel exists and Rys otherwise.
 * HGP: all_twoe_ints_chrr's algorithm (src/HGP.jl:22-242) wherever it exists, Rys for classes
 * with an f shell.  RYS: all_twoe_ints_rys's algorithm (src/Rys.jl:16-156) for every class
 * pair. */
enum molints_method { MOLINTS_METHOD_AUTO = 0, MOLINTS_METHOD_HGP = 1, MOLINTS_METHOD_RYS = 2 };
enum molints_precision { MOLINTS_FP64 = 0, MOLINTS_MIXED = 1 };
enum molints_boys {
    /* farray of src/Boys.jl:19-27: exact F_m below T = 30, the asymptotic form (without the
     * e^-T terms) from T = 30 up.  Matches the reference HGP bit for bit up to rounding. */
    MOLINTS_BOYS_REFERENCE = 0,
    /* exact F_m (table + Taylor + downward recursion) up to T = 40, asymptotic beyond. */
    MOLINTS_BOYS_EXACT = 1
};
/* How the class kernels reach the packed vector.  DIRECT: each integral is stored at its
 * iindex position.  For an output larger than L2 that costs one read-modify-write of a DRAM
 * sector per 8-byte store.  TWO_PHASE: each shell quartet's block is stored whole, coalesced,
 * into a class-major scratch held by the plan (about npacked doubles more); then one pass
 * writes the packed vector in order from it, an output row per thread block (whole-molecule
 * plans; shard plans stay DIRECT).  AUTO: TWO_PHASE for outputs of at least
 * MOLINTS_TWO_PHASE_MIN integrals (256 MB, twice L2) when its scratch fits the context's
 * budget and the device, else DIRECT; served requests (molints_submit) with AUTO run DIRECT.
 * An explicit TWO_PHASE whose scratch does not fit fails.  The values are the same either way,
 * bit for bit. */
enum molints_output { MOLINTS_OUTPUT_AUTO = 0, MOLINTS_OUTPUT_DIRECT = 1, MOLINTS_OUTPUT_TWO_PHASE = 2 };
/* Plans of at least this many integrals take TWO_PHASE under MOLINTS_OUTPUT_AUTO. */
#define MOLINTS_TWO_PHASE_MIN ((int64_t)1 << 25)

/* Largest shell angular momentum the engine accepts (g = 4), as the reference's tables
 * (shell_indices, src/Basis.jl:269-279).  Class pairs up to (ff|ff) run the generated HGP or Rys
 * kernels (n <= 7 roots); every shell quartet with a g shell runs one generic Rys kernel (n <= 9
 * roots, FP64, no screening), written for coverage rather than speed.  Plans with a g shell use
 * the direct output and support neither sharding, J/K digestion nor molints_plan_schwarz
 * (MOLINTS_ERR_UNSUPPORTED). */
#define MOLINTS_LMAX 4
/* Number of shell-pair classes, ordered by la+lb then la: ss ps pp ds dp fs dd fp df fd ff.
 * A pair is oriented with the larger L first, except that equal-L pairs and f-d pairs put the
 * tighter shell first (hence the class df). */
#define MOLINTS_NUM_PAIR_CLASSES 11

/* A basis set as flat shell arrays: what the reference's Basis/Shell hold
 * (src/Basis.jl:147-177).  Functions are numbered shell by shell, components in the
 * reference's shell_indices order (src/Basis.jl:269-279). */
typedef struct molints_basis {
    int32_t nshell;
    const double *xyz;       /* [3*nshell] centres, bohr */
    const int32_t *L;        /* [nshell] angular momentum, 0..MOLINTS_LMAX */
    const int32_t *nprim;    /* [nshell] primitives per shell, >= 1 */
    const int32_t *prim_off; /* [nshell] offset of the shell's first primitive */
    const double *expn;      /* primitive exponents (Shell.expns) */
    const double *coef;      /* raw contraction coefficients (Shell.coefs); the engine
                                applies primitive and contracted norms (src/Basis.jl:42-98) */
} molints_basis;

typedef struct molints_options {
    int32_t method;          /* enum molints_method */
    int32_t precision;       /* enum molints_precision */
    int32_t boys;            /* enum molints_boys; the Rys kernels always evaluate the exact
                                quadrature (there is no T >= 30 branch to follow) */
    int32_t output;          /* enum molints_output */
    /* Both cutoffs compare against B = Qabs_ab * Qabs_cd, where Qabs_ab is the sum over the
     * pair's primitive pairs i of sqrt(max |(a_i b_i|a_i b_i)|).  B bounds the sum of the
     * magnitudes of all primitive contributions to (ab|cd), not only |(ab|cd)|. */
    double fp32_cutoff;      /* MIXED: quartets with R_ab * R_cd below this run the VRR in
                                FP32 (FP64 Boys, prefactors, contraction and HRR); R_ab =
                                (1+|A-B|)^lb sum_i sqrt(max |[e0|e0]_ii|) bounds the VRR
                                output block the HRR combines */
    double screen_cutoff;    /* quartets with B below this are written as 0, and their work
                                is skipped: such plans order each class's pairs by Qabs and
                                end each bra's ket run after its last unscreened ket (a direct
                                output is cleared with one memset first, a two-phase one gets
                                the zeros from the gather).  The bra/ket roles of some
                                same-class quartets then differ from an unscreened plan's, so
                                the kept integrals agree with it to rounding, not bit for bit.
                                Shard plans keep the per-quartet test only. */
    double prim_cutoff;      /* primitive pairs i with b_i * max_cd Qabs_cd below this are
                                dropped, b_i = sqrt(max |(a_i b_i|a_i b_i)|); each dropped
                                contribution is below prim_cutoff.  Default 1e-18. */
} molints_options;

typedef struct molints_stats {
    int64_t n_eri;            /* packed integrals written */
    int64_t n_shell_quartets; /* unique shell quartets */
    int64_t n_prim_quartets;  /* primitive quartets in those */
    int64_t n_fp32_quartets;  /* quartets that ran an FP32 kernel variant: bound below
                                 fp32_cutoff, in a class pair whose plan launches its FP32
                                 variant (counted on the host) */
    int64_t n_screened;       /* quartets skipped by screen_cutoff (counted on the host) */
    int32_t n_kernel_launches;
    int32_t n_fp32_launches;  /* class-pair kernels of the last execute launched as their FP32
                                 variant (MIXED plans) */
    double device_ms;         /* device time of the last execute (CUDA events) */
    int64_t n_prim_pairs;     /* primitive pairs of all shell pairs */
    int64_t n_prim_pairs_kept;/* primitive pairs left after prim_cutoff */
    /* host wall time of plan creation, ms: [0] host tables (pair list, stage-1 primitive
     * pairs, gather tables), [1] uploads and the device build up to its one read-back
     * (normalisation, bound pass, screening, pair re-sort, work-queue sizes), [2] work-queue
     * emission and ordering (launches), [3] the rest (g-shell quartet lists) */
    double plan_ms[4];
} molints_stats;

typedef struct molints_ctx molints_ctx;
typedef struct molints_plan molints_plan;

/* Library version / ABI check. */
int molints_abi_version(void);

/* Fill opts with the defaults: AUTO, FP64, reference Boys, fp32_cutoff 0, screen_cutoff 0,
 * prim_cutoff 1e-18. */
void molints_default_options(molints_options *opts);

/* Number of basis functions of a basis, or a negative status. */
int64_t molints_nbf(const molints_basis *basis);
/* Length of the packed vector for n functions: n(n+1)(n^2+n+2)/8 (src/ERI.jl:106). */
int64_t molints_npacked(int64_t nbf);

/* Create a context on a CUDA device.  hbm_budget_bytes bounds the device memory the
 * context may hold (0 = no bound).  flags is reserved (0). */
int molints_create(molints_ctx **ctx, int device, int64_t hbm_budget_bytes, uint32_t flags);
int molints_destroy(molints_ctx *ctx);
const char *molints_last_error(const molints_ctx *ctx);

/* Per class pair method for MOLINTS_METHOD_AUTO plans created afterwards (the autotuner's
 * choice).  methods[x * MOLINTS_NUM_PAIR_CLASSES + y] for bra class x >= ket class y is
 * MOLINTS_METHOD_HGP, MOLINTS_METHOD_RYS or MOLINTS_METHOD_AUTO (HGP where it exists);
 * entries with y > x are ignored.  n must be MOLINTS_NUM_PAIR_CLASSES^2.  A new context starts
 * with the default table: on an NVIDIA B200 the class tuner's measured choices shipped with the
 * library (Rys for the heavy d and f classes, FP32 variants only where they measured faster),
 * elsewhere HGP everywhere.  methods == NULL restores that default.  No reference counterpart
 * (the reference picks its driver by function name). */
int molints_set_class_methods(molints_ctx *ctx, const int32_t *methods, int32_t n);
/* The context's current table, in the layout of molints_set_class_methods (n entries). */
int molints_get_class_methods(const molints_ctx *ctx, int32_t *methods, int32_t n);
/* Flag OR'ed into a molints_set_class_methods entry: MIXED plans run that class pair's FP64
 * kernel (its FP32 variant measured no faster).  It applies when the plan runs the entry's own
 * method (or the entry is AUTO); a plan whose options force the other method ignores it. */
#define MOLINTS_CLASS_NO_FP32 4

/* Work-queue schedule of the plans a context creates (no reference counterpart: the
 * reference evaluates one shell quartet at a time).  Plans created after the call use it.
 *   lane_cost     HGP lane split: a quartet's primitive quartets are spread over up to 32
 *                 lanes until one lane's share costs at most lane_cost (ss|ss)-equivalents
 *                 (default 80)
 *   hgp_widen     ket pairs of an unsplit HGP chunk, in units of 32 (one per lane) (default 1;
 *                 very large batches widen further to bound the queue length)
 *   rys_chunks    Rys chunks are as long as keeps about this many chunks in a class queue
 *                 (default 4096)
 *   rys_max_width the longest Rys chunk, in ket pairs (default 8)
 *   gather_blocks resident blocks per SM of the two-phase output's gather pass, in [1, 16]
 *                 (0 = default 5): its persistent grid is this many blocks per SM.  Fewer
 *                 blocks trade warps for L1 space per block.
 * On a B200 the defaults are the shipped tuned values (autotune.tune_schedule); s == NULL
 * restores them. */
typedef struct molints_schedule {
    double lane_cost;
    int32_t hgp_widen;
    int32_t rys_chunks;
    int32_t rys_max_width;
    int32_t gather_blocks;
} molints_schedule;
int molints_set_schedule(molints_ctx *ctx, const molints_schedule *s);
int molints_get_schedule(const molints_ctx *ctx, molints_schedule *s);

/* Set the CUDA stream (a cudaStream_t passed as void*) the context launches on.
 * NULL selects the context's own (non-blocking) stream; to launch on the legacy default
 * stream pass cudaStreamLegacy ((void*)0x1). */
int molints_set_stream(molints_ctx *ctx, void *stream);

/* One call, the drop-in for all_twoe_ints / all_twoe_ints_chrr: computes every unique
 * integral of the basis into out[molints_npacked(nbf)].  out is a host pointer (pinned or
 * pageable) when out_is_device == 0, a device pointer on the context's device otherwise.
 * The call returns when the result is in out.  stats may be NULL. */
int molints_eri_packed(molints_ctx *ctx, const molints_basis *basis,
                       const molints_options *opts, double *out, int out_is_device,
                       molints_stats *stats);

/* Plans: the device-resident form of one basis.  plan_create normalises the basis, builds
 * the primitive pairs and their Schwarz bounds on the device, drops negligible primitive
 * pairs (prim_cutoff), orders the shell pairs by class and kept contraction length and
 * uploads the pair tables (it synchronises the context's stream once).  plan_execute then
 * runs the device path -- primitive-pair records and every shell quartet -- into a device
 * vector of molints_npacked(nbf) doubles, on the context's stream, without host
 * synchronisation. */
int molints_plan_create(molints_ctx *ctx, const molints_basis *basis,
                        const molints_options *opts, molints_plan **plan);
/* A plan over nmol molecules at once (no reference counterpart; the batched form of
 * all_twoe_ints).  One execute computes every molecule; molecule m's packed vector starts at
 * out_device + sum over m' < m of molints_npacked(nbf(m')).  All shell quartets of all
 * molecules go through one work queue per class pair. */
int molints_plan_create_batch(molints_ctx *ctx, int32_t nmol, const molints_basis *bases,
                              const molints_options *opts, molints_plan **plan);
/* Sharding one basis over nshards devices (no reference counterpart).  Shard r owns the shell
 * quartets whose highest shell index lies in a contiguous shell range (split by estimated
 * cost), which are exactly the integrals of one contiguous slice [lo, hi) of the packed
 * vector.  molints_shard_range gives the slice (host only, no device needed);
 * molints_plan_create_shard makes a plan whose execute writes that slice into
 * out_device[0 .. hi-lo).  The slices of shards 0..nshards-1 tile the vector in order. */
int molints_shard_range(const molints_basis *basis, int32_t shard, int32_t nshards, int64_t *lo,
                        int64_t *hi);
int molints_plan_create_shard(molints_ctx *ctx, const molints_basis *basis,
                              const molints_options *opts, int32_t shard, int32_t nshards,
                              molints_plan **plan);
/* Doubles the plan writes per execute (all molecules; a shard plan: its slice), or a negative
 * status. */
int64_t molints_plan_npacked(const molints_plan *plan);
int molints_plan_execute(molints_plan *plan, double *out_device);
/* Coulomb and exchange matrices instead of the packed vector: one execute of a one-molecule
 * plan (or of a shard plan: that shard's share) digests every unique integral into
 * J_pq = sum_rs D_rs (pq|rs) and K_pr = sum_qs D_qs (pq|rs), n x n row-major device arrays
 * (zeroed by the call) for a symmetric device density D, on the context's stream.  No packed
 * vector is written.  The reference consumer is make2JmK (src/ERI.jl:114-128), which forms
 * 2J - K from the packed vector. */
int molints_plan_jk(molints_plan *plan, const double *D_device, double *J_device, double *K_device);
/* The same from host arrays in one synchronous call (plan, device buffers, copies). */
int molints_jk(molints_ctx *ctx, const molints_basis *basis, const molints_options *opts,
               const double *D_host, double *J_host, double *K_host);
/* enable != 0: the next execute captures the plan's whole device path (pair build, counter
 * reset, every class-pair kernel on the forked side streams) into a CUDA graph on the
 * context's stream, and later executes into the same out_device launch that graph (a new
 * out_device recaptures).  Not combined with profiling.  No reference counterpart. */
int molints_plan_set_graph(molints_plan *plan, int enable);
int molints_plan_stats(const molints_plan *plan, molints_stats *stats);
/* Per class pair x >= y (entry x * MOLINTS_NUM_PAIR_CLASSES + y, n = MOLINTS_NUM_PAIR_CLASSES^2):
 * the plan's shell quartets and the primitive quartets its kernels evaluate (the primitive
 * pairs kept after prim_cutoff; screen_cutoff not applied), for work accounting.  Host only.
 * No reference counterpart. */
int molints_plan_class_work(const molints_plan *plan, int64_t *quartets, double *prim_quartets,
                            int32_t n);
int molints_plan_destroy(molints_plan *plan);

/* Contracted Schwarz bounds Q_ab = sqrt(max |(ab|ab)|) of the plan's shell pairs (computed
 * on demand on the context's stream; the plan must have been executed once), in the
 * reference's pair order (shell i >= shell j, row-major): out[nshell*(nshell+1)/2], one such
 * block per molecule of a batch plan, in molecule order. */
int molints_plan_schwarz(molints_plan *plan, double *out_host);

/* Per-launch device times.  After molints_plan_set_profiling(plan, 1), every execute runs
 * its kernels one after another on the context's stream (no side streams) and records a CUDA
 * event pair around each launch; molints_plan_launch_times then waits for the
 * last execute and returns up to cap entries: names[k] (static strings such as
 * "eri_ssss", "schwarz_pp", "build_pairs") and ms[k].  Returns the number of launches of the
 * last execute, or a negative status. */
int molints_plan_set_profiling(molints_plan *plan, int enable);
int molints_plan_launch_times(molints_plan *plan, const char **names, float *ms, int cap);

/* F_m(T) for m = 0..mmax-1 at n values of T, evaluated by the device Boys function
 * (src/Boys.jl:19-27) in the given mode.  T and out are host arrays; out is [n][mmax]. */
int molints_boys_eval(molints_ctx *ctx, int32_t boys_mode, int32_t mmax, const double *T,
                      int64_t n, double *out);

/* The ERI path for callers that cannot allocate device memory where they need the
 * integrals: host programs whose own allocator has reserved the GPU's memory (a framework's
 * caching allocator, a simulation code's memory manager), and time-critical loops that cannot
 * take the device synchronisation a cudaMalloc or cudaFree may cause.  There is no counterpart
 * in the reference.  It needs no context and allocates nothing: the caller passes the basis
 * (host arrays, as for molints_eri_packed) and its own device vector out_device of
 * molints_npacked(nbf) doubles; the Boys table, the pair tables and the work queues live in
 * one static device array of 8 MiB that every GPU which loads the library holds until exit.
 * Bases whose tables do not fit are rejected with MOLINTS_ERR_UNSUPPORTED and a message in err
 * (err may be NULL).  FP64 without screening, shells up to d only (opts NULL = defaults;
 * prim_cutoff is ignored: every primitive pair is kept).  The first call on a device, with
 * that device current, looks the array up with cudaGetSymbolAddress and copies the Boys table
 * into it synchronously, so make that first call before any stream capture.  The call enqueues
 * its work on `stream` (a cudaStream_t; NULL is the legacy default stream) and returns; all
 * calls share the array, so calls whose GPU work overlaps race on it. */
int molints_eri_packed_noalloc(const molints_basis *basis, const molints_options *opts,
                               double *out_device, void *stream, char *err, size_t err_len);

/* The one-electron matrices of the basis, the drop-in for all_1e_ints(bfs, mol)
 * (src/OneInts.jl:267-290): overlap S, kinetic energy T and nuclear attraction V (summed over
 * natom point charges atom_charge[c] at atom_xyz[3c..3c+2], bohr), each n x n row-major in host
 * memory, for the same normalised functions as the ERIs.  Shells up to f.  Synchronous. */
int molints_one_e(molints_ctx *ctx, const molints_basis *basis, int32_t natom,
                  const double *atom_xyz, const double *atom_charge, double *S, double *T, double *V);

/* ------------------------------------------------------------------------------------------
 * Serving: molecules submitted as they arrive, computed concurrently, results kept on the
 * device until released.  No reference counterpart (the reference computes one basis per
 * blocking call); each request's vector is what molints_eri_packed would write for it.
 *
 * molints_serve_start gives the context a server of nslots slot workers (host threads, each
 * with its own engine context and stream on the context's device).  A free slot admits the
 * smallest queued request for which the server's HBM ledger -- resident result vectors plus
 * the pair tables of running plans -- has room under hbm_budget_bytes (0 = no bound); a
 * request that has waited 40 ms is admitted before any other (nothing else is admitted until it
 * fits), so none starves.  New requests join the ones already running and their kernels
 * overlap on the device.  A request larger than the whole budget fails with
 * MOLINTS_ERR_BUDGET.
 * submit, poll, result, release and request_info may be called from any host thread. */
typedef struct molints_request molints_request;

/* The slots take the context's per-class method table (molints_set_class_methods) as it is at
 * this call. */
int molints_serve_start(molints_ctx *ctx, int32_t nslots, int64_t hbm_budget_bytes);
/* Stop the server: queued requests fail, running ones finish; results stay valid until
 * released.  molints_destroy stops the context's server. */
int molints_serve_stop(molints_ctx *ctx);
/* Queue one basis (copied; the caller's arrays may be reused at once). */
int molints_submit(molints_ctx *ctx, const molints_basis *basis, const molints_options *opts,
                   molints_request **req);
/* Wait up to timeout_ms (0: do not wait, < 0: no limit) for the request: MOLINTS_OK when its
 * result is ready, MOLINTS_ERR_TIMEOUT if not yet, or the request's own error status. */
int molints_poll(molints_request *req, int32_t timeout_ms);
/* The finished request's packed vector: a device pointer of *len doubles on the server's
 * device, valid until molints_release. */
int molints_result(molints_request *req, double **out_device, int64_t *len);
/* Copy the finished request's vector (len == its length) into host memory. */
int molints_result_copy(molints_request *req, double *out_host, int64_t len);
/* Host steady-clock seconds of submission, admission and completion, and the slot that ran
 * the request (MOLINTS_ERR_TIMEOUT while it is not finished). */
int molints_request_info(molints_request *req, double *t_submit, double *t_admit, double *t_done,
                         int32_t *slot);
const char *molints_request_error(const molints_request *req);
/* Give the request back: frees its result (or withdraws it from the queue; a running request
 * is freed when it finishes).  The handle is invalid afterwards. */
int molints_release(molints_request *req);
/* Ledger bytes in use, queued, finished and failed request counts of the context's server. */
int molints_serve_stats(molints_ctx *ctx, int64_t *ledger_bytes, int64_t *queued, int64_t *done,
                        int64_t *failed);

#ifdef __cplusplus
}
#endif
#endif /* MOLINTS_H */

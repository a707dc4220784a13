// serve.cu -- the serving form of the ERI engine: molints_submit / poll / result / release.
//
// A context's server is a set of slot workers (host threads), each with its own engine
// context and stream on the same device.  Requests (a basis and options) wait in one queue.  A
// free worker admits the smallest queued request that the HBM budget ledger can hold -- its
// output vector plus its plan's pair tables -- or, once the oldest request has waited
// kMaxWait, that one (then nothing else is admitted before it, so no request starves).
// Requests that arrive while others are on the GPU join them: several plans execute at once on
// the workers' streams and their kernels share the device (continuous batching).  Taking the
// smallest first keeps small requests from queueing behind large ones when every slot is busy.  A finished request keeps
// its packed ERI vector resident on the device until the caller releases it; its plan tables
// are freed at completion.  The reference has no serving form; this is the batched,
// asynchronous counterpart of all_twoe_ints (src/ERI.jl:104-112).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/molints.h"

namespace molints {
int ctx_device_of(const molints_ctx *ctx);                          // molints.cu
void ctx_copy_methods(molints_ctx *dst, const molints_ctx *src);    // molints.cu
}  // namespace molints

namespace {

double now_s() {
    using namespace std::chrono;
    return duration_cast<duration<double>>(steady_clock::now().time_since_epoch()).count();
}

struct Server;

}  // namespace

struct molints_request {
    Server *srv = nullptr;
    // owned copy of the basis
    std::vector<double> xyz, expn, coef;
    std::vector<int32_t> L, nprim, prim_off;
    molints_basis basis{};
    molints_options opts{};
    int64_t npacked = 0;
    int64_t need_out = 0, need_plan = 0;  // ledger bytes: output vector, plan tables
    // state, guarded by the server mutex
    int state = 0;       // 0 queued, 1 running, 2 done, 3 failed
    int status = 0;      // final status of the request
    bool released = false;
    double *out = nullptr;  // device vector (done)
    std::string err;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int slot = -1;
};

namespace {

struct Server {
    int device = 0;
    int64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work;   // workers: a request or a release may let one proceed
    std::condition_variable cv_done;   // pollers
    std::deque<molints_request *> queue;
    int64_t ledger = 0;                // bytes admitted and not yet given back
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<molints_ctx *> ctxs;
    std::vector<cudaStream_t> streams;
    cudaMemPool_t pool = nullptr;      // output vectors
    cudaStream_t free_stream = nullptr;
    int64_t n_done = 0, n_failed = 0;
    int64_t live = 0;                  // request objects not yet deleted
    bool stopped = false;              // molints_serve_stop ran; the last release frees the rest

    void worker(int slot);
    void destroy_resources();
    molints_request *pick() const;
};

// Seconds after which the oldest queued request is admitted before any smaller one.
constexpr double kMaxWait = 0.040;

// The request a free worker admits now, or nullptr (called with mu held): the oldest once it
// has waited kMaxWait (if it does not fit, nothing is admitted until releases make room);
// otherwise the smallest one that fits, the oldest among equals.
molints_request *Server::pick() const {
    if (queue.empty()) return nullptr;
    auto fits = [&](const molints_request *r) {
        return budget <= 0 || ledger + r->need_out + r->need_plan <= budget;
    };
    molints_request *h = queue.front();
    if (now_s() - h->t_submit > kMaxWait) return fits(h) ? h : nullptr;
    molints_request *best = nullptr;
    for (molints_request *r : queue)
        if (fits(r) && (!best || r->need_out < best->need_out)) best = r;
    return best;
}

// Pool and free stream, once no request can reach them any more.
void Server::destroy_resources() {
    cudaSetDevice(device);
    cudaStreamSynchronize(free_stream);
    cudaStreamDestroy(free_stream);
    cudaMemPoolDestroy(pool);
}

// Device bytes a plan of this basis holds (an upper bound of molints_plan_create's tables:
// shells, primitives, pairs, primitive pairs, chunk queues, and for a two-phase output the
// scratch of quartet blocks: the sum over shell-pair pairs P >= Q of n_P n_Q components, at
// most (S^2 + S n_max) / 2 with S = sum_P n_P).
int64_t plan_bytes(const molints_basis &b, const molints_options &o, int64_t npacked) {
    int64_t nprim = 0, nall = 0;
    for (int s = 0; s < b.nshell; ++s) nprim = std::max<int64_t>(nprim, b.prim_off[s] + b.nprim[s]);
    for (int i = 0; i < b.nshell; ++i)
        for (int j = 0; j <= i; ++j) nall += (int64_t)b.nprim[i] * b.nprim[j];
    const int64_t npair = (int64_t)b.nshell * (b.nshell + 1) / 2;
    const int64_t nchunk = npair * (npair + 1) / 2 / 32 + npair * 2;
    int64_t scratch = 0;
    (void)npacked;  // the workers run AUTO requests DIRECT
    if (o.output == MOLINTS_OUTPUT_TWO_PHASE) {
        double S = 0.0;
        for (int i = 0; i < b.nshell; ++i)
            for (int j = 0; j <= i; ++j)
                S += (double)((b.L[i] + 1) * (b.L[i] + 2) / 2) * ((b.L[j] + 1) * (b.L[j] + 2) / 2);
        scratch = (int64_t)(8.0 * (S * S + S * 100.0) / 2.0) + 8 * nchunk;
    }
    return 40 * (int64_t)b.nshell + 24 * nprim + 88 * npair + 100 * nall + 16 * nchunk + scratch + (4 << 20);
}

void Server::worker(int slot) {
    cudaSetDevice(device);
    molints_ctx *ctx = ctxs[slot];
    cudaStream_t s = streams[slot];
    for (;;) {
        molints_request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            // woken by submits and releases; the timeout re-checks the oldest request's age
            while (!stop && !(r = pick())) cv_work.wait_for(lk, std::chrono::milliseconds(5));
            if (stop) return;
            queue.erase(std::find(queue.begin(), queue.end(), r));
            ledger += r->need_out + r->need_plan;
            r->state = 1;
            r->slot = slot;
            r->t_admit = now_s();
        }
        int rc = MOLINTS_OK;
        std::string msg;
        molints_plan *plan = nullptr;
        double *out = nullptr;
        // AUTO requests run DIRECT: with eight slots in flight, each large request's scratch (as
        // large as its output) raised the mean latency of the serving stream by 12 %
        molints_options popts = r->opts;
        if (popts.output == MOLINTS_OUTPUT_AUTO) popts.output = MOLINTS_OUTPUT_DIRECT;
        rc = molints_plan_create(ctx, &r->basis, &popts, &plan);
        if (rc) msg = molints_last_error(ctx);
        if (!rc && r->npacked > 0) {
            cudaError_t e = cudaMallocFromPoolAsync((void **)&out, (size_t)r->npacked * sizeof(double), pool, s);
            if (e != cudaSuccess) { rc = MOLINTS_ERR_CUDA; msg = cudaGetErrorString(e); out = nullptr; }
        }
        if (!rc) {
            rc = molints_plan_execute(plan, out);
            if (rc) msg = molints_last_error(ctx);
        }
        if (!rc) {
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) { rc = MOLINTS_ERR_CUDA; msg = cudaGetErrorString(e); }
        }
        if (plan) molints_plan_destroy(plan);
        if (rc && out) {
            cudaFreeAsync(out, s);
            out = nullptr;
        }
        bool free_now = false;
        {
            std::lock_guard<std::mutex> lk(mu);
            ledger -= r->need_plan;
            r->t_done = now_s();
            if (rc) {
                ledger -= r->need_out;
                r->state = 3;
                r->status = rc;
                r->err = msg;
                ++n_failed;
            } else {
                r->state = 2;
                r->out = out;
                ++n_done;
                if (r->released) {  // the caller gave the request up while it ran
                    ledger -= r->need_out;
                    free_now = true;
                }
            }
        }
        if (free_now) {
            if (out) cudaFreeAsync(out, s);
            delete r;
            std::lock_guard<std::mutex> lk(mu);
            --live;
        }
        cv_work.notify_all();
        cv_done.notify_all();
    }
}

Server *server_start(molints_ctx *ctx, int device, int nslots, int64_t budget, std::string &err) {
    Server *S = new (std::nothrow) Server();
    if (!S) return nullptr;
    S->device = device;
    S->budget = budget;
    if (cudaSetDevice(device) != cudaSuccess) { err = "cudaSetDevice"; delete S; return nullptr; }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&S->pool, &props) != cudaSuccess) { err = "cudaMemPoolCreate"; delete S; return nullptr; }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (cudaStreamCreateWithFlags(&S->free_stream, cudaStreamNonBlocking) != cudaSuccess) {
        err = "cudaStreamCreate";
        cudaMemPoolDestroy(S->pool);
        delete S;
        return nullptr;
    }
    for (int i = 0; i < nslots; ++i) {
        molints_ctx *c = nullptr;
        if (molints_create(&c, device, 0, 0) != MOLINTS_OK) break;
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            molints_destroy(c);
            break;
        }
        molints_set_stream(c, st);
        molints::ctx_copy_methods(c, ctx);  // the slots follow the owner's AUTO method table
        S->ctxs.push_back(c);
        S->streams.push_back(st);
    }
    if ((int)S->ctxs.size() != nslots) {
        for (size_t i = 0; i < S->ctxs.size(); ++i) {
            molints_destroy(S->ctxs[i]);
            cudaStreamDestroy(S->streams[i]);
        }
        cudaStreamDestroy(S->free_stream);
        cudaMemPoolDestroy(S->pool);
        err = "could not create the slot contexts";
        delete S;
        return nullptr;
    }
    for (int i = 0; i < nslots; ++i) S->workers.emplace_back(&Server::worker, S, i);
    return S;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
namespace {
std::mutex g_srv_mu;
std::vector<std::pair<molints_ctx *, Server *>> g_servers;

Server *find_server(molints_ctx *ctx) {
    for (auto &p : g_servers)
        if (p.first == ctx) return p.second;
    return nullptr;
}
}  // namespace

extern "C" {

int molints_serve_start(molints_ctx *ctx, int32_t nslots, int64_t hbm_budget_bytes) {
    if (!ctx || nslots < 1 || nslots > 64 || hbm_budget_bytes < 0) return MOLINTS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_srv_mu);
    if (find_server(ctx)) return MOLINTS_ERR_INVALID;
    const int dev = molints::ctx_device_of(ctx);
    std::string err;
    Server *S = server_start(ctx, dev, nslots, hbm_budget_bytes, err);
    if (!S) return MOLINTS_ERR_CUDA;
    g_servers.push_back({ctx, S});
    return MOLINTS_OK;
}

int molints_serve_stop(molints_ctx *ctx) {
    if (!ctx) return MOLINTS_ERR_INVALID;
    Server *S = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_srv_mu);
        for (size_t i = 0; i < g_servers.size(); ++i)
            if (g_servers[i].first == ctx) {
                S = g_servers[i].second;
                g_servers.erase(g_servers.begin() + i);
                break;
            }
    }
    if (!S) return MOLINTS_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        // queued requests fail; running ones finish
        for (molints_request *r : S->queue) {
            r->state = 3;
            r->status = MOLINTS_ERR_INVALID;
            r->err = "server stopped";
        }
        S->queue.clear();
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
    for (std::thread &t : S->workers) t.join();
    cudaSetDevice(S->device);
    for (size_t i = 0; i < S->ctxs.size(); ++i) {
        molints_destroy(S->ctxs[i]);
        cudaStreamDestroy(S->streams[i]);
    }
    // Results not yet released stay valid until their release, which then frees the rest.
    bool last = false;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopped = true;
        last = S->live == 0;
    }
    if (last) {
        S->destroy_resources();
        delete S;
    }
    return MOLINTS_OK;
}

int molints_submit(molints_ctx *ctx, const molints_basis *b, const molints_options *opts,
                   molints_request **out) {
    if (!ctx || !b || !out) return MOLINTS_ERR_INVALID;
    *out = nullptr;
    Server *S = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_srv_mu);
        S = find_server(ctx);
    }
    if (!S) return MOLINTS_ERR_INVALID;
    const int64_t nbf = molints_nbf(b);
    if (nbf < 0) return MOLINTS_ERR_INVALID;
    const int ns = b->nshell;
    if (ns > 0 && (!b->expn || !b->coef)) return MOLINTS_ERR_INVALID;
    molints_request *r = new (std::nothrow) molints_request();
    if (!r) return MOLINTS_ERR_NOMEM;
    r->srv = S;
    int64_t nprim = 0;
    for (int s = 0; s < ns; ++s) {
        if (b->nprim[s] < 1 || b->prim_off[s] < 0) { delete r; return MOLINTS_ERR_INVALID; }
        nprim = std::max<int64_t>(nprim, b->prim_off[s] + b->nprim[s]);
    }
    r->xyz.assign(b->xyz, b->xyz + 3 * (size_t)ns);
    r->L.assign(b->L, b->L + ns);
    r->nprim.assign(b->nprim, b->nprim + ns);
    r->prim_off.assign(b->prim_off, b->prim_off + ns);
    r->expn.assign(b->expn, b->expn + nprim);
    r->coef.assign(b->coef, b->coef + nprim);
    r->basis = molints_basis{ns, r->xyz.data(), r->L.data(), r->nprim.data(), r->prim_off.data(),
                             r->expn.data(), r->coef.data()};
    if (opts) r->opts = *opts; else molints_default_options(&r->opts);
    r->npacked = molints_npacked(nbf);
    r->need_out = r->npacked * (int64_t)sizeof(double);
    r->need_plan = plan_bytes(r->basis, r->opts, r->npacked);
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        ++S->live;
        if (S->budget > 0 && r->need_out + r->need_plan > S->budget) {
            r->state = 3;
            r->status = MOLINTS_ERR_BUDGET;
            r->err = "request larger than the serving HBM budget";
            r->t_done = r->t_submit;
        } else {
            S->queue.push_back(r);
        }
    }
    S->cv_work.notify_one();
    *out = r;
    return MOLINTS_OK;
}

int molints_poll(molints_request *r, int32_t timeout_ms) {
    if (!r) return MOLINTS_ERR_INVALID;
    Server *S = r->srv;
    std::unique_lock<std::mutex> lk(S->mu);
    auto ready = [&] { return r->state >= 2; };
    if (!ready()) {
        if (timeout_ms == 0) return MOLINTS_ERR_TIMEOUT;
        if (timeout_ms < 0) S->cv_done.wait(lk, ready);
        else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return MOLINTS_ERR_TIMEOUT;
    }
    return r->state == 2 ? MOLINTS_OK : r->status;
}

int molints_result(molints_request *r, double **out_device, int64_t *len) {
    if (!r || !out_device || !len) return MOLINTS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->srv->mu);
    if (r->state < 2) return MOLINTS_ERR_TIMEOUT;
    if (r->state == 3) return r->status;
    *out_device = r->out;
    *len = r->npacked;
    return MOLINTS_OK;
}

int molints_result_copy(molints_request *r, double *out_host, int64_t len) {
    if (!r || (!out_host && len > 0)) return MOLINTS_ERR_INVALID;
    double *src = nullptr;
    int64_t n = 0;
    int rc = molints_result(r, &src, &n);
    if (rc) return rc;
    if (len != n) return MOLINTS_ERR_INVALID;
    if (n == 0) return MOLINTS_OK;
    Server *S = r->srv;
    if (cudaSetDevice(S->device) != cudaSuccess) return MOLINTS_ERR_CUDA;
    if (cudaMemcpy(out_host, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MOLINTS_ERR_CUDA;
    return MOLINTS_OK;
}

int molints_request_info(molints_request *r, double *t_submit, double *t_admit, double *t_done,
                         int32_t *slot) {
    if (!r) return MOLINTS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->srv->mu);
    if (t_submit) *t_submit = r->t_submit;
    if (t_admit) *t_admit = r->t_admit;
    if (t_done) *t_done = r->t_done;
    if (slot) *slot = r->slot;
    return r->state >= 2 ? MOLINTS_OK : MOLINTS_ERR_TIMEOUT;
}

const char *molints_request_error(const molints_request *r) { return r ? r->err.c_str() : "no request"; }

int molints_release(molints_request *r) {
    if (!r) return MOLINTS_OK;
    Server *S = r->srv;
    double *out = nullptr;
    bool del = false;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (r->released) return MOLINTS_ERR_INVALID;
        r->released = true;
        if (r->state == 0) {  // still queued: withdraw it
            S->queue.erase(std::remove(S->queue.begin(), S->queue.end(), r), S->queue.end());
            del = true;
        } else if (r->state == 2) {
            out = r->out;
            S->ledger -= r->need_out;
            del = true;
        } else if (r->state == 3) {
            del = true;
        }  // running: the worker frees it at completion
    }
    if (out) {
        cudaSetDevice(S->device);
        cudaFreeAsync(out, S->free_stream);
    }
    bool last = false;
    if (del) {
        delete r;
        std::lock_guard<std::mutex> lk(S->mu);
        last = --S->live == 0 && S->stopped;
    }
    if (last) {
        S->destroy_resources();
        delete S;
        return MOLINTS_OK;
    }
    S->cv_work.notify_all();
    return MOLINTS_OK;
}

int molints_serve_stats(molints_ctx *ctx, int64_t *ledger_bytes, int64_t *queued, int64_t *done,
                        int64_t *failed) {
    if (!ctx) return MOLINTS_ERR_INVALID;
    Server *S = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_srv_mu);
        S = find_server(ctx);
    }
    if (!S) return MOLINTS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    if (ledger_bytes) *ledger_bytes = S->ledger;
    if (queued) *queued = (int64_t)S->queue.size();
    if (done) *done = S->n_done;
    if (failed) *failed = S->n_failed;
    return MOLINTS_OK;
}

}  // extern "C"

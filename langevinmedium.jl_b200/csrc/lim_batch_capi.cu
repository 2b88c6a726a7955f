// lim_batch_capi.cu — the batch entry points of the C-ABI (include/langevin_b200.h):
// many configured contexts advanced together, one persistent launch per chunk of
// steps, the chunk sequence captured once as a CUDA graph and replayed.
#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "lim_ctx.h"

using namespace lim;

namespace {
thread_local std::string g_batch_create_error;
}

struct lim_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    struct Ens {
        lim_ctx* c;
        int64_t first, nsteps;
        uint64_t gen;
    };
    std::vector<Ens> ens;
    lim_batch_shape shape{ 256, 0, 0, 0 };

    // prepared launch data (valid while `prepared` and no context changed)
    bool prepared = false;
    int prec = -1, dims = 0, pdim = 0;
    bool fo = false, cap = false;
    int block = 256, grid = 0;
    int64_t chunk = 0, nchunks = 0, max_steps = 0;
    std::vector<int64_t> chunk_first;     // item offset of every chunk (nchunks + 1)
    DevBuf d_kp, d_items, d_counters, d_status, d_tables;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    int64_t last_launches = 0, particle_steps = 0;
};

namespace {

int bfail(lim_batch* b, int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->err = buf; else g_batch_create_error = buf;
    return code;
}

#define LIM_BCUDA(b, call)                                                                      \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return bfail((b), LIM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));    \
    } while (0)

int balloc(lim_batch* b, DevBuf& d, size_t bytes)
{
    if (d.p && d.bytes >= bytes) return LIM_OK;
    if (d.p) { cudaFree(d.p); d.p = nullptr; d.bytes = 0; }
    if (!bytes) return LIM_OK;
    cudaError_t e = cudaMalloc(&d.p, bytes);
    if (e != cudaSuccess) {
        d.p = nullptr;
        return bfail(b, LIM_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    d.bytes = bytes;
    return LIM_OK;
}
void bfree(DevBuf& d)
{
    if (d.p) cudaFree(d.p);
    d.p = nullptr;
    d.bytes = 0;
}

void release_graph(lim_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->prepared = false;
}

bool stale(const lim_batch* b)
{
    if (!b->prepared) return true;
    for (const auto& e : b->ens)
        if (e.c->gen != e.gen) return true;
    return false;
}

int sync_contexts(lim_batch* b)
{
    for (const auto& e : b->ens) LIM_BCUDA(b, cudaStreamSynchronize(e.c->stream));
    return LIM_OK;
}

// Checks that the ensembles can share one launch; fills prec/dims/pdim/fo.
int check_uniform(lim_batch* b)
{
    if (b->ens.empty()) return bfail(b, LIM_ERR_STATE, "the batch has no ensembles (lim_batch_add)");
    const lim_ctx* c0 = b->ens[0].c;
    for (size_t k = 0; k < b->ens.size(); ++k) {
        lim_ctx* c = b->ens[k].c;
        if (ctx_check_ready(c)) return bfail(b, LIM_ERR_STATE, "ensemble %zu: %s", k, c->err.c_str());
        if (c->device != b->device)
            return bfail(b, LIM_ERR_ARG, "ensemble %zu lives on device %d, the batch on %d", k, c->device, b->device);
        if (c->P.coords != LIM_COORDS_CARTESIAN)
            return bfail(b, LIM_ERR_UNSUPPORTED, "ensemble %zu: batches run Cartesian coordinates only", k);
        if (c->P.precision != c0->P.precision || c->dims != c0->dims || c->pdim != c0->pdim)
            return bfail(b, LIM_ERR_ARG, "ensemble %zu: precision, dimensions and momentum_dimensions must match ensemble 0", k);
        if ((c->P.freezeout_capture != 0) != (c0->P.freezeout_capture != 0))
            return bfail(b, LIM_ERR_ARG, "ensemble %zu: freezeout_capture must match ensemble 0", k);
        if (c->P.seed != c0->P.seed)
            return bfail(b, LIM_ERR_ARG, "ensemble %zu: all ensembles share one seed (particle_offset keeps their noise apart)", k);
    }
    const int dp = c0->dims * 10 + c0->pdim;
    if (dp != 22 && dp != 23 && dp != 33)
        return bfail(b, LIM_ERR_UNSUPPORTED, "batches run (dimensions, momentum_dimensions) = (2,2), (2,3) or (3,3)");
    b->prec = (int)c0->P.precision;
    b->dims = c0->dims;
    b->pdim = c0->pdim;
    b->fo = c0->P.freezeout_capture != 0;
    return LIM_OK;
}

template <typename R>
int prepare_impl(lim_batch* b)
{
    const size_t E = b->ens.size();
    const lim_batch_shape& sh = b->shape;
    b->block = sh.block > 0 ? (int)sh.block : 256;
    b->cap = sizeof(R) == 4 && sh.reg_cap != 0;
    std::vector<KParams<R>> kps(E);
    std::vector<size_t> tab_off(E);
    size_t tab_bytes = 0;
    b->max_steps = 0;
    b->particle_steps = 0;
    for (size_t k = 0; k < E; ++k) {
        tab_off[k] = tab_bytes;
        tab_bytes += ((size_t)b->ens[k].nsteps * step_record_bytes<R>() + 255) & ~(size_t)255;
        b->max_steps = std::max(b->max_steps, b->ens[k].nsteps);
        b->particle_steps += b->ens[k].c->n * b->ens[k].nsteps;
    }
    int rc;
    if ((rc = balloc(b, b->d_tables, std::max<size_t>(tab_bytes, 256)))) return rc;
    if ((rc = balloc(b, b->d_status, E * sizeof(unsigned long long)))) return rc;
    for (size_t k = 0; k < E; ++k) {
        lim_ctx* c = b->ens[k].c;
        if (ctx_build_kparams<R>(c, kps[k])) return bfail(b, LIM_ERR_STATE, "ensemble %zu: %s", k, c->err.c_str());
        KParams<R>& kp = kps[k];
        kp.steps = (char*)b->d_tables.p + tab_off[k];
        kp.step_base = b->ens[k].first;
        kp.step_cap = b->ens[k].nsteps;
        kp.first_bad = (unsigned long long*)b->d_status.p + k;
        kp.rec = nullptr;
        kp.rec_steps = 0;
        LIM_BCUDA(b, launch_batch_table<R>(kp, kp.step_base, kp.step_cap, kp.steps, b->stream));
    }
    if ((rc = balloc(b, b->d_kp, E * sizeof(KParams<R>)))) return rc;
    LIM_BCUDA(b, cudaMemcpyAsync(b->d_kp.p, kps.data(), E * sizeof(KParams<R>), cudaMemcpyHostToDevice, b->stream));

    // work items, chunk by chunk, ensemble by ensemble
    b->chunk = sh.chunk_steps > 0 ? std::min<int64_t>(sh.chunk_steps, std::max<int64_t>(b->max_steps, 1)) : std::max<int64_t>(b->max_steps, 1);
    b->nchunks = (b->max_steps + b->chunk - 1) / b->chunk;
    std::vector<int2> items;
    b->chunk_first.assign(1, 0);
    for (int64_t ch = 0; ch < b->nchunks; ++ch) {
        for (size_t k = 0; k < E; ++k) {
            if (ch * b->chunk >= b->ens[k].nsteps) continue;
            const int64_t tiles = (b->ens[k].c->n + b->block - 1) / b->block;
            for (int64_t t = 0; t < tiles; ++t) items.push_back(make_int2((int)k, (int)t));
        }
        if (items.size() > (size_t)INT_MAX) return bfail(b, LIM_ERR_ARG, "too many work items (%zu)", items.size());
        b->chunk_first.push_back((int64_t)items.size());
    }
    if ((rc = balloc(b, b->d_items, std::max<size_t>(items.size(), 1) * sizeof(int2)))) return rc;
    if (!items.empty())
        LIM_BCUDA(b, cudaMemcpyAsync(b->d_items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    if ((rc = balloc(b, b->d_counters, std::max<int64_t>(b->nchunks, 1) * sizeof(unsigned)))) return rc;
    LIM_BCUDA(b, cudaStreamSynchronize(b->stream));   // host vectors go out of scope

    // persistent grid
    int per_sm = 0;
    LIM_BCUDA(b, batch_blocks_per_sm<R>(b->dims, b->pdim, b->fo, b->cap, b->block, &per_sm));
    if (per_sm < 1) return bfail(b, LIM_ERR_UNSUPPORTED, "the batch kernel does not fit %d threads per block", b->block);
    if (sh.blocks_per_sm > 0) per_sm = std::min<int>(per_sm, (int)sh.blocks_per_sm);
    int sms = 0;
    LIM_BCUDA(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    b->grid = per_sm * sms;

    // the chunk loop as one graph: zero the counters, reset the status, one launch per chunk
    BatchLaunch<R> bl;
    std::memset(&bl, 0, sizeof bl);
    bl.ens = (const KParams<R>*)b->d_kp.p;
    {
        uint32_t k0 = (uint32_t)(uint64_t)b->ens[0].c->P.seed, k1 = (uint32_t)((uint64_t)b->ens[0].c->P.seed >> 32);
        for (int r = 0; r < 10; ++r) { bl.rk[r] = make_uint2(k0, k1); k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
    LIM_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaMemsetAsync(b->d_counters.p, 0, std::max<int64_t>(b->nchunks, 1) * sizeof(unsigned), b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_status.p, 0xFF, E * sizeof(unsigned long long), b->stream);
    int64_t launches = 0;
    for (int64_t ch = 0; ch < b->nchunks && ce == cudaSuccess; ++ch) {
        const int64_t n_items = b->chunk_first[ch + 1] - b->chunk_first[ch];
        if (!n_items) continue;
        bl.items = (const int2*)b->d_items.p + b->chunk_first[ch];
        bl.counter = (unsigned*)b->d_counters.p + ch;
        bl.n_items = (int)n_items;
        bl.chunk_lo = ch * b->chunk;
        bl.chunk_len = b->chunk;
        const int g = (int)std::min<int64_t>(b->grid, n_items);
        ce = launch_batch<R>(bl, b->dims, b->pdim, b->fo, b->cap, g, b->block, b->stream);
        ++launches;
    }
    cudaGraph_t graph = nullptr;
    cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return bfail(b, LIM_ERR_CUDA, "capturing the chunk loop failed: %s",
                     cudaGetErrorString(ce != cudaSuccess ? ce : ee));
    }
    cudaGraphExec_t exec = nullptr;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return bfail(b, LIM_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ce));
    }
    b->graph = graph;
    b->exec = exec;
    b->last_launches = launches;
    for (auto& e : b->ens) e.gen = e.c->gen;
    b->prepared = true;
    return LIM_OK;
}

int prepare(lim_batch* b)
{
    release_graph(b);
    int rc = check_uniform(b);
    if (rc) return rc;
    cudaSetDevice(b->device);
    if ((rc = sync_contexts(b))) return rc;
    return b->prec == LIM_FP32 ? prepare_impl<float>(b) : prepare_impl<double>(b);
}

int run_graph(lim_batch* b)
{
    int rc;
    if (stale(b) && (rc = prepare(b))) return rc;
    cudaSetDevice(b->device);
    if ((rc = sync_contexts(b))) return rc;
    LIM_BCUDA(b, cudaEventRecord(b->ev0, b->stream));
    LIM_BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
    LIM_BCUDA(b, cudaEventRecord(b->ev1, b->stream));
    LIM_BCUDA(b, cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    LIM_BCUDA(b, cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    const size_t E = b->ens.size();
    std::vector<unsigned long long> st(E);
    LIM_BCUDA(b, cudaMemcpy(st.data(), b->d_status.p, E * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < E; ++k)
        if (st[k] != ULLONG_MAX)
            return bfail(b, LIM_ERR_NONFINITE, "Breaking simulation due to NaN/Inf at step %llu (ensemble %zu)", st[k], k);
    return LIM_OK;
}

bool valid_shape(const lim_batch_shape& s)
{
    return (s.block == 0 || s.block == 64 || s.block == 128 || s.block == 256) && s.chunk_steps >= 0 &&
           s.blocks_per_sm >= 0 && (s.reg_cap == 0 || s.reg_cap == 1);
}

}  // namespace

extern "C" {

int lim_batch_create(int device, void* stream, lim_batch** out)
{
    if (!out) return bfail(nullptr, LIM_ERR_ARG, "lim_batch_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return bfail(nullptr, LIM_ERR_CUDA, "cudaGetDeviceCount failed: %s", cudaGetErrorString(e));
    if (device < 0 || device >= ndev)
        return bfail(nullptr, LIM_ERR_ARG, "lim_batch_create: device %d out of range (%d devices)", device, ndev);
    lim_batch* b = new (std::nothrow) lim_batch();
    if (!b) return bfail(nullptr, LIM_ERR_NOMEM, "lim_batch_create: out of host memory");
    b->device = device;
    cudaSetDevice(device);
    // the chunk loop is captured into a graph, which needs a stream other than the
    // legacy default one
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        b->own_stream = e == cudaSuccess;
    }
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) {
        lim_batch_destroy(b);
        return bfail(nullptr, LIM_ERR_CUDA, "lim_batch_create: %s", cudaGetErrorString(e));
    }
    *out = b;
    return LIM_OK;
}

int lim_batch_destroy(lim_batch* b)
{
    if (!b) return LIM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    release_graph(b);
    bfree(b->d_kp); bfree(b->d_items); bfree(b->d_counters); bfree(b->d_status); bfree(b->d_tables);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return LIM_OK;
}

const char* lim_batch_last_error(const lim_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int lim_batch_add(lim_batch* b, lim_ctx* ensemble, int64_t first_step, int64_t nsteps, int64_t* index)
{
    if (!b) return LIM_ERR_ARG;
    if (!ensemble) return bfail(b, LIM_ERR_ARG, "lim_batch_add: ensemble is NULL");
    if (first_step < 0 || nsteps < 0) return bfail(b, LIM_ERR_ARG, "lim_batch_add: first_step and nsteps must be >= 0");
    if (first_step + nsteps > (int64_t)UINT32_MAX)
        return bfail(b, LIM_ERR_ARG, "lim_batch_add: steps beyond 2^32 - 1 (the noise counter's step word)");
    for (const auto& e : b->ens)
        if (e.c == ensemble) return bfail(b, LIM_ERR_ARG, "lim_batch_add: this context is already in the batch");
    if (b->ens.size() >= (size_t)INT_MAX) return bfail(b, LIM_ERR_ARG, "lim_batch_add: too many ensembles");
    b->ens.push_back({ ensemble, first_step, nsteps, ~0ull });
    release_graph(b);
    if (index) *index = (int64_t)b->ens.size() - 1;
    return LIM_OK;
}

int lim_batch_set_shape(lim_batch* b, const lim_batch_shape* shape)
{
    if (!b || !shape) return LIM_ERR_ARG;
    if (!valid_shape(*shape))
        return bfail(b, LIM_ERR_ARG, "lim_batch_set_shape: block must be 0, 64, 128 or 256; chunk_steps and "
                                     "blocks_per_sm >= 0; reg_cap 0 or 1");
    b->shape = *shape;
    release_graph(b);
    return LIM_OK;
}

int lim_batch_get_shape(const lim_batch* b, lim_batch_shape* shape)
{
    if (!b || !shape) return LIM_ERR_ARG;
    *shape = b->shape;
    return LIM_OK;
}

int lim_batch_run(lim_batch* b)
{
    if (!b) return LIM_ERR_ARG;
    return run_graph(b);
}

int lim_batch_tune(lim_batch* b, lim_batch_shape* best, double* best_ms)
{
    if (!b) return LIM_ERR_ARG;
    int rc = check_uniform(b);
    if (rc) return rc;
    for (size_t k = 0; k < b->ens.size(); ++k)
        if (lim_state_save(b->ens[k].c))
            return bfail(b, LIM_ERR_STATE, "ensemble %zu: %s", k, b->ens[k].c->err.c_str());
    const lim_batch_shape keep = b->shape;
    lim_batch_shape cand_best = keep;
    double t_best = -1.0;
    const int64_t chunks[4] = { 64, 256, 1024, 0 };
    const int caps = b->prec == LIM_FP32 ? 2 : 1;
    for (int64_t block : { 128, 256 })
        for (int64_t ch : chunks)
            for (int cap = 0; cap < caps; ++cap) {
                lim_batch_shape s{ block, ch, keep.blocks_per_sm, cap };
                b->shape = s;
                release_graph(b);
                for (const auto& e : b->ens)
                    if (lim_state_restore(e.c)) return bfail(b, LIM_ERR_STATE, "%s", e.c->err.c_str());
                if ((rc = run_graph(b))) { b->shape = keep; release_graph(b); return rc; }
                if (t_best < 0 || b->last_ms < t_best) { t_best = b->last_ms; cand_best = s; }
            }
    for (const auto& e : b->ens)
        if (lim_state_restore(e.c)) return bfail(b, LIM_ERR_STATE, "%s", e.c->err.c_str());
    b->shape = cand_best;
    release_graph(b);
    if (best) *best = cand_best;
    if (best_ms) *best_ms = t_best;
    return LIM_OK;
}

int lim_batch_stats(const lim_batch* b, double* ms, int64_t* launches, int64_t* particle_steps)
{
    if (!b) return LIM_ERR_ARG;
    if (ms) *ms = b->last_ms;
    if (launches) *launches = b->last_launches;
    if (particle_steps) *particle_steps = b->particle_steps;
    return LIM_OK;
}

}  // extern "C"

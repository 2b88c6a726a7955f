// lim_noalloc.cu — ensemble observables for callers that cannot allocate device memory.
//
// Some hosts embed the engine where cudaMalloc is not available to them: memory is
// handed out by the host's own pool (CUDA.jl or another framework's caching
// allocator), or the call sits on a real-time path that must not allocate.
// lim_observables_noalloc reduces a caller-owned device ensemble into a
// caller-owned device output and allocates nothing: its per-block FP64 partial
// sums live in a fixed file-scope device array (g_obs_scratch, 96 KiB), which every
// GPU that loads this library holds until the process exits.
#include <cstdio>
#include <mutex>
#include "../../include/langevin_b200.h"
#include "lim_internal.h"
#include "lim_obs.cuh"

namespace {

constexpr int kNAThreads = 256;
constexpr int kNABlocks = 1024;                  // rows of the scratch array
constexpr int kNAPerThread = 64;                 // particles per thread at the largest size
constexpr long long kNAMaxParticles = (long long)kNABlocks * kNAThreads * kNAPerThread;   // 16,777,216
constexpr int kNAObs = lim::kObsNum;

// One FP64 partial row per block.  Every call overwrites the rows it uses and reads
// only those, so nothing needs clearing.  All calls share it: calls that overlap on the
// GPU (for example on two streams) race on it, so the caller serialises them.
static __device__ __align__(256) double g_obs_scratch[kNABlocks * kNAObs];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_scratch_addr[kMaxDevices] = {};        // device address of g_obs_scratch, per device

__global__ void __launch_bounds__(kNAThreads)
k_obs_noalloc_partials(const double* __restrict__ p, int pdim, const double* __restrict__ x, int dims,
                       long long n, double m, double cut, double width, double* __restrict__ partials)
{
    __shared__ double sh[kNAThreads / 32][kNAObs];
    double v[kNAObs];
#pragma unroll
    for (int k = 0; k < kNAObs; ++k) v[k] = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double q[3] = { 0.0, 0.0, 0.0 }, y[3] = { 0.0, 0.0, 0.0 };
        for (int d = 0; d < pdim; ++d) q[d] = p[i * pdim + d];
        for (int d = 0; d < dims; ++d) y[d] = x[i * dims + d];
        lim::obs_add_terms(q, y, pdim, dims, m, cut, width, v);
    }
    lim::obs_block_sum(v, sh, partials + (long long)blockIdx.x * kNAObs);
}

__global__ void k_obs_noalloc_total(const double* __restrict__ partials, int nblocks, double* __restrict__ out)
{
    const int k = threadIdx.x;            // fixed summation order over the rows
    if (k >= kNAObs) return;
    double a = 0.0;
    for (int b = 0; b < nblocks; ++b) a += partials[b * kNAObs + k];
    out[k] = a;
}

int noalloc_fail(int code, const char* msg)
{
    lim::set_noctx_error(msg);
    return code;
}

}  // namespace

extern "C" int lim_observables_noalloc(int device, const double* p_dev, int64_t pdim, const double* x_dev,
                                       int64_t dims, int64_t n, double m, double pt_cut, double pt_width,
                                       double* out_dev, void* stream)
{
    char buf[256];
    if (pdim < 1 || pdim > 3) return noalloc_fail(LIM_ERR_ARG, "lim_observables_noalloc: pdim must be 1, 2 or 3");
    if (dims < 0 || dims > 3 || (dims > 0 && !x_dev))
        return noalloc_fail(LIM_ERR_ARG, "lim_observables_noalloc: dims must be 0..3 (0 or x_dev = NULL: no positions)");
    if (n < 0) return noalloc_fail(LIM_ERR_ARG, "lim_observables_noalloc: negative particle count");
    if (n > kNAMaxParticles) {
        snprintf(buf, sizeof buf, "lim_observables_noalloc: n = %lld exceeds the fixed scratch limit of %lld particles",
                 (long long)n, kNAMaxParticles);
        return noalloc_fail(LIM_ERR_ARG, buf);
    }
    if (!out_dev || (n > 0 && !p_dev)) return noalloc_fail(LIM_ERR_ARG, "lim_observables_noalloc: NULL device pointer");
    if (device < 0 || device >= kMaxDevices) return noalloc_fail(LIM_ERR_ARG, "lim_observables_noalloc: device out of range");
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return noalloc_fail(LIM_ERR_CUDA, cudaGetErrorString(e));
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return noalloc_fail(LIM_ERR_CUDA, cudaGetErrorString(e));
    double* scratch;
    {
        // Set-up, once per device, with that device current: the host-side name
        // g_obs_scratch is not a device address; ask the runtime for it.
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_addr[device]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_obs_scratch);
            if (e != cudaSuccess) {
                if (prev != device) cudaSetDevice(prev);
                snprintf(buf, sizeof buf, "lim_observables_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return noalloc_fail(LIM_ERR_CUDA, buf);
            }
            g_scratch_addr[device] = (double*)ptr;
        }
        scratch = g_scratch_addr[device];
    }
    long long blocks = (n + kNAThreads - 1) / kNAThreads;
    blocks = blocks < 1 ? 1 : (blocks > kNABlocks ? kNABlocks : blocks);
    cudaStream_t st = (cudaStream_t)stream;
    // an error left pending by earlier work on this thread is reported as such, so that
    // the status after the launches below belongs to this call
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        if (prev != device) cudaSetDevice(prev);
        snprintf(buf, sizeof buf, "lim_observables_noalloc: a CUDA error was pending before the call: %s",
                 cudaGetErrorString(e));
        return noalloc_fail(LIM_ERR_CUDA, buf);
    }
    k_obs_noalloc_partials<<<(unsigned)blocks, kNAThreads, 0, st>>>(p_dev, (int)pdim, x_dev, x_dev ? (int)dims : 0,
                                                                     (long long)n, m, pt_cut,
                                                                     pt_width > 0 ? pt_width : 1e-3, scratch);
    k_obs_noalloc_total<<<1, 32, 0, st>>>(scratch, (int)blocks, out_dev);
    e = cudaGetLastError();
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        snprintf(buf, sizeof buf, "lim_observables_noalloc: launch failed: %s", cudaGetErrorString(e));
        return noalloc_fail(LIM_ERR_CUDA, buf);
    }
    return LIM_OK;
}

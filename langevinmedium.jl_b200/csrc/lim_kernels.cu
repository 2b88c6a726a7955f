// lim_kernels.cu — the fused step kernels and their helpers.
//
// One thread owns one particle for a whole chunk of steps: the state is loaded
// once (coalesced structure-of-arrays loads), evolved in registers through every
// step of the chunk, and stored once.  This replaces the 5-7 launches per step of
// the reference GPU driver (simulate_gpu.jl:283-392), each of which re-streamed
// the state and its scratch arrays through HBM.
#include <climits>
#include "lim_internal.h"
#include "lim_step.cuh"
#include "lim_particle.cuh"
#include "lim_obs.cuh"

namespace lim {

template <typename R, int MED>
__global__ void k_step_table(const KParams<R> kp, int64_t s0, int64_t n)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    ((StepRec<R>*)kp.steps)[k] = make_step_rec<R, MED>(kp, s0 + k);
}

template <bool REC, bool FO, typename R, int MED, int DIMS, int PDIM>
__global__ void __launch_bounds__(256)
k_cart(const KParams<R> kp, int64_t s0, int64_t s1)
{
    if (FO && kp.live) {                  // compacted list of the particles not yet frozen out
        const unsigned cnt = *kp.live_n;
        for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x)
            cart_particle<REC, FO, R, MED, DIMS, PDIM>(kp, kp.rk, kp.live[k], s0, s1);
        return;
    }
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    cart_particle<REC, FO, R, MED, DIMS, PDIM>(kp, kp.rk, i, s0, s1);
}

// The FP32 grid kernel with the freeze-out latch, in blocks of 128 held to 72 registers
// so that seven blocks stay resident per SM (1.3 % faster on the 2+1D workloads than
// three blocks of 256 at 80 registers, 13 % faster than two at 128; the other
// instantiations lose by such a cap).
template <bool REC, int DIMS, int PDIM>
__global__ void __launch_bounds__(128, 7)
k_cart_grid_fo32(const KParams<float> kp, int64_t s0, int64_t s1)
{
    // one inlined copy of the particle loop for both forms (the live list, or every
    // particle with the grid covering them): half the code of two copies
    const int64_t cnt = kp.live ? (int64_t)*kp.live_n : kp.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += stride) {
        const int64_t i = kp.live ? (int64_t)kp.live[k] : k;
        cart_particle<REC, true, float, MED_GRID, DIMS, PDIM>(kp, kp.rk, i, s0, s1);
    }
}

// Ordered-within-block compaction of the particles whose freeze-out flag is clear:
// from `in` (or every index < n when in is NULL) to `out`; *out_n must be zero.
__global__ void __launch_bounds__(256)
k_compact_live(const double* __restrict__ flag, const int* __restrict__ in, const unsigned* in_n, int64_t n,
               int* __restrict__ out, unsigned* out_n)
{
    __shared__ unsigned warp_cnt[8];
    __shared__ unsigned base;
    const unsigned cnt = in ? *in_n : (unsigned)n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (unsigned t0 = blockIdx.x * blockDim.x; t0 < cnt; t0 += gridDim.x * blockDim.x) {
        const unsigned k = t0 + threadIdx.x;
        int idx = -1;
        if (k < cnt) idx = in ? in[k] : (int)k;
        const bool keep = idx >= 0 && flag[idx] == 0.0;
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) warp_cnt[warp] = __popc(ballot);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned tot = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { unsigned c = warp_cnt[w]; warp_cnt[w] = tot; tot += c; }
            base = tot ? atomicAdd(out_n, tot) : 0u;
        }
        __syncthreads();
        if (keep) out[base + warp_cnt[warp] + __popc(ballot & ((1u << lane) - 1u))] = idx;
        __syncthreads();
    }
}

template <bool REC, typename R>
__global__ void __launch_bounds__(256)
k_milne(const KParams<R> kp, int64_t s0, int64_t s1)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    R x[3];
    double p[3];
    float xl[3];
    load_state<R, 2, 2>(kp, i, x, xl, p);
    const NoiseKey nk{ kp.rk, (uint32_t)(kp.pid_offset + i) };
    const StepRec<R>* __restrict__ tab = (const StepRec<R>*)kp.steps - kp.step_base;
    for (int64_t s = s0; s < s1; ++s) {
        const StepRec<R> sr = tab[s];
        milne_step<REC, R>(kp, sr, i, s, nk, x, xl, p);
        if (!state_finite_all<R, 2, 2>(x, p)) {
            atomicMin(kp.first_bad, (unsigned long long)s);
            break;
        }
    }
    store_state<R, 2, 2>(kp, i, x, xl, p);
}

template <typename R, int MED, int DIMS, int PDIM>
__global__ void __launch_bounds__(256)
k_lab_boost(const KParams<R> kp)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    R x[3];
    double p[3];
    float xl[3];
    load_state<R, DIMS, PDIM>(kp, i, x, xl, p);
    const StepRec<R> sr = make_step_rec<R, MED>(kp, 0);
    const Local<R> L = local_medium<R, MED, DIMS>(kp, sr, x, nullptr, nullptr, xl);
    if (L.boost) boost<R, DIMS, PDIM>(kp, L, p, true);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) kp.p[d][i] = p[d];
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
static inline unsigned grid_of(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

template <bool REC, bool FO, typename R, int MED>
static cudaError_t launch_cart_fo(const KParams<R>& kp, int64_t s0, int64_t s1, int block, cudaStream_t st)
{
    unsigned g = grid_of(kp.n, block);
    if (FO && kp.live) {                  // grid-stride over the live list: a few waves of blocks
        int sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const unsigned cap = (unsigned)sms * (unsigned)(2048 / block);
        g = g < cap ? g : cap;
    }
    const int dp = kp.dims * 10 + kp.pdim;
    if (MED == MED_GRID) {
        if constexpr (FO && sizeof(R) == 4) {
            if (block <= 128) {
                const KParams<float>& kf = reinterpret_cast<const KParams<float>&>(kp);
                if (dp == 22) k_cart_grid_fo32<REC, 2, 2><<<g, block, 0, st>>>(kf, s0, s1);
                else if (dp == 23) k_cart_grid_fo32<REC, 2, 3><<<g, block, 0, st>>>(kf, s0, s1);
                else return cudaErrorInvalidValue;
                return cudaGetLastError();
            }
        }
        if (dp == 22) k_cart<REC, FO, R, MED, 2, 2><<<g, block, 0, st>>>(kp, s0, s1);
        else if (dp == 23) k_cart<REC, FO, R, MED, 2, 3><<<g, block, 0, st>>>(kp, s0, s1);
        else return cudaErrorInvalidValue;
        return cudaGetLastError();
    }
    switch (dp) {
    case 11: k_cart<REC, FO, R, MED, 1, 1><<<g, block, 0, st>>>(kp, s0, s1); break;
    case 22: k_cart<REC, FO, R, MED, 2, 2><<<g, block, 0, st>>>(kp, s0, s1); break;
    case 23: k_cart<REC, FO, R, MED, 2, 3><<<g, block, 0, st>>>(kp, s0, s1); break;
    case 33: k_cart<REC, FO, R, MED, 3, 3><<<g, block, 0, st>>>(kp, s0, s1); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <bool REC, typename R, int MED>
static cudaError_t launch_cart_med(const KParams<R>& kp, int64_t s0, int64_t s1, int block, cudaStream_t st)
{
    return kp.fo_capture ? launch_cart_fo<REC, true, R, MED>(kp, s0, s1, block, st)
                         : launch_cart_fo<REC, false, R, MED>(kp, s0, s1, block, st);
}

template <typename R, int MED>
static cudaError_t launch_table(const KParams<R>& kp, int64_t s0, int64_t s1, cudaStream_t st)
{
    const int64_t n = s1 - s0;
    k_step_table<R, MED><<<grid_of(n, 128), 128, 0, st>>>(kp, s0, n);
    return cudaGetLastError();
}

template <bool REC, typename R>
static cudaError_t launch_steps_rec(const KParams<R>& kp, int coords, int64_t s0, int64_t s1, int block, cudaStream_t st)
{
    cudaError_t e;
    if (coords == 1) {
        if ((e = launch_table<R, MED_MILNE_TABLE>(kp, s0, s1, st)) != cudaSuccess) return e;
        k_milne<REC, R><<<grid_of(kp.n, block), block, 0, st>>>(kp, s0, s1);
        return cudaGetLastError();
    }
    switch (kp.med.kind) {
    case MED_RT:
        if ((e = launch_table<R, MED_RT>(kp, s0, s1, st)) != cudaSuccess) return e;
        return launch_cart_med<REC, R, MED_RT>(kp, s0, s1, block, st);
    case MED_BJORKEN:
        if ((e = launch_table<R, MED_BJORKEN>(kp, s0, s1, st)) != cudaSuccess) return e;
        return launch_cart_med<REC, R, MED_BJORKEN>(kp, s0, s1, block, st);
    case MED_GRID:
        if ((e = launch_table<R, MED_GRID>(kp, s0, s1, st)) != cudaSuccess) return e;
        return launch_cart_med<REC, R, MED_GRID>(kp, s0, s1, block, st);
    }
    return cudaErrorInvalidValue;
}

// Steps [s0, s1) of a Cartesian run whose per-step table already holds them (no
// table launch): the sub-chunks of a live-list run and of a checkpointed forward pass.
template <typename R>
cudaError_t launch_steps_in_table(const KParams<R>& kp, int64_t s0, int64_t s1, int block, cudaStream_t st)
{
    if (kp.n == 0 || s1 <= s0) return cudaSuccess;
    if (!kp.steps || s0 < kp.step_base || s1 > kp.step_base + kp.step_cap) return cudaErrorInvalidValue;
    switch (kp.med.kind) {
    case MED_RT: return launch_cart_med<false, R, MED_RT>(kp, s0, s1, block, st);
    case MED_BJORKEN: return launch_cart_med<false, R, MED_BJORKEN>(kp, s0, s1, block, st);
    case MED_GRID: return launch_cart_med<false, R, MED_GRID>(kp, s0, s1, block, st);
    }
    return cudaErrorInvalidValue;
}

template <typename R>
cudaError_t launch_step_table(const KParams<R>& kp, int coords, int64_t s0, int64_t s1, cudaStream_t st)
{
    if (s1 <= s0) return cudaSuccess;
    if (!kp.steps || s0 != kp.step_base || s1 - s0 > kp.step_cap) return cudaErrorInvalidValue;
    if (coords == 1) return launch_table<R, MED_MILNE_TABLE>(kp, s0, s1, st);
    switch (kp.med.kind) {
    case MED_RT: return launch_table<R, MED_RT>(kp, s0, s1, st);
    case MED_BJORKEN: return launch_table<R, MED_BJORKEN>(kp, s0, s1, st);
    case MED_GRID: return launch_table<R, MED_GRID>(kp, s0, s1, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_compact_live(const double* flag, const int* in, const unsigned* in_n, int64_t n, int* out,
                                unsigned* out_n, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out_n, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    if (n <= 0) return cudaSuccess;
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    unsigned g = grid_of(n, 256);
    const unsigned cap = (unsigned)sms * 8u;
    g = g < cap ? g : cap;
    k_compact_live<<<g, 256, 0, st>>>(flag, in, in_n, n, out, out_n);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_steps(const KParams<R>& kp, int coords, int64_t s0, int64_t s1, int block, cudaStream_t st)
{
    if (kp.n == 0 || s1 <= s0) return cudaSuccess;
    // the per-step table of this launch holds steps [s0, s1) at [0, s1 - s0)
    if (!kp.steps || s0 != kp.step_base || s1 - s0 > kp.step_cap) return cudaErrorInvalidValue;
    const bool rec = kp.rec != nullptr && kp.rec_steps > 0;
    return rec ? launch_steps_rec<true, R>(kp, coords, s0, s1, block, st)
               : launch_steps_rec<false, R>(kp, coords, s0, s1, block, st);
}

template <typename R, int MED>
static cudaError_t launch_boost_med(const KParams<R>& kp, int block, cudaStream_t st)
{
    const unsigned g = grid_of(kp.n, block);
    const int dp = kp.dims * 10 + kp.pdim;
    if (MED == MED_GRID) {
        if (dp == 22) k_lab_boost<R, MED, 2, 2><<<g, block, 0, st>>>(kp);
        else if (dp == 23) k_lab_boost<R, MED, 2, 3><<<g, block, 0, st>>>(kp);
        else return cudaErrorInvalidValue;
        return cudaGetLastError();
    }
    switch (dp) {
    case 11: k_lab_boost<R, MED, 1, 1><<<g, block, 0, st>>>(kp); break;
    case 22: k_lab_boost<R, MED, 2, 2><<<g, block, 0, st>>>(kp); break;
    case 23: k_lab_boost<R, MED, 2, 3><<<g, block, 0, st>>>(kp); break;
    case 33: k_lab_boost<R, MED, 3, 3><<<g, block, 0, st>>>(kp); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_lab_boost(const KParams<R>& kp, int block, cudaStream_t st)
{
    if (kp.n == 0) return cudaSuccess;
    switch (kp.med.kind) {
    case MED_RT: return launch_boost_med<R, MED_RT>(kp, block, st);
    case MED_BJORKEN: return launch_boost_med<R, MED_BJORKEN>(kp, block, st);
    case MED_GRID: return launch_boost_med<R, MED_GRID>(kp, block, st);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------
struct RowPtrs3 { void* p[3]; float* lo[3]; };

template <typename R>
__global__ void k_aos_to_soa(const double* __restrict__ src, int rows, int64_t n, RowPtrs3 dst)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < rows; ++d) {
        double v = src[i * rows + d];
        R h = (R)v;
        ((R*)dst.p[d])[i] = h;
        if (dst.lo[d]) dst.lo[d][i] = (float)(v - (double)h);
    }
}

template <typename R>
__global__ void k_soa_to_aos(RowPtrs3 src, int rows, int64_t n, double* __restrict__ dst)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < rows; ++d) {
        double v = (double)((const R*)src.p[d])[i];
        if (src.lo[d]) v += (double)src.lo[d][i];
        dst[i * rows + d] = v;
    }
}

template <typename R>
cudaError_t launch_aos_to_soa(const double* src, int rows, int64_t n, R* const* dst, float* const* lo, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    RowPtrs3 rp{};
    for (int d = 0; d < 3; ++d) { rp.p[d] = d < rows ? (void*)dst[d] : nullptr; rp.lo[d] = (lo && d < rows) ? lo[d] : nullptr; }
    k_aos_to_soa<R><<<grid_of(n, 256), 256, 0, st>>>(src, rows, n, rp);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_soa_to_aos(R* const* src, float* const* lo, int rows, int64_t n, double* dst, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    RowPtrs3 rp{};
    for (int d = 0; d < 3; ++d) { rp.p[d] = d < rows ? (void*)src[d] : nullptr; rp.lo[d] = (lo && d < rows) ? lo[d] : nullptr; }
    k_soa_to_aos<R><<<grid_of(n, 256), 256, 0, st>>>(rp, rows, n, dst);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// observables: FP64 block partials, then a fixed-order sum (deterministic)
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
k_obs_partials(const KParams<R> kp, int from_fo, double cut, double width, double* __restrict__ partials)
{
    __shared__ double sh[8][kObsNum];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v[kObsNum];
#pragma unroll
    for (int k = 0; k < kObsNum; ++k) v[k] = 0.0;
    if (i < kp.n) obs_terms<R>(kp, i, from_fo, cut, width, v);
    obs_block_sum(v, sh, partials + (int64_t)blockIdx.x * kObsNum);
}

__global__ void __launch_bounds__(kObsNum * 32) k_obs_total(const double* __restrict__ partials, int64_t nblocks,
                                                             double* __restrict__ out)
{
    // one warp per observable: lane-strided sums combined by a fixed shuffle tree (a
    // fixed summation order for a given block count)
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= kObsNum) return;
    double a = 0.0;
    for (int64_t b = lane; b < nblocks; b += 32) a += partials[b * kObsNum + k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
    if (lane == 0) out[k] = a;
}

cudaError_t launch_obs_total(const double* partials, int64_t nblocks, double* out, cudaStream_t st)
{
    k_obs_total<<<1, kObsNum * 32, 0, st>>>(partials, nblocks, out);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_observables(const KParams<R>& kp, int from_fo, double cut, double width,
                               double* partials, int64_t nblocks_max, double* out, cudaStream_t st)
{
    const int64_t nb = kp.n == 0 ? 1 : (kp.n + 255) / 256;
    if (nb > nblocks_max) return cudaErrorInvalidValue;
    k_obs_partials<R><<<(unsigned)nb, 256, 0, st>>>(kp, from_fo, cut, width, partials);
    k_obs_total<<<1, kObsNum * 32, 0, st>>>(partials, nb, out);
    return cudaGetLastError();
}

// FP32 FMA issue-rate probe: 8 independent dependency chains per thread.
__global__ void __launch_bounds__(256) k_fma_probe(float* out, int iters, float b, float c)
{
    float a0 = threadIdx.x * 1e-3f, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t launch_fma_probe(float* out, int blocks, int iters, cudaStream_t st)
{
    k_fma_probe<<<blocks, 256, 0, st>>>(out, iters, 0.99999f, 1e-6f);
    return cudaGetLastError();
}

// Multi-function-unit (XU) probe: 8 independent chains of the hardware base-2
// exponential (ex2.approx, one MUFU instruction each) with one FP32 multiply to keep the
// values bounded; the XU pipe, with an eighth of the FMA pipe's lanes, is the bound.
__global__ void __launch_bounds__(256) k_mufu_probe(float* out, int iters, float b)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = -1e-3f * (float)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float e;
                asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(a[k]));
                a[k] = -b * e;
            }
        }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t launch_mufu_probe(float* out, int blocks, int iters, cudaStream_t st)
{
    k_mufu_probe<<<blocks, 256, 0, st>>>(out, iters, 0.5f);
    return cudaGetLastError();
}

__global__ void k_philox_probe(const uint32_t* ck, uint32_t* out)
{
    uint4 r = philox4x32_10(make_uint4(ck[0], ck[1], ck[2], ck[3]), make_uint2(ck[4], ck[5]));
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

cudaError_t launch_philox_probe(const uint32_t* ctr_key, uint32_t* out, cudaStream_t st)
{
    k_philox_probe<<<1, 1, 0, st>>>(ctr_key, out);
    return cudaGetLastError();
}

template <typename R>
size_t step_record_bytes() { return sizeof(StepRec<R>); }

// explicit instantiations
template size_t step_record_bytes<double>();
template size_t step_record_bytes<float>();
template cudaError_t launch_steps<double>(const KParams<double>&, int, int64_t, int64_t, int, cudaStream_t);
template cudaError_t launch_steps_in_table<double>(const KParams<double>&, int64_t, int64_t, int, cudaStream_t);
template cudaError_t launch_steps_in_table<float>(const KParams<float>&, int64_t, int64_t, int, cudaStream_t);
template cudaError_t launch_step_table<double>(const KParams<double>&, int, int64_t, int64_t, cudaStream_t);
template cudaError_t launch_step_table<float>(const KParams<float>&, int, int64_t, int64_t, cudaStream_t);
template cudaError_t launch_steps<float>(const KParams<float>&, int, int64_t, int64_t, int, cudaStream_t);
template cudaError_t launch_lab_boost<double>(const KParams<double>&, int, cudaStream_t);
template cudaError_t launch_lab_boost<float>(const KParams<float>&, int, cudaStream_t);
template cudaError_t launch_aos_to_soa<double>(const double*, int, int64_t, double* const*, float* const*, cudaStream_t);
template cudaError_t launch_aos_to_soa<float>(const double*, int, int64_t, float* const*, float* const*, cudaStream_t);
template cudaError_t launch_soa_to_aos<double>(double* const*, float* const*, int, int64_t, double*, cudaStream_t);
template cudaError_t launch_soa_to_aos<float>(float* const*, float* const*, int, int64_t, double*, cudaStream_t);
template cudaError_t launch_observables<double>(const KParams<double>&, int, double, double, double*, int64_t, double*, cudaStream_t);
template cudaError_t launch_observables<float>(const KParams<float>&, int, double, double, double*, int64_t, double*, cudaStream_t);

}  // namespace lim

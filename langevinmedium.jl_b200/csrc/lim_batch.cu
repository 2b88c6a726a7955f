// lim_batch.cu — many independent ensembles (own particle count, step range, mass,
// transport tables and medium) in one persistent launch per chunk of steps.
//
// The work of a chunk is a list of (ensemble, tile) items; a tile is one block's worth
// of particles of one ensemble, advanced through the chunk's step window in registers
// (the same per-particle code as the plain kernel).  Persistent blocks take items from
// an atomic counter, stage the item's ensemble parameters in shared memory and run
// it.  Items are ordered by ensemble, so the blocks in flight work on a few ensembles
// at a time and a grid medium's current time slices stay L2-resident.  Chunking the
// step range (the chunk loop is replayed as a CUDA graph) keeps every ensemble at the
// same step index across the device.
#include "lim_internal.h"
#include "lim_particle.cuh"

namespace lim {

static_assert(sizeof(KParams<float>) % 16 == 0 && sizeof(KParams<double>) % 16 == 0,
              "KParams is staged in shared memory with 16-byte copies");

template <bool FO, typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void batch_tile(const KParams<R>& kp, const uint2* __restrict__ rk, int tile,
                                           int64_t lo, int64_t len)
{
    const int64_t i = (int64_t)tile * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    const int64_t s0 = kp.step_base + lo;
    const int64_t end = kp.step_base + kp.step_cap;
    const int64_t s1 = s0 + len < end ? s0 + len : end;
    cart_particle<false, FO, R, MED, DIMS, PDIM>(kp, rk, i, s0, s1);
}

// CAP (FP32 only): at most 64 registers, so that four 256-thread blocks stay resident
// per SM (the plain kernel's occupancy) at the price of a few spills; the autotuner
// picks between the capped and the natural build.
template <bool FO, typename R, int DIMS, int PDIM, bool CAP>
__global__ void __launch_bounds__(256, CAP ? 4 : 1)
k_batch(const BatchLaunch<R> bl)
{
    __shared__ __align__(16) unsigned char raw[sizeof(KParams<R>)];
    __shared__ int2 item;
    const KParams<R>& kp = *reinterpret_cast<const KParams<R>*>(raw);
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned k = atomicAdd(bl.counter, 1u);
            item = k < (unsigned)bl.n_items ? bl.items[k] : make_int2(-1, 0);
        }
        __syncthreads();
        const int2 it = item;
        if (it.x < 0) return;                       // the same value in every thread
        const int4* __restrict__ src = reinterpret_cast<const int4*>(bl.ens + it.x);
        int4* dst = reinterpret_cast<int4*>(raw);
        for (int w = threadIdx.x; w < (int)(sizeof(KParams<R>) / 16); w += blockDim.x) dst[w] = src[w];
        __syncthreads();
        const int kind = kp.med.kind;
        if (kind == MED_BJORKEN) {
            batch_tile<FO, R, MED_BJORKEN, DIMS, PDIM>(kp, bl.rk, it.y, bl.chunk_lo, bl.chunk_len);
        } else if (kind == MED_RT) {
            batch_tile<FO, R, MED_RT, DIMS, PDIM>(kp, bl.rk, it.y, bl.chunk_lo, bl.chunk_len);
        } else {
            if constexpr (DIMS == 2) batch_tile<FO, R, MED_GRID, DIMS, PDIM>(kp, bl.rk, it.y, bl.chunk_lo, bl.chunk_len);
        }
        __syncthreads();                            // before the next item overwrites raw / item
    }
}

template <bool FO, typename R, bool CAP>
static const void* batch_kernel(int dp)
{
    if (dp == 22) return (const void*)k_batch<FO, R, 2, 2, CAP>;
    if (dp == 23) return (const void*)k_batch<FO, R, 2, 3, CAP>;
    if (dp == 33) return (const void*)k_batch<FO, R, 3, 3, CAP>;
    return nullptr;
}

template <typename R>
static const void* batch_kernel_of(int dims, int pdim, bool fo, bool cap)
{
    const int dp = dims * 10 + pdim;
    if (sizeof(R) == 8) cap = false;               // FP64 runs at its natural register count
    if (fo) return cap ? batch_kernel<true, R, true>(dp) : batch_kernel<true, R, false>(dp);
    return cap ? batch_kernel<false, R, true>(dp) : batch_kernel<false, R, false>(dp);
}

template <typename R>
cudaError_t launch_batch(const BatchLaunch<R>& bl, int dims, int pdim, bool fo, bool cap, int grid, int block,
                         cudaStream_t st)
{
    const void* k = batch_kernel_of<R>(dims, pdim, fo, cap);
    if (!k) return cudaErrorInvalidValue;
    void* args[] = { (void*)&bl };
    return cudaLaunchKernel(k, dim3(grid), dim3(block), args, 0, st);
}

template <typename R>
cudaError_t batch_blocks_per_sm(int dims, int pdim, bool fo, bool cap, int block, int* out)
{
    const void* k = batch_kernel_of<R>(dims, pdim, fo, cap);
    if (!k) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, k, block, 0);
}

// Per-step records of one ensemble for steps [s0, s0 + n) into `out`.
template <typename R, int MED>
__global__ void k_batch_table(const KParams<R> kp, int64_t s0, int64_t n, StepRec<R>* out)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[k] = make_step_rec<R, MED>(kp, s0 + k);
}

template <typename R>
cudaError_t launch_batch_table(const KParams<R>& kp, int64_t s0, int64_t n, void* out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const unsigned g = (unsigned)((n + 127) / 128);
    StepRec<R>* o = (StepRec<R>*)out;
    switch (kp.med.kind) {
    case MED_RT: k_batch_table<R, MED_RT><<<g, 128, 0, st>>>(kp, s0, n, o); break;
    case MED_BJORKEN: k_batch_table<R, MED_BJORKEN><<<g, 128, 0, st>>>(kp, s0, n, o); break;
    case MED_GRID: k_batch_table<R, MED_GRID><<<g, 128, 0, st>>>(kp, s0, n, o); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template cudaError_t launch_batch<double>(const BatchLaunch<double>&, int, int, bool, bool, int, int, cudaStream_t);
template cudaError_t launch_batch<float>(const BatchLaunch<float>&, int, int, bool, bool, int, int, cudaStream_t);
template cudaError_t batch_blocks_per_sm<double>(int, int, bool, bool, int, int*);
template cudaError_t batch_blocks_per_sm<float>(int, int, bool, bool, int, int*);
template cudaError_t launch_batch_table<double>(const KParams<double>&, int64_t, int64_t, void*, cudaStream_t);
template cudaError_t launch_batch_table<float>(const KParams<float>&, int64_t, int64_t, void*, cudaStream_t);

}  // namespace lim

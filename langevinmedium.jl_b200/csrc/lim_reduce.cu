// lim_reduce.cu — snapshot reductions on the device: instead of copying the
// (dims + pdim) x N FP64 state to the host at every save step (the reference's
// history of snapshots, simulate_cpu.jl:319-322), each snapshot is reduced in place to
// the observable sums and three histograms: the radial density n(r) (the n(r, t) that
// the reference exports as n_rt, LangevInMedium.jl:44), the p_T spectrum and the sum of
// cos 2 phi_p per p_T bin (the numerator of v2(p_T)).
//
// Counts are 64-bit integers and cos 2 phi enters as a 64-bit fixed-point number
// (rint(cos 2 phi * 2^32)), so the sums are exact and independent of the order in which
// particles are added: block histograms in shared memory, flushed with integer atomics.
#include <algorithm>
#include "lim_internal.h"
#include "lim_obs.cuh"

namespace lim {

namespace {

__device__ __forceinline__ int bin_of(double v, double scale, int nbins)
{
    // uniform bins [k w, (k+1) w) on [0, max); the last entry counts v >= max (and NaN)
    const double f = floor(__dmul_rn(v, scale));
    return (f >= 0.0 && f < (double)nbins) ? (int)f : nbins;
}

}  // namespace

// hist: (r_bins + 1) r counts, (pt_bins + 1) p_T counts, (pt_bins + 1) fixed-point sums of
// cos 2 phi, all unsigned 64-bit (the cos sums as two's complement).
// With the histograms, the block's sums of the observable terms go to partials[block]
// (a grid-stride loop over a grid that depends on n only: a fixed summation order).
template <typename R, bool MILNE>
__global__ void __launch_bounds__(256)
k_reduce_hist(const KParams<R> kp, const ReduceSpec rs, unsigned long long* __restrict__ hist, double cut,
              double width, double* __restrict__ partials)
{
    extern __shared__ unsigned long long sh[];
    __shared__ double sho[8][kObsTerms];
    double v[kObsTerms];
#pragma unroll
    for (int k = 0; k < kObsTerms; ++k) v[k] = 0.0;
    const int nr1 = rs.r_bins + 1, np1 = rs.pt_bins + 1, tot = nr1 + 2 * np1;
    for (int k = threadIdx.x; k < tot; k += blockDim.x) sh[k] = 0ull;
    __syncthreads();
    unsigned long long* shr = sh;
    unsigned long long* shp = sh + nr1;
    unsigned long long* shc = sh + nr1 + np1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < kp.n; i += (int64_t)gridDim.x * blockDim.x) {
        double x[3] = { 0.0, 0.0, 0.0 };
        for (int d = 0; d < kp.dims; ++d) {
            x[d] = (double)kp.x[d][i];
            if (sizeof(R) == 4) x[d] += (double)kp.xlo[d][i];
        }
        // every operation rounded on its own (no contraction), so a host restatement
        // reproduces the bins exactly
        double r, pt, c2 = 0.0;
        if (MILNE) {                                   // (tau, r), (p^tau, p^r)
            r = x[1];
            pt = fabs(kp.p[1][i]);
        } else {
            double r2 = 0.0;
            for (int d = 0; d < kp.dims; ++d) r2 = __dadd_rn(r2, __dmul_rn(x[d], x[d]));
            r = sqrt(r2);
            const double px = kp.p[0][i], py = kp.pdim >= 2 ? kp.p[1][i] : 0.0;
            const double px2 = __dmul_rn(px, px), py2 = __dmul_rn(py, py);
            const double pt2 = __dadd_rn(px2, py2);
            pt = sqrt(pt2);
            c2 = pt2 > 0.0 ? __ddiv_rn(__dsub_rn(px2, py2), pt2) : 0.0;
        }
        obs_terms<R>(kp, i, 0, cut, width, v);
        atomicAdd(&shr[bin_of(r, rs.r_scale, rs.r_bins)], 1ull);
        const int kb = bin_of(pt, rs.pt_scale, rs.pt_bins);
        atomicAdd(&shp[kb], 1ull);
        if (c2 != 0.0) atomicAdd(&shc[kb], (unsigned long long)__double2ll_rn(c2 * 4294967296.0));
    }
    obs_block_sum(v, sho, partials + (int64_t)blockIdx.x * kObsTerms);   // synchronises the block
    for (int k = threadIdx.x; k < tot; k += blockDim.x)
        if (sh[k]) atomicAdd(&hist[k], sh[k]);
}

int reduce_grid(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 8); }

template <typename R>
cudaError_t launch_reduce_hist(const KParams<R>& kp, bool milne, const ReduceSpec& rs, unsigned long long* hist,
                               double cut, double width, double* partials, double* obs_out, cudaStream_t st)
{
    const size_t smem = (size_t)(rs.r_bins + 1 + 2 * (rs.pt_bins + 1)) * sizeof(unsigned long long);
    const int grid = reduce_grid(kp.n);
    if (kp.n == 0) return cudaMemsetAsync(obs_out, 0, kObsTerms * sizeof(double), st);
    cudaError_t e;
    if (milne) {
        if ((e = cudaFuncSetAttribute(k_reduce_hist<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess) return e;
        k_reduce_hist<R, true><<<grid, 256, smem, st>>>(kp, rs, hist, cut, width, partials);
    } else {
        if ((e = cudaFuncSetAttribute(k_reduce_hist<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess) return e;
        k_reduce_hist<R, false><<<grid, 256, smem, st>>>(kp, rs, hist, cut, width, partials);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_obs_total(partials, grid, obs_out, st);
}

template cudaError_t launch_reduce_hist<double>(const KParams<double>&, bool, const ReduceSpec&, unsigned long long*,
                                                double, double, double*, double*, cudaStream_t);
template cudaError_t launch_reduce_hist<float>(const KParams<float>&, bool, const ReduceSpec&, unsigned long long*,
                                               double, double, double*, double*, cudaStream_t);

}  // namespace lim

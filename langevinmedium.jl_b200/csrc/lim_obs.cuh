// lim_obs.cuh — the per-particle terms of the observable sums (LIM_OBS_* in
// include/langevin_b200.h), shared by the observables kernel and the snapshot reduction.
#pragma once
#include "lim_common.cuh"

namespace lim {

constexpr int kObsTerms = 12;   // LIM_OBS_NUM

// Adds one particle's terms to v: count, pT, cos 2 phi, [pT > cut], sigmoid((pT - cut)/width),
// |p|^2, E, (m/E)|p|^2, p_x, (m/E) p_x, p_z^2, |x|^2, from its momentum p (pdim rows) and
// position x (dims rows, 0 for none).  Every entry point that reduces observables calls
// this one definition.
__device__ __forceinline__ void obs_add_terms(const double (&p)[3], const double (&x)[3], int pdim, int dims, double m,
                                              double cut, double width, double (&v)[kObsTerms])
{
    const double px = p[0], py = pdim >= 2 ? p[1] : 0.0;
    const double pt2 = px * px + py * py, pt = sqrt(pt2);
    double p2 = 0.0;
    for (int d = 0; d < pdim; ++d) p2 += p[d] * p[d];
    const double E = sqrt(m * m + p2), w = m / E;
    double x2 = 0.0;
    for (int d = 0; d < dims; ++d) x2 += x[d] * x[d];
    v[0] += 1.0;
    v[1] += pt;
    v[2] += pt2 > 0.0 ? (px * px - py * py) / pt2 : 0.0;
    v[3] += pt > cut ? 1.0 : 0.0;
    v[4] += 1.0 / (1.0 + exp(-(pt - cut) / width));
    v[5] += p2;
    v[6] += E;
    v[7] += w * p2;
    v[8] += px;
    v[9] += w * px;
    v[10] += pdim == 3 ? p[2] * p[2] : 0.0;
    v[11] += x2;
}

// Adds particle i's terms of an engine context (the freeze-out latch's values and only
// latched particles when from_fo).
template <typename R>
__device__ __forceinline__ void obs_terms(const KParams<R>& kp, int64_t i, int from_fo, double cut, double width,
                                          double (&v)[kObsTerms])
{
    double p[3] = { 0, 0, 0 }, x[3] = { 0, 0, 0 };
    if (from_fo) {
        if (kp.fo_flag[i] == 0.0) return;
        for (int d = 0; d < kp.pdim; ++d) p[d] = (double)kp.fo_mom[d][i];
        for (int d = 0; d < kp.dims; ++d) x[d] = (double)kp.fo_pos[d][i];
    } else {
        for (int d = 0; d < kp.pdim; ++d) p[d] = (double)kp.p[d][i];
        for (int d = 0; d < kp.dims; ++d) {
            x[d] = (double)kp.x[d][i];
            if (sizeof(R) == 4) x[d] += (double)kp.xlo[d][i];
        }
    }
    obs_add_terms(p, x, kp.pdim, kp.dims, (double)kp.m, cut, width, v);
}

// Block sum of v (blockDim.x a multiple of 32, at most 256) in a fixed order into out[0..11]
// (thread k < 12 writes out[k]); sh holds [8][kObsTerms] doubles.
__device__ __forceinline__ void obs_block_sum(const double (&v)[kObsTerms], double (*sh)[kObsTerms], double* out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kObsTerms; ++k) {
        double a = v[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if (lane == 0) sh[warp][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < kObsTerms) {
        double a = 0.0;
        const int nw = blockDim.x >> 5;
        for (int w = 0; w < nw; ++w) a += sh[w][threadIdx.x];
        out[threadIdx.x] = a;
    }
}

}  // namespace lim

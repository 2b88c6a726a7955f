// lim_sample.cu — initial heavy-quark states sampled on the device from a FONLL-type
// density table (utils.jl:33-172, sample_particles_from_FONLL) with the thermal
// longitudinal momentum of append_thermal_pz / sample_pz_conditional_juttner
// (utils.jl:499-551).  The host samplers draw from Julia's global RNG in rejection
// loops; here every draw comes from the counter-based Philox stream of the particle,
// counter (pid, draw, tag), so the restatement can repeat a particle's sampling.
//
// Per particle (or per antithetic pair, which shares the draws):
//   Cartesian mode: trial t proposes (x, y) uniform in [-rmax, rmax]^2 from block
//     (pid, t, SAMPLE_XY), rejects r > rmax and u * f_max > n(r) (n linear on the r grid,
//     0 outside); the accepted trial's block (pid, t, SAMPLE_P) gives |p| from the
//     conditional inverse CDF of p | r and the momentum angle.
//   polar mode: block (pid, 0, SAMPLE_XY) gives r (inverse CDF of the r marginal), the
//     position angle, |p| | r and the momentum angle.
//   p_z: trial t of block (pid, t, SAMPLE_PZ): y from the Gaussian envelope N(0, c/a) in
//     rapidity (Box–Muller of words 0, 1), accepted if u (word 2) <= the density ratio;
//     a <= 1.05 takes the Laplace envelope in p_z (words 0, 1, 2 and 3).
#include "lim_internal.h"
#include "lim_step.cuh"

namespace lim {

namespace {

// searchsortedlast on an ascending grid, capped to [0, n-2].
__device__ __forceinline__ int cell_of(const double* __restrict__ g, int n, double x)
{
    int lo = -1, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (g[mid] <= x) lo = mid; else hi = mid;
    }
    lo = lo < 0 ? 0 : lo;
    return lo > n - 2 ? n - 2 : lo;
}

// Interpolations.LinearInterpolation(cdf, grid, Flat()) evaluated at u in (0, 1).
__device__ __forceinline__ double inverse_cdf(const double* __restrict__ cdf, const double* __restrict__ grid, int n,
                                              double u)
{
    if (n < 2) return grid[0];
    if (u <= cdf[0]) return grid[0];
    if (u >= cdf[n - 1]) return grid[n - 1];
    const int k = cell_of(cdf, n, u);
    const double w = (u - cdf[k]) / (cdf[k + 1] - cdf[k]);
    return grid[k] + w * (grid[k + 1] - grid[k]);
}

// One exact draw of p_z ~ exp(-sqrt(mT^2 + p_z^2) / T) (utils.jl:499-528): 1e5 trials with the
// rapidity envelope, 1e6 with the Laplace one, as there.
__device__ double sample_pz(const NoiseKey& nk, double mT, double T, int max_trials)
{
    if (!(T > 0.0 && mT > 0.0)) return 0.0;
    const double a = mT / T;
    if (a > 1.05) {
        const double c = fmax(2.0, a / (a - 1.0));
        const double sig = sqrt(c / a);
        for (int t = 0; t < max_trials; ++t) {
            const uint4 w = philox_words(nk.rk, nk.pid, (uint32_t)t, TAG_SAMPLE_PZ);
            double z0, z1;
            box_muller(w.x, w.y, z0, z1);
            const double y = sig * z0;
            const double ch = cosh(y);
            const double acc = ch * exp(-a * (ch - 1.0) + a * y * y / (2.0 * c));
            if (u_exact(w.z) <= acc) return mT * sinh(y);
        }
        return 0.0;
    }
    const double b = sqrt(2.0) * T;
    for (int t = 0; t < 10 * max_trials; ++t) {             // 1e6 trials for the loose envelope
        const uint4 w = philox_words(nk.rk, nk.pid, (uint32_t)t, TAG_SAMPLE_PZ);
        const double pz = -b * log(u_exact(w.x)) * (u_exact(w.y) < 0.5 ? -1.0 : 1.0);
        const double acc = exp(-(sqrt(mT * mT + pz * pz) - (mT + fabs(pz)) / sqrt(2.0)) / T);
        if (u_exact(w.z) <= acc) return pz;
    }
    return 0.0;
}

}  // namespace

template <typename R>
__global__ void __launch_bounds__(128)
k_sample_fonll(const KParams<R> kp, const SampleTables st)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    // antithetic pairs (0,1), (2,3), ... share their draws; the second negates p
    int64_t draw = i;
    bool mirror = false;
    if (st.antithetic) {
        const int64_t half = kp.n / 2;
        if (i < 2 * half) { draw = i / 2; mirror = (i & 1) != 0; }
        else draw = half;
    }
    const NoiseKey nk{ kp.rk, (uint32_t)(kp.pid_offset + draw) };
    double x = 0.0, y = 0.0, r = 0.0, pmag = 0.0, phip = 0.0;
    bool ok = true;
    if (st.cartesian) {
        ok = false;
        for (int t = 0; t < st.max_trials; ++t) {
            const uint4 w = philox_words(nk.rk, nk.pid, (uint32_t)t, TAG_SAMPLE_XY);
            const double xt = st.rmax * (2.0 * u_exact(w.x) - 1.0);
            const double yt = st.rmax * (2.0 * u_exact(w.y) - 1.0);
            const double rt = sqrt(xt * xt + yt * yt);
            if (rt > st.rmax) continue;
            double nr = 0.0;                        // LinearInterpolation(r_grid, n, 0 outside)
            if (rt >= st.r_grid[0] && rt <= st.r_grid[st.nr - 1]) {
                const int k = cell_of(st.r_grid, st.nr, rt);
                const double wk = (rt - st.r_grid[k]) / (st.r_grid[k + 1] - st.r_grid[k]);
                nr = st.n_spatial[k] + wk * (st.n_spatial[k + 1] - st.n_spatial[k]);
            }
            if (u_exact(w.z) * st.f_max > nr) continue;
            x = xt; y = yt; r = rt;
            const uint4 v = philox_words(nk.rk, nk.pid, (uint32_t)t, TAG_SAMPLE_P);
            const double rc = fmin(fmax(r, st.r_grid[0]), st.r_grid[st.nr - 1]);
            const int j = cell_of(st.r_grid, st.nr, rc) + (rc >= st.r_grid[st.nr - 1] ? 1 : 0);
            pmag = st.p_mass[j] > 0 ? inverse_cdf(st.cdf_p + (size_t)j * st.np, st.p_grid, st.np, u_exact(v.x)) : 0.0;
            phip = 2.0 * M_PI * u_exact(v.y);
            ok = true;
            break;
        }
    } else {
        const uint4 w = philox_words(nk.rk, nk.pid, 0u, TAG_SAMPLE_XY);
        r = inverse_cdf(st.cdf_r, st.r_grid, st.nr, u_exact(w.x));
        r = fmin(fmax(r, st.r_grid[0]), st.r_grid[st.nr - 1]);
        const double phi = 2.0 * M_PI * u_exact(w.y);
        x = r * cos(phi);
        y = r * sin(phi);
        const int j = cell_of(st.r_grid, st.nr, r) + (r >= st.r_grid[st.nr - 1] ? 1 : 0);
        pmag = st.p_mass[j] > 0 ? inverse_cdf(st.cdf_p + (size_t)j * st.np, st.p_grid, st.np, u_exact(w.z)) : 0.0;
        phip = 2.0 * M_PI * u_exact(w.w);
    }
    if (!ok) atomicAdd(st.failed, 1ull);
    double px = pmag * cos(phip), py = pmag * sin(phip);
    double pz = 0.0;
    if (kp.pdim == 3 && st.with_pz) {
        // the local temperature at the initial time (the medium's own lookup, FP64)
        const StepRec<R> sr = st.med_kind == MED_GRID ? step_rec_at_time<R, MED_GRID>(kp, kp.t0)
                            : st.med_kind == MED_RT ? step_rec_at_time<R, MED_RT>(kp, kp.t0)
                                                    : step_rec_at_time<R, MED_BJORKEN>(kp, kp.t0);
        const double xd[3] = { x, y, 0.0 };
        double T = st.med_kind == MED_GRID ? temperature_fp64<R, MED_GRID, 2>(kp, sr, xd)
                 : st.med_kind == MED_RT ? temperature_fp64<R, MED_RT, 2>(kp, sr, xd)
                                         : temperature_fp64<R, MED_BJORKEN, 2>(kp, sr, xd);
        T = T > 0.0 ? T : 0.0;
        const double mT = sqrt((double)kp.m * (double)kp.m + px * px + py * py);
        pz = sample_pz(nk, mT, T, st.max_trials);
    }
    if (mirror) { px = -px; py = -py; pz = -pz; }
    kp.x[0][i] = (R)x;
    kp.x[1][i] = (R)y;
    if (sizeof(R) == 4) {
        kp.xlo[0][i] = (float)(x - (double)(R)x);
        kp.xlo[1][i] = (float)(y - (double)(R)y);
    }
    kp.p[0][i] = px;
    kp.p[1][i] = py;
    if (kp.pdim == 3) kp.p[2][i] = pz;
}

// sample_initial_particles_milne! (utils.jl:350-400): r by rejection against the binned
// Boltzmann density (trial t: block (pid, t, SAMPLE_XY), r = lo + (hi - lo) u0 accepted if
// u1 < pdf/max_pdf of the first bin center >= r), then p^r = sigma z with
// sigma = sqrt(m T(r)) and z from block (pid, 0, SAMPLE_P); the state is (tau0, r),
// (sqrt(m^2 + p_r^2), |p_r|).
template <typename R>
__global__ void __launch_bounds__(128)
k_sample_milne(const KParams<R> kp, const MilneTables mt)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    const NoiseKey nk{ kp.rk, (uint32_t)(kp.pid_offset + i) };
    double r = 0.0;
    bool ok = false;
    for (int t = 0; t < mt.max_trials; ++t) {
        const uint4 w = philox_words(nk.rk, nk.pid, (uint32_t)t, TAG_SAMPLE_XY);
        const double rt = mt.lo + (mt.hi - mt.lo) * u_exact(w.x);
        int lo = -1, hi = mt.nbins;                      // searchsortedfirst(centers, rt)
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (mt.centers[mid] >= rt) hi = mid; else lo = mid;
        }
        const double acc = hi < mt.nbins ? mt.ratio[hi] : 0.0;
        if (u_exact(w.y) < acc) { r = rt; ok = true; break; }
    }
    if (!ok) atomicAdd(mt.failed, 1ull);
    double T;
    {
        const double rq = fmin(fmax(r, mt.rT[0]), mt.rT[mt.nT - 1]);
        const int k = cell_of(mt.rT, mt.nT, rq);
        const double w = (rq - mt.rT[k]) / (mt.rT[k + 1] - mt.rT[k]);
        T = mt.TT[k] + w * (mt.TT[k + 1] - mt.TT[k]);
    }
    const double sigma = sqrt((double)kp.m * T);
    const uint4 v = philox_words(nk.rk, nk.pid, 0u, TAG_SAMPLE_P);
    double z0, z1;
    box_muller(v.x, v.y, z0, z1);
    const double pr = sigma * z0;
    const double tau0 = (double)kp.t0;
    kp.x[0][i] = (R)tau0;
    kp.x[1][i] = (R)r;
    if (sizeof(R) == 4) {
        kp.xlo[0][i] = (float)(tau0 - (double)(R)tau0);
        kp.xlo[1][i] = (float)(r - (double)(R)r);
    }
    kp.p[0][i] = sqrt((double)kp.m * (double)kp.m + pr * pr);
    kp.p[1][i] = fabs(pr);
}

template <typename R>
cudaError_t launch_sample_milne(const KParams<R>& kp, const MilneTables& mt, cudaStream_t s)
{
    if (kp.n == 0) return cudaSuccess;
    k_sample_milne<R><<<(unsigned)((kp.n + 127) / 128), 128, 0, s>>>(kp, mt);
    return cudaGetLastError();
}

template cudaError_t launch_sample_milne<double>(const KParams<double>&, const MilneTables&, cudaStream_t);
template cudaError_t launch_sample_milne<float>(const KParams<float>&, const MilneTables&, cudaStream_t);

template <typename R>
cudaError_t launch_sample_fonll(const KParams<R>& kp, const SampleTables& st, cudaStream_t s)
{
    if (kp.n == 0) return cudaSuccess;
    k_sample_fonll<R><<<(unsigned)((kp.n + 127) / 128), 128, 0, s>>>(kp, st);
    return cudaGetLastError();
}

template cudaError_t launch_sample_fonll<double>(const KParams<double>&, const SampleTables&, cudaStream_t);
template cudaError_t launch_sample_fonll<float>(const KParams<float>&, const SampleTables&, cudaStream_t);

}  // namespace lim

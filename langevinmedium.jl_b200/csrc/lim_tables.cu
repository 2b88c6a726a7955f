// lim_tables.cu — the transport tables built on the device: the uniform linear time
// splines of transport.jl:165-222 (drag time, diffusion-current time tau_n_main3, and
// the RTA time factor (eta/s)/T of the Langevin+RTA step) and the Jüttner inverse-CDF
// table of transport.jl:277-365, so that hosts running many ensembles (one spline per
// D_s variant) do not evaluate Bessel functions and CDFs node by node on the CPU.
//
// The scaled Bessel functions K_nu(z) e^z that tau_n_main3 needs come from the integral
// representation K_nu(z) = int_0^inf exp(-z cosh t) cosh(nu t) dt, evaluated as
// e^z K_nu(z) = int_0^inf exp(-z (cosh t - 1)) cosh(nu t) dt by the trapezoidal rule: the
// integrand is even and analytic in a strip about the real axis, so the rule converges
// geometrically in 1/h, and a step of min(1/8, 1/(2 sqrt z)) leaves an error far below
// FP64 rounding; the terms are positive, so the sum loses no digits.
#include <algorithm>
#include "lim_internal.h"

namespace lim {

namespace {

constexpr double kFmGeVd = 1.0 / 0.197327;   // constants.jl:13,23

__device__ double besselkx_dev(int nu, double z)
{
    // step 1/8, or 1/(2 sqrt z) where the integrand narrows to exp(-z t^2 / 2) (large z):
    // the trapezoid error then stays below exp(-2 pi^2 / (z h^2)) <= exp(-78)
    const double h = fmin(0.125, 0.5 / sqrt(z));
    double s = 0.5;                           // t = 0: exp(0) cosh(0), half weight
    for (int k = 1; k < 100000; ++k) {
        const double t = k * h;
        const double sh = sinh(0.5 * t);
        const double c = z * (2.0 * sh * sh);   // z (cosh t - 1) without cancellation at small t
        const double e = c - nu * t;          // term <= exp(-e), as cosh(nu t) <= exp(nu t)
        if (e > 745.0) break;
        const double term = exp(-c) * cosh(nu * t);
        s += term;
        if (e > 40.0 && term < 1e-18 * s) break;
    }
    return s * h;
}

__device__ double effective_DsT_dev(double T, double DsT, const TimeSplineSpec& sp)
{
    // transport.jl:139-156
    if (sp.quad) { const double x = T / sp.Tref; return DsT * x * x; }
    if (!sp.linear) return DsT;
    const double Tf = T > sp.Tfo ? T : sp.Tfo;
    return sp.slope * Tf + sp.offset;
}

// transport.jl:58-104 (tau_n_main3), :132-137 (tau_drag); the RTA time factor (eta/s)/T.
__device__ double time_of(int kind, double T, double m, double Ds, const TimeSplineSpec& sp)
{
    if (kind == TIME_TAUR) {
        if (!isfinite(T) || T <= 0.0) return 0.0;
        return sp.factor * sp.eta_over_s / T / kFmGeVd;
    }
    if (!isfinite(T) || !isfinite(m) || !isfinite(Ds) || T <= 0.0 || m <= 0.0 || Ds <= 0.0) return 0.0;
    if (kind == TIME_DRAG) return m * Ds / (T * T) / kFmGeVd;
    const double z = m / T;
    if (z <= 0.0) return 0.0;
    const double K2x = besselkx_dev(2, z), K3x = besselkx_dev(3, z);
    const double den = fabs(K2x) > 1e-300 ? fabs(K2x) : 1e-300;
    const double sgn = K2x == 0.0 ? 1.0 : copysign(1.0, K2x);
    if (z > 50.0) {
        const double tau = (Ds / T) * z * (K3x / den * sgn);
        return fmin(tau / kFmGeVd, 1e20);
    }
    const double num = 2.0 * besselkx_dev(1, z) - 3.0 * K3x + besselkx_dev(5, z);
    double z3T = z * z * z / T;
    if (!isfinite(z3T) || z3T > 1e50) z3T = 1e50;
    const double tau = (Ds / 48.0) * z3T * (num / den * sgn);
    if (!isfinite(tau) || fabs(tau) > 1e50) return 1e50 * copysign(1.0, tau);
    return tau / kFmGeVd;
}

}  // namespace

__global__ void k_time_spline(const TimeSplineSpec sp, double* __restrict__ vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.nT) return;
    const double dT = (sp.Tmax - sp.Tmin) / (sp.nT - 1);
    const double Ti = sp.Tmin + i * dT;
    const double Ds = effective_DsT_dev(Ti, sp.DsT, sp);
    vals[i] = time_of(sp.kind, Ti, sp.m, Ds, sp) * sp.scale;
}

// One block per temperature node jT: the trapezoid CDF of p^a exp(-(E - m)/T) on np
// momenta (a = dims - 1) in cdf[jT * np ...], a block scan of per-thread partial sums,
// then the inverse at nU uniform quantiles.
__global__ void __launch_bounds__(256) k_juttner_invcdf(const JuttnerSpec js, double* __restrict__ cdf_all,
                                                        double* __restrict__ inv)
{
    __shared__ double part[256];
    __shared__ double s_norm, s_phi;
    const int jT = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const int np = js.np, nU = js.nU, a = js.dims - 1;
    const double M = js.m, T = js.Tmin + jT * js.dT;
    const double pmax = 16.0 * sqrt(M * T) + 16.0 * T, dp = pmax / (np - 1);
    double* cdf = cdf_all + (size_t)jT * np;
    auto w = [&](int k) {
        if (k == 0) return a == 0 ? 1.0 : 0.0;
        const double p = k * dp, E = sqrt(M * M + p * p);
        const double pa = a == 0 ? 1.0 : (a == 1 ? p : p * p);
        return pa * exp(-(E - M) / T);
    };
    // increments inc_k = (w_k + w_{k+1}) dp / 2 for k = 0 .. np-2, into cdf[k+1]
    const int ninc = np - 1;
    const int per = (ninc + nth - 1) / nth;
    const int k0 = tid * per, k1 = min(k0 + per, ninc);
    double run = 0.0;
    for (int k = k0; k < k1; ++k) {
        run += 0.5 * (w(k) + w(k + 1)) * dp;
        cdf[k + 1] = run;                                   // local prefix
    }
    part[tid] = run;
    __syncthreads();
    if (tid == 0) {                                          // exclusive scan of the thread totals
        double acc = 0.0;
        for (int t = 0; t < nth; ++t) { const double v = part[t]; part[t] = acc; acc += v; }
        s_norm = acc;
        cdf[0] = 0.0;
    }
    __syncthreads();
    const double off = part[tid], norm = s_norm;
    const double invnorm = norm > 0.0 ? 1.0 / norm : 0.0;
    for (int k = k0; k < k1; ++k) cdf[k + 1] = (cdf[k + 1] + off) * invnorm;
    __syncthreads();
    if (tid == 0) {
        cdf[np - 1] = 1.0;
        const double thr = 1.0 - js.quantile_cap;           // first momentum whose CDF reaches thr
        int hit = np - 1;
        for (int k = 0; k < np; ++k) if (cdf[k] >= thr) { hit = k; break; }
        s_phi = hit * dp;
    }
    __syncthreads();
    const double p_hi = s_phi;
    for (int iu = tid; iu < nU; iu += nth) {
        const double u = (double)iu / (double)(nU - 1);
        // k = #{j >= 1 : cdf[j] < u} (searchsorted left in cdf[1:]), capped to np - 2
        int lo = 0, hi = np - 1;                             // search in cdf[1 .. np-1]
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf[1 + mid] < u) lo = mid + 1; else hi = mid;
        }
        const int k = min(lo, np - 2);
        const double c0 = cdf[k], c1 = cdf[k + 1];
        double frac = c1 > c0 ? (u - c0) / (c1 - c0) : 0.0;
        frac = fmin(fmax(frac, 0.0), 1.0);
        const double p0 = k * dp, p1 = (k + 1) * dp;
        const double pv = p0 + frac * (p1 - p0);
        inv[(size_t)jT * nU + iu] = pv < p_hi ? pv : p_hi;
    }
}

cudaError_t launch_time_spline(const TimeSplineSpec& sp, double* vals, cudaStream_t st)
{
    k_time_spline<<<(sp.nT + 127) / 128, 128, 0, st>>>(sp, vals);
    return cudaGetLastError();
}

cudaError_t launch_juttner_invcdf(const JuttnerSpec& js, double* cdf_scratch, double* inv, cudaStream_t st)
{
    k_juttner_invcdf<<<js.nT, 256, 0, st>>>(js, cdf_scratch, inv);
    return cudaGetLastError();
}

}  // namespace lim

// lim_common.cuh — device-side building blocks shared by every step kernel:
// kernel parameter blocks, counter-based Philox-4x32-10 variates, and the scalar
// semantics of the reference (Julia clamp / max / searchsortedlast).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lim {

constexpr double kEps = 2.220446049250313e-16;   // Julia eps()
constexpr double kFmGeV = 1.0 / 0.197327;        // constants.jl:13,23
constexpr int kNoiseSlots = 11;
enum { TAG_MOM = 1, TAG_RTA = 2, TAG_RTADIR = 3, TAG_DIFF = 4 };
enum { MED_RT = 0, MED_BJORKEN = 1, MED_GRID = 2 };
enum { COLL_LANGEVIN = 0, COLL_RTA = 1, COLL_LANGEVIN_RTA = 2, COLL_FLUID = 3 };

template <typename R> struct V2T;
template <> struct V2T<double> { using type = double2; };
template <> struct V2T<float>  { using type = float2; };

// ---------------------------------------------------------------------------
// Parameter blocks (passed by value to every step kernel)
// ---------------------------------------------------------------------------
template <typename R>
struct MediumDev {
    int kind;
    // (r, t) tables, kernels_cpu.jl:22-51: grids ascending, TV[i + nr*j] = (T, V)
    const R* xg; const R* tg; int nr, nt;
    R xg0, xinvd; int x_uniform;                 // O(1) first guess of searchsortedlast
    double tg0, tinvd; int t_uniform;
    const typename V2T<R>::type* TV;
    const R* V2; int use_v2;
    const double* tgd;                           // tgrid in FP64 (time cell is found in FP64)
    const double* xgd;                           // xgrid in FP64 (FP64 freeze-out temperature)
    // analytic Bjorken T(tau) = T0 (tau0/tau)^power
    double bj_T0, bj_tau0, bj_power;
    // 2+1D grid, float4 (T, ux, uy, 0) per node, [it][iy][ix]
    const float4* G; int gnx, gny, gnt;
    double gx0_d, gdx_d, gxl_d, gy0_d, gdy_d, gyl_d;   // node geometry (FP64)
    float ginvdx, ginvdy;                              // FP32 fast path
    double gt0, gdt_d, gtl;
    // geometry of the reflecting boundary (kernels_cpu.jl:528-534)
    R r_max, r_axis_eps;
    R T_scale;
};

template <typename R>
struct KParams {
    // run constants
    double dt, t0;
    R m, DsT, Tfo, psi2, sqrt_dt, dtR;
    int rel, collision, redshift, diffusion, reflect, integrator, fo_capture, fo_interp, stop_fo;
    uint32_t seed_lo, seed_hi;
    int64_t pid_offset;
    int64_t n;
    int dims, pdim;
    // transport splines (transport.jl:231-253) and Jüttner inverse CDF
    const R* drag; int n_drag; R drag_Tmin, drag_invdT;
    const R* rta;  int n_rta;  R rta_Tmin, rta_invdT;
    const R* icdf; int nU, nT; R ic_Tmin, ic_invdT;
    MediumDev<R> med;
    // particle state, structure of arrays.  Momenta are accumulated in FP64 in both
    // precisions (the FP32 path adds FP32-computed increments to an FP64 state).
    R* x[3]; float* xlo[3]; double* p[3];
    // freeze-out latch: outputs and the last-above cache (FP64 in both precisions:
    // the latch divides by a one-step temperature change)
    double* fo_pos[3]; double* fo_mom[3]; double* fo_tau; double* fo_flag;
    double* l_pos[3]; double* l_mom[3]; double* l_tau; double* l_T;
    // status and diagnostics
    unsigned long long* first_bad;   // atomicMin of the first non-finite step
    double* rec; int64_t rec_first, rec_steps;
    // per-step records (StepRec<R>, lim_step.cuh) for steps [step_base, step_base + step_cap)
    void* steps; int64_t step_base, step_cap;
};

// ---------------------------------------------------------------------------
// Julia scalar semantics on the device
// ---------------------------------------------------------------------------
template <typename R> __device__ __forceinline__ R jclamp(R x, R lo, R hi)
{
    return x > hi ? hi : (x < lo ? lo : x);   // Base.clamp
}
template <typename R> __device__ __forceinline__ R jmax0(R x)
{
    return (x != x) ? x : (x > R(0) ? x : R(0));   // Base.max(x, 0.0), NaN-propagating
}
template <typename R> __device__ __forceinline__ bool finite_(R x) { return isfinite(x); }

// Last 0-based index k with g[k] <= x, capped to [0, n-2] (the reference's
// i = clamp(searchsortedlast(g, x), 1, n-1) minus one).  x must already be
// clamped to [g[0], g[n-1]] by the caller when the reference clamps.
template <typename R>
__device__ __forceinline__ int cell_index(const R* __restrict__ g, int n, R x, int uniform, R g0, R invd)
{
    int k;
    if (uniform) {
        R f = (x - g0) * invd;
        k = f > R(0) ? (int)f : 0;
        k = k > n - 1 ? n - 1 : k;
        // exact correction to searchsortedlast semantics
        while (k + 1 < n && __ldg(g + k + 1) <= x) ++k;
        while (k > 0 && __ldg(g + k) > x) --k;
    } else {
        int lo = -1, hi = n;            // invariant: g[lo] <= x < g[hi]
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (__ldg(g + mid) <= x) lo = mid; else hi = mid;
        }
        k = lo < 0 ? 0 : lo;
    }
    return k > n - 2 ? n - 2 : k;
}

// transport.jl:231-253 — eval_tau_n_spline (0-based).
template <typename R>
__device__ __forceinline__ R eval_spline(R T, R Tmin, R invdT, const R* __restrict__ vals, int n)
{
    if (n < 2) return __ldg(vals);
    if (!isfinite(T)) return R(0);
    R u = (T - Tmin) * invdT;
    R fl = floor(u);
    int i = fl < R(0) ? 0 : (fl > R(n - 2) ? n - 2 : (int)fl);
    R t = u - R(i);
    R y0 = __ldg(vals + i), y1 = __ldg(vals + i + 1);
    if (sizeof(R) == 8) return (R(1) - t) * y0 + t * y1;   // the reference's form, for FP64 parity
    return y0 + t * (y1 - y0);                             // FP32: no cancellation when |t| is large
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter (pid, step, 2*tag+half, 0)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u; k.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ double u01_f64(uint32_t hi, uint32_t lo)
{
    unsigned long long v = ((unsigned long long)hi << 32) | (unsigned long long)lo | 1ull;
    return __ull2double_rz(v) * 0x1p-64;     // (0,1), exact truncation to 53 bits
}
__device__ __forceinline__ float u01_f32(uint32_t hi)
{
    return __uint2float_rz(hi | 1u) * 0x1p-32f;   // (0,1), tracks u01_f64 to 2^-23
}

template <typename R> struct Uni4 { R u[4]; };

// Four uniforms of `tag` for (pid, step).  FP64 combines the high words of block
// (tag, 0) with the low words of block (tag, 1); FP32 uses the high words only.
template <typename R>
__device__ __forceinline__ Uni4<R> uniforms4(uint32_t seed_lo, uint32_t seed_hi, uint32_t pid, uint32_t step, int tag);

template <>
__device__ __forceinline__ Uni4<double> uniforms4<double>(uint32_t slo, uint32_t shi, uint32_t pid, uint32_t step, int tag)
{
    uint2 key = make_uint2(slo, shi);
    uint4 h = philox4x32_10(make_uint4(pid, step, 2u * tag, 0u), key);
    uint4 l = philox4x32_10(make_uint4(pid, step, 2u * tag + 1u, 0u), key);
    Uni4<double> r;
    r.u[0] = u01_f64(h.x, l.x); r.u[1] = u01_f64(h.y, l.y);
    r.u[2] = u01_f64(h.z, l.z); r.u[3] = u01_f64(h.w, l.w);
    return r;
}
template <>
__device__ __forceinline__ Uni4<float> uniforms4<float>(uint32_t slo, uint32_t shi, uint32_t pid, uint32_t step, int tag)
{
    uint4 h = philox4x32_10(make_uint4(pid, step, 2u * tag, 0u), make_uint2(slo, shi));
    Uni4<float> r;
    r.u[0] = u01_f32(h.x); r.u[1] = u01_f32(h.y); r.u[2] = u01_f32(h.z); r.u[3] = u01_f32(h.w);
    return r;
}

// Box–Muller: (sqrt(-2 ln u0) cos 2πu1, sqrt(-2 ln u0) sin 2πu1).
__device__ __forceinline__ void box_muller(double u0, double u1, double& z0, double& z1)
{
    double rad = sqrt(-2.0 * log(u0));
    double th = 6.283185307179586 * u1;
    double s, c;
    sincos(th, &s, &c);
    z0 = rad * c; z1 = rad * s;
}
__device__ __forceinline__ void box_muller(float u0, float u1, float& z0, float& z1)
{
    float rad = sqrtf(-2.0f * logf(u0));
    float s, c;
    sincospif(2.0f * u1, &s, &c);
    z0 = rad * c; z1 = rad * s;
}

}  // namespace lim

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
enum { TAG_MOM = 1, TAG_RTA = 2, TAG_DIFF = 4,                   // (tag 3 unused)
       TAG_SAMPLE_XY = 5, TAG_SAMPLE_P = 6, TAG_SAMPLE_PZ = 7 };   // initial-state sampling (lim_sample.cu)
enum { MED_RT = 0, MED_BJORKEN = 1, MED_GRID = 2 };
// The adjoint's tape: float4 rows per particle-step, row k of step s at
// ((s - tape_first) * rows + k) * n + i.  Bjorken: (x0, x1, p0, p1), (p2, xi0, xi1, xi2).
// 2+1D grid: the pre-step momentum and the medium the step saw, with its gradient, so
// the reverse sweep needs no grid lookups:
//   (p0, p1, p2, T), (xi0, xi1, xi2, v^x), (v^y, dT/dx, dT/dy, dv^x/dx), (dv^x/dy, dv^y/dx, dv^y/dy, 0)
// (T before the medium scale, v the grid's flow velocity).
__host__ __device__ constexpr int tape_rows(int med) { return med == MED_GRID ? 4 : 2; }
constexpr int kTapeRowsMax = 4;
enum { COLL_LANGEVIN = 0, COLL_RTA = 1, COLL_LANGEVIN_RTA = 2, COLL_FLUID = 3 };

template <typename R> struct V2T;
template <> struct V2T<double> { using type = double2; };
template <> struct V2T<float>  { using type = float2; };
template <typename R> struct V4T;
template <> struct V4T<double> { using type = double4; };
template <> struct V4T<float>  { using type = float4; };

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
    // the same table per cell for the step's lookup: TVc[i + (nr-1) j] = (T_i, V_i,
    // T_i+1, V_i+1) of time row j, xc[i] = (x_i, x_i+1), and the clamp bounds x_0, x_nr-1
    const typename V4T<R>::type* TVc;
    const typename V2T<R>::type* xc;
    R xlo, xhi;
    const R* V2; int use_v2;
    const double* tgd;                           // tgrid in FP64 (time cell is found in FP64)
    const double* xgd;                           // xgrid in FP64 (FP64 freeze-out temperature)
    // analytic Bjorken T(tau) = T0 (tau0/tau)^power
    double bj_T0, bj_tau0, bj_power;
    // 2+1D grid, float4 (T, ux, uy, 0) per node, [it][iy][ix]
    const float4* G; int gnx, gny, gnt;
    double gx0_d, gdx_d, gxl_d, gy0_d, gdy_d, gyl_d;   // node geometry (FP64)
    float ginvdx, ginvdy;                              // FP32 fast path
    // FP32 cell location: the node nearest the grid's centre (index, coordinate as a
    // float pair) and the low words of 1/dx, 1/dy
    int gicx, gicy;
    float gxc, gxcl, gyc, gycl, ginvdx_lo, ginvdy_lo;
    double gt0, gdt_d, gtl;
    // geometry of the reflecting boundary (kernels_cpu.jl:528-534)
    R r_max, r_axis_eps;
    R T_scale;
};

// 16-byte aligned and sized, so that a kernel can stage it in shared memory with
// 128-bit copies.
template <typename R>
struct alignas(16) KParams {
    // run constants
    double dt, t0;
    R m, DsT, Tfo, psi2, sqrt_dt, dtR;
    int rel, collision, redshift, diffusion, reflect, integrator, fo_capture, fo_interp, stop_fo;
    uint32_t seed_lo, seed_hi;
    uint2 rk[10];          // Philox round keys of the seed (kernel-parameter constants)
    int spl_shared;        // drag and RTA splines share their T grid: one index for both
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
    // live list (runs that stop particles at freeze-out): when set, the step kernel
    // advances only particles live[0 .. *live_n) (grid-stride), so that warps stay full
    const int* live; const unsigned* live_n;
    // RTA decisions of steps [rta_first, rta_first + rta_steps): rta_mode 1 records them
    // (bit (s - rta_first) % 32 of word [(s - rta_first) / 32][particle], zeroed before),
    // 2 replays them instead of comparing u_collide with the collision probability
    uint32_t* rta_bits; int rta_mode; int64_t rta_first, rta_steps;
    // derivative tables of the drag spline w.r.t. two parameters of D_s(T) (same T grid);
    // for the adjoint: per drag cell two float4 (tau_i, dtau_i, a_i, da_i), (b_i, db_i,
    // dtau_i invdT, 0) with the differences to cell i+1 formed in FP64, the inverse
    // CDF's T differences, and the tape of steps [tape_first, ...)
    const R* drag_da; const R* drag_db;
    const float4* adj_drag; const R* icdf_dT;
    float* tape; int64_t tape_first;
    // FP32 runs: the RTA spline and the (r, t) temperature table in FP64, for collision
    // decisions that fall within FP32 rounding of the collision probability (decided
    // again in FP64, as the FP64 path decides them); NULL in FP64 runs
    const double* rta64; double rta_Tmin64, rta_invdT64; int n_rta64;
    const double* T64;
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

// transport.jl:231-253 — eval_tau_n_spline (0-based), split into the cell/weight
// lookup and the evaluation so that two splines on one T grid share the lookup.
template <typename R> struct SplIdx { int i; R t; int mode; };   // mode: 0 normal, 1 first value, 2 zero

template <typename R>
__device__ __forceinline__ SplIdx<R> spline_index(R T, R Tmin, R invdT, int n)
{
    SplIdx<R> s;
    s.i = 0; s.t = R(0);
    if (n < 2) { s.mode = 1; return s; }
    if (!isfinite(T)) { s.mode = 2; return s; }
    s.mode = 0;
    R u = (T - Tmin) * invdT;
    if constexpr (sizeof(R) == 4) {
        // floor(u) from one round-down add of 1.5 2^23 (exact for |u| < 2^22; beyond the
        // clamp the index is clamped to the table either way): no FP32 -> int conversion
        const float tf = __fadd_rd(jclamp(u, -4.0e6f, 4.0e6f), 12582912.0f);
        const int k = __float_as_int(tf) - 0x4B400000;
        s.i = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
        s.t = __fmaf_rn(T - Tmin, invdT, -(float)s.i);   // fused: one rounding in every instantiation
    } else {
        R fl = floor(u);
        s.i = fl < R(0) ? 0 : (fl > R(n - 2) ? n - 2 : (int)fl);
        s.t = u - R(s.i);
    }
    return s;
}

template <typename R>
__device__ __forceinline__ R spline_at(const R* __restrict__ vals, const SplIdx<R>& s)
{
    if (s.mode == 1) return __ldg(vals);
    if (s.mode == 2) return R(0);
    R y0 = __ldg(vals + s.i), y1 = __ldg(vals + s.i + 1);
    if (sizeof(R) == 8) return (R(1) - s.t) * y0 + s.t * y1;   // the reference's form, for FP64 parity
    return y0 + s.t * (y1 - y0);                               // FP32: no cancellation when |t| is large
}

template <typename R>
__device__ __forceinline__ R eval_spline(R T, R Tmin, R invdT, const R* __restrict__ vals, int n)
{
    return spline_at(vals, spline_index(T, Tmin, invdT, n));
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter (pid, step, tag, 0)
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

// The same block with the round keys precomputed (k_r = key + r (W0, W1)): the keys
// become constant operands instead of two additions per round.
__device__ __forceinline__ uint4 philox4x32_10_rk(uint4 c, const uint2* __restrict__ rk)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ rk[r].x, lo1, hi0 ^ c.w ^ rk[r].y, lo0);
    }
    return c;
}

// A particle's noise stream: the seed's round keys and the particle id.  The keys are
// passed apart from the rest of the parameters so that a kernel whose per-ensemble
// parameters live in shared memory still reads them as kernel-parameter constants.
struct NoiseKey { const uint2* rk; uint32_t pid; };

// The four words of `tag` for (pid, step): one Philox block, counter (pid, step, tag, 0).
__device__ __forceinline__ uint4 philox_words(const uint2* rk, uint32_t pid, uint32_t step, int tag)
{
    return philox4x32_10_rk(make_uint4(pid, step, (uint32_t)tag, 0u), rk);
}

// Uniform variates.  A word w stands for u = (w + 1/2) 2^-32 in (0, 1), the same value
// in both precisions.  FP64 holds u exactly.  FP32 evaluates the steep maps (log u near
// 1, the inverse normal CDF and the inverse Jüttner CDF near 0 and 1) on u folded about
// 1/2: u = mag (lower half) or 1 - mag (upper half), with
// mag = (2 min(w, ~w) + 1) 2^-33 in (0, 1/2], so both tails keep full relative precision.
__device__ __forceinline__ double u_exact(uint32_t w) { return fma((double)w, 0x1p-32, 0x1p-33); }
__device__ __forceinline__ bool u_upper(uint32_t w) { return (int32_t)w < 0; }

template <typename R> __device__ __forceinline__ R u_mag(uint32_t w);
template <> __device__ __forceinline__ double u_mag<double>(uint32_t w)
{
    const uint32_t m = u_upper(w) ? ~w : w;
    return (double)(2u * m + 1u) * 0x1p-33;
}
template <> __device__ __forceinline__ float u_mag<float>(uint32_t w)
{
    const uint32_t m = u_upper(w) ? ~w : w;
    return __uint2float_rn(2u * m + 1u) * 0x1p-33f;
}

template <typename R> __device__ __forceinline__ R u_value(uint32_t w);
template <> __device__ __forceinline__ double u_value<double>(uint32_t w) { return u_exact(w); }
template <> __device__ __forceinline__ float u_value<float>(uint32_t w)
{
    return fmaf(__uint2float_rn(w), 0x1p-32f, 0x1p-33f);
}

// -2 ln u.  FP32 upper half: ln(1 - mag) = ln(y) + r/y with y = fl(1 - mag) and the
// exact rounding error r = (1 - mag) - y (Fast2Sum), so one logf serves both halves.
__device__ __forceinline__ double neg2_log_u(uint32_t w, double) { return -2.0 * log(u_exact(w)); }
__device__ __forceinline__ float neg2_log_u(uint32_t w, float)
{
    const float mag = u_mag<float>(w);
    const bool up = u_upper(w);
    const float y = 1.0f - mag;
    const float r = -mag - (y - 1.0f);
    const float a = up ? y : mag;
    const float c = up ? __fdividef(r, y) : 0.0f;
    return -2.0f * (logf(a) + c);
}

// 2u - 1 = (2w + 1 - 2^32) 2^-32, the Box–Muller angle in units of pi.
__device__ __forceinline__ double u_centered(uint32_t w, double) { return fma((double)(int32_t)(w ^ 0x80000000u), 0x1p-31, 0x1p-32); }
__device__ __forceinline__ float u_centered(uint32_t w, float)
{
    return fmaf(__int2float_rn((int32_t)(w ^ 0x80000000u)), 0x1p-31f, 0x1p-32f);
}

// sin(pi a) and cos(pi a) for a in [-1, 1] in FP32: a = r + q/2 with q = rint(2a) and
// |r| <= 1/4 (exact), the Taylor series of sin(pi r) (through r^9) and cos(pi r)
// (through r^10) in r^2 by Horner's rule (truncation below 3e-9), then the quadrant
// q selects and signs them.  Absolute error about 1.5e-7 (the arguments' and results'
// FP32 rounding), against 2^-21.4 = 3.6e-7 of the hardware sine/cosine.
__device__ __forceinline__ void sincospi_f32(float a, float& s, float& c)
{
    const float q = rintf(2.0f * a);
    const float r = fmaf(-0.5f, q, a);
    const float z = r * r;
    float ps = fmaf(z, 0.08214588661112823f, -0.5992645293207921f);
    ps = fmaf(ps, z, 2.5501640398773455f);
    ps = fmaf(ps, z, -5.16771278004997f);
    ps = fmaf(ps, z, 3.141592653589793f);
    float pc = fmaf(z, -0.02580689139001406f, 0.2353306303588932f);
    pc = fmaf(pc, z, -1.3352627688545895f);
    pc = fmaf(pc, z, 4.0587121264167685f);
    pc = fmaf(pc, z, -4.934802200544679f);
    const float sn = r * ps, cs = fmaf(pc, z, 1.0f);
    const int qi = (int)q;
    const bool swap = (qi & 1) != 0;
    s = swap ? cs : sn;
    c = swap ? sn : cs;
    if ((qi + 4) & 2) s = -s;      // quadrants q = 2, -1, -2
    if ((qi + 5) & 2) c = -c;      // quadrants q = 1, 2, -2
}

// Box–Muller with the angle in (-pi, pi): (rad cos(pi(2u1-1)), rad sin(pi(2u1-1))),
// rad = sqrt(-2 ln u0); FP32 takes the sine and cosine from sincospi_f32.
__device__ __forceinline__ void box_muller(uint32_t w0, uint32_t w1, double& z0, double& z1)
{
    const double rad = sqrt(neg2_log_u(w0, 0.0));
    double s, c;
    sincospi(u_centered(w1, 0.0), &s, &c);
    z0 = rad * c; z1 = rad * s;
}
__device__ __forceinline__ void box_muller(uint32_t w0, uint32_t w1, float& z0, float& z1)
{
    const float rad = sqrtf(neg2_log_u(w0, 0.0f));
    float s, c;
    sincospi_f32(u_centered(w1, 0.0f), s, c);
    z0 = rad * c; z1 = rad * s;
}

// Inverse standard normal CDF of u (FP32: of the folded magnitude, sign restored).
__device__ __forceinline__ double norm_inv(uint32_t w, double) { return normcdfinv(u_exact(w)); }
__device__ __forceinline__ float norm_inv(uint32_t w, float)
{
    const float z = normcdfinvf(u_mag<float>(w));
    return u_upper(w) ? -z : z;
}

}  // namespace lim

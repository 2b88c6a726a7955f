// lim_step.cuh — one Langevin step of one particle, register-resident.
//
// The sequence is the reference's (simulate_cpu.jl:215-303):
//   noise -> rest-frame boost -> [Bjorken redshift] -> {fluid | OU kick | RTA
//   | OU kick + RTA} -> lab boost -> streaming (+diffusion, reflection)
// fused into one device function so that the state never leaves registers.
// Medium time at step s is s*dt + t0 (kernels_cpu.jl:67).
#pragma once
#include "lim_common.cuh"

namespace lim {

// Per-step values that are the same for every particle.
template <typename R>
struct StepU {
    double t;        // medium time s*dt + t0
    R tR;
    int kt; R wt;    // (r,t) table: time cell and weight
    R T_bj;          // Bjorken temperature at t
    int it; R wtg;       // grid: time cell and weight
};

template <typename R, int MED>
__device__ __forceinline__ StepU<R> step_uniforms(const KParams<R>& kp, int64_t s)
{
    StepU<R> u;
    u.t = __dadd_rn(__dmul_rn((double)s, kp.dt), kp.t0);
    u.tR = (R)u.t;
    u.kt = 0; u.wt = R(0); u.T_bj = R(0); u.it = 0; u.wtg = R(0);
    const MediumDev<R>& md = kp.med;
    if (MED == MED_RT) {
        const double* tg = md.tgd;
        int nt = md.nt;
        double tq = u.t > tg[nt - 1] ? tg[nt - 1] : (u.t < tg[0] ? tg[0] : u.t);
        int k;
        if (md.t_uniform) {
            double f = (tq - md.tg0) * md.tinvd;
            k = f > 0.0 ? (int)f : 0;
            k = k > nt - 1 ? nt - 1 : k;
            while (k + 1 < nt && __ldg(tg + k + 1) <= tq) ++k;
            while (k > 0 && __ldg(tg + k) > tq) --k;
        } else {
            int lo = -1, hi = nt;
            while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (__ldg(tg + mid) <= tq) lo = mid; else hi = mid; }
            k = lo < 0 ? 0 : lo;
        }
        k = k > nt - 2 ? nt - 2 : k;
        double y0 = __ldg(tg + k), y1 = __ldg(tg + k + 1), dy = y1 - y0;
        u.kt = k;
        u.wt = (R)(fabs(dy) < kEps ? 0.0 : (tq - y0) / dy);
    } else if (MED == MED_BJORKEN) {
        double T = (u.t > md.bj_tau0) ? md.bj_T0 * pow(md.bj_tau0 / u.t, md.bj_power) : md.bj_T0;
        u.T_bj = (R)T;
    } else {
        double tq = u.t > md.gtl ? md.gtl : (u.t < md.gt0 ? md.gt0 : u.t);
        double f = (tq - md.gt0) / md.gdt_d;
        double fl = floor(f);
        int it = fl < 0.0 ? 0 : (fl > (double)(md.gnt - 2) ? md.gnt - 2 : (int)fl);
        u.it = it;
        u.wtg = (R)(f - (double)it);
    }
    return u;
}

// (r, t) table: bilinear interpolation of (T, V) at radius r (clamped), time cell from StepU.
template <typename R>
__device__ __forceinline__ void rt_lookup(const MediumDev<R>& md, const StepU<R>& su, R r, R& T, R& V)
{
    R rq = jclamp(r, __ldg(md.xg), __ldg(md.xg + md.nr - 1));
    int i = cell_index(md.xg, md.nr, rq, md.x_uniform, md.xg0, md.xinvd);
    R x0 = __ldg(md.xg + i), x1 = __ldg(md.xg + i + 1);
    R dx = x1 - x0;
    R xd = fabs(dx) < R(kEps) ? R(0) : (rq - x0) / dx;
    const int nr = md.nr, j = su.kt;
    auto a00 = md.TV[i + nr * j],       a10 = md.TV[i + 1 + nr * j];
    auto a01 = md.TV[i + nr * (j + 1)], a11 = md.TV[i + 1 + nr * (j + 1)];
    R yd = su.wt;
    R c0 = a00.x * (R(1) - xd) + a10.x * xd;
    R c1 = a01.x * (R(1) - xd) + a11.x * xd;
    T = c0 * (R(1) - yd) + c1 * yd;
    c0 = a00.y * (R(1) - xd) + a10.y * xd;
    c1 = a01.y * (R(1) - xd) + a11.y * xd;
    V = c0 * (R(1) - yd) + c1 * yd;
}

template <typename R>
__device__ __forceinline__ R rt_lookup_scalar(const MediumDev<R>& md, const StepU<R>& su, const R* __restrict__ vals, R r)
{
    R rq = jclamp(r, __ldg(md.xg), __ldg(md.xg + md.nr - 1));
    int i = cell_index(md.xg, md.nr, rq, md.x_uniform, md.xg0, md.xinvd);
    R x0 = __ldg(md.xg + i), x1 = __ldg(md.xg + i + 1);
    R dx = x1 - x0;
    R xd = fabs(dx) < R(kEps) ? R(0) : (rq - x0) / dx;
    const int nr = md.nr, j = su.kt;
    R v00 = __ldg(vals + i + nr * j), v10 = __ldg(vals + i + 1 + nr * j);
    R v01 = __ldg(vals + i + nr * (j + 1)), v11 = __ldg(vals + i + 1 + nr * (j + 1));
    R yd = su.wt;
    R c0 = v00 * (R(1) - xd) + v10 * xd;
    R c1 = v01 * (R(1) - xd) + v11 * xd;
    return c0 * (R(1) - yd) + c1 * yd;
}

// 2+1D grid: trilinear of (T, ux, uy) at (x, y) clamped to the grid.  The
// FP32 path finds the cell in FP32; the FP64 path in FP64 from the same nodes.
template <typename R>
__device__ __forceinline__ void grid_cell(const MediumDev<R>& md, R xq, R yq, int& ix, int& iy, R& wx, R& wy)
{
    R x = xq > (R)md.gxl_d ? (R)md.gxl_d : (xq < (R)md.gx0_d ? (R)md.gx0_d : xq);
    R y = yq > (R)md.gyl_d ? (R)md.gyl_d : (yq < (R)md.gy0_d ? (R)md.gy0_d : yq);
    R fx, fy;
    if (sizeof(R) == 8) { fx = (x - (R)md.gx0_d) / (R)md.gdx_d; fy = (y - (R)md.gy0_d) / (R)md.gdy_d; }
    else { fx = (x - (R)md.gx0_d) * (R)md.ginvdx; fy = (y - (R)md.gy0_d) * (R)md.ginvdy; }
    R flx = floor(fx), fly = floor(fy);
    ix = flx < R(0) ? 0 : (flx > R(md.gnx - 2) ? md.gnx - 2 : (int)flx);
    iy = fly < R(0) ? 0 : (fly > R(md.gny - 2) ? md.gny - 2 : (int)fly);
    wx = fx - R(ix);
    wy = fy - R(iy);
}

template <typename R>
__device__ __forceinline__ void grid_lookup(const MediumDev<R>& md, const StepU<R>& su, R xq, R yq, R& T, R& ux, R& uy)
{
    int ix, iy;
    R Wx, Wy;
    grid_cell(md, xq, yq, ix, iy, Wx, Wy);
    const R Wt = su.wtg;
    const float4* s0 = md.G + ((size_t)su.it * md.gny + iy) * md.gnx + ix;
    const float4* s1 = s0 + (size_t)md.gny * md.gnx;
    float4 a00 = __ldg(s0), a10 = __ldg(s0 + 1), a01 = __ldg(s0 + md.gnx), a11 = __ldg(s0 + md.gnx + 1);
    float4 b00 = __ldg(s1), b10 = __ldg(s1 + 1), b01 = __ldg(s1 + md.gnx), b11 = __ldg(s1 + md.gnx + 1);
#define LIM_BILERP(c, A00, A10, A01, A11)                                              \
    ((((R)A00.c) * (R(1) - Wx) + ((R)A10.c) * Wx) * (R(1) - Wy) +                          \
     (((R)A01.c) * (R(1) - Wx) + ((R)A11.c) * Wx) * Wy)
    R T0 = LIM_BILERP(x, a00, a10, a01, a11), T1 = LIM_BILERP(x, b00, b10, b01, b11);
    R U0 = LIM_BILERP(y, a00, a10, a01, a11), U1 = LIM_BILERP(y, b00, b10, b01, b11);
    R V0 = LIM_BILERP(z, a00, a10, a01, a11), V1 = LIM_BILERP(z, b00, b10, b01, b11);
#undef LIM_BILERP
    T = T0 * (R(1) - Wt) + T1 * Wt;
    ux = U0 * (R(1) - Wt) + U1 * Wt;
    uy = V0 * (R(1) - Wt) + V1 * Wt;
}

// Flow seen by one particle this step: boost direction (nx, ny), signed speed v,
// and the local temperature T at the same point.
template <typename R>
struct Local {
    R T, v, nx, ny;
    bool active;      // false => no boost (r < eps, kernels_cpu.jl:75-77)
};

template <typename R, int MED, int DIMS>
__device__ __forceinline__ Local<R> local_medium(const KParams<R>& kp, const StepU<R>& su, const R (&x)[3])
{
    Local<R> L;
    L.nx = R(0); L.ny = R(0);
    if (MED == MED_GRID) {
        R ux, uy;
        grid_lookup(kp.med, su, x[0], x[1], L.T, ux, uy);
        R u = sqrt(ux * ux + uy * uy);
        L.active = !(u < R(kEps));
        L.v = u;
        if (L.active) { L.nx = ux / u; L.ny = uy / u; }
    } else {
        R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        R r = sqrt(r2);
        L.active = !(r < R(kEps));
        if (MED == MED_RT) {
            rt_lookup(kp.med, su, r, L.T, L.v);
            if (DIMS >= 2 && kp.med.use_v2 && L.active) {
                R v2m = rt_lookup_scalar(kp.med, su, kp.med.V2, r);
                R phi = atan2(x[1], x[0]);
                L.v *= (R(1) + R(2) * v2m * cos(R(2) * (phi - kp.psi2)));
            }
        } else {
            L.T = su.T_bj;
            L.v = R(0);
        }
        if (DIMS >= 2 && L.active) { L.nx = x[0] / r; L.ny = x[1] / r; }
    }
    if (kp.med.T_scale != R(1)) L.T *= kp.med.T_scale;
    return L;
}

// kernels_cpu.jl:89-145 (to_lab = false) and :188-241 (to_lab = true).
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ void boost(const KParams<R>& kp, const Local<R>& L, R (&p)[3], bool to_lab)
{
    if (!L.active) return;
    const R m = kp.m;
    R v = L.v;
    if (!kp.rel) {                     // Galilean p_par -/+ m v
        R mv = m * v;
        if (DIMS == 1) { p[0] = to_lab ? p[0] + mv : p[0] - mv; }
        else {
            R dx = mv * L.nx, dy = mv * L.ny;
            p[0] = to_lab ? p[0] + dx : p[0] - dx;
            p[1] = to_lab ? p[1] + dy : p[1] - dy;
        }
        return;
    }
    const R vmax = sizeof(R) == 8 ? R(0.9999999999995) : R(0.99999994f);   // sqrt(1 - 1e-12)
    v = jclamp(v, -vmax, vmax);
    R gam;
    if (sizeof(R) == 8) gam = R(1) / sqrt(R(1) - v * v + R(1e-10));
    else gam = rsqrt((R(1) - v) * (R(1) + v) + R(1e-10));
    R p2 = R(0);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p2 += p[d] * p[d];
    R E = sqrt(p2 + m * m);
    R vE = to_lab ? v * E : -(v * E);
    if (DIMS == 1) { p[0] = gam * (p[0] + vE); return; }
    R px = p[0], py = p[1];
    R ppar = px * L.nx + py * L.ny;
    R pperpx = px - ppar * L.nx;
    R pperpy = py - ppar * L.ny;
    R pnew = gam * (ppar + vE);
    p[0] = pnew * L.nx + pperpx;
    p[1] = pnew * L.ny + pperpy;
}

// Records the variates consumed by the step when noise recording is on.
template <typename R>
__device__ __forceinline__ void rec_slot(const KParams<R>& kp, int64_t s, int64_t i, int slot, R val)
{
    if (kp.rec && s >= kp.rec_first && s < kp.rec_first + kp.rec_steps)
        kp.rec[((s - kp.rec_first) * kNoiseSlots + slot) * kp.n + i] = (double)val;
}

// kernels_cpu.jl:246-357 + :406-417: exact-OU drag and kick in the LRF.
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ void langevin_kick(const KParams<R>& kp, R T, R (&p)[3], const R (&xi)[3])
{
    const R M = kp.m, dt = kp.dtR;
    const R DsT_safe = kp.DsT <= R(0) ? R(0) : kp.DsT;
    R tau = DsT_safe == R(0) ? R(0) : eval_spline(T, kp.drag_Tmin, kp.drag_invdT, kp.drag, kp.n_drag);
    const bool ok = tau > R(0) && isfinite(tau);
    R etaD = ok ? R(1) / tau : R(0);
    R kappa = ok ? (R(2) * M * T) / tau : R(0);
    R kT = sqrt(kappa);
    if (DIMS == 1) {
        R pm = fabs(p[0]);
        R E = sqrt(pm * pm + M * M);
        R eff = kp.rel ? etaD * M / E : etaD;
        p[0] += -eff * p[0] * dt + kp.sqrt_dt * (kT * xi[0]);
        return;
    }
    if (!(etaD > R(0))) {
#pragma unroll
        for (int d = 0; d < PDIM; ++d) p[d] += kp.sqrt_dt * (kT * xi[d]);
        return;
    }
    R p2 = R(0);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p2 += p[d] * p[d];
    R E = sqrt(p2 + M * M);
    R eff = kp.rel ? etaD * M / E : etaD;
    if (kp.integrator == 1) {          // kernels_gpu.jl:368-381 drift-midpoint
        R a_half = exp(-eff * (R(0.5) * dt));
        R p2m = R(0);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) { R pm = a_half * p[d]; p2m += pm * pm; }
        R Em = sqrt(p2m + M * M);
        eff = kp.rel ? etaD * M / Em : etaD;
    }
    if (sizeof(R) == 8) {
        R a = exp(-eff * dt);
        R np = (dt > R(0) && eff > R(0)) ? kT * sqrt((R(1) - a * a) / (R(2) * eff * dt)) : R(0);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) p[d] += (a - R(1)) * p[d] + kp.sqrt_dt * (np * xi[d]);
    } else {
        // FP32: a - 1 and 1 - a^2 from one expm1 (no cancellation); the noise
        // amplitude sqrt(dt)*kT*sqrt((1-a^2)/(2 eff dt)) = sqrt(kappa (1-a^2) / (2 eff)).
        R em1 = expm1(-eff * dt);
        R one_m_a2 = -em1 * (R(2) + em1);
        R amp = (dt > R(0) && eff > R(0)) ? sqrt(kappa * one_m_a2 / (R(2) * eff)) : R(0);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) p[d] += em1 * p[d] + amp * xi[d];
    }
}

// kernels_gpu.jl:88-117
template <typename R>
__device__ __forceinline__ R invcdf_lookup(const KParams<R>& kp, R u, R T)
{
    const int nU = kp.nU, nT = kp.nT;
    R uu = u < R(0) ? R(0) : (u > R(1) ? R(1) : u);
    R fu = uu * R(nU - 1);
    int iu = (int)floor(fu);
    iu = iu < 0 ? 0 : (iu > nU - 2 ? nU - 2 : iu);
    R tu = fu - R(iu);
    R fT = (T - kp.ic_Tmin) * kp.ic_invdT;
    R flT = floor(fT);
    int jT = flT < R(0) ? 0 : (flT > R(nT - 2) ? nT - 2 : (int)flT);
    R tT = fT - R(jT);
    tT = tT < R(0) ? R(0) : (tT > R(1) ? R(1) : tT);
    const R* b0 = kp.icdf + (size_t)jT * nU + iu;
    const R* b1 = b0 + nU;
    R v00 = __ldg(b0), v10 = __ldg(b0 + 1), v01 = __ldg(b1), v11 = __ldg(b1 + 1);
    R c0 = v00 * (R(1) - tu) + v10 * tu;
    R c1 = v01 * (R(1) - tu) + v11 * tu;
    return c0 * (R(1) - tT) + c1 * tT;
}

// kernels_gpu.jl:653-704 with Philox variates (tag RTA: u_collide, u_sample, g0, g1;
// tag RTADIR: g2).  Returns true when the particle was resampled.
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ bool rta_collide(const KParams<R>& kp, int64_t i, int64_t s, uint32_t pid,
                                            R T, R (&p)[3])
{
    Uni4<R> u = uniforms4<R>(kp.seed_lo, kp.seed_hi, pid, (uint32_t)s, TAG_RTA);
    rec_slot(kp, s, i, 3, u.u[0]);
    rec_slot(kp, s, i, 4, u.u[1]);
    R tn = (kp.DsT > R(0) && T > R(0)) ? eval_spline(T, kp.rta_Tmin, kp.rta_invdT, kp.rta, kp.n_rta) : R(0);
    R Pcol = (tn > R(0) && isfinite(tn)) ? jclamp(kp.dtR / tn, R(0), R(1)) : R(1);
    if (!(u.u[0] < Pcol)) return false;
    R pstar = invcdf_lookup(kp, u.u[1], T);
    R g[3];
    box_muller(u.u[2], u.u[3], g[0], g[1]);
    g[2] = R(0);
    if (PDIM == 3) {
        Uni4<R> w = uniforms4<R>(kp.seed_lo, kp.seed_hi, pid, (uint32_t)s, TAG_RTADIR);
        R z;
        box_muller(w.u[0], w.u[1], g[2], z);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) rec_slot(kp, s, i, 5 + d, g[d]);
    if (DIMS == 1) { p[0] = (g[0] < R(0) ? R(-1) : R(1)) * pstar; return true; }
    R nrm2 = R(0);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) nrm2 += g[d] * g[d];
    R inv = pstar / sqrt(nrm2 > R(1e-300) ? nrm2 : R(1e-300));
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p[d] = g[d] * inv;
    return true;
}

// kernels_cpu.jl:671-735 (momentum_langevin = false or DsT == 0).
template <typename R, int MED, int DIMS>
__device__ __forceinline__ void set_to_fluid(const KParams<R>& kp, const StepU<R>& su, const R (&x)[3], R (&p)[3])
{
    const R m = kp.m;
    const R vmax = sizeof(R) == 8 ? R(0.9999999999995) : R(0.99999994f);
    if (MED == MED_GRID) {
        R T, ux, uy;
        grid_lookup(kp.med, su, x[0], x[1], T, ux, uy);
        R u = sqrt(ux * ux + uy * uy);
        if (u < R(kEps)) { p[0] = R(0); p[1] = R(0); return; }
        R vc = kp.rel ? jclamp(u, -vmax, vmax) : u;
        R g = kp.rel ? R(1) / sqrt(R(1) - vc * vc + R(1e-10)) : R(1);
        p[0] = m * g * vc * (ux / u);
        p[1] = m * g * vc * (uy / u);
        return;
    }
    R r = DIMS == 1 ? x[0] : sqrt(x[0] * x[0] + x[1] * x[1]);
    if (r < R(kEps)) return;
    R v = R(0);
    if (MED == MED_RT) { R Tdummy; rt_lookup(kp.med, su, r, Tdummy, v); }
    if (!kp.rel) {
        if (DIMS == 1) p[0] = m * v;
        else { p[0] = m * v * (x[0] / r); p[1] = m * v * (x[1] / r); }
        return;
    }
    v = jclamp(v, -vmax, vmax);
    R gam = R(1) / sqrt(R(1) - v * v + R(1e-10));
    if (DIMS == 1) p[0] = m * gam * v;
    else { p[0] = m * gam * v * (x[0] / r); p[1] = m * gam * v * (x[1] / r); }
}

// Temperature at an arbitrary point of this step (diffusion, freeze-out).
template <typename R, int MED, int DIMS>
__device__ __forceinline__ R temperature_at(const KParams<R>& kp, const StepU<R>& su, const R (&x)[3], R r)
{
    R T;
    if (MED == MED_RT) { R V; rt_lookup(kp.med, su, r, T, V); }
    else if (MED == MED_BJORKEN) T = su.T_bj;
    else { R ux, uy; grid_lookup(kp.med, su, x[0], x[1], T, ux, uy); }
    if (kp.med.T_scale != R(1)) T *= kp.med.T_scale;
    return T;
}

// Compensated accumulation x += dx (FP32 keeps a float low word per component).
template <typename R>
__device__ __forceinline__ void acc_add(R& hi, float& lo, R dx)
{
    if (sizeof(R) == 8) { hi += dx; return; }
    float s = (float)hi + (float)dx;          // TwoSum (Knuth)
    float bp = s - (float)hi;
    float err = ((float)hi - (s - bp)) + ((float)dx - bp);
    lo += err;
    float h2 = s + lo;                        // renormalise
    lo = lo - (h2 - s);
    hi = (R)h2;
}

// kernels_cpu.jl:510-637
template <typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void stream_positions(const KParams<R>& kp, const StepU<R>& su, int64_t i, int64_t s,
                                                 uint32_t pid, R (&x)[3], float (&xl)[3], R (&p)[3])
{
    const R m = kp.m, dt = kp.dtR;
    R E2 = m * m;
#pragma unroll
    for (int d = 0; d < PDIM; ++d) E2 += p[d] * p[d];
    R E = kp.rel ? sqrt(E2) : m;
    const R r_max = kp.med.r_max, r_axis_eps = kp.med.r_axis_eps;
    if (DIMS == 1) {
        R r = x[0], pr = p[0];
        R r_abs = fabs(r);
        R r_safe = r_abs < r_axis_eps ? r_axis_eps : r_abs;
        R dr = (pr / E) * dt;
        if (kp.diffusion) {
            R xs[3] = { r_safe, R(0), R(0) };
            R T = temperature_at<R, MED, DIMS>(kp, su, xs, r_safe);
            R D = (kp.DsT / (T != T ? T : (T > R(kEps) ? T : R(kEps)))) / R(kFmGeV);
            if (D > R(0)) {
                Uni4<R> u = uniforms4<R>(kp.seed_lo, kp.seed_hi, pid, (uint32_t)s, TAG_DIFF);
                R z0, z1;
                box_muller(u.u[0], u.u[1], z0, z1);
                rec_slot(kp, s, i, 8, z0);
                dr += (D / r_safe) * dt + sqrt(R(2) * D * dt) * z0;
            }
        }
        R r_new = r + dr;
        if (r_new < R(0)) { r_new = -r_new; p[0] = -p[0]; }
        if (kp.reflect && r_max > R(0) && r_new > r_max) {
            r_new = R(2) * r_max - r_new;
            p[0] = -p[0];
            if (r_new < R(0)) { r_new = -r_new; p[0] = -p[0]; }
        }
        x[0] = r_new;
        return;
    }
    R invE = R(1) / E;
#pragma unroll
    for (int d = 0; d < DIMS; ++d) {
        R dx = sizeof(R) == 8 ? dt * p[d] / E : (dt * p[d]) * invE;
        acc_add(x[d], xl[d], dx);
    }
    if (kp.diffusion) {
        R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        R T = temperature_at<R, MED, DIMS>(kp, su, x, sqrt(r2));
        R D = (kp.DsT / (T != T ? T : (T > R(kEps) ? T : R(kEps)))) / R(kFmGeV);
        if (D > R(0)) {
            R sg = sqrt(R(2) * D * dt);
            Uni4<R> u = uniforms4<R>(kp.seed_lo, kp.seed_hi, pid, (uint32_t)s, TAG_DIFF);
            R z[4];
            box_muller(u.u[0], u.u[1], z[0], z[1]);
            box_muller(u.u[2], u.u[3], z[2], z[3]);
#pragma unroll
            for (int d = 0; d < DIMS; ++d) { rec_slot(kp, s, i, 8 + d, z[d]); acc_add(x[d], xl[d], sg * z[d]); }
        }
    }
    if (kp.reflect && r_max > R(0)) {
        R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        R r_now = sqrt(r2);
        if (r_now > r_max) {
            R invr = R(1) / (r_now > r_axis_eps ? r_now : r_axis_eps);
            R ppar = R(0);
#pragma unroll
            for (int d = 0; d < DIMS; ++d) ppar += p[d] * (x[d] * invr);
#pragma unroll
            for (int d = 0; d < DIMS; ++d) p[d] -= R(2) * ppar * (x[d] * invr);
            R scale = (R(2) * r_max - r_now) * invr;
#pragma unroll
            for (int d = 0; d < DIMS; ++d) { x[d] = (R)((double)x[d] + (double)xl[d]) * scale; xl[d] = 0.f; }
        }
    }
}

// Momentum noise: 4 normals from one uniform group (the first PDIM are used).
template <typename R, int PDIM>
__device__ __forceinline__ void momentum_noise(const KParams<R>& kp, int64_t i, int64_t s, uint32_t pid, R (&xi)[3])
{
    Uni4<R> u = uniforms4<R>(kp.seed_lo, kp.seed_hi, pid, (uint32_t)s, TAG_MOM);
    R z1;
    box_muller(u.u[0], u.u[1], xi[0], xi[1]);
    if (PDIM == 3) box_muller(u.u[2], u.u[3], xi[2], z1);
    else xi[2] = R(0);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) rec_slot(kp, s, i, d, xi[d]);
}

// One Cartesian step (simulate_cpu.jl:215-290).
template <typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void cart_step(const KParams<R>& kp, const StepU<R>& su, int64_t i, int64_t s,
                                          uint32_t pid, R (&x)[3], float (&xl)[3], R (&p)[3])
{
    Local<R> L = local_medium<R, MED, DIMS>(kp, su, x);
    boost<R, DIMS, PDIM>(kp, L, p, false);
    if (PDIM == 3 && kp.redshift) {
        double ta = kp.t0 + (double)(s - 1) * kp.dt;
        if (ta > 0.0) p[2] *= (R)(ta / (ta + kp.dt));
    }
    if (kp.collision == COLL_FLUID) {
        set_to_fluid<R, MED, DIMS>(kp, su, x, p);
    } else {
        R T = jmax0(L.T);
        if (kp.collision != COLL_RTA) {
            R xi[3];
            momentum_noise<R, PDIM>(kp, i, s, pid, xi);
            langevin_kick<R, DIMS, PDIM>(kp, T, p, xi);
        }
        if (kp.collision == COLL_RTA || kp.collision == COLL_LANGEVIN_RTA)
            rta_collide<R, DIMS, PDIM>(kp, i, s, pid, T, p);
        boost<R, DIMS, PDIM>(kp, L, p, true);
    }
    stream_positions<R, MED, DIMS, PDIM>(kp, su, i, s, pid, x, xl, p);
}

// Freeze-out latch after streaming (kernels_gpu.jl:588-635).
template <typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void freezeout_latch(const KParams<R>& kp, const StepU<R>& su, int64_t i,
                                                const R (&x)[3], const R (&p)[3],
                                                R& flag, R (&lpos)[3], R (&lmom)[3], R& ltau, R& lT)
{
    if (flag != R(0)) return;
    R r;
    if (DIMS == 1) r = fabs(x[0]);
    else { R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        r = sqrt(r2); }
    R T = temperature_at<R, MED, DIMS>(kp, su, x, r);
    R tau = su.tR;
    if (sizeof(R) == 4) tau = (R)su.t;
    if (T < kp.Tfo) {
        R frac = (kp.fo_interp && lT > kp.Tfo && lT > T) ? (lT - kp.Tfo) / (lT - T) : R(1);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) kp.fo_pos[d][i] = lpos[d] + frac * (x[d] - lpos[d]);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) kp.fo_mom[d][i] = lmom[d] + frac * (p[d] - lmom[d]);
        kp.fo_tau[i] = (R)((double)ltau + (double)frac * (su.t - (double)ltau));
        kp.fo_flag[i] = R(1);
        flag = R(1);
    } else {
#pragma unroll
        for (int d = 0; d < DIMS; ++d) lpos[d] = x[d];
#pragma unroll
        for (int d = 0; d < PDIM; ++d) lmom[d] = p[d];
        ltau = (R)su.t;
        lT = T;
    }
}

// ---------------------------------------------------------------------------
// Milne (tau, r) step (simulate_cpu_general_coords.jl:83-126).  The Milne
// interpolation neither clamps the query nor guards dx (kernels_cpu_GC.jl:37-57).
// ---------------------------------------------------------------------------
template <typename R>
struct StepMilne { double t; int kt; R wt; };

template <typename R>
__device__ __forceinline__ StepMilne<R> milne_uniforms(const KParams<R>& kp, int64_t s)
{
    StepMilne<R> u;
    u.t = __dadd_rn(__dmul_rn((double)s, kp.dt), kp.t0);
    const double* tg = kp.med.tgd;
    const int nt = kp.med.nt;
    int lo = -1, hi = nt;
    while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (__ldg(tg + mid) <= u.t) lo = mid; else hi = mid; }
    int k = lo < 0 ? 0 : lo;
    k = k > nt - 2 ? nt - 2 : k;
    double y0 = __ldg(tg + k), y1 = __ldg(tg + k + 1);
    u.kt = k;
    u.wt = (R)((u.t - y0) / (y1 - y0));
    return u;
}

template <typename R>
__device__ __forceinline__ void milne_lookup(const MediumDev<R>& md, const StepMilne<R>& su, R r, R& T, R& V)
{
    int i = cell_index(md.xg, md.nr, r, md.x_uniform, md.xg0, md.xinvd);
    R x0 = __ldg(md.xg + i), x1 = __ldg(md.xg + i + 1);
    R xd = (r - x0) / (x1 - x0);
    const int nr = md.nr, j = su.kt;
    auto a00 = md.TV[i + nr * j],       a10 = md.TV[i + 1 + nr * j];
    auto a01 = md.TV[i + nr * (j + 1)], a11 = md.TV[i + 1 + nr * (j + 1)];
    R yd = su.wt;
    R c0 = a00.x * (R(1) - xd) + a10.x * xd;
    R c1 = a01.x * (R(1) - xd) + a11.x * xd;
    T = c0 * (R(1) - yd) + c1 * yd;
    c0 = a00.y * (R(1) - xd) + a10.y * xd;
    c1 = a01.y * (R(1) - xd) + a11.y * xd;
    V = c0 * (R(1) - yd) + c1 * yd;
}

template <typename R>
__device__ __forceinline__ void milne_step(const KParams<R>& kp, const StepMilne<R>& su, int64_t i, int64_t s,
                                           uint32_t pid, R (&x)[3], float (&xl)[3], R (&p)[3])
{
    const R m = kp.m, dt = kp.dtR;
    R T, v;
    milne_lookup(kp.med, su, fabs(x[1]), T, v);       // same (r, t) for rest boost, forces, lab boost
    if (kp.med.T_scale != R(1)) T *= kp.med.T_scale;
    // kernels_cpu_GC.jl:64-82
    R g = R(1) / sqrt(R(1) - v * v + R(1e-10));
    R pt = p[0], pr = p[1];
    p[0] = g * (pt - v * pr);
    p[1] = g * (pr - v * pt);
    // kernels_cpu_GC.jl:110-174 (Christoffel term identically zero) + :244-256
    const R DsT_safe = kp.DsT <= R(0) ? R(0) : kp.DsT;
    R tn = DsT_safe == R(0) ? R(0) : eval_spline(T, kp.drag_Tmin, kp.drag_invdT, kp.drag, kp.n_drag);
    const bool ok = tn > R(0) && isfinite(tn);
    R etaD = ok ? R(1) / tn : R(0);
    R kappa = ok ? (R(2) * m * T) / tn : R(0);
    R kT = sqrt(kappa);
    Uni4<R> u = uniforms4<R>(kp.seed_lo, kp.seed_hi, pid, (uint32_t)s, TAG_MOM);
    R xi, z1;
    box_muller(u.u[0], u.u[1], xi, z1);
    rec_slot(kp, s, i, 0, xi);
    R det, sto;
    if (etaD > R(0) && dt > R(0)) {
        R a = exp(-etaD * dt);
        R np = kT * sqrt((R(1) - a * a) / (R(2) * etaD * dt));
        det = (a - R(1)) * p[1];
        sto = np * xi;
    } else {
        det = R(0);
        sto = kT * xi;
    }
    p[1] += det + kp.sqrt_dt * sto;
    p[0] = sqrt(m * m + p[1] * p[1]);
    // kernels_cpu_GC.jl:85-102
    g = R(1) / sqrt(R(1) - v * v + R(1e-8));
    pt = p[0]; pr = p[1];
    p[0] = g * (pt + v * pr);
    p[1] = g * (pr + v * pt);
    // kernels_cpu_GC.jl:259-274
    R E = p[0];
    acc_add(x[0], xl[0], sizeof(R) == 8 ? dt * p[0] / E : dt);
    acc_add(x[1], xl[1], dt * p[1] / E);
}

}  // namespace lim

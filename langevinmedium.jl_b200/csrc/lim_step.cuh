// lim_step.cuh — one Langevin step of one particle, register-resident.
//
// The sequence is the reference's (simulate_cpu.jl:215-303):
//   noise -> rest-frame boost -> [Bjorken redshift] -> {fluid | OU kick | RTA
//   | OU kick + RTA} -> lab boost -> streaming (+diffusion, reflection)
// fused into one device function so that the state never leaves registers.
// Medium time at step s is s*dt + t0 (kernels_cpu.jl:67).
//
// Variates per step (counter-based Philox, see lim_common.cuh), slot numbers as
// recorded by the noise-recording mode:
//   group MOM  u0..u3: momentum normals (u0,u1) -> Box-Muller (xi0,xi1),
//                      xi2 = Phi^-1(u2); RTA decision u_collide = u3 when pdim = 3,
//                      u2 when pdim < 3, u0 in pure RTA mode           [slots 0-3]
//   group RTA  (drawn only when a collision happens): u_sample = u0,
//                      (u1,u2) -> directions g0, g1, g2 = Phi^-1(u3)   [slots 4-7]
//   group DIFF position-diffusion normals                              [slots 8-10]
#pragma once
#include <type_traits>
#include "lim_common.cuh"

namespace lim {

// ---------------------------------------------------------------------------
// Per-step record, identical for every particle: computed once per launch by
// k_step_table and read by every thread with one broadcast load.
// ---------------------------------------------------------------------------
template <typename R>
struct __align__(16) StepRec {
    double t;    // medium time s*dt + t0
    double zf;   // Bjorken redshift factor tau_a/(tau_a+dt), 1 when not applied (FP64:
                 // the product over steps telescopes to tau_0/tau exactly)
    double wtd;  // time weight in FP64
    double Td;   // Bjorken temperature in FP64
    R tR;        // the medium time in R
    R wt;        // time weight of the (r,t) table, the grid or the Milne table
    R T_bj;      // Bjorken temperature at t
    int kt;      // time cell
};

enum { MED_MILNE_TABLE = 3 };   // Milne (tau, r): unclamped time interpolation

// t0 + s dt, rounded in this order wherever a step's time is needed
template <typename R>
__device__ __forceinline__ double step_time(const KParams<R>& kp, int64_t s)
{
    return __dadd_rn(__dmul_rn((double)s, kp.dt), kp.t0);
}

// The 2+1D grid's time cell of time t (clamped to the grid): the row kt and the weight.
template <typename R>
__device__ __forceinline__ int grid_time_cell(const MediumDev<R>& md, double t, double& w)
{
    const double tq = t > md.gtl ? md.gtl : (t < md.gt0 ? md.gt0 : t);
    const double f = (tq - md.gt0) / md.gdt_d;
    const double fl = floor(f);
    const int it = fl < 0.0 ? 0 : (fl > (double)(md.gnt - 2) ? md.gnt - 2 : (int)fl);
    w = f - (double)it;
    return it;
}

template <typename R, int MED>
__device__ __forceinline__ StepRec<R> make_step_rec(const KParams<R>& kp, int64_t s)
{
    StepRec<R> u;
    u.t = step_time(kp, s);
    u.tR = (R)u.t;
    u.kt = 0; u.wt = R(0); u.T_bj = R(0); u.zf = 1.0; u.wtd = 0.0; u.Td = 0.0;
    const MediumDev<R>& md = kp.med;
    if (MED == MED_RT || MED == MED_MILNE_TABLE) {
        const double* tg = md.tgd;
        const int nt = md.nt;
        const bool clamp = MED == MED_RT;
        double tq = u.t;
        if (clamp) tq = tq > tg[nt - 1] ? tg[nt - 1] : (tq < tg[0] ? tg[0] : tq);
        int lo = -1, hi = nt;          // last node <= tq (searchsortedlast)
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (tg[mid] <= tq) lo = mid; else hi = mid; }
        int k = lo < 0 ? 0 : lo;
        k = k > nt - 2 ? nt - 2 : k;
        double y0 = tg[k], y1 = tg[k + 1], dy = y1 - y0;
        u.kt = k;
        if (clamp) u.wtd = fabs(dy) < kEps ? 0.0 : (tq - y0) / dy;      // kernels_cpu.jl:45
        else u.wtd = (tq - y0) / dy;                                     // kernels_cpu_GC.jl:51
        u.wt = (R)u.wtd;
    } else if (MED == MED_BJORKEN) {
        double T = (u.t > md.bj_tau0) ? md.bj_T0 * pow(md.bj_tau0 / u.t, md.bj_power) : md.bj_T0;
        u.T_bj = (R)T;
        u.Td = T;
    } else {
        u.kt = grid_time_cell(md, u.t, u.wtd);
        u.wt = (R)u.wtd;
    }
    if (kp.redshift) {                 // kernels_cpu.jl:427-435
        double ta = kp.t0 + (double)(s - 1) * kp.dt;
        if (ta > 0.0) u.zf = ta / (ta + kp.dt);
    }
    return u;
}

// ---------------------------------------------------------------------------
// medium lookups
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 ldg_cell(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ldg_cell(const double4* p)
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// (r, t) table: bilinear interpolation of (T, V) at radius r (clamped).  The cell is
// searchsortedlast(x, r) capped to [0, nr-2] (kernels_cpu.jl:22-51): on a near-uniform
// grid a first guess corrected against the cell's own nodes (one load of xc), else a
// binary search; the values come from the two per-cell records of time rows kt, kt+1.
template <typename R>
__device__ __forceinline__ void rt_lookup(const MediumDev<R>& md, const StepRec<R>& sr, R r, R& T, R& V)
{
    const R rq = jclamp(r, md.xlo, md.xhi);
    const int nc = md.nr - 1;
    int i;
    if (md.x_uniform) {
        const R f = (rq - md.xg0) * md.xinvd;
        i = f > R(0) ? (int)f : 0;
        i = i > nc - 1 ? nc - 1 : i;
    } else {
        i = cell_index(md.xg, md.nr, rq, 0, md.xg0, md.xinvd);
    }
    auto xn = __ldg(md.xc + i);
    while (i < nc - 1 && xn.y <= rq) xn = __ldg(md.xc + ++i);
    while (i > 0 && xn.x > rq) xn = __ldg(md.xc + --i);
    const R dx = xn.y - xn.x;
    const R xd = fabs(dx) < R(kEps) ? R(0) : (rq - xn.x) / dx;
    const int j = sr.kt;
    const auto c0 = ldg_cell(md.TVc + i + nc * j), c1 = ldg_cell(md.TVc + i + nc * (j + 1));
    const R yd = sr.wt;
    R a = c0.x * (R(1) - xd) + c0.z * xd;
    R b = c1.x * (R(1) - xd) + c1.z * xd;
    T = a * (R(1) - yd) + b * yd;
    a = c0.y * (R(1) - xd) + c0.w * xd;
    b = c1.y * (R(1) - xd) + c1.w * xd;
    V = a * (R(1) - yd) + b * yd;
}

template <typename R>
__device__ __forceinline__ R rt_lookup_scalar(const MediumDev<R>& md, const StepRec<R>& sr, const R* __restrict__ vals, R r)
{
    R rq = jclamp(r, __ldg(md.xg), __ldg(md.xg + md.nr - 1));
    int i = cell_index(md.xg, md.nr, rq, md.x_uniform, md.xg0, md.xinvd);
    R x0 = __ldg(md.xg + i), x1 = __ldg(md.xg + i + 1);
    R dx = x1 - x0;
    R xd = fabs(dx) < R(kEps) ? R(0) : (rq - x0) / dx;
    const int nr = md.nr, j = sr.kt;
    R v00 = __ldg(vals + i + nr * j), v10 = __ldg(vals + i + 1 + nr * j);
    R v01 = __ldg(vals + i + nr * (j + 1)), v11 = __ldg(vals + i + 1 + nr * (j + 1));
    R yd = sr.wt;
    R c0 = v00 * (R(1) - xd) + v10 * xd;
    R c1 = v01 * (R(1) - xd) + v11 * xd;
    return c0 * (R(1) - yd) + c1 * yd;
}

// FP32 cell index i and weight w of the clamped coordinate q (low word ql) on a uniform
// axis of n nodes: the coordinate is taken relative to the node ic nearest the axis's
// centre (xc + xcl as a float pair) and scaled by 1/dx (inv + ilo), keeping the
// rounding of both steps (TwoSum of q - xc, the exact FMA remainder of the product), so
// the weight is the cell fraction rounded once.  Measured from the far origin instead,
// (q - x0) / dx rounds at the ulp of ~100 cells: a weight error of up to 1e-5, which the
// momentum of a slow heavy quark in a flowing cell follows (FP32 against FP64 per
// particle 1.1e-5 before, 3.6e-6 after, on the 201 x 201 grid of 0.1 fm).
__device__ __forceinline__ void cell_fp32(float q, float ql, int ic, float xc, float xcl, float inv, float ilo,
                                          int n, int& i, float& w)
{
    const float s = __fsub_rn(q, xc);
    const float bp = __fsub_rn(s, q);
    const float err = __fadd_rn(__fsub_rn(q, __fsub_rn(s, bp)), __fsub_rn(-xc, bp));
    const float dlo = __fadd_rn(__fsub_rn(err, xcl), ql);
    const float pr = __fmul_rn(s, inv);
    const float e = __fmaf_rn(s, inv, -pr);
    const float lo = __fadd_rn(e, __fmaf_rn(s, ilo, __fmul_rn(dlo, inv)));
    // floor(pr) from one round-down add: for |pr| < 2^22 the low mantissa bits of
    // pr + 1.5 2^23 rounded down hold floor(pr) (NaN gives a large index, clamped below)
    const float tf = __fadd_rd(pr, 12582912.0f);
    const float fl = __fsub_rn(tf, 12582912.0f);
    int k = ic + (__float_as_int(tf) - 0x4B400000);
    float base = fl;
    if (k < 0) { k = 0; base = (float)(-ic); }
    if (k > n - 2) { k = n - 2; base = (float)(n - 2 - ic); }
    i = k;
    w = __fadd_rn(__fsub_rn(pr, base), lo);
}

// 2+1D grid: trilinear of (T, ux, uy) at (x, y) clamped to the grid.  The FP32 path
// finds the cell with cell_fp32 (xlo, ylo: the position's low words, dropped where the
// query is clamped); the FP64 path in FP64 from the same nodes.
template <typename R>
__device__ __forceinline__ void grid_cell(const MediumDev<R>& md, R xq, R yq, int& ix, int& iy, R& wx, R& wy,
                                          float xlo = 0.0f, float ylo = 0.0f)
{
    if constexpr (sizeof(R) == 4) {
        // the query clamped to the grid through its cell: off the grid the cell index is
        // clamped to the edge cell and the weight to 0 or 1, the edge node's value exactly
        // (inside the grid nothing is clamped)
        float fwx, fwy;
        cell_fp32(xq, xlo, md.gicx, md.gxc, md.gxcl, md.ginvdx, md.ginvdx_lo, md.gnx, ix, fwx);
        cell_fp32(yq, ylo, md.gicy, md.gyc, md.gycl, md.ginvdy, md.ginvdy_lo, md.gny, iy, fwy);
        wx = fminf(fmaxf(fwx, 0.0f), 1.0f);
        wy = fminf(fmaxf(fwy, 0.0f), 1.0f);
    } else {
        R x = xq > (R)md.gxl_d ? (R)md.gxl_d : (xq < (R)md.gx0_d ? (R)md.gx0_d : xq);
        R y = yq > (R)md.gyl_d ? (R)md.gyl_d : (yq < (R)md.gy0_d ? (R)md.gy0_d : yq);
        R fx = (x - (R)md.gx0_d) / (R)md.gdx_d, fy = (y - (R)md.gy0_d) / (R)md.gdy_d;
        R flx = floor(fx), fly = floor(fy);
        ix = flx < R(0) ? 0 : (flx > R(md.gnx - 2) ? md.gnx - 2 : (int)flx);
        iy = fly < R(0) ? 0 : (fly > R(md.gny - 2) ? md.gny - 2 : (int)fly);
        wx = fx - R(ix);
        wy = fy - R(iy);
    }
}

// Products and fused multiply-adds with their rounding spelled out, for expressions
// with two products (a b + c d), where the compiler's contraction may otherwise pick a
// different product to fuse in different instantiations of the same step.
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Linear interpolation with the rounding spelled out, so the compiler may not contract
// it differently where it is inlined and the grid's interpolation gives the same bits in
// every kernel and at every call site.  FP32: a + w (b - a) as one subtraction and one
// fused multiply-add (b - a is exact for neighbouring nodes within a factor 2 of each
// other, so the result is rounded once); FP64: the reference's a (1 - w) + b w.
__device__ __forceinline__ float lerp_rn(float a, float b, float w)
{
    return __fmaf_rn(w, __fsub_rn(b, a), a);
}
__device__ __forceinline__ double lerp_rn(double a, double b, double w)
{
    return __fma_rn(b, w, __dmul_rn(a, __dsub_rn(1.0, w)));
}
template <typename R>
__device__ __forceinline__ R bilerp_rn(float a00, float a10, float a01, float a11, R wx, R wy)
{
    return lerp_rn(lerp_rn((R)a00, (R)a10, wx), lerp_rn((R)a01, (R)a11, wx), wy);
}

// The grid at a position, interpolated in space only: (T, v^x, v^y) on time rows kt
// (T0, U0, V0) and kt + 1 (T1, U1, V1), the two values grid_lookup blends in time.  The
// FP32 freeze-out kernel looks them up once per step, at the end of step s at the new
// position on the time row of step s + 1, and carries the result into step s + 1
// (cart_particle): blended in time at once, T0, U0, V0 then hold the medium of step
// s + 1 and T1 the latch's temperature screen of step s (-1 where the two steps do not
// share the time row: the FP64 test decides), so four values stay live across the step.
template <typename R>
struct GridRows {
    R T0, T1, U0, U1, V0, V1;
    int kt;
};

// The 2 x 2 x 2 grid nodes around (xq, yq) on time rows kt (a) and kt + 1 (b), in the
// order 00, 10, 01, 11 (x fastest), and the cell weights.
template <typename R>
__device__ __forceinline__ void grid_corners(const MediumDev<R>& md, int kt, R xq, R yq, float4 (&a)[4],
                                             float4 (&b)[4], R& Wx, R& Wy, float xlo = 0.0f, float ylo = 0.0f)
{
    int ix, iy;
    grid_cell(md, xq, yq, ix, iy, Wx, Wy, xlo, ylo);
    const float4* s0 = md.G + ((size_t)kt * md.gny + iy) * md.gnx + ix;
    const float4* s1 = s0 + (size_t)md.gny * md.gnx;
    a[0] = __ldg(s0); a[1] = __ldg(s0 + 1); a[2] = __ldg(s0 + md.gnx); a[3] = __ldg(s0 + md.gnx + 1);
    b[0] = __ldg(s1); b[1] = __ldg(s1 + 1); b[2] = __ldg(s1 + md.gnx); b[3] = __ldg(s1 + md.gnx + 1);
}

template <typename R>
__device__ __forceinline__ void rows_of(const float4 (&a)[4], const float4 (&b)[4], R Wx, R Wy, GridRows<R>& g)
{
    g.T0 = bilerp_rn(a[0].x, a[1].x, a[2].x, a[3].x, Wx, Wy); g.T1 = bilerp_rn(b[0].x, b[1].x, b[2].x, b[3].x, Wx, Wy);
    g.U0 = bilerp_rn(a[0].y, a[1].y, a[2].y, a[3].y, Wx, Wy); g.U1 = bilerp_rn(b[0].y, b[1].y, b[2].y, b[3].y, Wx, Wy);
    g.V0 = bilerp_rn(a[0].z, a[1].z, a[2].z, a[3].z, Wx, Wy); g.V1 = bilerp_rn(b[0].z, b[1].z, b[2].z, b[3].z, Wx, Wy);
}

template <typename R>
__device__ __forceinline__ void grid_rows(const MediumDev<R>& md, int kt, R xq, R yq, GridRows<R>& g,
                                          float xlo = 0.0f, float ylo = 0.0f)
{
    float4 a[4], b[4];
    R Wx, Wy;
    grid_corners(md, kt, xq, yq, a, b, Wx, Wy, xlo, ylo);
    rows_of(a, b, Wx, Wy, g);
    g.kt = kt;
}

// (T, v^x, v^y) at time weight Wt between the rows
template <typename R>
__device__ __forceinline__ void grid_combine(const GridRows<R>& g, R Wt, R& T, R& ux, R& uy)
{
    T = lerp_rn(g.T0, g.T1, Wt);
    ux = lerp_rn(g.U0, g.U1, Wt);
    uy = lerp_rn(g.V0, g.V1, Wt);
}

// The grid medium at the particle with its gradient in (x, y) (zero along an axis where
// the query is clamped to the grid), for the adjoint's tape.
struct MedGrad {
    float T, vx, vy, dT[2], dvx[2], dvy[2];
};

template <typename R, bool GRAD = false>
__device__ __forceinline__ void grid_lookup(const MediumDev<R>& md, const StepRec<R>& sr, R xq, R yq, R& T, R& ux, R& uy,
                                            MedGrad* mg = nullptr, float xlo = 0.0f, float ylo = 0.0f)
{
    float4 a[4], b[4];
    R Wx, Wy;
    grid_corners(md, sr.kt, xq, yq, a, b, Wx, Wy, xlo, ylo);
    const R Wt = sr.wt;
    GridRows<R> g;
    rows_of(a, b, Wx, Wy, g);
    grid_combine(g, Wt, T, ux, uy);
    if constexpr (GRAD) {
        const float4 &a00 = a[0], &a10 = a[1], &a01 = a[2], &a11 = a[3];
        const float4 &b00 = b[0], &b10 = b[1], &b01 = b[2], &b11 = b[3];
        const float wx = (float)Wx, wy = (float)Wy, wt = (float)Wt;
        const float kx = (xq > (R)md.gx0_d && xq < (R)md.gxl_d) ? md.ginvdx : 0.0f;
        const float ky = (yq > (R)md.gy0_d && yq < (R)md.gyl_d) ? md.ginvdy : 0.0f;
        // d/dx: x-differences bilinear in (y, t); d/dy: y-differences bilinear in (x, t)
        auto grad = [&](float A00, float A10, float A01, float A11, float B00, float B10, float B01, float B11,
                        float (&g)[2]) {
            const float xa = (A10 - A00) + wy * ((A11 - A01) - (A10 - A00));
            const float xb = (B10 - B00) + wy * ((B11 - B01) - (B10 - B00));
            const float ya = (A01 - A00) + wx * ((A11 - A10) - (A01 - A00));
            const float yb = (B01 - B00) + wx * ((B11 - B10) - (B01 - B00));
            g[0] = (xa + wt * (xb - xa)) * kx;
            g[1] = (ya + wt * (yb - ya)) * ky;
        };
        grad(a00.x, a10.x, a01.x, a11.x, b00.x, b10.x, b01.x, b11.x, mg->dT);
        grad(a00.y, a10.y, a01.y, a11.y, b00.y, b10.y, b01.y, b11.y, mg->dvx);
        grad(a00.z, a10.z, a01.z, a11.z, b00.z, b10.z, b01.z, b11.z, mg->dvy);
        mg->T = (float)T;
        mg->vx = (float)ux;
        mg->vy = (float)uy;
    }
}

// Flow seen by one particle this step: boost direction (nx, ny), signed speed v,
// the local temperature T at the same point, and whether the frame changes.
template <typename R>
struct Local {
    R T, v, nx, ny;
    bool boost;   // false: r < eps (kernels_cpu.jl:75-77), or FP32 with zero flow
};

template <typename R, int MED, int DIMS, bool GRAD = false>
__device__ __forceinline__ Local<R> local_medium(const KParams<R>& kp, const StepRec<R>& sr, const R (&x)[3],
                                                 MedGrad* mg = nullptr, GridRows<R>* carry = nullptr,
                                                 const float* xl = nullptr)
{
    constexpr bool fp32 = sizeof(R) == 4;
    Local<R> L;
    L.nx = R(0); L.ny = R(0); L.v = R(0);
    if (MED == MED_GRID) {
        // the grid holds the flow velocity (v^x, v^y), as the reference's (r, t) tables do
        R ux, uy;
        if (!GRAD && carry) {                 // looked up and blended at the end of the previous step
            L.T = carry->T0; ux = carry->U0; uy = carry->V0;
        } else {
            grid_lookup<R, GRAD>(kp.med, sr, x[0], x[1], L.T, ux, uy, mg, xl ? xl[0] : 0.0f, xl ? xl[1] : 0.0f);
        }
        R u = sqrt(fma_rn(ux, ux, mul_rn(uy, uy)));
        L.boost = !(u < R(kEps));
        L.v = u;
        if (L.boost) { L.nx = ux / u; L.ny = uy / u; }
    } else if (MED == MED_BJORKEN && fp32) {
        // zero flow: in FP32 the boost is the identity (gamma(0) rounds to 1)
        L.T = sr.T_bj;
        L.boost = false;
    } else {
        R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        R r = sqrt(r2);
        L.boost = !(r < R(kEps));
        if (MED == MED_RT) {
            rt_lookup(kp.med, sr, r, L.T, L.v);
            if (DIMS >= 2 && kp.med.use_v2 && L.boost) {
                R v2m = rt_lookup_scalar(kp.med, sr, kp.med.V2, r);
                R phi = atan2(x[1], x[0]);
                L.v *= (R(1) + R(2) * v2m * cos(R(2) * (phi - kp.psi2)));
            }
        } else {
            L.T = sr.T_bj;
        }
        // FP64 keeps the reference's gamma(0) = 1/sqrt(1+1e-10) factor at zero flow;
        // in FP32 that factor is 1 and the boost is skipped.
        if (fp32 && L.v == R(0)) L.boost = false;
        if (DIMS >= 2 && L.boost) { L.nx = x[0] / r; L.ny = x[1] / r; }
    }
    if (kp.med.T_scale != R(1)) L.T *= kp.med.T_scale;
    return L;
}

// 1/sqrt(s) and sqrt(s) for s > 0 in the FP32 kernels' FP64 frame change: the FP32
// hardware estimate refined by one Newton step in FP64 (relative error below 1e-13, far
// inside FP32 resolution; the FP64 kernels keep the correctly rounded forms for FP64
// parity).  Each is one FP32 estimate and three FP64 operations in place of a
// correctly rounded FP64 square root and division.
__device__ __forceinline__ double rsqrt_f32_newton(double s)
{
    const double r = (double)rsqrtf((float)s);
    const double h = 0.5 * fma(-s * r, r, 1.0);
    return fma(r, h, r);
}
__device__ __forceinline__ double sqrt_f32_newton(double s)
{
    const float sf = (float)s;
    if (!(sf > 0.0f && sf < 3.0e38f)) return sqrt(s);       // 0, FP32 overflow, NaN: the plain form
    const float r0 = rsqrtf(sf);
    const double e0 = (double)(sf * r0);
    return fma(0.5 * (double)r0, fma(-e0, e0, s), e0);
}

// kernels_cpu.jl:89-145 (to_lab = false) and :188-241 (to_lab = true).  The frame
// change is evaluated in FP64 in both precisions: with the momentum held in FP64,
// p_par - v E does not lose the LRF momentum to cancellation at large gamma, and no
// FP32 rounding of the momentum enters the state.  (The FP32 freeze-out kernel on the
// grid changes frames in FP32 below gamma = 2 instead, as an increment of the FP64
// state: step_rest_frame_incr.)  gamma = 1/sqrt(1 - v^2 + 1e-10) of the clamped local
// speed (kernels_cpu.jl:100-104), computed once per step for both frame changes.
template <typename R>
__device__ __forceinline__ double boost_gamma(const Local<R>& L)
{
    const double vmax = 0.9999999999995;   // sqrt(1 - 1e-12)
    const double v = jclamp((double)L.v, -vmax, vmax);
    if constexpr (sizeof(R) == 4) return rsqrt_f32_newton(1.0 - v * v + 1e-10);
    return 1.0 / sqrt(1.0 - v * v + 1e-10);
}

// gamp: boost_gamma(L) when the caller has it, else (<= 0) computed here.
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ void boost(const KParams<R>& kp, const Local<R>& L, double (&p)[3], bool to_lab,
                                      double gamp = -1.0)
{
    const double m = (double)kp.m;
    double v = (double)L.v;
    const double nx = (double)L.nx, ny = (double)L.ny;
    if (!kp.rel) {                     // Galilean p_par -/+ m v
        double mv = m * v;
        if (DIMS == 1) { p[0] = to_lab ? p[0] + mv : p[0] - mv; }
        else {
            double dx = mv * nx, dy = mv * ny;
            p[0] = to_lab ? p[0] + dx : p[0] - dx;
            p[1] = to_lab ? p[1] + dy : p[1] - dy;
        }
        return;
    }
    const double vmax = 0.9999999999995;   // sqrt(1 - 1e-12)
    v = jclamp(v, -vmax, vmax);
    double gam = gamp;
    if (!(gam > 0.0)) gam = sizeof(R) == 4 ? rsqrt_f32_newton(1.0 - v * v + 1e-10) : 1.0 / sqrt(1.0 - v * v + 1e-10);
    if constexpr (sizeof(R) == 4) {
        if (DIMS >= 2) {
            // p' = p + d n with d = p'_par - p_par = (gamma - 1) p_par +- gamma v E: the same
            // frame change as the reference's split into parallel and perpendicular parts,
            // in fewer FP64 operations (FP32 path only; the FP64 path keeps the reference's form)
            double q = m * m;
#pragma unroll
            for (int d = PDIM - 1; d >= 0; --d) q = fma(p[d], p[d], q);
            const double E = sqrt_f32_newton(q);
            const double ppar = fma(p[0], nx, p[1] * ny);
            const double gvE = (gam * v) * E;
            const double dd = fma(gam - 1.0, ppar, to_lab ? gvE : -gvE);
            p[0] = fma(dd, nx, p[0]);
            p[1] = fma(dd, ny, p[1]);
            return;
        }
    }
    double p2 = 0.0;
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p2 += p[d] * p[d];
    const double E = sizeof(R) == 4 ? sqrt_f32_newton(p2 + m * m) : sqrt(p2 + m * m);
    double vE = to_lab ? v * E : -(v * E);
    if (DIMS == 1) { p[0] = gam * (p[0] + vE); return; }
    double px = p[0], py = p[1];
    double ppar = fma_rn(px, nx, mul_rn(py, ny));
    double pperpx = px - ppar * nx;
    double pperpy = py - ppar * ny;
    double pnew = gam * (ppar + vE);
    p[0] = pnew * nx + pperpx;
    p[1] = pnew * ny + pperpy;
}

// Records a consumed variate.  REC = 1: the noise-recording instantiation (every
// slot, FP64); REC = 2: the adjoint's tape (the momentum normals, FP32).
template <int REC, typename R>
__device__ __forceinline__ void rec_slot(const KParams<R>& kp, int64_t s, int64_t i, int slot, double val)
{
    if (REC == 1 && s >= kp.rec_first && s < kp.rec_first + kp.rec_steps)
        kp.rec[((s - kp.rec_first) * kNoiseSlots + slot) * kp.n + i] = (double)val;
    if (REC == 2 && slot < 3)
        reinterpret_cast<float*>(reinterpret_cast<float4*>(kp.tape) + ((s - kp.tape_first) * 2 + 1) * kp.n + i)[1 + slot] =
            (float)val;
}

// expm1(-x) for x >= 0: Taylor series below 0.05 (truncation < 1e-11 relative),
// the library function above.
__device__ __forceinline__ float expm1_neg(float x)
{
    if (x < 0.05f) {
        float p = 1.0f / 720.0f;
        p = fmaf(p, -x, 1.0f / 120.0f);
        p = fmaf(p, -x, 1.0f / 24.0f);
        p = fmaf(p, -x, 1.0f / 6.0f);
        p = fmaf(p, -x, 0.5f);
        p = fmaf(p, -x, 1.0f);
        return -x * p;
    }
    return expm1f(-x);
}

// kernels_cpu.jl:246-357 + :406-417: exact-OU drag and kick in the LRF.
// tau: the drag time from the drag spline (0 when DsT <= 0), kernels_cpu.jl:270-281.
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ void langevin_kick(const KParams<R>& kp, R T, R tau, double (&p)[3], const R (&xi)[3])
{
    const R M = kp.m, dt = kp.dtR;
    const bool ok = tau > R(0) && isfinite(tau);
    if (sizeof(R) == 4) {
        // FP32: with kappa = 2MT/tau and eta_eff = (M/E)/tau the kick amplitude
        // sqrt(dt) kT sqrt((1-a^2)/(2 eta_eff dt)) is sqrt(T E (1-a^2)) (M in place of E
        // when non-relativistic); a - 1 and 1 - a^2 come from one expm1 (no
        // cancellation).  The FP32 increment is added to the FP64 momentum.
        if (!ok) return;                                   // kT = 0: no drag, no kick
        R pf[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) pf[d] = (R)p[d];
        if (DIMS == 1) {
            R E = sqrt(pf[0] * pf[0] + M * M);
            R eff = kp.rel ? M / (E * tau) : R(1) / tau;
            R kT = sqrt((R(2) * M * T) / tau);
            p[0] += (double)(-eff * pf[0] * dt + kp.sqrt_dt * (kT * xi[0]));
            return;
        }
        R p2 = R(0);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) p2 = fma_rn(pf[d], pf[d], p2);
        R E = sqrt(fma_rn(M, M, p2));
        R Ew = kp.rel ? E : M;
        if (kp.integrator == 1) {
            R a_half = R(1) + expm1_neg((M / (Ew * tau)) * (R(0.5) * dt));
            R p2m = R(0);
#pragma unroll
            for (int d = 0; d < PDIM; ++d) { R q = a_half * pf[d]; p2m += q * q; }
            R Em = sqrt(p2m + M * M);
            Ew = kp.rel ? Em : M;
        }
        R x = (M / (Ew * tau)) * dt;                         // eta_eff * dt
        R em1 = expm1_neg(x);
        R one_m_a2 = -em1 * (R(2) + em1);
        R amp = (dt > R(0) && x > R(0)) ? sqrt(T * Ew * one_m_a2) : R(0);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) p[d] += (double)fma_rn(amp, xi[d], mul_rn(em1, pf[d]));   // the kick fused
        return;
    }
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
        for (int d = 0; d < PDIM; ++d) { R q = a_half * p[d]; p2m += q * q; }
        R Em = sqrt(p2m + M * M);
        eff = kp.rel ? etaD * M / Em : etaD;
    }
    R a = exp(-eff * dt);
    R np = (dt > R(0) && eff > R(0)) ? kT * sqrt((R(1) - a * a) / (R(2) * eff * dt)) : R(0);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p[d] += (a - R(1)) * p[d] + kp.sqrt_dt * (np * xi[d]);
}

// kernels_gpu.jl:88-117.  The u-cell is located from the nearer end of the u grid
// (u or 1 - u, both exact), so the steep tail cells of p*(u) near u = 1 are resolved as
// finely as those near 0; FP32 adds the FMA residual of mag*(nU-1), which restores the
// cell weight exactly.
template <typename R>
__device__ __forceinline__ R invcdf_lookup(const KParams<R>& kp, uint32_t w, R T)
{
    const int nU = kp.nU, nT = kp.nT;
    const R mag = u_mag<R>(w);
    const R fm = mag * R(nU - 1);
    const R k = floor(fm);
    R fr = fm - k;
    if (sizeof(R) == 4) fr += fma(mag, R(nU - 1), -fm);
    const bool up = u_upper(w);
    int iu = up ? nU - 2 - (int)k : (int)k;
    iu = iu < 0 ? 0 : (iu > nU - 2 ? nU - 2 : iu);
    const R tu = up ? R(1) - fr : fr;
    R fT = (T - kp.ic_Tmin) * kp.ic_invdT;
    R flT = floor(fT);
    int jT = flT < R(0) ? 0 : (flT > R(nT - 2) ? nT - 2 : (int)flT);
    R tT = fT - R(jT);
    tT = tT < R(0) ? R(0) : (tT > R(1) ? R(1) : tT);
    const R* b0 = kp.icdf + (size_t)jT * nU + iu;
    const R* b1 = b0 + nU;
    R v00 = __ldg(b0), v10 = __ldg(b0 + 1), v01 = __ldg(b1), v11 = __ldg(b1 + 1);
    R c0 = fma_rn(v10, tu, mul_rn(v00, R(1) - tu));
    R c1 = fma_rn(v11, tu, mul_rn(v01, R(1) - tu));
    return fma_rn(c1, tT, mul_rn(c0, R(1) - tT));
}

template <typename R, int MED, int DIMS>
__device__ __forceinline__ double temperature_fp64(const KParams<R>& kp, const StepRec<R>& sr, const double (&xd)[3]);

// The collision decision of the FP64 path, for an FP32 step whose collision uniform falls
// within 1e-5 (relative) of its FP32 collision probability: the medium temperature at the
// pre-step position, the RTA time and the probability in FP64 (kernels_gpu.jl:675-688),
// compared with the uniform's exact value.  This gives the FP64 path's decision up to
// the FP64 rounding of the temperature (the FP32 decision alone would flip wherever the
// two probabilities straddle the uniform: a few per 1e9 particle-steps).
template <typename R, int MED, int DIMS>
__device__ __forceinline__ bool rta_decide_fp64(const KParams<R>& kp, const StepRec<R>& sr, const R (&x)[3],
                                                const float (&xl)[3], uint32_t wc)
{
    const double xd[3] = { (double)x[0] + (double)xl[0], (double)x[1] + (double)xl[1], (double)x[2] + (double)xl[2] };
    const double T = jmax0(temperature_fp64<R, MED, DIMS>(kp, sr, xd));
    double tn = 0.0;
    if ((double)kp.DsT > 0.0 && T > 0.0)
        tn = spline_at(kp.rta64, spline_index(T, kp.rta_Tmin64, kp.rta_invdT64, kp.n_rta64));
    const double Pcol = (tn > 0.0 && isfinite(tn)) ? jclamp(kp.dt / tn, 0.0, 1.0) : 1.0;
    return u_exact(wc) < Pcol || Pcol >= 1.0;
}

// kernels_gpu.jl:653-704: with probability Pcol = clamp(dt/tau, 0, 1) re-draw |p*|
// from the Jüttner inverse CDF and an isotropic direction.  The collision
// uniform u_collide comes with the step's momentum variates; the sample and the
// direction are drawn only when the particle collides.
// tn: the RTA relaxation time (0 when DsT <= 0 or T <= 0), kernels_gpu.jl:675-679.
// wc: the collision word (uc = u_value<R>(wc)); sr, x, xl: the step record and the
// pre-step position (for the FP32 path's near-threshold FP64 decision).
template <int REC, typename R, int MED, int DIMS, int PDIM, typename PT = double>
__device__ __forceinline__ bool rta_collide(const KParams<R>& kp, int64_t i, int64_t s, const NoiseKey& nk,
                                            R T, R tn, uint32_t wc, const StepRec<R>& sr, const R (&x)[3],
                                            const float (&xl)[3], PT (&p)[3])
{
    const R uc = u_value<R>(wc);
    R Pcol = (tn > R(0) && isfinite(tn)) ? jclamp(kp.dtR / tn, R(0), R(1)) : R(1);
    bool collide = uc < Pcol || Pcol >= R(1);
    if constexpr (sizeof(R) == 4) {
        if (kp.rta64 && fabsf(uc - Pcol) <= 1e-5f * Pcol) collide = rta_decide_fp64<R, MED, DIMS>(kp, sr, x, xl, wc);
    }
    if (kp.rta_mode && s >= kp.rta_first && s < kp.rta_first + kp.rta_steps) {
        uint32_t* w = kp.rta_bits + ((s - kp.rta_first) >> 5) * kp.n + i;
        const uint32_t bit = 1u << ((s - kp.rta_first) & 31);
        if (kp.rta_mode == 2) collide = (*w & bit) != 0u;
        else if (collide) *w |= bit;
    }
    if (!collide) return false;
    const uint4 u = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_RTA);
    R pstar = invcdf_lookup(kp, u.x, T);
    R g[3];
    box_muller(u.y, u.z, g[0], g[1]);
    g[2] = PDIM == 3 ? norm_inv(u.w, R(0)) : R(0);      // one block serves the whole collision
    rec_slot<REC>(kp, s, i, 4, u_exact(u.x));
#pragma unroll
    for (int d = 0; d < 3; ++d) rec_slot<REC>(kp, s, i, 5 + d, g[d]);
    if (DIMS == 1) { p[0] = (PT)((g[0] < R(0) ? R(-1) : R(1)) * pstar); return true; }
    R nrm2 = R(0);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) nrm2 += g[d] * g[d];
    const R tiny = (R)(sizeof(R) == 8 ? 1e-300 : 1e-30);   // the reference's 1e-300 guard, FP32-representable
    R inv = pstar / sqrt(nrm2 > tiny ? nrm2 : tiny);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p[d] = (PT)(g[d] * inv);
    return true;
}

// kernels_cpu.jl:671-735 (momentum_langevin = false or DsT == 0).
template <typename R, int MED, int DIMS>
__device__ __forceinline__ void set_to_fluid(const KParams<R>& kp, const StepRec<R>& sr, const R (&x)[3], double (&p)[3])
{
    const R m = kp.m;
    const R vmax = sizeof(R) == 8 ? R(0.9999999999995) : R(0.99999994f);
    if (MED == MED_GRID) {
        R T, ux, uy;
        grid_lookup(kp.med, sr, x[0], x[1], T, ux, uy);
        R u = sqrt(ux * ux + uy * uy);
        if (u < R(kEps)) { p[0] = 0.0; p[1] = 0.0; return; }
        R vc = kp.rel ? jclamp(u, -vmax, vmax) : u;
        R g = kp.rel ? R(1) / sqrt(R(1) - vc * vc + R(1e-10)) : R(1);
        p[0] = (double)(m * g * vc * (ux / u));
        p[1] = (double)(m * g * vc * (uy / u));
        return;
    }
    R r = DIMS == 1 ? x[0] : sqrt(x[0] * x[0] + x[1] * x[1]);
    if (r < R(kEps)) return;
    R v = R(0);
    if (MED == MED_RT) { R Tdummy; rt_lookup(kp.med, sr, r, Tdummy, v); }
    if (!kp.rel) {
        if (DIMS == 1) p[0] = (double)(m * v);
        else { p[0] = (double)(m * v * (x[0] / r)); p[1] = (double)(m * v * (x[1] / r)); }
        return;
    }
    v = jclamp(v, -vmax, vmax);
    R gam = R(1) / sqrt(R(1) - v * v + R(1e-10));
    if (DIMS == 1) p[0] = (double)(m * gam * v);
    else { p[0] = (double)(m * gam * v * (x[0] / r)); p[1] = (double)(m * gam * v * (x[1] / r)); }
}

// Temperature at an arbitrary point of this step (diffusion, freeze-out).
template <typename R, int MED, int DIMS>
__device__ __forceinline__ R temperature_at(const KParams<R>& kp, const StepRec<R>& sr, const R (&x)[3], R r)
{
    R T;
    if (MED == MED_RT) { R V; rt_lookup(kp.med, sr, r, T, V); }
    else if (MED == MED_BJORKEN) T = sr.T_bj;
    else { R ux, uy; grid_lookup(kp.med, sr, x[0], x[1], T, ux, uy); }
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
// pf_out (optional): the lab momentum after the step rounded to FP32, taken from the
// rounding streaming makes anyway (three fewer FP64 -> FP32 conversions per step, and
// fewer spills, in the freeze-out kernel: 4 % on fixed work); redone where a reflection
// changes the momentum.
template <int REC, typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void stream_positions(const KParams<R>& kp, const StepRec<R>& sr, int64_t i, int64_t s,
                                                 const NoiseKey& nk, R (&x)[3], float (&xl)[3], double (&p)[3],
                                                 float* pf_out = nullptr)
{
    const R m = kp.m, dt = kp.dtR;
    R pr_[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) pr_[d] = (R)p[d];
    if (pf_out) {
#pragma unroll
        for (int d = 0; d < 3; ++d) pf_out[d] = (float)pr_[d];
    }
    R E2 = mul_rn(m, m);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) E2 = fma_rn(pr_[d], pr_[d], E2);
    R E = kp.rel ? sqrt(E2) : m;
    const R r_max = kp.med.r_max, r_axis_eps = kp.med.r_axis_eps;
    if (DIMS == 1) {
        R r = x[0], pr = pr_[0];
        R r_abs = fabs(r);
        R r_safe = r_abs < r_axis_eps ? r_axis_eps : r_abs;
        R dr = (pr / E) * dt;
        if (kp.diffusion) {
            R xs[3] = { r_safe, R(0), R(0) };
            R T = temperature_at<R, MED, DIMS>(kp, sr, xs, r_safe);
            R D = (kp.DsT / (T != T ? T : (T > R(kEps) ? T : R(kEps)))) / R(kFmGeV);
            if (D > R(0)) {
                const uint4 u = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_DIFF);
                R z0, z1;
                box_muller(u.x, u.y, z0, z1);
                rec_slot<REC>(kp, s, i, 8, z0);
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
        if (pf_out) pf_out[0] = (float)p[0];
        return;
    }
    R invE = R(1) / E;
#pragma unroll
    for (int d = 0; d < DIMS; ++d) {
        R dx = sizeof(R) == 8 ? dt * pr_[d] / E : (dt * pr_[d]) * invE;
        acc_add(x[d], xl[d], dx);
    }
    if (kp.diffusion) {
        R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        R T = temperature_at<R, MED, DIMS>(kp, sr, x, sqrt(r2));
        R D = (kp.DsT / (T != T ? T : (T > R(kEps) ? T : R(kEps)))) / R(kFmGeV);
        if (D > R(0)) {
            R sg = sqrt(R(2) * D * dt);
            const uint4 u = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_DIFF);
            R z[4];
            box_muller(u.x, u.y, z[0], z[1]);
            box_muller(u.z, u.w, z[2], z[3]);
#pragma unroll
            for (int d = 0; d < DIMS; ++d) { rec_slot<REC>(kp, s, i, 8 + d, z[d]); acc_add(x[d], xl[d], sg * z[d]); }
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
            for (int d = 0; d < DIMS; ++d) ppar += pr_[d] * (x[d] * invr);
#pragma unroll
            for (int d = 0; d < DIMS; ++d) p[d] -= (double)(R(2) * ppar * (x[d] * invr));
            if (pf_out) {
#pragma unroll
                for (int d = 0; d < DIMS; ++d) pf_out[d] = (float)p[d];
            }
            R scale = (R(2) * r_max - r_now) * invr;
#pragma unroll
            for (int d = 0; d < DIMS; ++d) { x[d] = (R)((double)x[d] + (double)xl[d]) * scale; xl[d] = 0.f; }
        }
    }
}

// FP32 step on the 2+1D grid with the frame changes as FP32 increments (flow speed
// below kVIncr, gamma <= 2; faster flows take the FP64 frame change of cart_step).  The
// lab momentum p stays FP64.  The rest-frame momentum p* = L(p) is formed in FP32 from
// p rounded to FP32 (kernels_cpu.jl:89-145); the Bjorken redshift of its p_z, the kick
// and the RTA resample change it by dl (FP32, as in cart_step); the lab momentum then
// moves by
//     L^-1(p* + dl) - L^-1(p*) = dl + n [(gamma - 1) (dl . n) + gamma v (E1 - E0)],
// E1 - E0 = dl . (2 p* + dl) / (E1 + E0), the exact difference of the two lab-frame
// changes (kernels_cpu.jl:188-241) without cancellation, added to p in FP64.  The FP32
// rounding of p* enters only the increment, so the state keeps the FP64 frame change's
// accuracy at a fraction of its FP64 work.
constexpr float kVIncr = 0.8660254f;   // gamma = 2

template <int REC, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void step_rest_frame_incr(const KParams<float>& kp, const StepRec<float>& sr, int64_t i,
                                                     int64_t s, const NoiseKey& nk, const float (&x)[3],
                                                     const float (&xl)[3], double (&p)[3], const Local<float>& L,
                                                     const float* pin)
{
    const float m = kp.m;
    float pl[3] = { 0.0f, 0.0f, 0.0f };           // p rounded to FP32 (pin: the caller's copy)
#pragma unroll
    for (int d = 0; d < PDIM; ++d) pl[d] = pin ? pin[d] : (float)p[d];
    const float v = L.v, vv = mul_rn(v, v);
    const float g = rsqrtf(1.0f - vv);
    const float gm1 = __fdividef(mul_rn(vv, mul_rn(g, g)), 1.0f + g);     // gamma - 1 = gamma^2 v^2 / (1 + gamma)
    const float gv = mul_rn(g, v);
    const float nx = L.nx, ny = L.ny;
    float q = mul_rn(m, m);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) q = fma_rn(pl[d], pl[d], q);
    const float El = sqrtf(q);
    const float dpar = fma_rn(gm1, fma_rn(pl[0], nx, mul_rn(pl[1], ny)), -mul_rn(gv, El));
    float ps[3] = { fma_rn(dpar, nx, pl[0]), fma_rn(dpar, ny, pl[1]), pl[2] };
    float E0 = mul_rn(m, m);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) E0 = fma_rn(ps[d], ps[d], E0);
    E0 = sqrtf(E0);
    // the change dl of p*, kept apart from p* so that its FP32 rounding is that of the
    // change: the redshift of p*_z (kernels_cpu.jl:427-435), then the kick on the
    // redshifted p* (pr), or the RTA resample in place of both
    float dl[3] = { 0.0f, 0.0f, 0.0f };
    float pr[3] = { ps[0], ps[1], ps[2] };
    float Er = E0;
    if (PDIM == 3 && kp.redshift) {
        dl[2] = mul_rn((float)(sr.zf - 1.0), ps[2]);
        pr[2] = ps[2] + dl[2];
        float qr = mul_rn(m, m);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) qr = fma_rn(pr[d], pr[d], qr);
        Er = sqrtf(qr);
    }
    const float T = jmax0(L.T);
    const uint4 u = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_MOM);
    const bool kick = kp.collision != COLL_RTA;
    const bool rta = kp.collision == COLL_RTA || kp.collision == COLL_LANGEVIN_RTA;
    const SplIdx<float> sd = spline_index(T, kp.drag_Tmin, kp.drag_invdT, kp.n_drag);
    uint32_t wc = u.x;
    if (kick) {
        float xi[3];
        box_muller(u.x, u.y, xi[0], xi[1]);
        if (PDIM == 3) { xi[2] = norm_inv(u.z, 0.0f); wc = u.w; }
        else { xi[2] = 0.0f; wc = u.z; }
#pragma unroll
        for (int d = 0; d < PDIM; ++d) rec_slot<REC>(kp, s, i, d, xi[d]);
        const float tau = kp.DsT <= 0.0f ? 0.0f : spline_at(kp.drag, sd);
        const float M = m, dt = kp.dtR;
        if (tau > 0.0f && isfinite(tau)) {               // as langevin_kick's FP32 form, on p*
            float Ew = Er;
            if (kp.integrator == 1) {
                const float a_half = 1.0f + expm1_neg((M / (Ew * tau)) * (0.5f * dt));
                float p2m = 0.0f;
#pragma unroll
                for (int d = 0; d < PDIM; ++d) { const float qd = a_half * pr[d]; p2m += qd * qd; }
                Ew = sqrtf(p2m + M * M);
            }
            const float xx = (M / (Ew * tau)) * dt;
            const float em1 = expm1_neg(xx);
            const float one_m_a2 = -em1 * (2.0f + em1);
            const float amp = (dt > 0.0f && xx > 0.0f) ? sqrtf(T * Ew * one_m_a2) : 0.0f;
#pragma unroll
            for (int d = 0; d < PDIM; ++d) dl[d] += fma_rn(amp, xi[d], mul_rn(em1, pr[d]));
        }
    }
    if (rta) {
        rec_slot<REC>(kp, s, i, 3, u_exact(wc));
        float tn = 0.0f;
        if (kp.DsT > 0.0f && T > 0.0f)
            tn = spline_at(kp.rta, kp.spl_shared ? sd : spline_index(T, kp.rta_Tmin, kp.rta_invdT, kp.n_rta));
        float pc[3] = { 0.0f, 0.0f, 0.0f };
        if (rta_collide<REC, float, MED, DIMS, PDIM, float>(kp, i, s, nk, T, tn, wc, sr, x, xl, pc)) {
#pragma unroll
            for (int d = 0; d < 3; ++d) dl[d] = pc[d] - ps[d];
        }
    }
    float sm[3];
    float E1 = mul_rn(m, m);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float pn = ps[d] + dl[d];
        sm[d] = ps[d] + pn;
        if (d < PDIM) E1 = fma_rn(pn, pn, E1);
    }
    E1 = sqrtf(E1);
    float dd = mul_rn(dl[0], sm[0]);
#pragma unroll
    for (int d = 1; d < PDIM; ++d) dd = fma_rn(dl[d], sm[d], dd);
    const float dE = __fdividef(dd, E0 + E1);
    const float c = fma_rn(gm1, fma_rn(dl[0], nx, mul_rn(dl[1], ny)), mul_rn(gv, dE));
    p[0] += (double)fma_rn(c, nx, dl[0]);
    p[1] += (double)fma_rn(c, ny, dl[1]);
    if (PDIM == 3) p[2] += (double)dl[2];
}

// One Cartesian step (simulate_cpu.jl:215-290).
// pf_out (optional): the lab momentum after the step, rounded to FP32; with INCR (the
// FP32 grid freeze-out kernel) it holds the lab momentum before the step, rounded the
// same way, on entry.
template <int REC, typename R, int MED, int DIMS, int PDIM, bool INCR = false>
__device__ __forceinline__ void cart_step(const KParams<R>& kp, const StepRec<R>& sr, int64_t i, int64_t s,
                                          const NoiseKey& nk, R (&x)[3], float (&xl)[3], double (&p)[3],
                                          GridRows<R>* carry = nullptr, float* pf_out = nullptr)
{
    // the grid medium's tape rows 0, 2, 3 (pre-step momentum, medium and gradient); row 1
    // (the normals and v^x) follows the kick
    constexpr bool kTapeGrid = REC == 2 && MED == MED_GRID;
    MedGrad mg;
    float4* trow = nullptr;
    if constexpr (kTapeGrid) trow = reinterpret_cast<float4*>(kp.tape) + (s - kp.tape_first) * 4 * kp.n + i;
    const Local<R> L = local_medium<R, MED, DIMS, kTapeGrid>(kp, sr, x, &mg, carry, xl);
    if constexpr (kTapeGrid) {
        trow[0] = make_float4((float)p[0], (float)p[1], (float)p[2], mg.T);
        trow[2 * kp.n] = make_float4(mg.vy, mg.dT[0], mg.dT[1], mg.dvx[0]);
        trow[3 * kp.n] = make_float4(mg.dvx[1], mg.dvy[0], mg.dvy[1], 0.0f);
    }
    if constexpr (INCR && MED == MED_GRID && sizeof(R) == 4 && DIMS == 2) {
        if (kp.rel && kp.collision != COLL_FLUID && L.v < kVIncr) {
            step_rest_frame_incr<REC, MED, DIMS, PDIM>(kp, sr, i, s, nk, x, xl, p, L, pf_out);
            stream_positions<REC, R, MED, DIMS, PDIM>(kp, sr, i, s, nk, x, xl, p, pf_out);
            return;
        }
    }
    // on the grid gamma is computed once for both frame changes (measured 2 % faster
    // there; the (r, t) and Bjorken kernels keep their own form, measured faster for them)
    double gam = -1.0;                                      // -1: computed in boost()
    if (L.boost) {
        if constexpr (MED == MED_GRID) gam = boost_gamma(L);
        boost<R, DIMS, PDIM>(kp, L, p, false, gam);
    }
    if (PDIM == 3 && kp.redshift) p[2] *= sr.zf;
    if (kp.collision == COLL_FLUID) {
        set_to_fluid<R, MED, DIMS>(kp, sr, x, p);
    } else {
        const R T = jmax0(L.T);
        const uint4 u = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_MOM);
        const bool kick = kp.collision != COLL_RTA;
        if constexpr (kTapeGrid) {
            if (!kick) trow[kp.n] = make_float4(0.0f, 0.0f, 0.0f, mg.vx);
        }
        const bool rta = kp.collision == COLL_RTA || kp.collision == COLL_LANGEVIN_RTA;
        // one T-grid lookup for both splines when they share the grid
        const SplIdx<R> sd = spline_index(T, kp.drag_Tmin, kp.drag_invdT, kp.n_drag);
        uint32_t wc = u.x;                   // the collision word
        if (kick) {
            R xi[3];
            box_muller(u.x, u.y, xi[0], xi[1]);
            if (PDIM == 3) {
                xi[2] = norm_inv(u.z, R(0));
                wc = u.w;
            } else {
                xi[2] = R(0);
                wc = u.z;
            }
            if constexpr (kTapeGrid) {
                trow[kp.n] = make_float4((float)xi[0], (float)xi[1], (float)xi[2], mg.vx);
            } else {
#pragma unroll
                for (int d = 0; d < PDIM; ++d) rec_slot<REC>(kp, s, i, d, xi[d]);
            }
            const R tau = kp.DsT <= R(0) ? R(0) : spline_at(kp.drag, sd);
            langevin_kick<R, DIMS, PDIM>(kp, T, tau, p, xi);
        }
        if (rta) {
            rec_slot<REC>(kp, s, i, 3, u_exact(wc));
            R tn = R(0);
            if (kp.DsT > R(0) && T > R(0))
                tn = spline_at(kp.rta, kp.spl_shared ? sd : spline_index(T, kp.rta_Tmin, kp.rta_invdT, kp.n_rta));
            rta_collide<REC, R, MED, DIMS, PDIM>(kp, i, s, nk, T, tn, wc, sr, x, xl, p);
        }
        if (L.boost) boost<R, DIMS, PDIM>(kp, L, p, true, gam);
    }
    stream_positions<REC, R, MED, DIMS, PDIM>(kp, sr, i, s, nk, x, xl, p, pf_out);
}

// Temperature at the particle in FP64 arithmetic (FP64 weights over the stored
// field values), for the freeze-out latch of the FP32 path.
template <typename R, int MED, int DIMS>
__device__ __forceinline__ double temperature_fp64(const KParams<R>& kp, const StepRec<R>& sr, const double (&xd)[3])
{
    const MediumDev<R>& md = kp.med;
    double T;
    if (MED == MED_BJORKEN) {
        T = sr.Td;
    } else if (MED == MED_RT) {
        double r;
        if (DIMS == 1) r = fabs(xd[0]);
        else { double r2 = 0.0;
#pragma unroll
            for (int d = 0; d < DIMS; ++d) r2 += xd[d] * xd[d];
            r = sqrt(r2); }
        const double* g = md.xgd;
        const int nr = md.nr;
        double rq = r > g[nr - 1] ? g[nr - 1] : (r < g[0] ? g[0] : r);
        int i = cell_index(g, nr, rq, md.x_uniform, (double)md.xg0, (double)md.xinvd);
        double x0 = g[i], x1 = g[i + 1], dx = x1 - x0;
        double w = fabs(dx) < kEps ? 0.0 : (rq - x0) / dx;
        const int j = sr.kt;
        double v00, v10, v01, v11;
        if (kp.T64) {                    // FP32 runs: the FP64 table the FP64 path interpolates
            v00 = kp.T64[i + nr * j]; v10 = kp.T64[i + 1 + nr * j];
            v01 = kp.T64[i + nr * (j + 1)]; v11 = kp.T64[i + 1 + nr * (j + 1)];
        } else {
            v00 = (double)md.TV[i + nr * j].x; v10 = (double)md.TV[i + 1 + nr * j].x;
            v01 = (double)md.TV[i + nr * (j + 1)].x; v11 = (double)md.TV[i + 1 + nr * (j + 1)].x;
        }
        double c0 = v00 * (1.0 - w) + v10 * w, c1 = v01 * (1.0 - w) + v11 * w;
        T = c0 * (1.0 - sr.wtd) + c1 * sr.wtd;
    } else {
        int ix, iy;
        double wx, wy;
        {
            double xq = xd[0] > md.gxl_d ? md.gxl_d : (xd[0] < md.gx0_d ? md.gx0_d : xd[0]);
            double yq = xd[1] > md.gyl_d ? md.gyl_d : (xd[1] < md.gy0_d ? md.gy0_d : xd[1]);
            double fx = (xq - md.gx0_d) / md.gdx_d, fy = (yq - md.gy0_d) / md.gdy_d;
            double flx = floor(fx), fly = floor(fy);
            ix = flx < 0.0 ? 0 : (flx > (double)(md.gnx - 2) ? md.gnx - 2 : (int)flx);
            iy = fly < 0.0 ? 0 : (fly > (double)(md.gny - 2) ? md.gny - 2 : (int)fly);
            wx = fx - (double)ix;
            wy = fy - (double)iy;
        }
        const float4* s0 = md.G + ((size_t)sr.kt * md.gny + iy) * md.gnx + ix;
        const float4* s1 = s0 + (size_t)md.gny * md.gnx;
        double c[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float4* q = k ? s1 : s0;
            double a00 = __ldg(q).x, a10 = __ldg(q + 1).x, a01 = __ldg(q + md.gnx).x, a11 = __ldg(q + md.gnx + 1).x;
            // the FP64 path's interpolation (bilerp_rn, grid_combine), rounding for rounding
            c[k] = lerp_rn(lerp_rn(a00, a10, wx), lerp_rn(a01, a11, wx), wy);
        }
        T = lerp_rn(c[0], c[1], sr.wtd);
    }
    if (md.T_scale != R(1)) T *= (double)md.T_scale;
    return T;
}

// The time record of medium time t (the FP64 fields make_step_rec derives from the
// same t, so a temperature re-evaluated from it is bit-identical).
template <typename R, int MED>
__device__ __forceinline__ StepRec<R> step_rec_at_time(const KParams<R>& kp, double t)
{
    StepRec<R> u;
    u.t = t; u.tR = (R)t; u.kt = 0; u.wt = R(0); u.T_bj = R(0); u.zf = 1.0; u.wtd = 0.0; u.Td = 0.0;
    const MediumDev<R>& md = kp.med;
    if (MED == MED_RT) {
        const double* tg = md.tgd;
        const int nt = md.nt;
        double tq = t > tg[nt - 1] ? tg[nt - 1] : (t < tg[0] ? tg[0] : t);
        int lo = -1, hi = nt;
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (tg[mid] <= tq) lo = mid; else hi = mid; }
        int k = lo < 0 ? 0 : lo;
        k = k > nt - 2 ? nt - 2 : k;
        double y0 = tg[k], y1 = tg[k + 1], dy = y1 - y0;
        u.kt = k;
        u.wtd = fabs(dy) < kEps ? 0.0 : (tq - y0) / dy;
    } else if (MED == MED_BJORKEN) {
        u.Td = (t > md.bj_tau0) ? md.bj_T0 * pow(md.bj_tau0 / t, md.bj_power) : md.bj_T0;
    } else {
        u.kt = grid_time_cell(md, t, u.wtd);
    }
    return u;
}

// FP32 screen of the temperature at the particle: T in FP32 from the same nodes, off
// from the FP64 value by far less than the latch's screening margin.
template <typename R, int MED, int DIMS>
__device__ __forceinline__ float temperature_screen(const KParams<R>& kp, const StepRec<R>& sr, const R (&x)[3])
{
    const MediumDev<R>& md = kp.med;
    if (MED == MED_BJORKEN) return (float)sr.T_bj * (float)md.T_scale;
    if (MED == MED_GRID) {
        int ix, iy;
        R wx, wy;
        grid_cell(md, x[0], x[1], ix, iy, wx, wy);
        const float4* s0 = md.G + ((size_t)sr.kt * md.gny + iy) * md.gnx + ix;
        const float4* s1 = s0 + (size_t)md.gny * md.gnx;
        const float* q0 = reinterpret_cast<const float*>(s0);
        const float* q1 = reinterpret_cast<const float*>(s1);
        const int rowf = 4 * md.gnx;
        const float fx = (float)wx, fy = (float)wy;
        float a00 = __ldg(q0), a10 = __ldg(q0 + 4), a01 = __ldg(q0 + rowf), a11 = __ldg(q0 + rowf + 4);
        float b00 = __ldg(q1), b10 = __ldg(q1 + 4), b01 = __ldg(q1 + rowf), b11 = __ldg(q1 + rowf + 4);
        const float ra = a00 + fx * (a10 - a00), rb = b00 + fx * (b10 - b00);
        const float c0 = ra + fy * ((a01 + fx * (a11 - a01)) - ra);
        const float c1 = rb + fy * ((b01 + fx * (b11 - b01)) - rb);
        return (c0 + (float)sr.wt * (c1 - c0)) * (float)md.T_scale;
    }
    R r;
    if (DIMS == 1) r = fabs(x[0]);
    else { R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        r = sqrt(r2); }
    return (float)temperature_at<R, MED, DIMS>(kp, sr, x, r);
}

// The FP64 latch's last-above record: the position and the lab momentum of the last
// step the particle ended above Tfo (FP64 runs; the FP32 kernels keep no record,
// freezeout_latch_pre).
template <typename R>
struct LatchPos {
    R h[3];
    __device__ __forceinline__ double at(int d) const { return (double)h[d]; }
};

template <typename R>
struct LatchMom {
    double m[3];
    __device__ __forceinline__ double at(int d) const { return m[d]; }
};

// Freeze-out latch after streaming (kernels_gpu.jl:588-635), FP64 runs: the temperature
// at the particle in FP64 every step; the last-above state and temperature lT are kept
// (a particle already below Tfo at its first step latches with frac = 1, as with lT = 0
// in the reference).
template <typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void freezeout_latch(const KParams<R>& kp, const StepRec<R>& sr, int64_t i,
                                                const R (&x)[3], const double (&p)[3], bool& frozen,
                                                LatchPos<R>& lpos, LatchMom<R>& lmom, double& ltau, double& lT)
{
    static_assert(sizeof(R) == 8, "the FP32 kernels latch with freezeout_latch_pre");
    if (frozen) return;
    const double Tfo = (double)kp.Tfo;
    double T;
    double xd[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) xd[d] = (double)x[d];
    R r;
    if (DIMS == 1) r = fabs(x[0]);
    else { R r2 = R(0);
#pragma unroll
        for (int d = 0; d < DIMS; ++d) r2 += x[d] * x[d];
        r = sqrt(r2); }
    T = (double)temperature_at<R, MED, DIMS>(kp, sr, x, r);
    if (T < Tfo) {
        const double frac = (kp.fo_interp && lT > Tfo && lT > T) ? (lT - Tfo) / (lT - T) : 1.0;
#pragma unroll
        for (int d = 0; d < DIMS; ++d) kp.fo_pos[d][i] = lpos.at(d) + frac * (xd[d] - lpos.at(d));
#pragma unroll
        for (int d = 0; d < PDIM; ++d) kp.fo_mom[d][i] = lmom.at(d) + frac * (p[d] - lmom.at(d));
        kp.fo_tau[i] = ltau + frac * (sr.t - ltau);
        kp.fo_flag[i] = 1.0;
        frozen = true;
    } else {
#pragma unroll
        for (int d = 0; d < DIMS; ++d) lpos.h[d] = xd[d];
#pragma unroll
        for (int d = 0; d < PDIM; ++d) lmom.m[d] = p[d];
        ltau = sr.t;
        lT = T;
    }
}

// The FP32 freeze-out latch without a last-above record.  A particle that is not frozen
// at step s was above Tfo after every step before (else it would have latched there), so
// its last-above state is the state before step s: the position pair (xp, xlp), the lab
// momentum as streaming rounded it (pfp) and the time of step s - 1.  The caller keeps
// them through the step (they are the registers the step starts from) instead of a
// record copied every step.  have_last: the particle has run a step before this one (a
// particle already below Tfo at its first step latches with frac = 1).  The temperature
// is screened in FP32 (kScreen: FP32 and FP64 temperatures differ by < 1e-6) and tested
// in FP64 only near Tfo; at a crossing the last-above temperature is evaluated in FP64
// from the pre-step position and the time of step s - 1, the crossing interpolated in
// FP64 (frac = (T_last - Tfo)/(T_last - T)).
template <typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void freezeout_latch_pre(const KParams<R>& kp, const StepRec<R>& sr, int64_t i, int64_t s,
                                                    const R (&x)[3], const float (&xl)[3], const double (&p)[3],
                                                    const R (&xp)[3], const float (&xlp)[3], const float (&pfp)[3],
                                                    bool& frozen, bool& have_last, const GridRows<R>* carry)
{
    constexpr float kScreen = 1e-4f;     // GeV; FP32 and FP64 temperatures differ by < 1e-6
    if (frozen) return;
    const double Tfo = (double)kp.Tfo;
    float Ts;
    if (MED == MED_GRID && carry) Ts = carry->T1;      // from the lookup at the new position (GridRows)
    else Ts = temperature_screen<R, MED, DIMS>(kp, sr, x);
    if (!(Ts >= (float)Tfo + kScreen)) {
        double xd[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) xd[d] = (double)x[d] + (double)xl[d];
        const double T = temperature_fp64<R, MED, DIMS>(kp, sr, xd);
        if (T < Tfo) {
            double lp[3] = { 0.0, 0.0, 0.0 }, lm[3] = { 0.0, 0.0, 0.0 }, lt = 0.0, lTv = 0.0;
            if (have_last) {
#pragma unroll
                for (int d = 0; d < DIMS; ++d) lp[d] = (double)xp[d] + (double)xlp[d];
#pragma unroll
                for (int d = 0; d < PDIM; ++d) lm[d] = (double)pfp[d];
                lt = step_time(kp, s - 1);
                const StepRec<R> pr = step_rec_at_time<R, MED>(kp, lt);
                lTv = temperature_fp64<R, MED, DIMS>(kp, pr, lp);
            }
            const double frac = (kp.fo_interp && lTv > Tfo && lTv > T) ? (lTv - Tfo) / (lTv - T) : 1.0;
#pragma unroll
            for (int d = 0; d < DIMS; ++d) kp.fo_pos[d][i] = lp[d] + frac * (xd[d] - lp[d]);
#pragma unroll
            for (int d = 0; d < PDIM; ++d) kp.fo_mom[d][i] = lm[d] + frac * (p[d] - lm[d]);
            kp.fo_tau[i] = lt + frac * (sr.t - lt);
            kp.fo_flag[i] = 1.0;
            frozen = true;
            return;
        }
    }
    have_last = true;
}

// ---------------------------------------------------------------------------
// Milne (tau, r) step (simulate_cpu_general_coords.jl:83-126).  The Milne
// interpolation neither clamps the query nor guards dx (kernels_cpu_GC.jl:37-57).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void milne_lookup(const MediumDev<R>& md, const StepRec<R>& sr, R r, R& T, R& V)
{
    int i = cell_index(md.xg, md.nr, r, md.x_uniform, md.xg0, md.xinvd);
    R x0 = __ldg(md.xg + i), x1 = __ldg(md.xg + i + 1);
    R xd = (r - x0) / (x1 - x0);
    const int nr = md.nr, j = sr.kt;
    auto a00 = md.TV[i + nr * j],       a10 = md.TV[i + 1 + nr * j];
    auto a01 = md.TV[i + nr * (j + 1)], a11 = md.TV[i + 1 + nr * (j + 1)];
    R yd = sr.wt;
    R c0 = a00.x * (R(1) - xd) + a10.x * xd;
    R c1 = a01.x * (R(1) - xd) + a11.x * xd;
    T = c0 * (R(1) - yd) + c1 * yd;
    c0 = a00.y * (R(1) - xd) + a10.y * xd;
    c1 = a01.y * (R(1) - xd) + a11.y * xd;
    V = c0 * (R(1) - yd) + c1 * yd;
}

template <int REC, typename R>
__device__ __forceinline__ void milne_step(const KParams<R>& kp, const StepRec<R>& sr, int64_t i, int64_t s,
                                           const NoiseKey& nk, R (&x)[3], float (&xl)[3], double (&p)[3])
{
    const double m = (double)kp.m;
    const R dt = kp.dtR;
    R T, vR;
    milne_lookup(kp.med, sr, fabs(x[1]), T, vR);      // same (r, t) for rest boost, forces, lab boost
    if (kp.med.T_scale != R(1)) T *= kp.med.T_scale;
    const double v = (double)vR;
    // kernels_cpu_GC.jl:64-82
    double g = 1.0 / sqrt(1.0 - v * v + 1e-10);
    double pt = p[0], pr = p[1];
    p[0] = g * (pt - v * pr);
    p[1] = g * (pr - v * pt);
    // kernels_cpu_GC.jl:110-174 (Christoffel term identically zero) + :244-256
    const R DsT_safe = kp.DsT <= R(0) ? R(0) : kp.DsT;
    R tn = DsT_safe == R(0) ? R(0) : eval_spline(T, kp.drag_Tmin, kp.drag_invdT, kp.drag, kp.n_drag);
    const bool ok = tn > R(0) && isfinite(tn);
    R etaD = ok ? R(1) / tn : R(0);
    R kappa = ok ? (R(2) * kp.m * T) / tn : R(0);
    R kT = sqrt(kappa);
    const uint4 u = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_MOM);
    R xi, z1;
    box_muller(u.x, u.y, xi, z1);
    rec_slot<REC>(kp, s, i, 0, xi);
    if (sizeof(R) == 8) {
        R det, sto;
        if (etaD > R(0) && dt > R(0)) {
            R a = exp(-etaD * dt);
            R np = kT * sqrt((R(1) - a * a) / (R(2) * etaD * dt));
            det = (a - R(1)) * (R)p[1];
            sto = np * xi;
        } else {
            det = R(0);
            sto = kT * xi;
        }
        p[1] += (double)(det + kp.sqrt_dt * sto);
    } else if (etaD > R(0) && dt > R(0)) {
        R em1 = expm1_neg(etaD * dt);
        R amp = sqrt(m * T * (-em1 * (R(2) + em1)));     // sqrt(kappa (1-a^2) / (2 eta_D))
        p[1] += (double)(em1 * (R)p[1] + amp * xi);
    } else {
        p[1] += (double)(kp.sqrt_dt * (kT * xi));
    }
    p[0] = sqrt(m * m + p[1] * p[1]);
    // kernels_cpu_GC.jl:85-102
    g = 1.0 / sqrt(1.0 - v * v + 1e-8);
    pt = p[0]; pr = p[1];
    p[0] = g * (pt + v * pr);
    p[1] = g * (pr + v * pt);
    // kernels_cpu_GC.jl:259-274
    if (sizeof(R) == 8) {
        double E = p[0];
        acc_add(x[0], xl[0], (R)(dt * p[0] / E));
        acc_add(x[1], xl[1], (R)(dt * p[1] / E));
    } else {
        acc_add(x[0], xl[0], dt);
        acc_add(x[1], xl[1], (R)((double)dt * p[1] / p[0]));
    }
}

}  // namespace lim

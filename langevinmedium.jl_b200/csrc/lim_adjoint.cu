// lim_adjoint.cu — reverse-mode (adjoint) pathwise derivatives of final-state
// observables with respect to the drag parametrisation (a, b) of D_s(T) and the
// medium temperature scale s, with the noise and the RTA indicators held fixed.
//
// The forward pass checkpoints the state every K steps and tapes the last segment.
// The reverse sweep then takes the segments from the last: k_tape recomputes a segment
// from its checkpoint with the primal step (RTA decisions replayed from the forward
// pass's record), writing to a tape what the reverse step needs: the pre-step momentum,
// the momentum normals and, on the 2+1D grid, the medium the step saw with its
// gradient (so the reverse needs no grid lookups); k_adjoint_rev walks
// the segment backwards, applying the hand-derived vector-Jacobian product of each step
// to two cotangents carried between segments in HBM.  All three observables are
// functions of the final (p_x, p_y), so the cotangents start as the unit vectors of
// p_x and p_y: the sweep yields d p_x / d theta and d p_y / d theta per particle, which
// k_adjoint_gsum contracts with each observable's gradient.  Each step is written in
// the form
//   A medium (T, u) at x          B rest boost  p1 = p + c (p.u) u - E u
//   C Bjorken redshift of p_z     D OU kick     p3 = a(p2) p2 + amp(p2, T, tau) xi
//   E RTA resample (fixed)        F lab boost   p5 = p4 + c (p4.u) u + E u
//   G streaming                   x' = x + dt p5 / E5
// with u = g V the spatial fluid four-velocity formed from the grid's flow velocity V
// (g = 1/sqrt(1 - V.V)), gamma = sqrt(1 + u.u) = g, c = 1/(1 + gamma): the step of
// lim_step.cuh (its frame change is this map, up to the reference's 1e-10 under the
// square root of gamma), smooth in V at V = 0; the cotangent of u maps back to the
// velocity field through du/dV = g I + g^3 V V^T.
// Intermediates are re-evaluated in FP32 from the taped values; slopes of the
// tabulated functions come from tables differenced in FP64 on the host.
#include "lim_internal.h"
#include "lim_particle.cuh"

namespace lim {

namespace {

// The Jüttner inverse CDF at (word w, T) as invcdf_lookup computes it, with its
// derivative in T (zero where the T weight is clamped).
__device__ __forceinline__ float invcdf_lookup_dT(const KParams<float>& kp, uint32_t w, float T, float& dpdT)
{
    const int nU = kp.nU, nT = kp.nT;
    const float mag = u_mag<float>(w);
    const float fm = mag * (float)(nU - 1);
    const float k = floorf(fm);
    float fr = fm - k;
    fr += fmaf(mag, (float)(nU - 1), -fm);
    const bool up = u_upper(w);
    int iu = up ? nU - 2 - (int)k : (int)k;
    iu = iu < 0 ? 0 : (iu > nU - 2 ? nU - 2 : iu);
    const float tu = up ? 1.0f - fr : fr;
    const float fT = (T - kp.ic_Tmin) * kp.ic_invdT;
    const float flT = floorf(fT);
    const int jT = flT < 0.0f ? 0 : (flT > (float)(nT - 2) ? nT - 2 : (int)flT);
    float tT = fT - (float)jT;
    const bool inside = tT > 0.0f && tT < 1.0f;
    tT = tT < 0.0f ? 0.0f : (tT > 1.0f ? 1.0f : tT);
    const float* b0 = kp.icdf + (size_t)jT * nU + iu;
    const float* b1 = b0 + nU;
    const float v00 = __ldg(b0), v10 = __ldg(b0 + 1), v01 = __ldg(b1), v11 = __ldg(b1 + 1);
    const float c0 = v00 * (1.0f - tu) + v10 * tu;
    const float c1 = v01 * (1.0f - tu) + v11 * tu;
    const float* d0 = kp.icdf_dT + (size_t)jT * nU + iu;     // (v[jT+1] - v[jT]) invdT, from FP64
    dpdT = inside ? __ldg(d0) * (1.0f - tu) + __ldg(d0 + 1) * tu : 0.0f;
    return c0 * (1.0f - tT) + c1 * tT;
}

// Vector-Jacobian product of the boost p' = p + c (p.u) u + sg E u (u in the x-y plane):
// b (the cotangent of p') -> the cotangent of p, and the cotangent of u added to ub.
__device__ __forceinline__ void boost_vjp(float sg, const float (&p)[3], float E, float iE, float ux, float uy,
                                          float gam, float c, const float (&b)[3], float (&bp)[3], float (&ub)[2])
{
    const float A = b[0] * ux + b[1] * uy;
    const float pu = p[0] * ux + p[1] * uy;
    const float sAE = sg * A * iE;
    bp[0] = b[0] + c * A * ux + sAE * p[0];
    bp[1] = b[1] + c * A * uy + sAE * p[1];
    bp[2] = b[2] + sAE * p[2];
    const float k1 = -c * c * pu / gam;
    const float k2 = c * pu + sg * E;
    ub[0] += A * (k1 * ux + c * p[0]) + b[0] * k2;
    ub[1] += A * (k1 * uy + c * p[1]) + b[1] * k2;
}

__device__ __forceinline__ void boost_fwd(float sg, const float (&p)[3], float m, float ux, float uy, float c,
                                          float (&q)[3], float& E)
{
    E = sqrtf(p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + m * m);
    const float pu = p[0] * ux + p[1] * uy;
    const float f = c * pu + sg * E;
    q[0] = p[0] + f * ux;
    q[1] = p[1] + f * uy;
    q[2] = p[2];
}

// The reverse of step s for NC cotangents: lx, lp (of the post-step state) become
// those of the pre-step state (xs, ps); g[o][k] accumulates the parameter part.
// mg: the medium the step saw (from the tape; T only for Bjorken); zf: the step's
// Bjorken redshift factor of p_z.
template <int MED, int NC>
__device__ __forceinline__ void adjoint_step(const KParams<float>& kp, int64_t s, int64_t i, const NoiseKey& nk,
                                             const MedGrad& mg, float zf, const float (&ps)[3], const float (&xi)[3],
                                             float (&lx)[NC][2], float (&lp)[NC][3], float (&g)[NC][3])
{
    const float m = kp.m, dt = kp.dtR;
    // ---- A. medium
    float ux = 0.0f, uy = 0.0f;
    const float Tf = mg.T;
    const float vx = MED == MED_GRID ? mg.vx : 0.0f, vy = MED == MED_GRID ? mg.vy : 0.0f;
    const float dT[2] = { mg.dT[0], mg.dT[1] }, dux[2] = { mg.dvx[0], mg.dvx[1] }, duy[2] = { mg.dvy[0], mg.dvy[1] };
    const float sc = kp.med.T_scale;
    const float T = Tf * sc;
    const bool flow = MED == MED_GRID && !(sqrtf(vx * vx + vy * vy) < (float)kEps);
    const float gam = rsqrtf(1.0f - (vx * vx + vy * vy)), c = 1.0f / (1.0f + gam);
    ux = gam * vx;                              // four-velocity
    uy = gam * vy;
    // ---- B. rest boost
    float p1[3], E0 = 0.0f;
    if (flow) boost_fwd(-1.0f, ps, m, ux, uy, c, p1, E0);
    else { p1[0] = ps[0]; p1[1] = ps[1]; p1[2] = ps[2]; }
    // ---- C. redshift
    float p2[3] = { p1[0], p1[1], p1[2] };
    if (kp.redshift) p2[2] *= zf;
    // ---- D. kick
    const float Tk = jmax0(T);
    const SplIdx<float> sd = spline_index(Tk, kp.drag_Tmin, kp.drag_invdT, kp.n_drag);
    float tau = 0.0f, slope = 0.0f, dta = 0.0f, dtb = 0.0f;
    if (sd.mode != 2 && kp.DsT > 0.0f) {       // one cell record: value, slope, d/da, d/db
        const bool lin = sd.mode == 0;
        const float4* c = kp.adj_drag + (lin ? 2 * sd.i : 0);
        const float4 q0 = __ldg(c), q1 = __ldg(c + 1);
        const float t = lin ? sd.t : 0.0f;
        tau = q0.x + t * q0.y;
        dta = q0.z + t * q0.w;
        dtb = q1.x + t * q1.y;
        slope = lin ? q1.z : 0.0f;
    }
    const bool ok = tau > 0.0f && isfinite(tau);
    float E1 = 0.0f, xk = 0.0f, a = 1.0f, q = 0.0f, amp = 0.0f;
    float p3[3] = { p2[0], p2[1], p2[2] };
    if (ok) {
        E1 = sqrtf(p2[0] * p2[0] + p2[1] * p2[1] + p2[2] * p2[2] + m * m);
        xk = (m / (E1 * tau)) * dt;
        const float em1 = expm1_neg(xk);
        a = 1.0f + em1;
        q = -em1 * (2.0f + em1);
        amp = (dt > 0.0f && xk > 0.0f) ? sqrtf(Tk * E1 * q) : 0.0f;
#pragma unroll
        for (int d = 0; d < 3; ++d) p3[d] = p2[d] + em1 * p2[d] + amp * xi[d];
    }
    // ---- E. RTA with the recorded indicator
    bool col = false;
    if (kp.collision == COLL_LANGEVIN_RTA && kp.rta_bits && s >= kp.rta_first && s < kp.rta_first + kp.rta_steps)
        col = (kp.rta_bits[((s - kp.rta_first) >> 5) * kp.n + i] >> ((s - kp.rta_first) & 31)) & 1u;
    float p4[3] = { p3[0], p3[1], p3[2] }, gh[3] = { 0.0f, 0.0f, 0.0f }, dpsT = 0.0f;
    if (col) {
        const uint4 w = philox_words(nk.rk, nk.pid, (uint32_t)s, TAG_RTA);
        const float pstar = invcdf_lookup_dT(kp, w.x, Tk, dpsT);
        float gv[3];
        box_muller(w.y, w.z, gv[0], gv[1]);
        gv[2] = norm_inv(w.w, 0.0f);
        const float n2 = gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2];
        const float inv = 1.0f / sqrtf(n2 > 1e-30f ? n2 : 1e-30f);
#pragma unroll
        for (int d = 0; d < 3; ++d) { gh[d] = gv[d] * inv; p4[d] = pstar * gh[d]; }
    }
    // ---- F. lab boost
    float p5[3], E4 = 0.0f;
    if (flow) boost_fwd(1.0f, p4, m, ux, uy, c, p5, E4);
    else { p5[0] = p4[0]; p5[1] = p4[1]; p5[2] = p4[2]; }
    // ---- G. streaming
    const float E5 = sqrtf(p5[0] * p5[0] + p5[1] * p5[1] + p5[2] * p5[2] + m * m);
    const float iE5 = 1.0f / E5;

    // partials shared by the cotangents
    const float iE0 = flow ? 1.0f / E0 : 0.0f, iE4 = flow ? 1.0f / E4 : 0.0f;
    const float iE1 = ok ? 1.0f / E1 : 0.0f, itau = ok ? 1.0f / tau : 0.0f;
    const float aaxq = (ok && q > 0.0f) ? amp * a * a * xk / q : 0.0f;     // amp a^2 x / q
    const float da_dE1 = a * xk * iE1;
    const float damp_dE1 = (0.5f * amp - aaxq) * iE1;
    const float da_dtau = a * xk * itau;
    const float damp_dtau = -aaxq * itau;
    const float damp_dT = (ok && Tk > 0.0f) ? 0.5f * amp / Tk : 0.0f;
#pragma unroll
    for (int o = 0; o < NC; ++o) {
        // G^T
        float b[3] = { lp[o][0], lp[o][1], lp[o][2] };
        const float tx = (lx[o][0] * p5[0] + lx[o][1] * p5[1]) * iE5 * iE5;
        b[0] += dt * iE5 * (lx[o][0] - tx * p5[0]);
        b[1] += dt * iE5 * (lx[o][1] - tx * p5[1]);
        b[2] += dt * iE5 * (-tx * p5[2]);
        // F^T
        float ub[2] = { 0.0f, 0.0f };
        float b4[3];
        if (flow) boost_vjp(1.0f, p4, E4, iE4, ux, uy, gam, c, b, b4, ub);
        else { b4[0] = b[0]; b4[1] = b[1]; b4[2] = b[2]; }
        // E^T
        float Tb = 0.0f, b3[3];
        if (col) {
            Tb += (b4[0] * gh[0] + b4[1] * gh[1] + b4[2] * gh[2]) * dpsT;
            b3[0] = b3[1] = b3[2] = 0.0f;
        } else {
            b3[0] = b4[0]; b3[1] = b4[1]; b3[2] = b4[2];
        }
        // D^T
        float b2[3] = { b3[0], b3[1], b3[2] };
        if (ok) {
            const float Sa = b3[0] * p2[0] + b3[1] * p2[1] + b3[2] * p2[2];
            const float Sx = b3[0] * xi[0] + b3[1] * xi[1] + b3[2] * xi[2];
            const float cE = (Sa * da_dE1 + Sx * damp_dE1) * iE1;
#pragma unroll
            for (int d = 0; d < 3; ++d) b2[d] = a * b3[d] + cE * p2[d];
            const float taub = Sa * da_dtau + Sx * damp_dtau;
            g[o][0] += taub * dta;
            g[o][1] += taub * dtb;
            Tb += Sx * damp_dT + taub * slope;
        }
        // C^T
        float b1[3] = { b2[0], b2[1], kp.redshift ? b2[2] * zf : b2[2] };
        // B^T
        float b0[3];
        if (flow) boost_vjp(-1.0f, ps, E0, iE0, ux, uy, gam, c, b1, b0, ub);
        else { b0[0] = b1[0]; b0[1] = b1[1]; b0[2] = b1[2]; }
        // T = s Tf, Tk = max(T, 0)
        if (!(T > 0.0f)) Tb = 0.0f;
        g[o][2] += Tb * Tf;
        const float Tfb = Tb * sc;
        // u = g V: the cotangent of the velocity is g ub + g^3 V (ub . V)
        const float uV = gam * gam * gam * (ub[0] * vx + ub[1] * vy);
        const float vb0 = gam * ub[0] + uV * vx, vb1 = gam * ub[1] + uV * vy;
        // A^T
        lx[o][0] += Tfb * dT[0] + vb0 * dux[0] + vb1 * duy[0];
        lx[o][1] += Tfb * dT[1] + vb0 * dux[1] + vb1 * duy[1];
        lp[o][0] = b0[0]; lp[o][1] = b0[1]; lp[o][2] = b0[2];
    }
}

// The observables of the final (lab) momentum and their gradients in (p_x, p_y).
__device__ __forceinline__ void final_observables(double px, double py, double cut, double width, double (&ov)[3],
                                                  double (&dx)[3], double (&dy)[3])
{
    const double pt2 = px * px + py * py, pt = sqrt(pt2);
    const double sig = 1.0 / (1.0 + exp(-(pt - cut) / width));
    ov[0] = pt;
    ov[1] = pt2 > 0.0 ? (px * px - py * py) / pt2 : 0.0;
    ov[2] = sig;
    const double ex = pt > 0.0 ? px / pt : 0.0, ey = pt > 0.0 ? py / pt : 0.0;
    const double ip4 = pt2 > 0.0 ? 1.0 / (pt2 * pt2) : 0.0;
    const double ds = sig * (1.0 - sig) / width;
    dx[0] = ex; dy[0] = ey;
    dx[1] = 4.0 * px * py * py * ip4; dy[1] = -4.0 * px * px * py * ip4;
    dx[2] = ds * ex; dy[2] = ds * ey;
}

}  // namespace

// Recomputes steps [s0, s1) from the checkpoint the parameters point at, taping them.
template <int MED>
__global__ void __launch_bounds__(256, 4)
k_tape(const KParams<float> kp, int64_t s0, int64_t s1)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kp.n) return;
    cart_particle<2, false, float, MED, 2, 3>(kp, kp.rk, i, s0, s1);
}

// The two cotangents the reverse sweep starts from (lam[(o*5 + c)*n + i], c = x0, x1,
// p0, p1, p2): the unit vectors of the final p_x and p_y; gacc[(o*3 + k)*n + i] zeroed.
__global__ void __launch_bounds__(kAdjBlock)
k_adjoint_seed(const KParams<float> kp, const AdjointArgs aa)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = kp.n;
    if (i >= n) return;
#pragma unroll
    for (int o = 0; o < kAdjCot; ++o) {
        float* l = aa.lam + (size_t)o * 5 * n + i;
        l[0] = 0.0f; l[n] = 0.0f; l[2 * n] = o == 0 ? 1.0f : 0.0f; l[3 * n] = o == 1 ? 1.0f : 0.0f; l[4 * n] = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) aa.gacc[(size_t)(o * 3 + k) * n + i] = 0.0;
    }
}

// Steps [s0, s1) backwards from the tape (index s - s0).
// At most 102 registers (five 128-thread blocks per SM): 6 % faster than the natural
// 124 on the 2+1D workload.
template <int MED>
__global__ void __launch_bounds__(kAdjBlock, 5)
k_adjoint_rev(const KParams<float> kp, const AdjointArgs aa, int64_t s0, int64_t s1)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = kp.n;
    if (i >= n) return;
    float lx[kAdjCot][2], lp[kAdjCot][3];
    float g[kAdjCot][3];                  // this segment's parameter sums (FP32), added to FP64 at the end
#pragma unroll
    for (int o = 0; o < kAdjCot; ++o) {
        const float* l = aa.lam + (size_t)o * 5 * n + i;
        lx[o][0] = l[0]; lx[o][1] = l[n]; lp[o][0] = l[2 * n]; lp[o][1] = l[3 * n]; lp[o][2] = l[4 * n];
#pragma unroll
        for (int k = 0; k < 3; ++k) g[o][k] = 0.0f;
    }
    const NoiseKey nk{ kp.rk, (uint32_t)(kp.pid_offset + i) };
    const StepRec<float>* __restrict__ tab = (const StepRec<float>*)kp.steps - kp.step_base;
    constexpr int rows = tape_rows(MED);
    const float4* t = reinterpret_cast<const float4*>(kp.tape) + (size_t)(s1 - 1 - s0) * rows * n + i;
    // the next (earlier) step's first two rows are loaded while the current step is
    // differentiated
    float4 na = __ldg(t), nb = __ldg(t + n);
    for (int64_t s = s1 - 1; s >= s0; --s) {
        const float4 ta = na, tb = nb;
        MedGrad mg;
        float ps[3];
        if (MED == MED_GRID) {
            const float4 tc = __ldg(t + 2 * n), td = __ldg(t + 3 * n);
            ps[0] = ta.x; ps[1] = ta.y; ps[2] = ta.z;
            mg.T = ta.w; mg.vx = tb.w; mg.vy = tc.x;
            mg.dT[0] = tc.y; mg.dT[1] = tc.z; mg.dvx[0] = tc.w;
            mg.dvx[1] = td.x; mg.dvy[0] = td.y; mg.dvy[1] = td.z;
        } else {
            ps[0] = ta.z; ps[1] = ta.w; ps[2] = tb.x;
            mg.T = tab[s].T_bj; mg.vx = mg.vy = 0.0f;
            mg.dT[0] = mg.dT[1] = mg.dvx[0] = mg.dvx[1] = mg.dvy[0] = mg.dvy[1] = 0.0f;
        }
        const float xib[3] = { MED == MED_GRID ? tb.x : tb.y, MED == MED_GRID ? tb.y : tb.z,
                               MED == MED_GRID ? tb.z : tb.w };
        if (s > s0) {
            t -= (size_t)rows * n;
            na = __ldg(t);
            nb = __ldg(t + n);
        }
        adjoint_step<MED, kAdjCot>(kp, s, i, nk, mg, (float)tab[s].zf, ps, xib, lx, lp, g);
    }
#pragma unroll
    for (int o = 0; o < kAdjCot; ++o) {
        float* l = aa.lam + (size_t)o * 5 * n + i;
        l[0] = lx[o][0]; l[n] = lx[o][1]; l[2 * n] = lp[o][0]; l[3 * n] = lp[o][1]; l[4 * n] = lp[o][2];
#pragma unroll
        for (int k = 0; k < 3; ++k) aa.gacc[(size_t)(o * 3 + k) * n + i] += (double)g[o][k];
    }
}

// Per particle: the observables and d obs_o / d theta_k = (d obs_o / d p_x) d p_x / d theta_k
// + (d obs_o / d p_y) d p_y / d theta_k; block sums in FP64 into partials[0..11].
__global__ void __launch_bounds__(kAdjBlock)
k_adjoint_gsum(const KParams<float> kp, const AdjointArgs aa)
{
    __shared__ double sh[kAdjBlock / 32][kAdjOut];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = kp.n;
    double v[kAdjOut];
#pragma unroll
    for (int k = 0; k < kAdjOut; ++k) v[k] = 0.0;
    if (i < n) {
        double ov[3], dx[3], dy[3];
        final_observables(kp.p[0][i], kp.p[1][i], aa.cut, aa.width, ov, dx, dy);
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            v[o] = ov[o];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                v[3 + 3 * o + k] = dx[o] * aa.gacc[(size_t)k * n + i] + dy[o] * aa.gacc[(size_t)(3 + k) * n + i];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kAdjOut; ++k) {
        double t = v[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
        if (lane == 0) sh[warp][k] = t;
    }
    __syncthreads();
    if (threadIdx.x < kAdjOut) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w][threadIdx.x];
        aa.partials[(size_t)blockIdx.x * kAdjOut + threadIdx.x] = t;
    }
}

// Fixed-order total of the block partials: one warp per output, lane-strided sums
// combined by a fixed shuffle tree.
__global__ void k_adjoint_total(const double* __restrict__ partials, int64_t nblocks, double* out)
{
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= kAdjOut) return;
    double t = 0.0;
    for (int64_t b = lane; b < nblocks; b += 32) t += partials[b * kAdjOut + k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    if (lane == 0) out[k] = t;
}

static unsigned blocks_of(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

cudaError_t launch_adjoint_seed(const KParams<float>& kp, const AdjointArgs& aa, cudaStream_t st)
{
    if (kp.n == 0) return cudaSuccess;
    k_adjoint_seed<<<blocks_of(kp.n, kAdjBlock), kAdjBlock, 0, st>>>(kp, aa);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_tape(const KParams<float>& kp, int64_t s0, int64_t s1, cudaStream_t st)
{
    if (kp.n == 0) return cudaSuccess;
    if (kp.med.kind == MED_GRID) k_tape<MED_GRID><<<blocks_of(kp.n, 256), 256, 0, st>>>(kp, s0, s1);
    else if (kp.med.kind == MED_BJORKEN) k_tape<MED_BJORKEN><<<blocks_of(kp.n, 256), 256, 0, st>>>(kp, s0, s1);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_adjoint_rev(const KParams<float>& kp, const AdjointArgs& aa, int64_t s0, int64_t s1, cudaStream_t st)
{
    if (kp.n == 0) return cudaSuccess;
    if (kp.med.kind == MED_GRID) k_adjoint_rev<MED_GRID><<<blocks_of(kp.n, kAdjBlock), kAdjBlock, 0, st>>>(kp, aa, s0, s1);
    else if (kp.med.kind == MED_BJORKEN)
        k_adjoint_rev<MED_BJORKEN><<<blocks_of(kp.n, kAdjBlock), kAdjBlock, 0, st>>>(kp, aa, s0, s1);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_adjoint_total(const KParams<float>& kp, const AdjointArgs& aa, double* out, cudaStream_t st)
{
    const int64_t n = kp.n;
    const int64_t nb = n > 0 ? (int64_t)blocks_of(n, kAdjBlock) : 0;
    if (nb == 0) return cudaMemsetAsync(out, 0, kAdjOut * sizeof(double), st);
    k_adjoint_gsum<<<(unsigned)nb, kAdjBlock, 0, st>>>(kp, aa);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_adjoint_total<<<1, 32 * kAdjOut, 0, st>>>(aa.partials, nb, out);
    return cudaGetLastError();
}

}  // namespace lim

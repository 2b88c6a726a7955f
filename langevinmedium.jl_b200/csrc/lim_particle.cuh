// lim_particle.cuh — one particle through a range of Cartesian steps: state loaded
// once, every step of the range evolved in registers, state stored once.  Shared by
// the plain step kernel (one ensemble per launch) and the batched persistent kernel
// (many ensembles per launch, parameters staged in shared memory).
#pragma once
#include "lim_step.cuh"

namespace lim {

template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ void load_state(const KParams<R>& kp, int64_t i, R (&x)[3], float (&xl)[3], double (&p)[3])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) { x[d] = R(0); xl[d] = 0.f; p[d] = 0.0; }
#pragma unroll
    for (int d = 0; d < DIMS; ++d) {
        x[d] = kp.x[d][i];
        if (sizeof(R) == 4) xl[d] = kp.xlo[d][i];
    }
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p[d] = kp.p[d][i];
}

template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ void store_state(const KParams<R>& kp, int64_t i, const R (&x)[3], const float (&xl)[3], const double (&p)[3])
{
#pragma unroll
    for (int d = 0; d < DIMS; ++d) {
        kp.x[d][i] = x[d];
        if (sizeof(R) == 4) kp.xlo[d][i] = xl[d];
    }
#pragma unroll
    for (int d = 0; d < PDIM; ++d) kp.p[d][i] = p[d];
}

// Every component of the state is finite (the Milne kernel's test).
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ bool state_finite_all(const R (&x)[3], const double (&p)[3])
{
    bool ok = true;
#pragma unroll
    for (int d = 0; d < DIMS; ++d) ok &= (bool)isfinite(x[d]);
#pragma unroll
    for (int d = 0; d < PDIM; ++d) ok &= (bool)isfinite(p[d]);
    return ok;
}

// The Cartesian state after a step is finite.  In relativistic runs the position
// decides: the step's streaming moves x by dt p / E with E = sqrt(m^2 + p.p) over every
// momentum component, so a non-finite momentum makes x non-finite in the same step
// (NaN or Inf in p gives NaN in p / E).  Galilean streaming divides by m and never sees
// the components beyond DIMS, so there the momentum is checked as well.
template <typename R, int DIMS, int PDIM>
__device__ __forceinline__ bool state_finite(const KParams<R>& kp, const R (&x)[3], const double (&p)[3])
{
    bool ok = true;
#pragma unroll
    for (int d = 0; d < DIMS; ++d) ok &= (bool)isfinite(x[d]);
    if (!kp.rel) {
#pragma unroll
        for (int d = 0; d < PDIM; ++d) ok &= (bool)isfinite(p[d]);
    }
    return ok;
}

// Steps [s0, s1) of particle i.  rk: the Philox round keys (kernel-parameter
// constants in both kernels); kp: the ensemble's parameters.
template <int REC, bool FO, typename R, int MED, int DIMS, int PDIM>
__device__ __forceinline__ void cart_particle(const KParams<R>& kp, const uint2* __restrict__ rk, int64_t i,
                                              int64_t s0, int64_t s1)
{
    R x[3];
    double p[3];
    float xl[3];
    load_state<R, DIMS, PDIM>(kp, i, x, xl, p);
    bool frozen = false, have_last = false;
    double ltau = 0.0, lT = 0.0;
    LatchPos<R> lpos;
    LatchMom<R> lmom;
#pragma unroll
    for (int d = 0; d < 3; ++d) { lpos.h[d] = R(0); lmom.m[d] = 0.0; }
    if (FO) {
        // the latch state of the previous launch: l_T = 0 until a particle has a last-above
        // state (FP32 runs hold -1 there; their last-above state is the state itself)
        frozen = kp.fo_flag[i] != 0.0;
        lT = kp.l_T[i];
        have_last = lT != 0.0;
        if (sizeof(R) == 8) {
            ltau = kp.l_tau[i];
#pragma unroll
            for (int d = 0; d < DIMS; ++d) lpos.h[d] = (R)kp.l_pos[d][i];
#pragma unroll
            for (int d = 0; d < PDIM; ++d) lmom.m[d] = kp.l_mom[d][i];
        }
    }
    const NoiseKey nk{ rk, (uint32_t)(kp.pid_offset + i) };
    const StepRec<R>* __restrict__ tab = (const StepRec<R>*)kp.steps - kp.step_base;
    // FP32 grid runs with the freeze-out latch: one spatial lookup per step, at the end
    // of the step at the new position on the next step's time row, serves both the next
    // step (its medium, blended in time at once into rows.T0, U0, V0) and the latch's
    // screen (rows.T1).  The first step's medium is looked up here, and the last step of
    // a launch looks up its own time row for the screen only; every step takes its
    // medium from the same code whether or not a launch boundary falls before it, so a
    // run split into more launches gives the same bits.
    constexpr bool kCarry = FO && MED == MED_GRID && sizeof(R) == 4;
    GridRows<R> rows;
    rows.kt = -1;
    GridRows<R>* carry = kCarry ? &rows : nullptr;
    if (kCarry && s0 < s1) {
        grid_rows(kp.med, tab[s0].kt, x[0], x[1], rows, xl[0], xl[1]);
        const R w0 = tab[s0].wt;
        grid_combine(rows, w0, rows.T0, rows.U0, rows.V0);
    }
    // the lab momentum rounded to FP32, as streaming leaves it at the end of each step: the
    // FP32 grid kernel's next step starts its frame change from it (the same values as
    // rounding p again)
    float pf[3] = { 0.0f, 0.0f, 0.0f };
#pragma unroll
    for (int d = 0; d < PDIM; ++d) pf[d] = (float)p[d];
    // steps lie in [0, 2^32) (lim_run checks): a 32-bit loop counter
    const uint32_t se = (uint32_t)s1;
    for (uint32_t s = (uint32_t)s0; s < se; ++s) {
        if (FO && kp.stop_fo && frozen) break;
        const StepRec<R> sr = tab[s];
        if (REC == 2 && MED != MED_GRID) {   // the adjoint's tape: the pre-step state (the normals follow)
            float4* t = reinterpret_cast<float4*>(kp.tape) + (s - kp.tape_first) * 2 * kp.n + i;
            *t = make_float4((float)x[0], (float)x[1], (float)p[0], (float)p[1]);
            reinterpret_cast<float*>(t + kp.n)[0] = (float)p[2];
        }
        // FP32 latch: the state the step starts from is the last-above record
        R xp[3];
        float xlp[3], pfp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) { xp[d] = x[d]; xlp[d] = xl[d]; pfp[d] = pf[d]; }
        cart_step<REC, R, MED, DIMS, PDIM, kCarry>(kp, sr, i, s, nk, x, xl, p, carry, FO && sizeof(R) == 4 ? pf : nullptr);
        if constexpr (kCarry) {
            const bool more = s + 1 < s1;
            int kn = sr.kt;
            R wn = R(0);
            if (more) { kn = tab[s + 1].kt; wn = tab[s + 1].wt; }
            grid_rows(kp.med, kn, x[0], x[1], rows, xl[0], xl[1]);
            const float scr = kn == sr.kt ? (float)lerp_rn(rows.T0, rows.T1, sr.wt) * (float)kp.med.T_scale : -1.0f;
            if (more) grid_combine(rows, wn, rows.T0, rows.U0, rows.V0);
            rows.T1 = scr;
        }
        if constexpr (FO && sizeof(R) == 4) {
            freezeout_latch_pre<R, MED, DIMS, PDIM>(kp, sr, i, s, x, xl, p, xp, xlp, pfp, frozen, have_last, carry);
        } else if constexpr (FO) {
            freezeout_latch<R, MED, DIMS, PDIM>(kp, sr, i, x, p, frozen, lpos, lmom, ltau, lT);
        }
        if (!state_finite<R, DIMS, PDIM>(kp, x, p)) {
            atomicMin(kp.first_bad, (unsigned long long)s);
            break;
        }
    }
    store_state<R, DIMS, PDIM>(kp, i, x, xl, p);
    if constexpr (FO && sizeof(R) == 4) {
        kp.l_T[i] = have_last ? -1.0 : 0.0;      // the record is the state itself (freezeout_latch_pre)
    } else if constexpr (FO) {
        kp.l_tau[i] = ltau;
        kp.l_T[i] = lT;
#pragma unroll
        for (int d = 0; d < DIMS; ++d) kp.l_pos[d][i] = lpos.at(d);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) kp.l_mom[d][i] = lmom.at(d);
    }
}

}  // namespace lim

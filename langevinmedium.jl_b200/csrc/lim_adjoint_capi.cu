// lim_adjoint_capi.cu — lim_adjoint (include/langevin_b200.h): checkpointed forward
// pass, then the reverse sweep of lim_adjoint.cu segment by segment.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>
#include "lim_ctx.h"

using namespace lim;

#define LIM_ACUDA(ctx, call)                                                                          \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return ctx_fail((ctx), LIM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));    \
    } while (0)

namespace {

int check_adjoint_config(lim_ctx* c)
{
    const lim_params& P = c->P;
    if (P.precision != LIM_FP32) return ctx_fail(c, LIM_ERR_UNSUPPORTED, "lim_adjoint: FP32 state only");
    if (P.coords != LIM_COORDS_CARTESIAN || c->dims != 2 || c->pdim != 3)
        return ctx_fail(c, LIM_ERR_UNSUPPORTED, "lim_adjoint: Cartesian coordinates with dimensions=2, momentum_dimensions=3");
    if (c->med_kind != MED_GRID && c->med_kind != MED_BJORKEN)
        return ctx_fail(c, LIM_ERR_UNSUPPORTED, "lim_adjoint: the 2+1D grid or the analytic Bjorken medium");
    if (P.collision != LIM_COLL_LANGEVIN && P.collision != LIM_COLL_LANGEVIN_RTA)
        return ctx_fail(c, LIM_ERR_UNSUPPORTED, "lim_adjoint: collision :langevin or :langevin_rta");
    if (!P.relativistic || P.integrator_mode != 0 || P.position_diffusion || P.reflecting_boundary || P.freezeout_capture)
        return ctx_fail(c, LIM_ERR_UNSUPPORTED, "lim_adjoint: relativistic pre-point steps without position diffusion, "
                                                 "reflection or freeze-out");
    if (!(P.DsT > 0)) return ctx_fail(c, LIM_ERR_UNSUPPORTED, "lim_adjoint: needs DsT > 0");
    for (int w = 2; w < 4; ++w)
        if (c->spl[w].size() != c->spl[0].size() || c->spl_Tmin[w] != c->spl_Tmin[0] || c->spl_invdT[w] != c->spl_invdT[0])
            return ctx_fail(c, LIM_ERR_STATE, "lim_adjoint: set LIM_SPLINE_DRAG_DA and _DB on the drag spline's grid");
    if (!(P.obs_pt_width > 0)) return ctx_fail(c, LIM_ERR_ARG, "lim_adjoint: obs_pt_width must be > 0");
    return LIM_OK;
}

}  // namespace

extern "C" {

int lim_adjoint(lim_ctx* c, int64_t first_step, int64_t nsteps, int64_t checkpoint_every, double* obs, double* grad)
{
    if (!c) return LIM_ERR_ARG;
    int rc = ctx_check_ready(c);
    if (rc) return rc;
    if ((rc = check_adjoint_config(c))) return rc;
    if (first_step < 0 || nsteps < 1 || checkpoint_every < 1)
        return ctx_fail(c, LIM_ERR_ARG, "lim_adjoint: need first_step >= 0, nsteps >= 1, checkpoint_every >= 1");
    if (first_step + nsteps > (int64_t)UINT32_MAX) return ctx_fail(c, LIM_ERR_ARG, "lim_adjoint: steps beyond 2^32 - 1");
    cudaSetDevice(c->device);
    const int64_t n = c->n, K = checkpoint_every, nseg = (nsteps + K - 1) / K;
    // record the RTA decisions of this run; the reverse sweep replays them
    if ((rc = lim_rta_decisions(c, 1, first_step, nsteps))) return rc;
    KParams<float> kp;
    if ((rc = ctx_build_kparams<float>(c, kp))) return rc;
    const size_t seg_bytes = (size_t)n * (4 * sizeof(float) + 3 * sizeof(double));
    const size_t nn = (size_t)std::max<int64_t>(n, 1);
    if ((rc = ctx_alloc(c, c->d_adj_ckpt, std::max<size_t>(seg_bytes * (size_t)nseg, 16)))) return rc;
    if ((rc = ctx_alloc(c, c->d_adj_tape, (size_t)std::min(K, nsteps) * tape_rows(c->med_kind) * nn * sizeof(float4))))
        return rc;
    if ((rc = ctx_alloc(c, c->d_adj_table, (size_t)nsteps * step_record_bytes<float>()))) return rc;
    const int64_t nblocks = std::max<int64_t>((n + kAdjBlock - 1) / kAdjBlock, 1);
    if ((rc = ctx_alloc(c, c->d_adj_part, (size_t)nblocks * kAdjOut * sizeof(double)))) return rc;
    if ((rc = ctx_alloc(c, c->d_adj_out, kAdjOut * sizeof(double)))) return rc;
    if ((rc = ctx_alloc(c, c->d_adj_lam, kAdjCot * 5 * nn * sizeof(float)))) return rc;
    if ((rc = ctx_alloc(c, c->d_adj_gacc, kAdjCot * 3 * nn * sizeof(double)))) return rc;
    // slopes of the tabulated functions, differenced in FP64 (FP32 node differences
    // lose ~eps / (relative step) to cancellation)
    {
        // per drag cell: (tau_i, tau_i+1 - tau_i, a_i, a_i+1 - a_i), (b_i, b_i+1 - b_i, slope_i, 0)
        const std::vector<double>& v = c->spl[0];
        const std::vector<double>& A = c->spl[2];
        const std::vector<double>& B = c->spl[3];
        const size_t cells = std::max<size_t>(v.size(), 2) - 1;
        std::vector<float4> tab(2 * cells);
        for (size_t k = 0; k < cells; ++k) {
            const size_t k1 = std::min(k + 1, v.size() - 1);
            const double dv = v[k1] - v[k], da = A[k1] - A[k], dbv = B[k1] - B[k];
            tab[2 * k] = make_float4((float)v[k], (float)dv, (float)A[k], (float)da);
            tab[2 * k + 1] = make_float4((float)B[k], (float)dbv, (float)(dv * c->spl_invdT[0]), 0.0f);
        }
        if ((rc = ctx_alloc(c, c->d_adj_slope, tab.size() * sizeof(float4)))) return rc;
        LIM_ACUDA(c, cudaMemcpy(c->d_adj_slope.p, tab.data(), tab.size() * sizeof(float4), cudaMemcpyHostToDevice));
        const int64_t nU = c->nU, nT = c->nT;
        std::vector<float> dT((size_t)std::max<int64_t>(nT - 1, 1) * (size_t)std::max<int64_t>(nU, 1), 0.0f);
        if (!c->icdf.empty())
            for (int64_t j = 0; j + 1 < nT; ++j)
                for (int64_t u = 0; u < nU; ++u)
                    dT[(size_t)j * nU + u] = (float)((c->icdf[(size_t)(j + 1) * nU + u] - c->icdf[(size_t)j * nU + u]) * c->ic_invdT);
        if ((rc = ctx_alloc(c, c->d_adj_icdt, dT.size() * sizeof(float)))) return rc;
        LIM_ACUDA(c, cudaMemcpy(c->d_adj_icdt.p, dT.data(), dT.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    LIM_ACUDA(c, cudaMemsetAsync(c->d_status.p, 0xff, sizeof(unsigned long long), c->stream));
    kp.steps = c->d_adj_table.p;
    kp.step_base = first_step;
    kp.step_cap = nsteps;
    kp.adj_drag = (const float4*)c->d_adj_slope.p;
    kp.icdf_dT = (const float*)c->d_adj_icdt.p;
    LIM_ACUDA(c, launch_step_table<float>(kp, 0, first_step, first_step + nsteps, c->stream));
    const int block = c->P.block_size > 0 ? (int)c->P.block_size : 256;
    cudaEvent_t e0 = c->ev0, e1 = c->ev1, e2 = nullptr;
    LIM_ACUDA(c, cudaEventCreate(&e2));
    LIM_ACUDA(c, cudaEventRecord(e0, c->stream));
    // forward: checkpoint, then the segment's steps (one launch per segment: measured
    // faster than one launch that checkpoints from inside, whose extra live values cost
    // occupancy).  The last segment, the first one the reverse sweep needs, is taped
    // directly instead of checkpointed and recomputed.
    const size_t fb = (size_t)n * sizeof(float), db = (size_t)n * sizeof(double);
    for (int64_t seg = 0; seg < nseg; ++seg) {
        if (seg == nseg - 1) {
            const int64_t s0 = first_step + seg * K, s1 = first_step + nsteps;
            KParams<float> kt = kp;
            kt.tape = (float*)c->d_adj_tape.p;
            kt.tape_first = s0;
            LIM_ACUDA(c, launch_adjoint_tape(kt, s0, s1, c->stream));
            break;
        }
        char* cb = (char*)c->d_adj_ckpt.p + (size_t)seg * seg_bytes;
        for (int d = 0; d < 2; ++d) {
            LIM_ACUDA(c, cudaMemcpyAsync(cb + d * fb, kp.x[d], fb, cudaMemcpyDeviceToDevice, c->stream));
            LIM_ACUDA(c, cudaMemcpyAsync(cb + (2 + d) * fb, kp.xlo[d], fb, cudaMemcpyDeviceToDevice, c->stream));
        }
        for (int d = 0; d < 3; ++d)
            LIM_ACUDA(c, cudaMemcpyAsync(cb + 4 * fb + d * db, kp.p[d], db, cudaMemcpyDeviceToDevice, c->stream));
        const int64_t s0 = first_step + seg * K, s1 = std::min(s0 + K, first_step + nsteps);
        LIM_ACUDA(c, launch_steps_in_table<float>(kp, s0, s1, block, c->stream));
    }
    LIM_ACUDA(c, cudaEventRecord(e1, c->stream));
    // reverse sweep: seeds at the final state, then segment by segment from the last
    AdjointArgs aa;
    std::memset(&aa, 0, sizeof aa);
    aa.lam = (float*)c->d_adj_lam.p;
    aa.gacc = (double*)c->d_adj_gacc.p;
    aa.cut = c->P.obs_pt_cut;
    aa.width = c->P.obs_pt_width;
    aa.partials = (double*)c->d_adj_part.p;
    LIM_ACUDA(c, launch_adjoint_seed(kp, aa, c->stream));
    KParams<float> kq = kp;                // the segment's state lives in its checkpoint
    kq.rta_mode = 2;                       // replay the forward pass's RTA decisions
    kq.tape = (float*)c->d_adj_tape.p;
    for (int64_t seg = nseg - 1; seg >= 0; --seg) {
        char* cb = (char*)c->d_adj_ckpt.p + (size_t)seg * seg_bytes;
        for (int d = 0; d < 2; ++d) {
            kq.x[d] = (float*)(cb + d * fb);
            kq.xlo[d] = (float*)(cb + (2 + d) * fb);
        }
        for (int d = 0; d < 3; ++d) kq.p[d] = (double*)(cb + 4 * fb + d * db);
        const int64_t s0 = first_step + seg * K, s1 = std::min(s0 + K, first_step + nsteps);
        kq.tape_first = s0;
        if (seg < nseg - 1) LIM_ACUDA(c, launch_adjoint_tape(kq, s0, s1, c->stream));
        LIM_ACUDA(c, launch_adjoint_rev(kq, aa, s0, s1, c->stream));
    }
    LIM_ACUDA(c, launch_adjoint_total(kp, aa, (double*)c->d_adj_out.p, c->stream));
    LIM_ACUDA(c, cudaEventRecord(e2, c->stream));
    LIM_ACUDA(c, cudaEventSynchronize(e2));
    float f_ms = 0.f, r_ms = 0.f;
    cudaEventElapsedTime(&f_ms, e0, e1);
    cudaEventElapsedTime(&r_ms, e1, e2);
    cudaEventDestroy(e2);
    c->adj_fwd_ms = f_ms;
    c->adj_rev_ms = r_ms;
    c->rta_mode = 2;                       // the run's decisions stay available for replay
    double out[kAdjOut];
    LIM_ACUDA(c, cudaMemcpy(out, c->d_adj_out.p, sizeof out, cudaMemcpyDeviceToHost));
    unsigned long long bad = ULLONG_MAX;
    LIM_ACUDA(c, cudaMemcpy(&bad, c->d_status.p, sizeof bad, cudaMemcpyDeviceToHost));
    if (bad != ULLONG_MAX) return ctx_fail(c, LIM_ERR_NONFINITE, "Breaking simulation due to NaN/Inf at step %llu", bad);
    const double inv = n > 0 ? 1.0 / (double)n : 0.0;
    if (obs) for (int o = 0; o < 3; ++o) obs[o] = out[o] * inv;
    if (grad) for (int k = 0; k < 9; ++k) grad[k] = out[3 + k] * inv;
    return LIM_OK;
}

int lim_adjoint_stats(lim_ctx* c, double* forward_ms, double* reverse_ms)
{
    if (!c) return LIM_ERR_ARG;
    if (forward_ms) *forward_ms = c->adj_fwd_ms;
    if (reverse_ms) *reverse_ms = c->adj_rev_ms;
    return LIM_OK;
}

}  // extern "C"

// lim_capi.cu — the C-ABI (include/langevin_b200.h) over the fused step kernels.
//
// Validation mirrors the reference's errors (check_momentum_dims, utils.jl:561-573;
// collision_mode, simulate_gpu_wrapper.jl:54-55; spline range, transport.jl:182-184).
// No exception crosses the ABI: every entry point returns a status and keeps the
// message for lim_last_error().
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <climits>
#include <new>
#include <string>
#include <vector>
#include "../../include/langevin_b200.h"
#include "../../include/langevin_b200_diag.h"
#include "lim_ctx.h"

using namespace lim;

namespace {

thread_local std::string g_create_error;

}  // namespace

namespace {

int fail(lim_ctx* c, int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf; else g_create_error = buf;
    return code;
}

#define LIM_CUDA(ctx, call)                                                                     \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail((ctx), LIM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

int dev_alloc(lim_ctx* c, DevBuf& b, size_t bytes)
{
    if (b.bytes >= bytes && b.p) return LIM_OK;
    if (b.p) { cudaFree(b.p); b.p = nullptr; b.bytes = 0; }
    if (bytes == 0) return LIM_OK;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return fail(c, LIM_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    b.bytes = bytes;
    return LIM_OK;
}
void dev_free(DevBuf& b)
{
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

template <typename T>
int upload(lim_ctx* c, DevBuf& b, const T* src, size_t count)
{
    int rc = dev_alloc(c, b, count * sizeof(T));
    if (rc) return rc;
    if (count) LIM_CUDA(c, cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));   // the host vectors may be released afterwards
    return LIM_OK;
}

bool all_finite(const double* v, size_t n)
{
    for (size_t i = 0; i < n; ++i) if (!std::isfinite(v[i])) return false;
    return true;
}
bool ascending(const double* v, size_t n)
{
    for (size_t i = 1; i < n; ++i) if (!(v[i] > v[i - 1])) return false;
    return true;
}
// A grid is "uniform" when node k lies within half a spacing of x0 + k h: the
// O(1) guess of the cell search then needs at most one correction step.
bool near_uniform(const std::vector<double>& g, double& x0, double& inv)
{
    size_t n = g.size();
    x0 = g[0];
    double h = (g[n - 1] - g[0]) / (double)(n - 1);
    inv = h > 0 ? 1.0 / h : 0.0;
    if (!(h > 0)) return false;
    for (size_t k = 0; k < n; ++k)
        if (std::fabs(g[k] - (x0 + (double)k * h)) > 0.5 * h) return false;
    return true;
}

int state_rows_ok(lim_ctx* c)
{
    if (!c->have_params) return fail(c, LIM_ERR_STATE, "lim_set_params must be called first");
    return LIM_OK;
}

template <typename R>
int ensure_device_medium(lim_ctx* c)
{
    const int prec = sizeof(R) == 8 ? LIM_FP64 : LIM_FP32;
    if (!c->dev_dirty && c->dev_prec == prec) return LIM_OK;
    int rc;
    if (c->med_kind == MED_RT) {
        size_t nr = c->xg.size(), nt = c->tg.size();
        std::vector<R> xr(nr), tr(nt);
        for (size_t k = 0; k < nr; ++k) xr[k] = (R)c->xg[k];
        for (size_t k = 0; k < nt; ++k) tr[k] = (R)c->tg[k];
        std::vector<R> tv(2 * nr * nt);
        for (size_t k = 0; k < nr * nt; ++k) { tv[2 * k] = (R)c->T[k]; tv[2 * k + 1] = (R)c->V[k]; }
        if ((rc = upload(c, c->d_xg, xr.data(), nr))) return rc;
        if ((rc = upload(c, c->d_tg, tr.data(), nt))) return rc;
        if ((rc = upload(c, c->d_tgd, c->tg.data(), nt))) return rc;
        if ((rc = upload(c, c->d_xgd, c->xg.data(), nr))) return rc;
        if ((rc = upload(c, c->d_TV, tv.data(), tv.size()))) return rc;
        // per-cell records: (T_i, V_i, T_i+1, V_i+1) of each time row, and (x_i, x_i+1)
        std::vector<R> tvc(4 * (nr - 1) * nt), xc(2 * (nr - 1));
        for (size_t j = 0; j < nt; ++j)
            for (size_t i = 0; i + 1 < nr; ++i) {
                R* q = tvc.data() + 4 * (i + (nr - 1) * j);
                q[0] = tv[2 * (i + nr * j)]; q[1] = tv[2 * (i + nr * j) + 1];
                q[2] = tv[2 * (i + 1 + nr * j)]; q[3] = tv[2 * (i + 1 + nr * j) + 1];
            }
        for (size_t i = 0; i + 1 < nr; ++i) { xc[2 * i] = xr[i]; xc[2 * i + 1] = xr[i + 1]; }
        if ((rc = upload(c, c->d_TVc, tvc.data(), tvc.size()))) return rc;
        if ((rc = upload(c, c->d_xc, xc.data(), xc.size()))) return rc;
        if (!c->V2.empty()) {
            std::vector<R> v2(c->V2.size());
            for (size_t k = 0; k < v2.size(); ++k) v2[k] = (R)c->V2[k];
            if ((rc = upload(c, c->d_V2, v2.data(), v2.size()))) return rc;
        }
    } else if (c->med_kind == MED_GRID) {
        size_t nn = (size_t)(c->gnx * c->gny * c->gnt);
        std::vector<float4> g(nn);
        for (size_t k = 0; k < nn; ++k) g[k] = make_float4(c->gT[k], c->gux[k], c->guy[k], 0.f);
        if ((rc = upload(c, c->d_G, g.data(), nn))) return rc;
    }
    for (int w = 0; w < 4; ++w) {
        if (c->spl[w].empty()) continue;
        std::vector<R> s(c->spl[w].size());
        for (size_t k = 0; k < s.size(); ++k) s[k] = (R)c->spl[w][k];
        if ((rc = upload(c, c->d_spl[w], s.data(), s.size()))) return rc;
    }
    if (!c->icdf.empty()) {
        std::vector<R> s(c->icdf.size());
        for (size_t k = 0; k < s.size(); ++k) s[k] = (R)c->icdf[k];
        if ((rc = upload(c, c->d_icdf, s.data(), s.size()))) return rc;
    }
    if (sizeof(R) == 4) {                 // FP64 copies for the FP32 path's near-threshold RTA decisions
        if (!c->spl[1].empty() && (rc = upload(c, c->d_rta64, c->spl[1].data(), c->spl[1].size()))) return rc;
        if (c->med_kind == MED_RT && (rc = upload(c, c->d_T64, c->T.data(), c->T.size()))) return rc;
    }
    c->dev_prec = prec;
    c->dev_dirty = false;
    return LIM_OK;
}

template <typename R>
int build_kparams(lim_ctx* c, KParams<R>& kp)
{
    int rc = ensure_device_medium<R>(c);
    if (rc) return rc;
    std::memset(&kp, 0, sizeof kp);
    const lim_params& P = c->P;
    kp.dt = P.dt; kp.t0 = P.t0;
    kp.m = (R)P.m; kp.DsT = (R)P.DsT; kp.Tfo = (R)P.Tfo; kp.psi2 = (R)P.psi2;
    kp.sqrt_dt = (R)std::sqrt(P.dt); kp.dtR = (R)P.dt;
    kp.rel = P.relativistic != 0; kp.collision = (int)P.collision; kp.redshift = P.bjorken_redshift != 0;
    kp.diffusion = P.position_diffusion != 0; kp.reflect = P.reflecting_boundary != 0;
    kp.integrator = (int)P.integrator_mode; kp.fo_capture = P.freezeout_capture != 0;
    kp.fo_interp = P.freezeout_interp != 0; kp.stop_fo = P.stop_after_freezeout != 0 && P.freezeout_capture != 0;
    kp.seed_lo = (uint32_t)(uint64_t)P.seed; kp.seed_hi = (uint32_t)((uint64_t)P.seed >> 32);
    {
        uint32_t k0 = kp.seed_lo, k1 = kp.seed_hi;       // Philox-4x32-10 key schedule
        for (int r = 0; r < 10; ++r) { kp.rk[r] = make_uint2(k0, k1); k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
    kp.pid_offset = P.particle_offset;
    kp.n = c->n; kp.dims = c->dims; kp.pdim = c->pdim;
    kp.drag = (const R*)c->d_spl[0].p; kp.n_drag = (int)c->spl[0].size();
    kp.drag_Tmin = (R)c->spl_Tmin[0]; kp.drag_invdT = (R)c->spl_invdT[0];
    kp.rta = (const R*)c->d_spl[1].p; kp.n_rta = (int)c->spl[1].size();
    kp.rta_Tmin = (R)c->spl_Tmin[1]; kp.rta_invdT = (R)c->spl_invdT[1];
    if (sizeof(R) == 4) {
        // A spline whose whole T range is narrower than FP32 resolves (the drivers build
        // [Tmin, Tmin + eps] for a uniform field, simulate_cpu.jl:191-192) is a constant
        // to FP32 accuracy; evaluating it as one avoids extrapolating over ~1e11 cells.
        for (int w = 0; w < 2; ++w) {
            const size_t n = c->spl[w].size();
            if (n >= 2) {
                const double width = (double)(n - 1) / c->spl_invdT[w];
                if (std::fabs(width) <= 1e-6 * std::fabs(c->spl_Tmin[w])) {
                    if (w == 0) kp.n_drag = 1; else kp.n_rta = 1;
                }
            }
        }
    }
    kp.spl_shared = kp.n_drag == kp.n_rta && kp.drag_Tmin == kp.rta_Tmin && kp.drag_invdT == kp.rta_invdT;
    kp.drag_da = c->spl[2].empty() ? nullptr : (const R*)c->d_spl[2].p;
    kp.drag_db = c->spl[3].empty() ? nullptr : (const R*)c->d_spl[3].p;
    kp.rta_bits = (uint32_t*)c->d_rta_bits.p;
    kp.rta_mode = c->d_rta_bits.p ? c->rta_mode : 0;
    kp.rta_first = c->rta_first;
    kp.rta_steps = c->rta_steps;
    if (sizeof(R) == 4) {
        kp.rta64 = c->spl[1].empty() ? nullptr : (const double*)c->d_rta64.p;
        kp.rta_Tmin64 = c->spl_Tmin[1];
        kp.rta_invdT64 = c->spl_invdT[1];
        kp.n_rta64 = (int)c->spl[1].size();
        kp.T64 = c->med_kind == MED_RT ? (const double*)c->d_T64.p : nullptr;
    }
    kp.icdf = (const R*)c->d_icdf.p; kp.nU = (int)c->nU; kp.nT = (int)c->nT;
    kp.ic_Tmin = (R)c->ic_Tmin; kp.ic_invdT = (R)c->ic_invdT;
    MediumDev<R>& md = kp.med;
    md.kind = c->med_kind;
    md.T_scale = (R)c->T_scale;
    if (c->med_kind == MED_RT) {
        md.xg = (const R*)c->d_xg.p; md.tg = (const R*)c->d_tg.p; md.tgd = (const double*)c->d_tgd.p;
        md.xgd = (const double*)c->d_xgd.p;
        md.nr = (int)c->xg.size(); md.nt = (int)c->tg.size();
        double x0, xi, t0g, ti;
        md.x_uniform = near_uniform(c->xg, x0, xi); md.xg0 = (R)x0; md.xinvd = (R)xi;
        md.t_uniform = near_uniform(c->tg, t0g, ti); md.tg0 = t0g; md.tinvd = ti;
        md.TV = (const typename V2T<R>::type*)c->d_TV.p;
        md.TVc = (const typename V4T<R>::type*)c->d_TVc.p;
        md.xc = (const typename V2T<R>::type*)c->d_xc.p;
        md.xlo = (R)c->xg.front(); md.xhi = (R)c->xg.back();
        md.V2 = (const R*)c->d_V2.p; md.use_v2 = !c->V2.empty();
        md.r_max = (R)c->xg.back();
        md.r_axis_eps = (R)std::max(1e-12, 0.5 * std::fabs(c->xg[1] - c->xg[0]));
    } else if (c->med_kind == MED_BJORKEN) {
        md.bj_T0 = c->bj_T0; md.bj_tau0 = c->bj_tau0; md.bj_power = c->bj_power;
        md.r_max = (R)c->bj_rmax; md.r_axis_eps = (R)1e-6;
    } else {
        md.G = (const float4*)c->d_G.p;
        md.gnx = (int)c->gnx; md.gny = (int)c->gny; md.gnt = (int)c->gnt;
        md.gx0_d = c->gx0; md.gdx_d = c->gdx; md.gxl_d = c->gx0 + (double)(c->gnx - 1) * c->gdx;
        md.gy0_d = c->gy0; md.gdy_d = c->gdy; md.gyl_d = c->gy0 + (double)(c->gny - 1) * c->gdy;
        md.ginvdx = (float)(1.0 / c->gdx); md.ginvdy = (float)(1.0 / c->gdy);
        md.ginvdx_lo = (float)(1.0 / c->gdx - (double)md.ginvdx);
        md.ginvdy_lo = (float)(1.0 / c->gdy - (double)md.ginvdy);
        md.gicx = (int)((c->gnx - 1) / 2); md.gicy = (int)((c->gny - 1) / 2);
        const double xcd = c->gx0 + (double)md.gicx * c->gdx, ycd = c->gy0 + (double)md.gicy * c->gdy;
        md.gxc = (float)xcd; md.gxcl = (float)(xcd - (double)md.gxc);
        md.gyc = (float)ycd; md.gycl = (float)(ycd - (double)md.gyc);
        md.gt0 = c->gt0; md.gdt_d = c->gdt; md.gtl = c->gt0 + (double)(c->gnt - 1) * c->gdt;
        double r = std::fabs(md.gx0_d);
        r = std::min(r, std::fabs(md.gxl_d)); r = std::min(r, std::fabs(md.gy0_d)); r = std::min(r, std::fabs(md.gyl_d));
        md.r_max = (R)r; md.r_axis_eps = (R)1e-6;
    }
    for (int d = 0; d < 3; ++d) {
        kp.x[d] = (R*)c->d_x[d].p; kp.xlo[d] = (float*)c->d_xlo[d].p; kp.p[d] = (double*)c->d_p[d].p;
        kp.fo_pos[d] = (double*)c->d_fo_pos[d].p; kp.fo_mom[d] = (double*)c->d_fo_mom[d].p;
        kp.l_pos[d] = (double*)c->d_l_pos[d].p; kp.l_mom[d] = (double*)c->d_l_mom[d].p;
    }
    kp.fo_tau = (double*)c->d_fo_tau.p; kp.fo_flag = (double*)c->d_fo_flag.p;
    kp.l_tau = (double*)c->d_l_tau.p; kp.l_T = (double*)c->d_l_T.p;
    kp.first_bad = (unsigned long long*)c->d_status.p;
    kp.rec = (double*)c->d_rec.p; kp.rec_first = c->rec_first; kp.rec_steps = c->d_rec.p ? c->rec_steps : 0;
    return LIM_OK;
}

int check_ready(lim_ctx* c)
{
    if (!c->have_params) return fail(c, LIM_ERR_STATE, "lim_set_params must be called before running");
    if (c->med_kind < 0) return fail(c, LIM_ERR_STATE, "no medium set (lim_set_medium_rt/_bjorken/_grid)");
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "no particle state uploaded (lim_upload_state)");
    if (c->P.coords == LIM_COORDS_MILNE && c->med_kind != MED_RT)
        return fail(c, LIM_ERR_UNSUPPORTED, "Milne (tau, r) coordinates need the (r, t) table medium");
    if (c->med_kind == MED_GRID && c->dims != 2)
        return fail(c, LIM_ERR_UNSUPPORTED, "the 2+1D grid medium needs dimensions=2 (got %d)", c->dims);
    const int coll = (int)c->P.collision;
    const bool langevin = coll == LIM_COLL_LANGEVIN || coll == LIM_COLL_LANGEVIN_RTA || c->P.coords == LIM_COORDS_MILNE;
    const bool rta = coll == LIM_COLL_RTA || coll == LIM_COLL_LANGEVIN_RTA;
    if (langevin && c->P.DsT > 0 && c->spl[0].empty())
        return fail(c, LIM_ERR_STATE, "drag spline not set (lim_set_spline LIM_SPLINE_DRAG) but DsT > 0");
    if (rta && c->P.coords != LIM_COORDS_MILNE) {
        if (c->P.DsT > 0 && c->spl[1].empty())
            return fail(c, LIM_ERR_STATE, "RTA spline not set (lim_set_spline LIM_SPLINE_RTA)");
        if (c->icdf.empty()) return fail(c, LIM_ERR_STATE, "RTA needs the Juttner inverse CDF (lim_set_invcdf)");
    }
    if (c->state_prec != (int)c->P.precision)
        return fail(c, LIM_ERR_STATE, "state was uploaded in another precision; upload it again");
    return LIM_OK;
}

// Threads per block of the step kernels: the caller's choice, else 128 for the FP32
// Cartesian kernels of the (r, t) and Bjorken media and for the grid with freeze-out
// (1 % faster than 256 on the benchmark workloads: the same residency in finer blocks
// balances the last wave), 256 for the rest (the grid without freeze-out measured 0.7 %
// faster at 256).
int block_of(const lim_ctx* c)
{
    int b = (int)c->P.block_size;
    if (b > 0) return b;
    const bool fp32_cart = c->P.precision == LIM_FP32 && c->P.coords == LIM_COORDS_CARTESIAN;
    if (fp32_cart && (c->med_kind != MED_GRID || c->P.freezeout_capture)) return 128;
    return 256;
}

constexpr int64_t kLiveSteps = 32;   // steps between compactions of the live list

// A snapshot reduced on the device into slot `slot` of the reduction buffers (observable
// sums and histograms; see lim_run_reduced).
struct SnapshotReduce {
    ReduceSpec rs;
    int64_t nslots;
};

template <typename R>
int reduce_snapshot(lim_ctx* c, const KParams<R>& kp, const SnapshotReduce& red, int64_t slot)
{
    double* obs = (double*)c->d_red_obs.p + slot * kObsNum;
    unsigned long long* hist = (unsigned long long*)c->d_red_hist.p + slot * reduce_hist_len(red.rs);
    LIM_CUDA(c, launch_reduce_hist<R>(kp, c->P.coords == LIM_COORDS_MILNE, red.rs, hist, c->P.obs_pt_cut,
                                      c->P.obs_pt_width > 0 ? c->P.obs_pt_width : 1e-3, (double*)c->d_partials.p, obs,
                                      c->stream));
    return LIM_OK;
}

// Copies the snapshot staged in buffer b (once its staging kernels have run) into slot
// `slot` of the host history, on the copy stream; the host waits for the copy, while
// the compute stream goes on with the next interval.
int copy_snapshot(lim_ctx* c, int b, int64_t slot, double* hist_x, double* hist_p, DevBuf* const* stage_x,
                  DevBuf* const* stage_p)
{
    LIM_CUDA(c, cudaStreamWaitEvent(c->copy_stream, c->ev_snap[b], 0));
    if (hist_x)
        LIM_CUDA(c, cudaMemcpyAsync(hist_x + slot * c->n * c->dims, stage_x[b]->p, sizeof(double) * c->n * c->dims,
                                    cudaMemcpyDeviceToHost, c->copy_stream));
    if (hist_p)
        LIM_CUDA(c, cudaMemcpyAsync(hist_p + slot * c->n * c->pdim, stage_p[b]->p, sizeof(double) * c->n * c->pdim,
                                    cudaMemcpyDeviceToHost, c->copy_stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->copy_stream));
    return LIM_OK;
}

template <typename R>
int run_impl(lim_ctx* c, int64_t first_step, int64_t nsteps, int64_t save_every, int64_t first_slot,
             double* hist_x, double* hist_p, const SnapshotReduce* red = nullptr)
{
    KParams<R> kp;
    int rc = build_kparams<R>(c, kp);
    if (rc) return rc;
    const int block = block_of(c);
    const bool saving = save_every > 0 && (hist_x || hist_p || red);
    const int64_t end = first_step + nsteps;
    const int64_t chunk_max = saving ? std::min<int64_t>(nsteps, save_every) : nsteps;
    if ((rc = dev_alloc(c, c->d_steps, (size_t)std::max<int64_t>(chunk_max, 1) * step_record_bytes<R>()))) return rc;
    kp.steps = c->d_steps.p;
    int64_t launches = 0;
    // stop-at-freeze-out runs of the Cartesian kernels advance a compacted live list
    const bool live_mode = c->P.coords == LIM_COORDS_CARTESIAN && kp.fo_capture && kp.stop_fo && kp.rec_steps == 0 &&
                           c->n > 0 && c->n <= (int64_t)INT_MAX;
    int cur = 0;
    bool live_valid = false;
    if (live_mode) {
        if ((rc = dev_alloc(c, c->d_live[0], (size_t)c->n * sizeof(int)))) return rc;
        if ((rc = dev_alloc(c, c->d_live[1], (size_t)c->n * sizeof(int)))) return rc;
        if ((rc = dev_alloc(c, c->d_live_n, 2 * sizeof(unsigned)))) return rc;
    }
    // snapshot staging: two buffers, copied to the host on the copy stream
    const bool to_host = saving && !red;
    DevBuf* stage_x[2] = { &c->d_stage_x, &c->d_stage2_x };
    DevBuf* stage_p[2] = { &c->d_stage_p, &c->d_stage2_p };
    int sb = 0;
    int64_t pending = -1;                  // slot staged in buffer 1 - sb, not yet copied
    if (to_host) {
        if (!c->copy_stream) LIM_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (cudaEvent_t& e : c->ev_snap)
            if (!e) LIM_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        const size_t nn = (size_t)std::max<int64_t>(c->n, 1);
        for (int b = 0; b < 2; ++b) {
            if ((rc = dev_alloc(c, *stage_x[b], nn * c->dims * sizeof(double)))) return rc;
            if ((rc = dev_alloc(c, *stage_p[b], nn * c->pdim * sizeof(double)))) return rc;
        }
    }
    LIM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    int64_t s = first_step;
    while (s < end) {
        int64_t chunk_end = end;
        if (saving) {   // run through the next save step (inclusive), then snapshot
            const int64_t next_save = ((s + save_every - 1) / save_every) * save_every;   // s >= 0
            if (next_save + 1 < chunk_end) chunk_end = next_save + 1;
        }
        kp.step_base = s;
        kp.step_cap = chunk_end - s;
        if (!live_mode) {
            LIM_CUDA(c, launch_steps<R>(kp, (int)c->P.coords, s, chunk_end, block, c->stream));
            launches += 2;                 // the per-step table, then the fused step kernel
        } else {
            // Particles stop at freeze-out: advance the chunk in sub-chunks of kLiveSteps
            // over a list of the live particles, compacted after each sub-chunk, so that
            // the frozen ones do not idle the lanes of warps that still run.
            LIM_CUDA(c, launch_step_table<R>(kp, 0, s, chunk_end, c->stream));
            ++launches;
            for (int64_t ss = s; ss < chunk_end; ss += kLiveSteps) {
                const int64_t se = std::min<int64_t>(ss + kLiveSteps, chunk_end);
                kp.live = live_valid ? (const int*)c->d_live[cur].p : nullptr;
                kp.live_n = live_valid ? (const unsigned*)c->d_live_n.p + cur : nullptr;
                LIM_CUDA(c, launch_steps_in_table<R>(kp, ss, se, block, c->stream));
                LIM_CUDA(c, launch_compact_live(kp.fo_flag, kp.live, kp.live_n, c->n, (int*)c->d_live[cur ^ 1].p,
                                                (unsigned*)c->d_live_n.p + (cur ^ 1), c->stream));
                launches += 2;
                cur ^= 1;
                live_valid = true;
            }
            kp.live = nullptr;
            kp.live_n = nullptr;
        }
        const int64_t last = chunk_end - 1;
        if (red && saving && last % save_every == 0 && last >= 0) {
            const int64_t slot = last / save_every - first_slot;
            if (slot >= 0 && slot < red->nslots) {
                if ((rc = reduce_snapshot<R>(c, kp, *red, slot))) return rc;
                launches += 2;
            }
        } else if (saving && last % save_every == 0 && last >= 0) {
            const int64_t slot = last / save_every - first_slot;
            if (slot >= 0) {
                // stage the snapshot (SoA -> the Julia layout) in buffer sb and copy the
                // previous one to the host while this interval's successor runs
                R* xs[3] = { kp.x[0], kp.x[1], kp.x[2] };
                double* ps[3] = { kp.p[0], kp.p[1], kp.p[2] };
                if (hist_x)
                    LIM_CUDA(c, launch_soa_to_aos<R>(xs, sizeof(R) == 4 ? kp.xlo : nullptr, c->dims, c->n,
                                                     (double*)stage_x[sb]->p, c->stream));
                if (hist_p)
                    LIM_CUDA(c, launch_soa_to_aos<double>(ps, nullptr, c->pdim, c->n, (double*)stage_p[sb]->p, c->stream));
                LIM_CUDA(c, cudaEventRecord(c->ev_snap[sb], c->stream));
                launches += 2;
                if (pending >= 0 && (rc = copy_snapshot(c, 1 - sb, pending, hist_x, hist_p, stage_x, stage_p))) return rc;
                pending = slot;
                sb = 1 - sb;
            }
        }
        s = chunk_end;
    }
    LIM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    if (pending >= 0 && (rc = copy_snapshot(c, 1 - sb, pending, hist_x, hist_p, stage_x, stage_p))) return rc;
    LIM_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    LIM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    c->last_launches = launches;
    unsigned long long bad = ULLONG_MAX;
    LIM_CUDA(c, cudaMemcpy(&bad, c->d_status.p, sizeof bad, cudaMemcpyDeviceToHost));
    if (bad != ULLONG_MAX)
        return fail(c, LIM_ERR_NONFINITE, "Breaking simulation due to NaN/Inf at step %llu", bad);
    return LIM_OK;
}

template <typename R>
int alloc_state(lim_ctx* c, int64_t n)
{
    int rc;
    const size_t nb = (size_t)n * sizeof(R);
    // buffers are reused when large enough (dev_alloc keeps a sufficient allocation)
    if (n == 0) return LIM_OK;
    for (int d = 0; d < c->dims; ++d) {
        if ((rc = dev_alloc(c, c->d_x[d], nb))) return rc;
        if (sizeof(R) == 4 && (rc = dev_alloc(c, c->d_xlo[d], (size_t)n * sizeof(float)))) return rc;
    }
    for (int d = 0; d < c->pdim; ++d)     // momenta are FP64 in both precisions
        if ((rc = dev_alloc(c, c->d_p[d], (size_t)n * sizeof(double)))) return rc;
    if (c->P.freezeout_capture) {
        const size_t nd = (size_t)n * sizeof(double);   // the latch is FP64 in both precisions
        for (int d = 0; d < c->dims; ++d) {
            if ((rc = dev_alloc(c, c->d_fo_pos[d], nd))) return rc;
            if ((rc = dev_alloc(c, c->d_l_pos[d], nd))) return rc;
            LIM_CUDA(c, cudaMemsetAsync(c->d_fo_pos[d].p, 0, nd, c->stream));
            LIM_CUDA(c, cudaMemsetAsync(c->d_l_pos[d].p, 0, nd, c->stream));
        }
        for (int d = 0; d < c->pdim; ++d) {
            if ((rc = dev_alloc(c, c->d_fo_mom[d], nd))) return rc;
            if ((rc = dev_alloc(c, c->d_l_mom[d], nd))) return rc;
            LIM_CUDA(c, cudaMemsetAsync(c->d_fo_mom[d].p, 0, nd, c->stream));
            LIM_CUDA(c, cudaMemsetAsync(c->d_l_mom[d].p, 0, nd, c->stream));
        }
        DevBuf* bufs[4] = { &c->d_fo_tau, &c->d_fo_flag, &c->d_l_tau, &c->d_l_T };
        for (DevBuf* b : bufs) {
            if ((rc = dev_alloc(c, *b, nd))) return rc;
            LIM_CUDA(c, cudaMemsetAsync(b->p, 0, nd, c->stream));
        }
    }
    return LIM_OK;
}

template <typename R>
int upload_state_impl(lim_ctx* c, const double* x, const double* p, int64_t n)
{
    int rc;
    if ((rc = alloc_state<R>(c, n))) return rc;
    if ((rc = dev_alloc(c, c->d_stage_x, (size_t)std::max<int64_t>(n, 1) * c->dims * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_stage_p, (size_t)std::max<int64_t>(n, 1) * c->pdim * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_status, sizeof(unsigned long long)))) return rc;
    LIM_CUDA(c, cudaMemsetAsync(c->d_status.p, 0xff, sizeof(unsigned long long), c->stream));
    c->n = n;
    if (n > 0) {
        LIM_CUDA(c, cudaMemcpyAsync(c->d_stage_x.p, x, sizeof(double) * n * c->dims, cudaMemcpyHostToDevice, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(c->d_stage_p.p, p, sizeof(double) * n * c->pdim, cudaMemcpyHostToDevice, c->stream));
        R* xs[3] = { (R*)c->d_x[0].p, (R*)c->d_x[1].p, (R*)c->d_x[2].p };
        double* ps[3] = { (double*)c->d_p[0].p, (double*)c->d_p[1].p, (double*)c->d_p[2].p };
        float* lo[3] = { (float*)c->d_xlo[0].p, (float*)c->d_xlo[1].p, (float*)c->d_xlo[2].p };
        LIM_CUDA(c, launch_aos_to_soa<R>((const double*)c->d_stage_x.p, c->dims, n, xs, sizeof(R) == 4 ? lo : nullptr, c->stream));
        LIM_CUDA(c, launch_aos_to_soa<double>((const double*)c->d_stage_p.p, c->pdim, n, ps, nullptr, c->stream));
    }
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    c->state_prec = (int)c->P.precision;
    c->have_state = true;
    return LIM_OK;
}

template <typename R>
int download_state_impl(lim_ctx* c, double* x, double* p)
{
    if (c->n == 0) return LIM_OK;
    R* xs[3] = { (R*)c->d_x[0].p, (R*)c->d_x[1].p, (R*)c->d_x[2].p };
    double* ps[3] = { (double*)c->d_p[0].p, (double*)c->d_p[1].p, (double*)c->d_p[2].p };
    float* lo[3] = { (float*)c->d_xlo[0].p, (float*)c->d_xlo[1].p, (float*)c->d_xlo[2].p };
    if (x) {
        LIM_CUDA(c, launch_soa_to_aos<R>(xs, sizeof(R) == 4 ? lo : nullptr, c->dims, c->n, (double*)c->d_stage_x.p, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(x, c->d_stage_x.p, sizeof(double) * c->n * c->dims, cudaMemcpyDeviceToHost, c->stream));
    }
    if (p) {
        LIM_CUDA(c, launch_soa_to_aos<double>(ps, nullptr, c->pdim, c->n, (double*)c->d_stage_p.p, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(p, c->d_stage_p.p, sizeof(double) * c->n * c->pdim, cudaMemcpyDeviceToHost, c->stream));
    }
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return LIM_OK;
}

template <typename R>
int download_fo_impl(lim_ctx* c, double* fo_pos, double* fo_mom, double* fo_tau, double* fo_flag)
{
    if (!c->P.freezeout_capture) return fail(c, LIM_ERR_STATE, "freezeout_capture is off");
    if (c->n == 0) return LIM_OK;
    double* fp[3] = { (double*)c->d_fo_pos[0].p, (double*)c->d_fo_pos[1].p, (double*)c->d_fo_pos[2].p };
    double* fm[3] = { (double*)c->d_fo_mom[0].p, (double*)c->d_fo_mom[1].p, (double*)c->d_fo_mom[2].p };
    double* ft[1] = { (double*)c->d_fo_tau.p };
    double* ff[1] = { (double*)c->d_fo_flag.p };
    if (fo_pos) {
        LIM_CUDA(c, launch_soa_to_aos<double>(fp, nullptr, c->dims, c->n, (double*)c->d_stage_x.p, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(fo_pos, c->d_stage_x.p, sizeof(double) * c->n * c->dims, cudaMemcpyDeviceToHost, c->stream));
    }
    if (fo_mom) {
        LIM_CUDA(c, launch_soa_to_aos<double>(fm, nullptr, c->pdim, c->n, (double*)c->d_stage_p.p, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(fo_mom, c->d_stage_p.p, sizeof(double) * c->n * c->pdim, cudaMemcpyDeviceToHost, c->stream));
    }
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    if (fo_tau) {
        LIM_CUDA(c, launch_soa_to_aos<double>(ft, nullptr, 1, c->n, (double*)c->d_stage_x.p, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(fo_tau, c->d_stage_x.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
        LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    if (fo_flag) {
        LIM_CUDA(c, launch_soa_to_aos<double>(ff, nullptr, 1, c->n, (double*)c->d_stage_x.p, c->stream));
        LIM_CUDA(c, cudaMemcpyAsync(fo_flag, c->d_stage_x.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
        LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return LIM_OK;
}

template <typename R>
int observables_impl(lim_ctx* c, int from_fo, double* out)
{
    KParams<R> kp;
    int rc = build_kparams<R>(c, kp);
    if (rc) return rc;
    if (from_fo && !c->P.freezeout_capture) return fail(c, LIM_ERR_STATE, "freezeout_capture is off");
    const int64_t nb = c->n == 0 ? 1 : (c->n + 255) / 256;
    if ((rc = dev_alloc(c, c->d_partials, (size_t)nb * kObsNum * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_obs, kObsNum * sizeof(double)))) return rc;
    LIM_CUDA(c, launch_observables<R>(kp, from_fo, c->P.obs_pt_cut, c->P.obs_pt_width > 0 ? c->P.obs_pt_width : 1e-3,
                                      (double*)c->d_partials.p, nb, (double*)c->d_obs.p, c->stream));
    LIM_CUDA(c, cudaMemcpyAsync(out, c->d_obs.p, kObsNum * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return LIM_OK;
}

}  // namespace

void lim::set_noctx_error(const char* msg) { g_create_error = msg; }

namespace lim {

int ctx_fail(lim_ctx* c, int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return fail(c, code, "%s", buf);
}
int ctx_check_ready(lim_ctx* c) { return check_ready(c); }
int ctx_alloc(lim_ctx* c, DevBuf& b, size_t bytes) { return dev_alloc(c, b, bytes); }
template <typename R> int ctx_build_kparams(lim_ctx* c, KParams<R>& kp) { return build_kparams<R>(c, kp); }
template int ctx_build_kparams<double>(lim_ctx*, KParams<double>&);
template int ctx_build_kparams<float>(lim_ctx*, KParams<float>&);

}  // namespace lim

namespace {

// Allocates the state for n particles and fills it with launch(kp) (a sampling kernel
// that counts particles without an accepted trial in *failed).
template <typename R, typename F>
int sample_state(lim_ctx* c, int64_t n, unsigned long long* failed_dev, int max_trials, const char* who, F&& launch)
{
    int rc;
    if ((rc = alloc_state<R>(c, n))) return rc;
    if ((rc = dev_alloc(c, c->d_stage_x, (size_t)std::max<int64_t>(n, 1) * c->dims * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_stage_p, (size_t)std::max<int64_t>(n, 1) * c->pdim * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_status, sizeof(unsigned long long)))) return rc;
    LIM_CUDA(c, cudaMemsetAsync(c->d_status.p, 0xff, sizeof(unsigned long long), c->stream));
    c->n = n;
    c->state_prec = (int)c->P.precision;
    c->have_state = true;                 // the kernel parameters need the state buffers
    KParams<R> kp;
    if ((rc = build_kparams<R>(c, kp))) { c->have_state = false; return rc; }
    LIM_CUDA(c, cudaMemsetAsync(failed_dev, 0, sizeof(unsigned long long), c->stream));
    LIM_CUDA(c, launch(kp));
    unsigned long long failed = 0;
    LIM_CUDA(c, cudaMemcpyAsync(&failed, failed_dev, sizeof failed, cudaMemcpyDeviceToHost, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    if (failed) {
        c->have_state = false;
        return fail(c, LIM_ERR_STATE, "%s: %llu particles found no accepted trial in %d trials", who, failed,
                    max_trials);
    }
    return LIM_OK;
}

template <typename R>
int sample_impl(lim_ctx* c, const SampleTables& st, int64_t n)
{
    return sample_state<R>(c, n, st.failed, st.max_trials, "lim_sample_fonll",
                           [&](const KParams<R>& kp) { return launch_sample_fonll<R>(kp, st, c->stream); });
}

template <typename R>
int sample_milne_impl(lim_ctx* c, const MilneTables& mt, int64_t n)
{
    return sample_state<R>(c, n, mt.failed, mt.max_trials, "lim_sample_milne",
                           [&](const KParams<R>& kp) { return launch_sample_milne<R>(kp, mt, c->stream); });
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

int lim_abi_version(void) { return LIM_ABI_VERSION; }

int lim_create(int device, void* stream, lim_ctx** out)
{
    if (!out) return fail(nullptr, LIM_ERR_ARG, "lim_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return fail(nullptr, LIM_ERR_CUDA, "cudaGetDeviceCount failed: %s", cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(nullptr, LIM_ERR_ARG, "lim_create: device %d out of range (%d devices)", device, ndev);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, LIM_ERR_CUDA, "cudaSetDevice failed: %s", cudaGetErrorString(e));
    lim_ctx* c = new (std::nothrow) lim_ctx();
    if (!c) return fail(nullptr, LIM_ERR_NOMEM, "lim_create: out of host memory");
    c->device = device;
    if (stream) c->stream = (cudaStream_t)stream;
    else {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete c; return fail(nullptr, LIM_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e)); }
        c->own_stream = true;
    }
    if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        delete c;
        return fail(nullptr, LIM_ERR_CUDA, "cudaEventCreate failed");
    }
    *out = c;
    return LIM_OK;
}

int lim_destroy(lim_ctx* c)
{
    if (!c) return LIM_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    DevBuf* all[] = { &c->d_xg, &c->d_tg, &c->d_tgd, &c->d_xgd, &c->d_TV, &c->d_TVc, &c->d_xc, &c->d_V2, &c->d_G, &c->d_spl[0], &c->d_spl[1], &c->d_spl[2], &c->d_spl[3], &c->d_icdf,
                      &c->d_fo_tau, &c->d_fo_flag, &c->d_l_tau, &c->d_l_T, &c->d_status, &c->d_stage_x, &c->d_stage_p,
                      &c->d_partials, &c->d_obs, &c->d_probe, &c->d_rec, &c->d_steps, &c->d_ckpt,
                      &c->d_live[0], &c->d_live[1], &c->d_live_n, &c->d_rta_bits,
                      &c->d_adj_ckpt, &c->d_adj_tape, &c->d_adj_table, &c->d_adj_part, &c->d_adj_out,
                      &c->d_adj_lam, &c->d_adj_gacc, &c->d_adj_slope, &c->d_adj_icdt, &c->d_sample,
                      &c->d_red_obs, &c->d_red_hist, &c->d_stage2_x, &c->d_stage2_p, &c->d_pmag_hist,
                      &c->d_rta64, &c->d_T64 };
    for (DevBuf* b : all) dev_free(*b);
    for (int d = 0; d < 3; ++d) {
        dev_free(c->d_x[d]); dev_free(c->d_xlo[d]); dev_free(c->d_p[d]);
        dev_free(c->d_fo_pos[d]); dev_free(c->d_fo_mom[d]); dev_free(c->d_l_pos[d]); dev_free(c->d_l_mom[d]);
    }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (cudaEvent_t e : c->ev_snap) if (e) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return LIM_OK;
}

const char* lim_last_error(const lim_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int lim_synchronize(lim_ctx* c)
{
    if (!c) return LIM_ERR_ARG;
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return LIM_OK;
}

int lim_device_bytes(const lim_ctx* c, int64_t* bytes)
{
    if (!c || !bytes) return LIM_ERR_ARG;
    const DevBuf* all[] = { &c->d_xg, &c->d_tg, &c->d_tgd, &c->d_xgd, &c->d_TV, &c->d_TVc, &c->d_xc, &c->d_V2, &c->d_G, &c->d_spl[0], &c->d_spl[1], &c->d_spl[2], &c->d_spl[3], &c->d_icdf,
                            &c->d_fo_tau, &c->d_fo_flag, &c->d_l_tau, &c->d_l_T, &c->d_status, &c->d_stage_x, &c->d_stage_p,
                            &c->d_partials, &c->d_obs, &c->d_probe, &c->d_rec, &c->d_steps, &c->d_ckpt,
                      &c->d_live[0], &c->d_live[1], &c->d_live_n, &c->d_rta_bits,
                      &c->d_adj_ckpt, &c->d_adj_tape, &c->d_adj_table, &c->d_adj_part, &c->d_adj_out,
                      &c->d_adj_lam, &c->d_adj_gacc, &c->d_adj_slope, &c->d_adj_icdt, &c->d_sample,
                      &c->d_red_obs, &c->d_red_hist, &c->d_stage2_x, &c->d_stage2_p, &c->d_pmag_hist,
                      &c->d_rta64, &c->d_T64 };
    int64_t t = 0;
    for (const DevBuf* b : all) t += (int64_t)b->bytes;
    for (int d = 0; d < 3; ++d)
        t += (int64_t)(c->d_x[d].bytes + c->d_xlo[d].bytes + c->d_p[d].bytes + c->d_fo_pos[d].bytes +
                       c->d_fo_mom[d].bytes + c->d_l_pos[d].bytes + c->d_l_mom[d].bytes);
    *bytes = t;
    return LIM_OK;
}

int lim_set_params(lim_ctx* c, const lim_params* P)
{
    if (!c || !P) return LIM_ERR_ARG;
    ++c->gen;
    lim_params q = *P;
    if (!std::isfinite(q.dt) || !std::isfinite(q.t0) || !std::isfinite(q.m))
        return fail(c, LIM_ERR_ARG, "dt, t0 and m must be finite");
    if (q.pdim <= 0) q.pdim = q.dims;                          // momentum_dimensions = 0 => dimensions
    if (q.coords != LIM_COORDS_CARTESIAN && q.coords != LIM_COORDS_MILNE)
        return fail(c, LIM_ERR_ARG, "coords=%lld is not a valid coordinate system", (long long)q.coords);
    if (q.coords == LIM_COORDS_MILNE) {
        if (q.dims != 2 || q.pdim != 2)
            return fail(c, LIM_ERR_ARG, "Milne coordinates evolve (tau, r) and (p^tau, p^r): dims = pdim = 2");
    } else {
        if (q.dims < 1 || q.dims > 3) return fail(c, LIM_ERR_ARG, "dimensions=%lld is not supported (1, 2 or 3)", (long long)q.dims);
        const bool radial = q.dims == 1;
        // utils.jl:561-573 check_momentum_dims
        if (q.pdim != q.dims && !(q.dims == 2 && q.pdim == 3 && !radial))
            return fail(c, LIM_ERR_ARG,
                        "momentum_dimensions=%lld with dimensions=%lld is not supported: only (dimensions=2, "
                        "momentum_dimensions=3) differs from the coupled default.", (long long)q.pdim, (long long)q.dims);
        if (q.bjorken_redshift) {
            if (!(q.dims == 2 && q.pdim == 3))
                return fail(c, LIM_ERR_ARG, "bjorken_redshift requires dimensions=2 and momentum_dimensions=3 (p_z is row 3).");
            if (!(q.t0 > 0))
                return fail(c, LIM_ERR_ARG, "bjorken_redshift needs initial_time > 0 (Milne tau; dp_z/dtau = -p_z/tau).");
        }
    }
    if (q.collision < LIM_COLL_LANGEVIN || q.collision > LIM_COLL_FLUID)
        return fail(c, LIM_ERR_ARG, "collision_mode=%lld is not supported (only :langevin, :rta, :langevin_rta, :fluid).", (long long)q.collision);
    if (q.integrator_mode != 0 && q.integrator_mode != 1)
        return fail(c, LIM_ERR_ARG, "integrator_mode must be 0 or 1");
    if (q.precision != LIM_FP64 && q.precision != LIM_FP32) return fail(c, LIM_ERR_ARG, "precision must be LIM_FP64 or LIM_FP32");
    if (q.block_size < 0 || q.block_size > 256 || (q.block_size % 32) != 0)
        return fail(c, LIM_ERR_ARG, "block_size must be a multiple of 32 in [32, 256] (or 0)");
    // A state of another shape or precision, or without latch buffers (they are
    // allocated at upload), no longer matches: it is dropped and must be uploaded again.
    const bool stale = c->have_state &&
        (q.dims != c->dims || q.pdim != c->pdim || (int)q.precision != c->state_prec ||
         (q.freezeout_capture && !c->P.freezeout_capture));
    c->P = q;
    c->have_params = true;
    if (stale) c->have_state = false;
    return LIM_OK;
}

int lim_set_medium_rt(lim_ctx* c, const double* xgrid, int64_t nr, const double* tgrid, int64_t nt,
                      const double* T, const double* V, const double* V2)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    if (!xgrid || !tgrid || !T || !V) return fail(c, LIM_ERR_ARG, "lim_set_medium_rt: NULL grid or field");
    if (nr < 2 || nt < 2) return fail(c, LIM_ERR_ARG, "lim_set_medium_rt: need at least 2 nodes per axis (got %lld x %lld)", (long long)nr, (long long)nt);
    if (!all_finite(xgrid, nr) || !all_finite(tgrid, nt)) return fail(c, LIM_ERR_ARG, "lim_set_medium_rt: non-finite grid node");
    if (!ascending(xgrid, nr) || !ascending(tgrid, nt)) return fail(c, LIM_ERR_ARG, "lim_set_medium_rt: grids must be strictly ascending");
    size_t nn = (size_t)(nr * nt);
    c->xg.assign(xgrid, xgrid + nr);
    c->tg.assign(tgrid, tgrid + nt);
    c->T.assign(T, T + nn);
    c->V.assign(V, V + nn);
    if (V2) c->V2.assign(V2, V2 + nn); else c->V2.clear();
    c->med_kind = MED_RT;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_set_medium_bjorken(lim_ctx* c, double T0, double tau0, double power, double r_max)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    if (!(T0 >= 0) || !(tau0 > 0) || !std::isfinite(power) || !std::isfinite(r_max))
        return fail(c, LIM_ERR_ARG, "lim_set_medium_bjorken: need T0 >= 0, tau0 > 0, finite power and r_max");
    c->bj_T0 = T0; c->bj_tau0 = tau0; c->bj_power = power; c->bj_rmax = r_max;
    c->med_kind = MED_BJORKEN;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_set_medium_grid(lim_ctx* c, int64_t nx, int64_t ny, int64_t nt, double x0, double dx, double y0, double dy,
                        double tau0, double dtau, const float* T, const float* ux, const float* uy)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    if (!T || !ux || !uy) return fail(c, LIM_ERR_ARG, "lim_set_medium_grid: NULL field");
    if (nx < 2 || ny < 2 || nt < 2) return fail(c, LIM_ERR_ARG, "lim_set_medium_grid: need at least 2 nodes per axis");
    if (!(dx > 0) || !(dy > 0) || !(dtau > 0)) return fail(c, LIM_ERR_ARG, "lim_set_medium_grid: spacings must be positive");
    if (!std::isfinite(x0) || !std::isfinite(y0) || !std::isfinite(tau0)) return fail(c, LIM_ERR_ARG, "lim_set_medium_grid: non-finite origin");
    if ((double)nx * ny * nt > 4.0e9) return fail(c, LIM_ERR_ARG, "lim_set_medium_grid: grid too large");
    size_t nn = (size_t)(nx * ny * nt);
    c->gT.assign(T, T + nn); c->gux.assign(ux, ux + nn); c->guy.assign(uy, uy + nn);
    c->gnx = nx; c->gny = ny; c->gnt = nt;
    c->gx0 = x0; c->gdx = dx; c->gy0 = y0; c->gdy = dy; c->gt0 = tau0; c->gdt = dtau;
    c->med_kind = MED_GRID;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_set_spline(lim_ctx* c, int which, double Tmin, double invdT, const double* vals, int64_t n)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    if (which < LIM_SPLINE_DRAG || which > LIM_SPLINE_DRAG_DB) return fail(c, LIM_ERR_ARG, "lim_set_spline: unknown spline %d", which);
    if (!vals || n < 1) return fail(c, LIM_ERR_ARG, "lim_set_spline: empty spline");
    if (!std::isfinite(Tmin) || !std::isfinite(invdT)) return fail(c, LIM_ERR_ARG, "lim_set_spline: non-finite Tmin/invdT");
    c->spl[which].assign(vals, vals + n);
    c->spl_Tmin[which] = Tmin;
    c->spl_invdT[which] = invdT;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_build_time_spline(lim_ctx* c, int which, int kind, double m, double DsT, const lim_dsform* form,
                          double Tmin, double Tmax, int64_t nT, double eta_over_s, double factor, double scale)
{
    if (!c) return LIM_ERR_ARG;
    if (which < LIM_SPLINE_DRAG || which > LIM_SPLINE_RTA)
        return fail(c, LIM_ERR_ARG, "lim_build_time_spline: which must be LIM_SPLINE_DRAG or LIM_SPLINE_RTA");
    if (kind < LIM_TIME_DRAG || kind > LIM_TIME_TAUR) return fail(c, LIM_ERR_ARG, "lim_build_time_spline: unknown kind %d", kind);
    // transport.jl:165-196 argument checks (and effective_DsT's, :139-156)
    if (nT < 2) return fail(c, LIM_ERR_ARG, "nT must be >= 2");
    if (nT > (1 << 24)) return fail(c, LIM_ERR_ARG, "lim_build_time_spline: at most 2^24 nodes");
    if (!(Tmin > 0.0)) return fail(c, LIM_ERR_ARG, "Tmin must be > 0");
    if (!(Tmax > Tmin) || !std::isfinite(Tmax)) return fail(c, LIM_ERR_ARG, "Tmax must be > Tmin");
    TimeSplineSpec sp;
    std::memset(&sp, 0, sizeof sp);
    if (form) {
        if (form->quad && form->linear)
            return fail(c, LIM_ERR_ARG, "effective_DsT: DsT_quad and DsT_linear are mutually exclusive");
        if (form->quad && !(form->Tref > 0.0)) return fail(c, LIM_ERR_ARG, "effective_DsT: DsT_quad requires DsT_Tref > 0");
        sp.linear = form->linear != 0; sp.quad = form->quad != 0;
        sp.slope = form->slope; sp.offset = form->offset; sp.Tfo = form->Tfo; sp.Tref = form->Tref;
    }
    sp.kind = kind; sp.nT = (int)nT; sp.m = m; sp.DsT = DsT; sp.Tmin = Tmin; sp.Tmax = Tmax; sp.scale = scale;
    sp.eta_over_s = eta_over_s; sp.factor = factor;
    cudaSetDevice(c->device);
    DevBuf tmp;
    int rc = dev_alloc(c, tmp, (size_t)nT * sizeof(double));
    if (rc) return rc;
    std::vector<double> vals((size_t)nT);
    cudaError_t e = launch_time_spline(sp, (double*)tmp.p, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vals.data(), tmp.p, vals.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dev_free(tmp);
    if (e != cudaSuccess) return fail(c, LIM_ERR_CUDA, "lim_build_time_spline: %s", cudaGetErrorString(e));
    const double dT = (Tmax - Tmin) / (double)(nT - 1);
    ++c->gen;
    c->spl[which] = std::move(vals);
    c->spl_Tmin[which] = Tmin;
    c->spl_invdT[which] = 1.0 / dT;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_build_juttner_invcdf(lim_ctx* c, double m, int64_t dims, double Tmin, double Tmax, int64_t nT, int64_t nU,
                             int64_t np, double quantile_cap)
{
    if (!c) return LIM_ERR_ARG;
    if (nT < 2) return fail(c, LIM_ERR_ARG, "nT must be >= 2");
    if (nU < 2) return fail(c, LIM_ERR_ARG, "nU must be >= 2");
    if (np < 2) return fail(c, LIM_ERR_ARG, "np must be >= 2");
    if (dims < 1 || dims > 3) return fail(c, LIM_ERR_ARG, "lim_build_juttner_invcdf: dimensions must be 1, 2 or 3");
    if (nT > 65535 || nU > (1 << 24) || np > (1 << 24) || (double)nT * (double)np > 1e9)
        return fail(c, LIM_ERR_ARG, "lim_build_juttner_invcdf: table too large");
    // transport.jl:277-300: the T range padded by 2 % on both sides, kept above 1e-4
    double Tmin_f = std::max(Tmin, 1e-4);
    double Tmax_f = std::max(Tmax, Tmin_f * (1.0 + 1e-6));
    const double span = Tmax_f - Tmin_f;
    Tmin_f = std::max(Tmin_f - 0.02 * span, 1e-4);
    Tmax_f = Tmax_f + 0.02 * span;
    JuttnerSpec js;
    js.dims = (int)dims; js.nT = (int)nT; js.nU = (int)nU; js.np = (int)np;
    js.m = m; js.Tmin = Tmin_f; js.dT = (Tmax_f - Tmin_f) / (double)(nT - 1); js.quantile_cap = quantile_cap;
    cudaSetDevice(c->device);
    DevBuf scratch, inv;
    int rc = dev_alloc(c, scratch, (size_t)nT * np * sizeof(double));
    if (!rc) rc = dev_alloc(c, inv, (size_t)nT * nU * sizeof(double));
    if (rc) { dev_free(scratch); dev_free(inv); return rc; }
    std::vector<double> vals((size_t)(nT * nU));
    cudaError_t e = launch_juttner_invcdf(js, (double*)scratch.p, (double*)inv.p, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vals.data(), inv.p, vals.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dev_free(scratch);
    dev_free(inv);
    if (e != cudaSuccess) return fail(c, LIM_ERR_CUDA, "lim_build_juttner_invcdf: %s", cudaGetErrorString(e));
    ++c->gen;
    c->icdf = std::move(vals);
    c->nU = nU; c->nT = nT; c->ic_Tmin = Tmin_f; c->ic_invdT = 1.0 / js.dT;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_get_spline(lim_ctx* c, int which, double* Tmin, double* invdT, double* vals, int64_t cap, int64_t* n)
{
    if (!c) return LIM_ERR_ARG;
    if (which < LIM_SPLINE_DRAG || which > LIM_SPLINE_DRAG_DB) return fail(c, LIM_ERR_ARG, "lim_get_spline: unknown spline %d", which);
    const std::vector<double>& v = c->spl[which];
    if (n) *n = (int64_t)v.size();
    if (Tmin) *Tmin = c->spl_Tmin[which];
    if (invdT) *invdT = c->spl_invdT[which];
    if (vals) {
        if (cap < (int64_t)v.size()) return fail(c, LIM_ERR_ARG, "lim_get_spline: buffer of %lld values for %zu",
                                                 (long long)cap, v.size());
        std::copy(v.begin(), v.end(), vals);
    }
    return LIM_OK;
}

int lim_get_invcdf(lim_ctx* c, double* vals, int64_t cap, int64_t* nU, int64_t* nT, double* Tmin, double* invdT)
{
    if (!c) return LIM_ERR_ARG;
    if (nU) *nU = c->nU;
    if (nT) *nT = c->nT;
    if (Tmin) *Tmin = c->ic_Tmin;
    if (invdT) *invdT = c->ic_invdT;
    if (vals) {
        if (cap < (int64_t)c->icdf.size()) return fail(c, LIM_ERR_ARG, "lim_get_invcdf: buffer too small");
        std::copy(c->icdf.begin(), c->icdf.end(), vals);
    }
    return LIM_OK;
}

int lim_set_medium_scale(lim_ctx* c, double s)
{
    if (!c) return LIM_ERR_ARG;
    if (!std::isfinite(s) || !(s > 0)) return fail(c, LIM_ERR_ARG, "lim_set_medium_scale: scale must be finite and > 0");
    ++c->gen;
    c->T_scale = s;
    return LIM_OK;
}

int lim_rta_decisions(lim_ctx* c, int mode, int64_t first_step, int64_t nsteps)
{
    if (!c) return LIM_ERR_ARG;
    if (mode < 0 || mode > 2) return fail(c, LIM_ERR_ARG, "lim_rta_decisions: mode must be 0 (off), 1 (record) or 2 (replay)");
    ++c->gen;
    if (mode == 0) { dev_free(c->d_rta_bits); c->rta_mode = 0; c->rta_steps = 0; return LIM_OK; }
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "upload the state before recording or replaying RTA decisions");
    if (first_step < 0 || nsteps < 1) return fail(c, LIM_ERR_ARG, "lim_rta_decisions: need first_step >= 0 and nsteps >= 1");
    const size_t words = (size_t)((nsteps + 31) / 32) * (size_t)c->n;
    if (mode == 1) {
        int rc = dev_alloc(c, c->d_rta_bits, std::max<size_t>(words, 1) * sizeof(uint32_t));
        if (rc) return rc;
        LIM_CUDA(c, cudaMemsetAsync(c->d_rta_bits.p, 0, std::max<size_t>(words, 1) * sizeof(uint32_t), c->stream));
        c->rta_first = first_step;
        c->rta_steps = nsteps;
    } else {
        if (!c->d_rta_bits.p || c->rta_first != first_step || c->rta_steps != nsteps || c->d_rta_bits.bytes < words * sizeof(uint32_t))
            return fail(c, LIM_ERR_STATE, "lim_rta_decisions: replay needs decisions recorded for the same steps and particles");
    }
    c->rta_mode = mode;
    return LIM_OK;
}

int lim_copy_rta_decisions(lim_ctx* dst, const lim_ctx* src)
{
    if (!dst || !src) return LIM_ERR_ARG;
    if (!src->d_rta_bits.p || src->n != dst->n)
        return fail(dst, LIM_ERR_STATE, "lim_copy_rta_decisions: the source holds no decisions for this particle count");
    ++dst->gen;
    int rc = dev_alloc(dst, dst->d_rta_bits, src->d_rta_bits.bytes);
    if (rc) return rc;
    LIM_CUDA(dst, cudaStreamSynchronize(src->stream));
    LIM_CUDA(dst, cudaMemcpyAsync(dst->d_rta_bits.p, src->d_rta_bits.p, src->d_rta_bits.bytes, cudaMemcpyDeviceToDevice, dst->stream));
    dst->rta_first = src->rta_first;
    dst->rta_steps = src->rta_steps;
    dst->rta_mode = 2;
    return LIM_OK;
}

int lim_set_invcdf(lim_ctx* c, const double* vals, int64_t nU, int64_t nT, double Tmin, double invdT)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    if (!vals || nU < 2 || nT < 2) return fail(c, LIM_ERR_ARG, "lim_set_invcdf: need nU >= 2 and nT >= 2");
    if (!std::isfinite(Tmin) || !std::isfinite(invdT)) return fail(c, LIM_ERR_ARG, "lim_set_invcdf: non-finite Tmin/invdT");
    c->icdf.assign(vals, vals + nU * nT);
    c->nU = nU; c->nT = nT; c->ic_Tmin = Tmin; c->ic_invdT = invdT;
    c->dev_dirty = true;
    return LIM_OK;
}

int lim_upload_state(lim_ctx* c, const double* x, int64_t dims, const double* p, int64_t pdim, int64_t n)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    int rc = state_rows_ok(c);
    if (rc) return rc;
    if (n < 0) return fail(c, LIM_ERR_ARG, "lim_upload_state: negative particle count");
    if (n > (int64_t)UINT32_MAX) return fail(c, LIM_ERR_ARG, "lim_upload_state: at most 2^32-1 particles per context");
    if (dims != c->P.dims || pdim != c->P.pdim)
        return fail(c, LIM_ERR_ARG, "momentum rows %lld / position rows %lld differ from the parameters (%lld, %lld)",
                    (long long)pdim, (long long)dims, (long long)c->P.pdim, (long long)c->P.dims);
    if (n > 0 && (!x || !p)) return fail(c, LIM_ERR_ARG, "lim_upload_state: NULL state");
    cudaSetDevice(c->device);
    c->dims = (int)dims; c->pdim = (int)pdim;
    c->have_state = false;
    return c->P.precision == LIM_FP32 ? upload_state_impl<float>(c, x, p, n) : upload_state_impl<double>(c, x, p, n);
}


int lim_sample_fonll(lim_ctx* c, const double* r_grid, int64_t nr, const double* p_grid, int64_t np,
                     const double* f, int64_t n, int cartesian, int antithetic, int thermal_pz)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    int rc = state_rows_ok(c);
    if (rc) return rc;
    if (c->P.coords != LIM_COORDS_CARTESIAN || c->P.dims != 2 || (c->P.pdim != 2 && c->P.pdim != 3))
        return fail(c, LIM_ERR_UNSUPPORTED, "lim_sample_fonll samples the transverse plane: dimensions=2, "
                                             "momentum_dimensions 2 or 3, Cartesian coordinates");
    if (n < 0 || n > (int64_t)UINT32_MAX) return fail(c, LIM_ERR_ARG, "lim_sample_fonll: particle count out of range");
    if (!r_grid || !p_grid || !f || nr < 2 || np < 2 || nr > INT32_MAX || np > INT32_MAX ||
        nr * np > (int64_t)1 << 31)
        return fail(c, LIM_ERR_ARG, "lim_sample_fonll: need r and p grids of 2 to 2^31 nodes and the density table");
    if (!ascending(r_grid, (size_t)nr) || !ascending(p_grid, (size_t)np))
        return fail(c, LIM_ERR_ARG, "lim_sample_fonll: r_grid and p_grid must be strictly ascending");
    if (c->P.pdim == 3 && thermal_pz && c->med_kind < 0)
        return fail(c, LIM_ERR_STATE, "lim_sample_fonll: the thermal p_z needs the medium (set it first)");
    // utils.jl:33-172, in FP64 on the host: f[ip + np*ir] is f(r_ir, p_ip) (an Np x Nr Matrix)
    double dr = 0.0, dp = 0.0;
    for (int64_t k = 1; k < nr; ++k) dr += r_grid[k] - r_grid[k - 1];
    for (int64_t k = 1; k < np; ++k) dp += p_grid[k] - p_grid[k - 1];
    dr /= (double)(nr - 1);
    dp /= (double)(np - 1);
    const double eps = 2.220446049250313e-16;
    std::vector<double> cdf_p((size_t)(nr * np), 0.0), nsp((size_t)nr, 0.0), cdf_r((size_t)nr, 0.0);
    std::vector<int> mass((size_t)nr, 0);
    for (int64_t ir = 0; ir < nr; ++ir) {
        double tot = 0.0;
        for (int64_t ip = 0; ip < np; ++ip) tot += p_grid[ip] * f[ip + np * ir];
        nsp[ir] = tot * dp;                                    // n(r) = int p f dp (Cartesian mode)
        if (!(tot > 0)) continue;
        mass[ir] = 1;
        double* row = cdf_p.data() + (size_t)ir * np;
        double acc = 0.0;
        for (int64_t ip = 0; ip < np; ++ip) { acc += p_grid[ip] * f[ip + np * ir]; row[ip] = acc * dp; }
        row[0] = 0.0;
        for (int64_t k = 1; k < np; ++k) row[k] = std::max(row[k], row[k - 1] + eps);
        const double last = row[np - 1];
        for (int64_t k = 0; k < np; ++k) row[k] /= last;
        row[np - 1] = 1.0;
    }
    double fmax = 0.0;
    for (double v : nsp) fmax = std::max(fmax, v);
    fmax += eps;
    if (!cartesian) {                                          // polar: P(r, p) ~ r p f
        double Z = 0.0;
        for (int64_t ir = 0; ir < nr; ++ir)
            for (int64_t ip = 0; ip < np; ++ip) Z += r_grid[ir] * p_grid[ip] * f[ip + np * ir];
        Z *= dr * dp;
        if (Z == 0.0) return fail(c, LIM_ERR_ARG, "Distribution normalization is zero.");
        double acc = 0.0;
        for (int64_t ir = 0; ir < nr; ++ir) {
            double pr = 0.0;
            for (int64_t ip = 0; ip < np; ++ip) pr += r_grid[ir] * p_grid[ip] * f[ip + np * ir] / Z;
            acc += pr * dp;
            cdf_r[ir] = acc * dr;
        }
        cdf_r[0] = 0.0;
        for (int64_t k = 1; k < nr; ++k) cdf_r[k] = std::max(cdf_r[k], cdf_r[k - 1] + eps);
        const double last = cdf_r[nr - 1];
        for (int64_t k = 0; k < nr; ++k) cdf_r[k] /= last;
        cdf_r[nr - 1] = 1.0;
    }
    // one device block: r grid, p grid, cdf_r, n(r), cdf_p, mass, failure count
    const size_t doubles = (size_t)(nr + np + nr + nr + nr * np);
    const size_t bytes = doubles * sizeof(double) + (size_t)nr * sizeof(int) + 64;
    cudaSetDevice(c->device);
    if ((rc = dev_alloc(c, c->d_sample, bytes))) return rc;
    double* d = (double*)c->d_sample.p;
    size_t off = 0;
    auto put = [&](const double* src, size_t cnt) {
        double* dst = d + off;
        off += cnt;
        return cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyHostToDevice, c->stream) == cudaSuccess ? dst : nullptr;
    };
    SampleTables st;
    std::memset(&st, 0, sizeof st);
    st.r_grid = put(r_grid, (size_t)nr);
    st.p_grid = put(p_grid, (size_t)np);
    st.cdf_r = put(cdf_r.data(), (size_t)nr);
    st.n_spatial = put(nsp.data(), (size_t)nr);
    st.cdf_p = put(cdf_p.data(), cdf_p.size());
    if (!st.r_grid || !st.p_grid || !st.cdf_r || !st.n_spatial || !st.cdf_p)
        return fail(c, LIM_ERR_CUDA, "lim_sample_fonll: table upload failed");
    int* dm = (int*)(d + off);
    LIM_CUDA(c, cudaMemcpyAsync(dm, mass.data(), mass.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    st.p_mass = dm;
    st.failed = (unsigned long long*)(((uintptr_t)(dm + nr) + 15) & ~(uintptr_t)15);
    st.nr = (int)nr; st.np = (int)np;
    st.f_max = fmax;
    st.rmax = r_grid[nr - 1];
    st.cartesian = cartesian != 0;
    st.antithetic = antithetic != 0;
    st.with_pz = thermal_pz != 0;
    st.med_kind = c->med_kind;
    st.max_trials = 100000;
    c->dims = 2;
    c->pdim = (int)c->P.pdim;
    c->have_state = false;
    rc = c->P.precision == LIM_FP32 ? sample_impl<float>(c, st, n) : sample_impl<double>(c, st, n);
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));    // the host tables are released on return
    return rc;
}

int lim_sample_milne(lim_ctx* c, double x_lo, double x_hi, int64_t nbins, const double* T_c, const double* ur_c,
                     const double* mu_c, const double* r_T, const double* T_r, int64_t nT, int64_t n)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    int rc = state_rows_ok(c);
    if (rc) return rc;
    if (c->P.coords != LIM_COORDS_MILNE || c->P.dims != 2 || c->P.pdim != 2)
        return fail(c, LIM_ERR_UNSUPPORTED, "Milne sampling requires dim = 2 (τ, r)");
    if (n < 0 || n > (int64_t)UINT32_MAX) return fail(c, LIM_ERR_ARG, "lim_sample_milne: particle count out of range");
    if (!T_c || !ur_c || !mu_c || !r_T || !T_r || nbins < 1 || nbins > INT32_MAX || nT < 2 || nT > INT32_MAX ||
        !(x_hi > x_lo) || !std::isfinite(x_lo) || !std::isfinite(x_hi))
        return fail(c, LIM_ERR_ARG, "lim_sample_milne: need x_lo < x_hi, nbins >= 1 profile values and a T(r) "
                                    "table of at least 2 nodes");
    if (!ascending(r_T, (size_t)nT)) return fail(c, LIM_ERR_ARG, "lim_sample_milne: r_T must be strictly ascending");
    // utils.jl:356-373 in FP64: bin centers, n_boltz = T^(3/2)/gamma exp((mu - m gamma)/T), pdf = n/sum(n)/dx
    const double m = c->P.m;
    const double dx = (x_hi - x_lo) / (double)nbins;
    std::vector<double> centers((size_t)nbins), nb((size_t)nbins), ratio((size_t)nbins);
    double sum = 0.0;
    for (int64_t k = 0; k < nbins; ++k) {
        const double e0 = x_lo + dx * (double)k, e1 = x_lo + dx * (double)(k + 1);
        centers[k] = (e0 + e1) / 2.0;
        const double g = std::sqrt(1.0 + ur_c[k] * ur_c[k]);
        nb[k] = std::pow(T_c[k], 1.5) / g * std::exp((mu_c[k] - m * g) / T_c[k]);
        sum += nb[k];
    }
    double pmax = 0.0;
    for (int64_t k = 0; k < nbins; ++k) { ratio[k] = nb[k] / sum / dx; pmax = std::max(pmax, ratio[k]); }
    if (!(pmax > 0.0) || !std::isfinite(pmax))
        return fail(c, LIM_ERR_ARG, "lim_sample_milne: the binned density has no positive finite maximum");
    for (int64_t k = 0; k < nbins; ++k) ratio[k] /= pmax;
    const size_t doubles = (size_t)(3 * nbins + 2 * nT);
    cudaSetDevice(c->device);
    if ((rc = dev_alloc(c, c->d_sample, doubles * sizeof(double) + 64))) return rc;
    double* d = (double*)c->d_sample.p;
    MilneTables mt;
    std::memset(&mt, 0, sizeof mt);
    mt.centers = d;
    mt.ratio = d + nbins;
    mt.rT = d + 2 * nbins;
    mt.TT = d + 2 * nbins + nT;
    mt.failed = (unsigned long long*)(((uintptr_t)(d + 2 * nbins + 2 * nT) + 15) & ~(uintptr_t)15);
    LIM_CUDA(c, cudaMemcpyAsync((void*)mt.centers, centers.data(), nbins * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    LIM_CUDA(c, cudaMemcpyAsync((void*)mt.ratio, ratio.data(), nbins * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    LIM_CUDA(c, cudaMemcpyAsync((void*)mt.rT, r_T, nT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    LIM_CUDA(c, cudaMemcpyAsync((void*)mt.TT, T_r, nT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    mt.nbins = (int)nbins;
    mt.nT = (int)nT;
    mt.lo = x_lo;
    mt.hi = x_hi;
    mt.max_trials = 100000;
    c->dims = 2;
    c->pdim = 2;
    c->have_state = false;
    rc = c->P.precision == LIM_FP32 ? sample_milne_impl<float>(c, mt, n) : sample_milne_impl<double>(c, mt, n);
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return rc;
}

int lim_download_state(lim_ctx* c, double* x, double* p)
{
    if (!c) return LIM_ERR_ARG;
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "no particle state uploaded");
    cudaSetDevice(c->device);
    return c->state_prec == LIM_FP32 ? download_state_impl<float>(c, x, p) : download_state_impl<double>(c, x, p);
}

namespace {
// The buffers a checkpoint covers, with their sizes for the current state.
int state_buffers(lim_ctx* c, DevBuf** bufs, size_t* sizes)
{
    int k = 0;
    const size_t n = (size_t)c->n;
    const size_t rb = c->state_prec == LIM_FP32 ? sizeof(float) : sizeof(double);
    for (int d = 0; d < c->dims; ++d) {
        bufs[k] = &c->d_x[d]; sizes[k++] = n * rb;
        if (c->state_prec == LIM_FP32) { bufs[k] = &c->d_xlo[d]; sizes[k++] = n * sizeof(float); }
    }
    for (int d = 0; d < c->pdim; ++d) { bufs[k] = &c->d_p[d]; sizes[k++] = n * sizeof(double); }
    if (c->P.freezeout_capture) {
        for (int d = 0; d < c->dims; ++d) {
            bufs[k] = &c->d_fo_pos[d]; sizes[k++] = n * sizeof(double);
            bufs[k] = &c->d_l_pos[d]; sizes[k++] = n * sizeof(double);
        }
        for (int d = 0; d < c->pdim; ++d) {
            bufs[k] = &c->d_fo_mom[d]; sizes[k++] = n * sizeof(double);
            bufs[k] = &c->d_l_mom[d]; sizes[k++] = n * sizeof(double);
        }
        DevBuf* f[4] = { &c->d_fo_tau, &c->d_fo_flag, &c->d_l_tau, &c->d_l_T };
        for (DevBuf* b : f) { bufs[k] = b; sizes[k++] = n * sizeof(double); }
    }
    bufs[k] = &c->d_status; sizes[k++] = sizeof(unsigned long long);
    return k;
}
}  // namespace

int lim_state_save(lim_ctx* c)
{
    if (!c) return LIM_ERR_ARG;
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "no particle state uploaded");
    cudaSetDevice(c->device);
    DevBuf* bufs[40];
    size_t sizes[40];
    const int k = state_buffers(c, bufs, sizes);
    size_t total = 0;
    for (int j = 0; j < k; ++j) total += (sizes[j] + 255) & ~(size_t)255;
    int rc = dev_alloc(c, c->d_ckpt, total);
    if (rc) return rc;
    size_t off = 0;
    for (int j = 0; j < k; ++j) {
        if (sizes[j]) LIM_CUDA(c, cudaMemcpyAsync((char*)c->d_ckpt.p + off, bufs[j]->p, sizes[j], cudaMemcpyDeviceToDevice, c->stream));
        off += (sizes[j] + 255) & ~(size_t)255;
    }
    c->ckpt_n = c->n;
    return LIM_OK;
}

int lim_state_restore(lim_ctx* c)
{
    if (!c) return LIM_ERR_ARG;
    if (!c->have_state || !c->d_ckpt.p || c->ckpt_n != c->n)
        return fail(c, LIM_ERR_STATE, "no checkpoint of the current state (lim_state_save)");
    cudaSetDevice(c->device);
    DevBuf* bufs[40];
    size_t sizes[40];
    const int k = state_buffers(c, bufs, sizes);
    size_t off = 0;
    for (int j = 0; j < k; ++j) {
        if (sizes[j]) LIM_CUDA(c, cudaMemcpyAsync(bufs[j]->p, (char*)c->d_ckpt.p + off, sizes[j], cudaMemcpyDeviceToDevice, c->stream));
        off += (sizes[j] + 255) & ~(size_t)255;
    }
    return LIM_OK;
}

int lim_initial_lab_boost(lim_ctx* c)
{
    if (!c) return LIM_ERR_ARG;
    int rc = check_ready(c);
    if (rc) return rc;
    if (c->P.coords == LIM_COORDS_MILNE) return LIM_OK;   // the Milne CPU driver has no step-0 boost
    cudaSetDevice(c->device);
    if (c->state_prec == LIM_FP32) {
        KParams<float> kp;
        if ((rc = build_kparams<float>(c, kp))) return rc;
        LIM_CUDA(c, launch_lab_boost<float>(kp, block_of(c), c->stream));
    } else {
        KParams<double> kp;
        if ((rc = build_kparams<double>(c, kp))) return rc;
        LIM_CUDA(c, launch_lab_boost<double>(kp, block_of(c), c->stream));
    }
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return LIM_OK;
}

int lim_run(lim_ctx* c, int64_t first_step, int64_t nsteps, int64_t save_every, int64_t first_slot,
            double* hist_x, double* hist_p)
{
    if (!c) return LIM_ERR_ARG;
    int rc = check_ready(c);
    if (rc) return rc;
    if (nsteps < 0) return fail(c, LIM_ERR_ARG, "lim_run: negative step count");
    if (first_step < 0 || first_step + nsteps > (int64_t)UINT32_MAX) return fail(c, LIM_ERR_ARG, "lim_run: steps must lie in [0, 2^32)");
    if (save_every < 0) return fail(c, LIM_ERR_ARG, "lim_run: negative save_every");
    cudaSetDevice(c->device);
    return c->state_prec == LIM_FP32 ? run_impl<float>(c, first_step, nsteps, save_every, first_slot, hist_x, hist_p)
                                     : run_impl<double>(c, first_step, nsteps, save_every, first_slot, hist_x, hist_p);
}

}  // extern "C"

namespace {

int reduce_setup(lim_ctx* c, const lim_reduce_spec* spec, int64_t nslots, SnapshotReduce& red)
{
    if (!spec || spec->r_bins < 1 || spec->r_bins > kReduceBinsMax || spec->pt_bins < 1 ||
        spec->pt_bins > kReduceBinsMax || !(spec->r_max > 0.0) || !(spec->pt_max > 0.0) ||
        !std::isfinite(spec->r_max) || !std::isfinite(spec->pt_max))
        return fail(c, LIM_ERR_ARG, "lim_reduce_spec: need 1..%d bins and finite positive r_max, pt_max",
                    kReduceBinsMax);
    red.rs.r_bins = (int)spec->r_bins;
    red.rs.pt_bins = (int)spec->pt_bins;
    red.rs.r_scale = (double)spec->r_bins / spec->r_max;
    red.rs.pt_scale = (double)spec->pt_bins / spec->pt_max;
    red.nslots = nslots;
    const int64_t nb = c->n == 0 ? 1 : (c->n + 255) / 256;
    int rc;
    if ((rc = dev_alloc(c, c->d_partials, (size_t)nb * kObsNum * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_red_obs, (size_t)nslots * kObsNum * sizeof(double)))) return rc;
    if ((rc = dev_alloc(c, c->d_red_hist, (size_t)nslots * reduce_hist_len(red.rs) * sizeof(unsigned long long))))
        return rc;
    LIM_CUDA(c, cudaMemsetAsync(c->d_red_obs.p, 0, (size_t)nslots * kObsNum * sizeof(double), c->stream));
    LIM_CUDA(c, cudaMemsetAsync(c->d_red_hist.p, 0, (size_t)nslots * reduce_hist_len(red.rs) * sizeof(unsigned long long),
                                c->stream));
    return LIM_OK;
}

// The device slots into out (host): per slot LIM_OBS_NUM sums, then the histograms as
// doubles (counts exact; the cos 2 phi sums from their 2^-32 fixed point).
int reduce_download(lim_ctx* c, const SnapshotReduce& red, double* out)
{
    const int64_t hl = reduce_hist_len(red.rs), stride = kObsNum + hl;
    std::vector<double> obs((size_t)red.nslots * kObsNum);
    std::vector<unsigned long long> hist((size_t)(red.nslots * hl));
    LIM_CUDA(c, cudaMemcpyAsync(obs.data(), c->d_red_obs.p, obs.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    LIM_CUDA(c, cudaMemcpyAsync(hist.data(), c->d_red_hist.p, hist.size() * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    const int64_t ncount = red.rs.r_bins + 1 + red.rs.pt_bins + 1;
    for (int64_t k = 0; k < red.nslots; ++k) {
        double* o = out + k * stride;
        for (int j = 0; j < kObsNum; ++j) o[j] = obs[(size_t)(k * kObsNum + j)];
        const unsigned long long* h = hist.data() + k * hl;
        for (int64_t j = 0; j < hl; ++j)
            o[kObsNum + j] = j < ncount ? (double)h[j] : (double)(long long)h[j] * 0x1p-32;
    }
    return LIM_OK;
}

}  // namespace

extern "C" {

int64_t lim_reduce_stride(const lim_reduce_spec* spec)
{
    if (!spec || spec->r_bins < 1 || spec->pt_bins < 1) return -1;
    return LIM_OBS_NUM + spec->r_bins + 1 + 2 * (spec->pt_bins + 1);
}

int lim_reduce_state(lim_ctx* c, const lim_reduce_spec* spec, double* out)
{
    if (!c || !out) return LIM_ERR_ARG;
    int rc = check_ready(c);
    if (rc) return rc;
    cudaSetDevice(c->device);
    SnapshotReduce red;
    if ((rc = reduce_setup(c, spec, 1, red))) return rc;
    if (c->state_prec == LIM_FP32) {
        KParams<float> kp;
        if ((rc = build_kparams<float>(c, kp)) || (rc = reduce_snapshot<float>(c, kp, red, 0))) return rc;
    } else {
        KParams<double> kp;
        if ((rc = build_kparams<double>(c, kp)) || (rc = reduce_snapshot<double>(c, kp, red, 0))) return rc;
    }
    return reduce_download(c, red, out);
}

int lim_run_static_T(lim_ctx* c, double T, int64_t first_step, int64_t nsteps, int64_t save_every,
                     int64_t first_slot, int64_t nslots, double* hist_pmag)
{
    if (!c) return LIM_ERR_ARG;
    if (!c->have_params) return fail(c, LIM_ERR_STATE, "lim_set_params must be called before running");
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "no particle state uploaded (lim_upload_state)");
    if (c->state_prec != (int)c->P.precision)
        return fail(c, LIM_ERR_STATE, "state was uploaded in another precision; upload it again");
    if (c->P.coords != LIM_COORDS_CARTESIAN)
        return fail(c, LIM_ERR_UNSUPPORTED, "lim_run_static_T: the static-temperature path is Cartesian");
    if (nsteps < 0) return fail(c, LIM_ERR_ARG, "lim_run_static_T: negative step count");
    if (first_step < 0 || first_step + nsteps > (int64_t)UINT32_MAX)
        return fail(c, LIM_ERR_ARG, "lim_run_static_T: steps must lie in [0, 2^32)");
    if (save_every < 0 || nslots < 0) return fail(c, LIM_ERR_ARG, "lim_run_static_T: negative save_every or nslots");
    const bool saving = save_every > 0 && nslots > 0 && hist_pmag;
    const double hist_bytes = saving ? (double)nslots * (double)c->n * sizeof(double) : 0.0;
    if (hist_bytes > 16.0e9) return fail(c, LIM_ERR_ARG, "lim_run_static_T: history of %.3g bytes is too large", hist_bytes);
    cudaSetDevice(c->device);
    StaticRun sr{};
    for (int d = 0; d < 3; ++d) sr.p[d] = d < c->pdim ? (double*)c->d_p[d].p : nullptr;
    sr.n = c->n;
    sr.pid_offset = c->P.particle_offset;
    sr.T = T;
    sr.m = c->P.m;
    sr.dt = c->P.dt;
    {
        uint32_t k0 = (uint32_t)(uint64_t)c->P.seed, k1 = (uint32_t)((uint64_t)c->P.seed >> 32);
        for (int r = 0; r < 10; ++r) { sr.rk[r] = make_uint2(k0, k1); k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
    sr.save_every = saving ? save_every : 0;
    sr.first_slot = first_slot;
    sr.nslots = saving ? nslots : 0;
    if (saving && c->n > 0) {
        int rc = dev_alloc(c, c->d_pmag_hist, (size_t)hist_bytes);
        if (rc) return rc;
        LIM_CUDA(c, cudaMemcpyAsync(c->d_pmag_hist.p, hist_pmag, (size_t)hist_bytes, cudaMemcpyHostToDevice, c->stream));
        sr.hist = (double*)c->d_pmag_hist.p;
    }
    LIM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    LIM_CUDA(c, c->state_prec == LIM_FP32 ? launch_static_T<float>(sr, c->pdim, first_step, first_step + nsteps, c->stream)
                                          : launch_static_T<double>(sr, c->pdim, first_step, first_step + nsteps, c->stream));
    LIM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    if (saving && c->n > 0)
        LIM_CUDA(c, cudaMemcpyAsync(hist_pmag, c->d_pmag_hist.p, (size_t)hist_bytes, cudaMemcpyDeviceToHost, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.0f;
    LIM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    c->last_launches = (c->n > 0 && nsteps > 0) ? 1 : 0;
    return LIM_OK;
}

int lim_run_reduced(lim_ctx* c, int64_t first_step, int64_t nsteps, int64_t save_every, int64_t first_slot,
                    int64_t nslots, const lim_reduce_spec* spec, double* out)
{
    if (!c || !out) return LIM_ERR_ARG;
    int rc = check_ready(c);
    if (rc) return rc;
    if (nsteps < 0) return fail(c, LIM_ERR_ARG, "lim_run_reduced: negative step count");
    if (first_step < 0 || first_step + nsteps > (int64_t)UINT32_MAX)
        return fail(c, LIM_ERR_ARG, "lim_run_reduced: steps must lie in [0, 2^32)");
    if (save_every < 1 || nslots < 1) return fail(c, LIM_ERR_ARG, "lim_run_reduced: need save_every >= 1 and nslots >= 1");
    cudaSetDevice(c->device);
    SnapshotReduce red;
    if ((rc = reduce_setup(c, spec, nslots, red))) return rc;
    rc = c->state_prec == LIM_FP32 ? run_impl<float>(c, first_step, nsteps, save_every, first_slot, nullptr, nullptr, &red)
                                   : run_impl<double>(c, first_step, nsteps, save_every, first_slot, nullptr, nullptr, &red);
    if (rc) return rc;
    return reduce_download(c, red, out);
}

int lim_host_alloc(int64_t bytes, void** out)
{
    if (!out || bytes < 0) {
        lim::set_noctx_error("lim_host_alloc: need a size >= 0 and an output pointer");
        return LIM_ERR_ARG;
    }
    *out = nullptr;
    if (bytes == 0) return LIM_OK;
    const cudaError_t e = cudaHostAlloc(out, (size_t)bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        *out = nullptr;
        lim::set_noctx_error((std::string("lim_host_alloc: cudaHostAlloc failed: ") + cudaGetErrorString(e)).c_str());
        return LIM_ERR_NOMEM;
    }
    return LIM_OK;
}

int lim_host_free(void* ptr)
{
    if (ptr && cudaFreeHost(ptr) != cudaSuccess) {
        lim::set_noctx_error("lim_host_free: cudaFreeHost failed");
        return LIM_ERR_CUDA;
    }
    return LIM_OK;
}

int lim_status(lim_ctx* c, int64_t* first_bad_step)
{
    if (!c || !first_bad_step) return LIM_ERR_ARG;
    *first_bad_step = -1;
    if (!c->d_status.p) return LIM_OK;
    unsigned long long bad = ULLONG_MAX;
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    LIM_CUDA(c, cudaMemcpy(&bad, c->d_status.p, sizeof bad, cudaMemcpyDeviceToHost));
    if (bad != ULLONG_MAX) *first_bad_step = (int64_t)bad;
    return LIM_OK;
}

int lim_download_freezeout(lim_ctx* c, double* fo_pos, double* fo_mom, double* fo_tau, double* fo_flag)
{
    if (!c) return LIM_ERR_ARG;
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "no particle state uploaded");
    cudaSetDevice(c->device);
    return c->state_prec == LIM_FP32 ? download_fo_impl<float>(c, fo_pos, fo_mom, fo_tau, fo_flag)
                                     : download_fo_impl<double>(c, fo_pos, fo_mom, fo_tau, fo_flag);
}

int lim_observables(lim_ctx* c, int from_freezeout, double* out)
{
    if (!c || !out) return LIM_ERR_ARG;
    int rc = check_ready(c);
    if (rc) return rc;
    cudaSetDevice(c->device);
    return c->state_prec == LIM_FP32 ? observables_impl<float>(c, from_freezeout, out)
                                     : observables_impl<double>(c, from_freezeout, out);
}

int lim_record_noise(lim_ctx* c, int64_t first_step, int64_t nsteps)
{
    if (!c) return LIM_ERR_ARG;
    ++c->gen;
    if (nsteps <= 0) { dev_free(c->d_rec); c->rec_steps = 0; return LIM_OK; }
    if (!c->have_state) return fail(c, LIM_ERR_STATE, "upload the state before enabling noise recording");
    const double bytes = (double)nsteps * kNoiseSlots * (double)c->n * sizeof(double);
    if (bytes > 8.0e9) return fail(c, LIM_ERR_ARG, "lim_record_noise: buffer of %.3g bytes is too large", bytes);
    cudaSetDevice(c->device);
    int rc = dev_alloc(c, c->d_rec, (size_t)bytes);
    if (rc) return rc;
    LIM_CUDA(c, cudaMemsetAsync(c->d_rec.p, 0, (size_t)bytes, c->stream));
    c->rec_first = first_step;
    c->rec_steps = nsteps;
    return LIM_OK;
}

int lim_download_noise(lim_ctx* c, double* out)
{
    if (!c || !out) return LIM_ERR_ARG;
    if (!c->d_rec.p) return fail(c, LIM_ERR_STATE, "noise recording is off");
    const size_t bytes = (size_t)c->rec_steps * kNoiseSlots * (size_t)c->n * sizeof(double);
    LIM_CUDA(c, cudaMemcpyAsync(out, c->d_rec.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return LIM_OK;
}

int lim_philox_device(lim_ctx* c, const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    if (!c || !ctr || !key || !out) return LIM_ERR_ARG;
    cudaSetDevice(c->device);
    int rc = dev_alloc(c, c->d_probe, 16 * sizeof(uint32_t));
    if (rc) return rc;
    uint32_t ck[6] = { ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1] };
    LIM_CUDA(c, cudaMemcpyAsync(c->d_probe.p, ck, sizeof ck, cudaMemcpyHostToDevice, c->stream));
    LIM_CUDA(c, launch_philox_probe((const uint32_t*)c->d_probe.p, (uint32_t*)c->d_probe.p + 8, c->stream));
    LIM_CUDA(c, cudaMemcpyAsync(out, (uint32_t*)c->d_probe.p + 8, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    LIM_CUDA(c, cudaStreamSynchronize(c->stream));
    return LIM_OK;
}

int lim_probe_fma_rate(lim_ctx* c, double* thread_fma_per_s, double* ms_out)
{
    if (!c || !thread_fma_per_s) return LIM_ERR_ARG;
    cudaSetDevice(c->device);
    int nsm = 0;
    LIM_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const int blocks = nsm * 8, iters = 4096;
    int rc = dev_alloc(c, c->d_probe, (size_t)blocks * 256 * sizeof(float));
    if (rc) return rc;
    LIM_CUDA(c, launch_fma_probe((float*)c->d_probe.p, blocks, 64, c->stream));   // warm-up
    LIM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    LIM_CUDA(c, launch_fma_probe((float*)c->d_probe.p, blocks, iters, c->stream));
    LIM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    LIM_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    LIM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *thread_fma_per_s = (double)blocks * 256.0 * iters * 64.0 / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return LIM_OK;
}

int lim_probe_mufu_rate(lim_ctx* c, double* thread_mufu_per_s, double* ms_out)
{
    if (!c || !thread_mufu_per_s) return LIM_ERR_ARG;
    cudaSetDevice(c->device);
    int nsm = 0;
    LIM_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const int blocks = nsm * 8, iters = 512;
    int rc = dev_alloc(c, c->d_probe, (size_t)blocks * 256 * sizeof(float));
    if (rc) return rc;
    LIM_CUDA(c, launch_mufu_probe((float*)c->d_probe.p, blocks, 16, c->stream));   // warm-up
    LIM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    LIM_CUDA(c, launch_mufu_probe((float*)c->d_probe.p, blocks, iters, c->stream));
    LIM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    LIM_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    LIM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *thread_mufu_per_s = (double)blocks * 256.0 * iters * 64.0 / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return LIM_OK;
}

int lim_last_run_stats(lim_ctx* c, double* kernel_ms, int64_t* launches)
{
    if (!c) return LIM_ERR_ARG;
    if (kernel_ms) *kernel_ms = c->last_ms;
    if (launches) *launches = c->last_launches;
    return LIM_OK;
}

}  // extern "C"

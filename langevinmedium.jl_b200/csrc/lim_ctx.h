// lim_ctx.h — the engine context behind the C-ABI handle `lim_ctx`, shared by the
// translation units of the C-ABI (single-ensemble runs and batches).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/langevin_b200.h"
#include "lim_internal.h"

namespace lim {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace lim

struct lim_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    lim_params P{};
    bool have_params = false;

    // host copy of the medium
    int med_kind = -1;
    std::vector<double> xg, tg, T, V, V2;
    double bj_T0 = 0, bj_tau0 = 0, bj_power = 0, bj_rmax = 0;
    int64_t gnx = 0, gny = 0, gnt = 0;
    double gx0 = 0, gdx = 0, gy0 = 0, gdy = 0, gt0 = 0, gdt = 0;
    std::vector<float> gT, gux, guy;
    std::vector<double> spl[4];           // drag, RTA, d(drag)/da, d(drag)/db
    double spl_Tmin[4] = { 0, 0, 0, 0 }, spl_invdT[4] = { 1, 1, 1, 1 };
    std::vector<double> icdf;
    int64_t nU = 0, nT = 0;
    double ic_Tmin = 0, ic_invdT = 1;
    double T_scale = 1.0;

    // device copy of the medium for `dev_prec`
    int dev_prec = -1;
    bool dev_dirty = true;
    lim::DevBuf d_xg, d_tg, d_tgd, d_xgd, d_TV, d_V2, d_G, d_spl[4], d_icdf;
    lim::DevBuf d_TVc, d_xc;              // per-cell (r, t) records for the step's lookup

    // particle state (structure of arrays, precision `state_prec`)
    int64_t n = 0;
    int dims = 0, pdim = 0, state_prec = -1;
    bool have_state = false;
    lim::DevBuf d_x[3], d_xlo[3], d_p[3];
    lim::DevBuf d_fo_pos[3], d_fo_mom[3], d_fo_tau, d_fo_flag, d_l_pos[3], d_l_mom[3], d_l_tau, d_l_T;
    lim::DevBuf d_status, d_stage_x, d_stage_p, d_partials, d_obs, d_probe, d_steps;
    lim::DevBuf d_rec, d_ckpt;
    lim::DevBuf d_live[2], d_live_n;      // live lists of a stop-at-freeze-out run
    lim::DevBuf d_rta_bits;               // recorded / replayed RTA decisions
    lim::DevBuf d_sample;                 // sampling tables (lim_sample_fonll)
    lim::DevBuf d_red_obs, d_red_hist;    // snapshot reductions (lim_run_reduced)
    lim::DevBuf d_pmag_hist;              // |p| history of lim_run_static_T
    lim::DevBuf d_rta64, d_T64;           // FP32 runs: FP64 RTA spline and (r, t) T table
    int rta_mode = 0;
    int64_t rta_first = 0, rta_steps = 0;
    lim::DevBuf d_adj_ckpt, d_adj_tape, d_adj_table, d_adj_part, d_adj_out;   // lim_adjoint
    lim::DevBuf d_adj_lam, d_adj_gacc, d_adj_slope, d_adj_icdt;
    double adj_fwd_ms = 0.0, adj_rev_ms = 0.0;
    int64_t rec_first = 0, rec_steps = 0, ckpt_n = -1;

    // bumped by every call that may move or re-shape a device buffer, so that a batch
    // holding this context's parameters knows to rebuild them
    uint64_t gen = 0;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // snapshot copies to the host overlap the next interval's steps: a copy stream, two
    // staging buffers (d_stage_* and d_stage2_*) and their "staged" events (made on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_snap[2] = { nullptr, nullptr };
    lim::DevBuf d_stage2_x, d_stage2_p;
    double last_ms = 0.0;
    int64_t last_launches = 0;
};


namespace lim {

// Context services used by the batch entry points (defined in lim_capi.cu).
int ctx_fail(lim_ctx* c, int code, const char* fmt, ...);
int ctx_alloc(lim_ctx* c, DevBuf& b, size_t bytes);
int ctx_check_ready(lim_ctx* c);
template <typename R> int ctx_build_kparams(lim_ctx* c, KParams<R>& kp);

}  // namespace lim

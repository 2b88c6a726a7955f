/*
 * langevin_b200.h — C-ABI of the B200 (sm_100a) heavy-quark Langevin engine.
 *
 * Drop-in boundary for the per-particle Langevin time loop of LangevInMedium.jl.
 * Every entry point takes plain pointers and sizes, returns an int status
 * (0 = LIM_OK, negative = error class) and never throws across the ABI.  The
 * text of the last error is returned by lim_last_error().
 *
 * Host-side array layout is the reference's Julia layout: a (rows, N) matrix in
 * column-major order, i.e. one particle's components are contiguous:
 *     x[d + rows * i]   for component d of particle i.
 * Medium tables (Nr, Nt) are column-major too: T[i + Nr * j] is T(xgrid[i], tgrid[j]).
 * Host memory is always owned by the caller; device memory is owned by the
 * context until lim_destroy().
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   - src/simulate.jl:21-87 and src/simulate_gpu_wrapper.jl:15-72
 *       simulate_ensemble_bulk(::CPUBackend / ::GPUBackend, r_grid, p_grid,
 *       dens, Tfield, Vfield, (xgrid, tgrid); kwargs...)
 *   - src/simulate.jl:117-141 (CPU_GCBackend, Milne (tau, r) coordinates)
 *   - src/simulate_cpu.jl:215-316 / src/simulate_gpu.jl:283-392 (the step loop)
 *   - src/simulate_cpu_general_coords.jl:83-126 (the Milne step loop)
 * A Julia caller reaches these through ccall with the signatures below.
 */
#ifndef LANGEVIN_B200_H
#define LANGEVIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LIM_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------- */
enum {
    LIM_OK              = 0,
    LIM_ERR_ARG         = -1,  /* invalid argument (the reference's error(...) on bad input) */
    LIM_ERR_CUDA        = -2,  /* a CUDA runtime call failed */
    LIM_ERR_STATE       = -3,  /* call out of order (e.g. run before upload) */
    LIM_ERR_NONFINITE   = -4,  /* NaN/Inf in the particle state (simulate_cpu.jl:293-303) */
    LIM_ERR_TIMEOUT     = -5,  /* a bounded device-side wait gave up */
    LIM_ERR_UNSUPPORTED = -6,  /* option combination the engine does not provide */
    LIM_ERR_NOMEM       = -7   /* device or host allocation failed */
};

/* ---- enumerations used in lim_params -------------------------------------- */
enum { LIM_FP64 = 0, LIM_FP32 = 1 };                    /* precision of the particle arithmetic */
enum { LIM_COORDS_CARTESIAN = 0, LIM_COORDS_MILNE = 1 }; /* kernels_cpu.jl vs kernels_cpu_GC.jl */
enum {
    LIM_COLL_LANGEVIN     = 0,  /* exact-OU drag + kick (simulate_cpu.jl:252-277) */
    LIM_COLL_RTA          = 1,  /* BGK/RTA resampling (simulate_cpu.jl:234-251, GPU form kernels_gpu.jl:653-704) */
    LIM_COLL_LANGEVIN_RTA = 2,  /* OU kick then RTA resample in the same LRF step (new; not a reference mode) */
    LIM_COLL_FLUID        = 3   /* momentum_langevin=false or DsT==0: set_to_fluid_velocity (simulate_cpu.jl:229-233) */
};
enum {
    LIM_MEDIUM_RT      = 0,     /* reference (r, t) tables, bilinear (kernels_cpu.jl:22-51) */
    LIM_MEDIUM_BJORKEN = 1,     /* analytic T(tau) = T0 (tau0/tau)^p, zero transverse flow */
    LIM_MEDIUM_GRID    = 2      /* 2+1D grid T, u^x, u^y on (tau, x, y), trilinear */
};
enum { LIM_SPLINE_DRAG = 0, LIM_SPLINE_RTA = 1,         /* transport.jl:208-222 */
       LIM_SPLINE_DRAG_DA = 2, LIM_SPLINE_DRAG_DB = 3 }; /* d(drag time)/da, /db (lim_adjoint) */
enum {                                                   /* observables reduced in FP64 on device */
    LIM_OBS_COUNT = 0,        /* number of particles counted (alive, or frozen-out when fo mode) */
    LIM_OBS_MEAN_PT,          /* <sqrt(px^2+py^2)> */
    LIM_OBS_MEAN_COS2PHI,     /* <cos 2 phi_p> = <(px^2-py^2)/pT^2> */
    LIM_OBS_FRAC_PT_GT,       /* fraction with pT > obs_pt_cut (sharp) */
    LIM_OBS_FRAC_PT_GT_SMOOTH,/* <sigmoid((pT - cut)/width)> */
    LIM_OBS_MEAN_P2,          /* <|p|^2> over all momentum rows */
    LIM_OBS_MEAN_E,           /* <sqrt(m^2+|p|^2)> */
    LIM_OBS_MEAN_LAM1_NUM,    /* <(m/E) |p|^2> (lambda_1 numerator, test_momentum_dims3.jl:74-78) */
    LIM_OBS_MEAN_PX,          /* <p_x> */
    LIM_OBS_MEAN_WPX,         /* <(m/E) p_x> */
    LIM_OBS_MEAN_PZ2,         /* <p_z^2> (row 3) */
    LIM_OBS_MEAN_X2,          /* <sum_d x_d^2> over position rows */
    LIM_OBS_NUM               /* number of observables written by lim_observables */
};

/*
 * Run configuration.  Every field is 8 bytes wide so that the struct has the
 * same layout in C, Julia (an isbits struct of Float64/Int64) and Python ctypes.
 * Field meanings follow the reference keyword arguments
 * (simulate_gpu_wrapper.jl:23-52).
 */
typedef struct lim_params {
    double  dt;                 /* Δt [fm/c] */
    double  t0;                 /* initial_time; medium time at step s is s*dt + t0 */
    double  m;                  /* heavy-quark mass [GeV] */
    double  DsT;                /* DsT; <= 0 disables the drag (kernels_cpu.jl:270) */
    double  Tfo;                /* freeze-out temperature for the latch (kernels_gpu.jl:588-635) */
    double  psi2;               /* event-plane angle of the optional v2 modulation */
    double  obs_pt_cut;         /* pT threshold of LIM_OBS_FRAC_PT_GT[_SMOOTH] [GeV] */
    double  obs_pt_width;       /* sigmoid width of LIM_OBS_FRAC_PT_GT_SMOOTH [GeV] */
    int64_t dims;               /* position rows: 1 (radial mode), 2 or 3; Milne: 2 = (tau, r) */
    int64_t pdim;               /* momentum rows (momentum_dimensions resolved; 0 => dims) */
    int64_t coords;             /* LIM_COORDS_* */
    int64_t collision;          /* LIM_COLL_* */
    int64_t relativistic;       /* 1: Lorentz boosts, drag eta*m/E, stream p/E; 0: Galilean, eta, p/m */
    int64_t bjorken_redshift;   /* 1: p_z *= tau_a/(tau_a+dt) in the LRF (kernels_cpu.jl:427-435) */
    int64_t position_diffusion; /* 1: x += sqrt(2 D dt) xi with D = DsT/T/fmGeV (kernels_cpu.jl:592-607) */
    int64_t reflecting_boundary;/* 1: reflect at r_max = last(xgrid) (kernels_cpu.jl:609-634) */
    int64_t integrator_mode;    /* 0: pre-point exact OU; 1: drift-midpoint (kernels_gpu.jl:368-381) */
    int64_t freezeout_capture;  /* 1: latch state at the first T < Tfo */
    int64_t freezeout_interp;   /* 1: interpolate the latch linearly in T to T = Tfo */
    int64_t precision;          /* LIM_FP64 or LIM_FP32 */
    int64_t seed;               /* Philox-4x32-10 key (64 bit) */
    int64_t particle_offset;    /* global id of particle 0 (shards keep the global noise stream) */
    int64_t stop_after_freezeout; /* 1: stop evolving a particle once latched (fo outputs unchanged) */
    int64_t block_size;         /* threads per block of the step kernel, a multiple of 32 up to 256;
                                   0 = the measured default (128 or 256 by kernel) */
} lim_params;

typedef struct lim_ctx lim_ctx;

/* ---- context ---------------------------------------------------------------- */
int         lim_abi_version(void);
/* Create a context on CUDA device `device`.  `stream` is a cudaStream_t (may be
 * NULL for a private stream), so the engine can share a caller's stream
 * (CUDA.jl: CUDA.stream().handle). */
int         lim_create(int device, void* stream, lim_ctx** out);
int         lim_destroy(lim_ctx* ctx);
/* Text of the last error on this context (or of the last failed lim_create when
 * ctx is NULL).  Valid until the next call on the same context. */
const char* lim_last_error(const lim_ctx* ctx);
int         lim_synchronize(lim_ctx* ctx);
/* Bytes of device memory the context currently holds. */
int         lim_device_bytes(const lim_ctx* ctx, int64_t* bytes);

/* ---- configuration ------------------------------------------------------------ */
int lim_set_params(lim_ctx* ctx, const lim_params* params);

/* Reference (r, t) medium: xgrid (nr, ascending), tgrid (nt, ascending),
 * T and V column-major (nr, nt); V2 (nr, nt) or NULL (no v2 modulation).
 * Replaces the CuArray uploads of simulate_gpu.jl:81-88. */
int lim_set_medium_rt(lim_ctx* ctx,
                      const double* xgrid, int64_t nr,
                      const double* tgrid, int64_t nt,
                      const double* T, const double* V, const double* V2);

/* Analytic Bjorken medium: T(tau) = T0 * (tau0 / tau)^power for tau >= tau0
 * (T0 for tau < tau0), zero transverse flow.  r_max bounds reflection. */
int lim_set_medium_bjorken(lim_ctx* ctx, double T0, double tau0, double power, double r_max);

/* 2+1D medium on a uniform grid: fields in FP32, row-major [it][iy][ix]
 * (ix fastest), node (ix, iy, it) at (x0 + ix*dx, y0 + iy*dy, tau0 + it*dtau).
 * u^x, u^y are the flow velocity components (as the reference's VelocityEvolution is a
 * velocity, kernels_cpu.jl:80,105): speed |u| along u / |u|. */
int lim_set_medium_grid(lim_ctx* ctx,
                        int64_t nx, int64_t ny, int64_t nt,
                        double x0, double dx, double y0, double dy,
                        double tau0, double dtau,
                        const float* T, const float* ux, const float* uy);

/* Uniform-grid linear spline of a transport time in fm (transport.jl:165-253):
 * vals[k] at T = Tmin + k/invdT, k = 0..n-1.  which = LIM_SPLINE_DRAG (the drag
 * time 1/eta_D) or LIM_SPLINE_RTA (the RTA relaxation time); LIM_SPLINE_DRAG_DA and
 * LIM_SPLINE_DRAG_DB hold the derivatives of the drag values w.r.t. two parameters
 * (a, b) of D_s(T) on the drag spline's grid, for lim_adjoint. */
int lim_set_spline(lim_ctx* ctx, int which, double Tmin, double invdT,
                   const double* vals, int64_t n);

/* ---- transport tables built on the device ------------------------------------------
 * The reference builds its tables on the host (transport.jl:165-365); these entry
 * points build the same tables on the device (one thread per T node; one block per T
 * node of the inverse CDF) and install them in the context like lim_set_spline /
 * lim_set_invcdf, for hosts that configure many ensembles (one spline per D_s variant).
 *
 * lim_build_time_spline: vals[i] = time(T_i, m, effective_DsT(T_i)) * scale on
 * T_i = Tmin + i (Tmax - Tmin)/(nT - 1) into spline `which` (LIM_SPLINE_DRAG or
 * LIM_SPLINE_RTA), time = tau_drag (transport.jl:132-137, build_tau_drag_spline),
 * tau_n_main3 (:58-104, build_taun_current_spline) or factor (eta/s)/T (the RTA time of
 * the Langevin+RTA step; m and D_s unused).  form: effective_DsT's options
 * (transport.jl:139-156), NULL for a constant D_s; scale: LV_TAUN_SCALE (1 normally).
 * Errors as the reference's: "nT must be >= 2", "Tmin must be > 0", "Tmax must be > Tmin". */
enum { LIM_TIME_DRAG = 0, LIM_TIME_TAUN = 1, LIM_TIME_TAUR = 2 };
typedef struct lim_dsform {
    int64_t linear;         /* DsT_linear: DsT_slope max(T, Tfo) + DsT_offset */
    double slope, offset, Tfo;
    int64_t quad;           /* DsT_quad: DsT (T / DsT_Tref)^2 */
    double Tref;
} lim_dsform;
int lim_build_time_spline(lim_ctx* ctx, int which, int kind, double m, double DsT, const lim_dsform* form,
                          double Tmin, double Tmax, int64_t nT, double eta_over_s, double factor, double scale);
/* build_juttner_invcdf (transport.jl:277-365) on the device: T range padded by 2 %,
 * nT x nU table of the inverse CDF of p^(dims-1) exp(-(E - m)/T) from an np-point
 * trapezoid CDF, capped at the (1 - quantile_cap) quantile; installed as lim_set_invcdf. */
int lim_build_juttner_invcdf(lim_ctx* ctx, double m, int64_t dims, double Tmin, double Tmax, int64_t nT, int64_t nU,
                             int64_t np, double quantile_cap);
/* The installed tables (n / nU, nT always written; vals when not NULL, cap values). */
int lim_get_spline(lim_ctx* ctx, int which, double* Tmin, double* invdT, double* vals, int64_t cap, int64_t* n);
int lim_get_invcdf(lim_ctx* ctx, double* vals, int64_t cap, int64_t* nU, int64_t* nT, double* Tmin, double* invdT);

/* Medium temperature scale s: every medium temperature is s * T (default 1).  No
 * counterpart in the reference; the third parameter of lim_adjoint. */
int lim_set_medium_scale(lim_ctx* ctx, double s);

/* RTA decisions of steps [first_step, first_step + nsteps): mode 1 records the
 * decisions of the following lim_run calls, mode 2 replays them (the collision
 * indicator is taken from the record instead of comparing u_collide with dt/tau_R),
 * mode 0 drops the record.  With the counter-based noise this fixes the whole random
 * path of a run, as pathwise derivatives and their finite-difference checks need.  No
 * counterpart in the reference.  lim_copy_rta_decisions copies a record between two
 * contexts of the same particle count and sets the destination to replay. */
int lim_rta_decisions(lim_ctx* ctx, int mode, int64_t first_step, int64_t nsteps);
int lim_copy_rta_decisions(lim_ctx* dst, const lim_ctx* src);

/* Jüttner inverse-CDF table (transport.jl:277-365): vals[jT*nU + iu] = p*(u_iu; T_jT). */
int lim_set_invcdf(lim_ctx* ctx, const double* vals, int64_t nU, int64_t nT,
                   double Tmin, double invdT);

/* ---- particle state ----------------------------------------------------------- */
/* x: (dims, n) and p: (pdim, n) column-major host arrays (the Julia layout).
 * Resets the freeze-out latch and the non-finite status. */
int lim_upload_state(lim_ctx* ctx, const double* x, int64_t dims,
                     const double* p, int64_t pdim, int64_t n);
int lim_download_state(lim_ctx* ctx, double* x, double* p);

/* Device-side checkpoint of the particle state (and freeze-out latch): save
 * copies it into a device buffer owned by the context, restore copies it back.
 * With the counter-based noise, (state, step) fully determines the continuation,
 * so a restore followed by lim_run(step, ...) reproduces the original run. */
int lim_state_save(lim_ctx* ctx);
int lim_state_restore(lim_ctx* ctx);

/* The step-0 lab boost applied before the loop (simulate_cpu.jl:160-163). */
int lim_initial_lab_boost(lim_ctx* ctx);

/* Advance steps first_step .. first_step+nsteps-1 (medium time s*dt + t0).
 * When save_every > 0 and hist_x / hist_p are not NULL, the state after every
 * step s with s % save_every == 0 is written to snapshot slot
 * (s / save_every) - first_slot of the host arrays hist_x (dims, n, nslots)
 * and hist_p (pdim, n, nslots), column-major.  Returns LIM_ERR_NONFINITE (and
 * the first bad step in lim_status) if any particle became NaN/Inf. */
int lim_run(lim_ctx* ctx, int64_t first_step, int64_t nsteps,
            int64_t save_every, int64_t first_slot,
            double* hist_x, double* hist_p);

/* The static-temperature momentum-only path: simulate_ensemble_bulk(::CPUBackend,
 * T::Float64; ...) (src/simulate.jl:89-109 -> src/simulate_cpu.jl:325-404) with its
 * legacy force (src/kernels_cpu.jl:359-404): kappa = 2.5 T^3, eta_D = kappa / (2 T m),
 * Euler drag -eta_D p dt and the kick sqrt(dt) sqrt(kappa) xi on the uploaded momenta
 * (pdim rows; the positions and any medium are not used), with the context's dt, m,
 * precision, seed and particle_offset.  |p| after every step s with s % save_every == 0
 * goes to hist_pmag[(s / save_every - first_slot) * n + i] for slots in [0, nslots)
 * (the host array is copied in first, so slots not written keep their values: the
 * reference's slot 0, the initial |p|, is the caller's).  As in the reference driver,
 * no non-finite check. */
int lim_run_static_T(lim_ctx* ctx, double T, int64_t first_step, int64_t nsteps, int64_t save_every,
                     int64_t first_slot, int64_t nslots, double* hist_pmag);

/* ---- snapshots reduced on the device ---------------------------------------------
 * In place of the FP64 snapshot history (simulate_cpu.jl:319-322: pdim x N x nslots
 * momenta and positions, 38 GB for 1e7 particles and 95 saves), each snapshot is
 * reduced on the device to, per slot (stride = lim_reduce_stride(spec) doubles):
 *   [0, LIM_OBS_NUM)            the observable sums of lim_observables
 *   r_bins + 1                  counts of r = |x| (Milne: the r row) in uniform bins on
 *                               [0, r_max), the last entry counting r >= r_max: the
 *                               radial density n(r, t) (exported as n_rt, LangevInMedium.jl:44)
 *   pt_bins + 1                 counts of p_T = |(p_x, p_y)| (Milne: |p^r|), same binning
 *   pt_bins + 1                 sums of cos 2 phi_p per p_T bin (0 for Milne), each term
 *                               rounded to 2^-32: the numerator of v2(p_T)
 * Counts are exact; the cos 2 phi sums are exact sums of the rounded terms, so the
 * result does not depend on the order of summation. */
typedef struct lim_reduce_spec {
    int64_t r_bins;         /* 1 .. 4096 */
    double r_max;           /* fm */
    int64_t pt_bins;        /* 1 .. 4096 */
    double pt_max;          /* GeV */
} lim_reduce_spec;
int64_t lim_reduce_stride(const lim_reduce_spec* spec);
/* Reduce the current state into out[lim_reduce_stride(spec)]. */
int lim_reduce_state(lim_ctx* ctx, const lim_reduce_spec* spec, double* out);
/* lim_run whose snapshots (steps s with s % save_every == 0, slot s / save_every -
 * first_slot, slots outside [0, nslots) skipped) are reduced on the device instead of
 * copied; out holds nslots x lim_reduce_stride(spec) doubles, written once at the end. */
int lim_run_reduced(lim_ctx* ctx, int64_t first_step, int64_t nsteps, int64_t save_every, int64_t first_slot,
                    int64_t nslots, const lim_reduce_spec* spec, double* out);

/* Page-locked host memory for snapshot histories (and any other host buffer of the
 * engine): lim_run copies each snapshot on a copy stream while the next interval's
 * steps run, at the full host-link rate when hist_x / hist_p lie in page-locked memory
 * (about 3x the rate into pageable memory).  Allocate once and reuse: locking pages
 * costs time of its own.  No counterpart in the reference. */
int lim_host_alloc(int64_t bytes, void** out);
int lim_host_free(void* ptr);

/* First step at which a particle became non-finite, or -1. */
int lim_status(lim_ctx* ctx, int64_t* first_bad_step);

/* Freeze-out latch outputs (simulate_gpu.jl:395-396): fo_pos (dims, n),
 * fo_mom (pdim, n), fo_tau (n), fo_flag (n, 1.0 = latched). */
int lim_download_freezeout(lim_ctx* ctx, double* fo_pos, double* fo_mom,
                           double* fo_tau, double* fo_flag);

/* FP64 device reduction of the current state (or of the freeze-out latch when
 * from_freezeout != 0): out[LIM_OBS_NUM] (see the LIM_OBS_* enumeration). */
int lim_observables(lim_ctx* ctx, int from_freezeout, double* out);

/* Observables of a caller-owned device ensemble without allocating anything.
 * No counterpart in the reference: it serves hosts that cannot call cudaMalloc
 * (memory comes from their own pool, e.g. CUDA.jl's, or the call runs where
 * allocation is not allowed).  p_dev: (pdim, n) column-major doubles on `device`;
 * x_dev: (dims, n) or NULL; out_dev: LIM_OBS_NUM doubles on the device receiving
 * the SUMS (out[LIM_OBS_COUNT] = n; divide for means).  pt_width <= 0 means 1e-3
 * (as in lim_observables).  Enqueued on `stream`
 * (NULL = default stream); read out_dev after the stream reaches the call.
 * Limits and sharing: n <= 16,777,216; the per-block partial sums live in one
 * fixed 96 KiB device array of the library, held by every GPU that loads it until
 * the process exits, shared by all calls: calls that overlap on the GPU (e.g. on
 * two streams at once) race.  The first call on a device looks up that array's
 * device address; make it before any stream capture.  A CUDA error left pending by
 * earlier work on the calling thread is reported (LIM_ERR_CUDA) before anything is
 * launched.  Errors: lim_last_error(NULL). */
int lim_observables_noalloc(int device, const double* p_dev, int64_t pdim, const double* x_dev,
                            int64_t dims, int64_t n, double m, double pt_cut, double pt_width,
                            double* out_dev, void* stream);

/* Debug/parity mode: record every random variate the kernel consumes into a
 * device buffer of nsteps * LIM_NOISE_SLOTS * n doubles, laid out
 * [step - first_step][slot][particle]; lim_download_noise copies it out.
 * Pass nsteps = 0 to switch recording off. */
#define LIM_NOISE_SLOTS 11
int lim_record_noise(lim_ctx* ctx, int64_t first_step, int64_t nsteps);
int lim_download_noise(lim_ctx* ctx, double* out);

/* Philox-4x32-10 block as the device computes it (for host-side parity checks):
 * out[4] = philox(ctr[4], key[2]). */
int lim_philox_device(lim_ctx* ctx, const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- timing helpers (bench) ---------------------------------------------------- */
/* Device time of the last lim_run's step kernels in ms (CUDA events on the
 * context stream) and the number of kernel launches it issued. */
int lim_last_run_stats(lim_ctx* ctx, double* kernel_ms, int64_t* launches);

/* ---- pathwise gradients ----------------------------------------------------------
 * lim_adjoint advances the state through steps [first_step, first_step + nsteps)
 * exactly as lim_run does (checkpointing it every `checkpoint_every` steps, recording
 * the RTA decisions), evaluates three final-state observables
 *   obs[0] = <pT>, obs[1] = <cos 2 phi>, obs[2] = <sigmoid((pT - obs_pt_cut)/obs_pt_width)>
 * and, with a hand-written reverse (adjoint) sweep that recomputes each segment from
 * its checkpoint, their pathwise derivatives with the noise and the RTA indicators held
 * fixed: grad[3*o + k] = d obs[o] / d theta_k for theta = (a, b, s), where a and b are
 * the parameters of D_s(T) whose drag-spline derivatives were set with
 * LIM_SPLINE_DRAG_DA / _DB and s is the medium scale (lim_set_medium_scale).  The
 * run's RTA decisions stay recorded (replay mode) for finite-difference checks.
 * Supported: FP32, Cartesian, dims 2, pdim 3, grid or analytic Bjorken medium,
 * collision :langevin or :langevin_rta, relativistic, pre-point, no position
 * diffusion, reflection or freeze-out.  No counterpart in the reference. */
int lim_adjoint(lim_ctx* ctx, int64_t first_step, int64_t nsteps, int64_t checkpoint_every,
                double* obs, double* grad);
/* Device time (ms) of the last lim_adjoint: checkpointed forward and reverse sweep. */
int lim_adjoint_stats(lim_ctx* ctx, double* forward_ms, double* reverse_ms);

/* ---- initial states -------------------------------------------------------------
 * Samples n heavy quarks on the device from a FONLL-type density f(r, p) on an r grid
 * (nr nodes) and a |p_T| grid (np nodes), f[ip + np*ir] = f(r_grid[ir], p_grid[ip])
 * (Julia's Np x Nr matrix, column-major), into the context's state (replacing an
 * uploaded one); then lim_initial_lab_boost / lim_run proceed as after lim_upload_state.
 * Replaces sample_particles_from_FONLL (utils.jl:33-172): cartesian != 0 is its
 * rejection sampling in (x, y) with |p| from the conditional inverse CDF of p | r,
 * cartesian == 0 its polar mode (r from the r marginal, uniform angle); antithetic
 * pairs (0,1), (2,3), ... share their draws, the second with -p.  thermal_pz != 0 (pdim
 * 3) appends p_z from the local temperature of the context's medium at t0 as
 * append_thermal_pz / sample_pz_conditional_juttner (utils.jl:499-551).  The draws come
 * from the particle's Philox stream (seed, particle_offset + pair index, trial, tag),
 * not a global RNG: the result depends on (seed, particle_offset) only.
 * Needs Cartesian coordinates, dimensions 2 and pdim 2 or 3; a set medium when
 * thermal_pz.  LIM_ERR_STATE when a particle found no accepted trial in 100000. */
int lim_sample_fonll(lim_ctx* ctx, const double* r_grid, int64_t nr, const double* p_grid, int64_t np,
                     const double* f, int64_t n, int cartesian, int antithetic, int thermal_pz);

/* Samples n heavy quarks in Milne coordinates on the device into the state, replacing
 * sample_initial_particles_milne! (utils.jl:350-400): nbins radial bins over
 * [x_lo, x_hi] with the profiles T, u^r, mu evaluated at the bin centers
 * (T_c, ur_c, mu_c: the host evaluates the reference's profile functions there), the
 * binned Boltzmann density T^(3/2)/gamma exp((mu - m gamma)/T) sampled by rejection
 * against the first bin center >= r, and p^r = sqrt(m T(r)) z with T(r) linear on the
 * table (r_T, T_r) of nT ascending nodes.  State: (t0, r), (sqrt(m^2 + p_r^2), |p_r|).
 * Draws: trial t from (seed, particle_offset + i, t, SAMPLE_XY), z from
 * (seed, particle_offset + i, 0, SAMPLE_P).  Needs Milne coordinates (dimensions 2,
 * pdim 2).  LIM_ERR_STATE when a particle found no accepted trial in 100000. */
int lim_sample_milne(lim_ctx* ctx, double x_lo, double x_hi, int64_t nbins, const double* T_c, const double* ur_c,
                     const double* mu_c, const double* r_T, const double* T_r, int64_t nT, int64_t n);

/* ---- batches ------------------------------------------------------------------
 * Many independent ensembles — each a configured context with its own particle
 * count, step range, mass, transport tables and medium — advanced together: every
 * chunk of steps is one persistent launch over all ensembles' particle tiles, and the
 * chunk sequence is captured once as a CUDA graph and replayed.  No counterpart in
 * the reference (one ensemble per simulate_ensemble_bulk call); a batch gives the
 * same per-particle results as running each context with lim_run (same noise: a
 * particle's variates depend on (seed, particle_offset + index, step) only).
 *
 * Every ensemble of a batch shares the precision, dims/pdim, the seed, Cartesian
 * coordinates and the freeze-out switch; noise recording is ignored.  Contexts are
 * referenced, not copied: they must outlive the batch, and their state is advanced
 * in place (read it with lim_download_state).  A change to a context (parameters,
 * medium, tables, a new upload) is picked up by the next lim_batch_run. */
typedef struct lim_batch lim_batch;

typedef struct lim_batch_shape {
    int64_t block;          /* threads (particles) per block: 64, 128 or 256; 0 = 256 */
    int64_t chunk_steps;    /* steps per chunk launch; 0 = the longest ensemble's range */
    int64_t blocks_per_sm;  /* persistent blocks per SM; 0 = the occupancy maximum */
    int64_t reg_cap;        /* FP32: 1 caps registers for four 256-thread blocks per SM */
} lim_batch_shape;

int lim_batch_create(int device, void* stream, lim_batch** out);
int lim_batch_destroy(lim_batch* b);
const char* lim_batch_last_error(const lim_batch* b);   /* b = NULL: the last create error */
/* Adds `ensemble` advancing steps [first_step, first_step + nsteps); *index = its position. */
int lim_batch_add(lim_batch* b, lim_ctx* ensemble, int64_t first_step, int64_t nsteps, int64_t* index);
int lim_batch_set_shape(lim_batch* b, const lim_batch_shape* shape);
int lim_batch_get_shape(const lim_batch* b, lim_batch_shape* shape);
/* Runs every ensemble through its range: one graph replay.  LIM_ERR_NONFINITE names the
 * first ensemble and step that produced NaN/Inf. */
int lim_batch_run(lim_batch* b);
/* Autotuner: times each candidate shape on the batch itself (every ensemble's state
 * is saved first and restored before each trial and at the end) and keeps the
 * fastest.  Candidates: block {128, 256} x chunk {64, 256, 1024, whole range} x
 * reg_cap {0, 1} (FP32).  *best and *best_ms (may be NULL) receive the choice. */
int lim_batch_tune(lim_batch* b, lim_batch_shape* best, double* best_ms);
/* Device time of the last lim_batch_run (ms), its kernel launches and particle-steps. */
int lim_batch_stats(const lim_batch* b, double* ms, int64_t* launches, int64_t* particle_steps);

#ifdef __cplusplus
}
#endif
#endif /* LANGEVIN_B200_H */

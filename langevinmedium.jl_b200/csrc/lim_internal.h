// lim_internal.h — launchers shared between the kernel and C-ABI translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "lim_common.cuh"

namespace lim {

constexpr int kObsNum = 12;   // LIM_OBS_NUM

// Fused step kernels over steps [s0, s1).  coords: 0 Cartesian, 1 Milne.
template <typename R>
cudaError_t launch_steps(const KParams<R>& kp, int coords, int64_t s0, int64_t s1, int block, cudaStream_t st);

// The per-step table alone (steps [s0, s1), s0 = kp.step_base), and Cartesian steps
// [s0, s1) inside an already computed table (no table launch).
template <typename R>
cudaError_t launch_step_table(const KParams<R>& kp, int coords, int64_t s0, int64_t s1, cudaStream_t st);
template <typename R>
cudaError_t launch_steps_in_table(const KParams<R>& kp, int64_t s0, int64_t s1, int block, cudaStream_t st);
// Compacts the not-frozen particles of `in` (every index < n when in is NULL) into `out`.
cudaError_t launch_compact_live(const double* flag, const int* in, const unsigned* in_n, int64_t n, int* out,
                                unsigned* out_n, cudaStream_t st);

// Bytes of one per-step record (the step table holds one per step of a launch).
template <typename R>
size_t step_record_bytes();

// The static-temperature momentum-only run (simulate_cpu.jl:325-404): the FP64 momenta
// p[d][i], the run constants and the |p| history hist[(s / save_every - first_slot) n + i].
struct StaticRun {
    double* p[3];
    int64_t n, pid_offset;
    double T, m, dt;
    uint2 rk[10];
    double* hist;
    int64_t save_every, first_slot, nslots;
};
template <typename R>
cudaError_t launch_static_T(const StaticRun& sr, int pdim, int64_t s0, int64_t s1, cudaStream_t st);

// Step-0 lab boost (simulate_cpu.jl:160-163).
template <typename R>
cudaError_t launch_lab_boost(const KParams<R>& kp, int block, cudaStream_t st);

// Host layout (rows, n) column-major doubles <-> device structure of arrays.
template <typename R>
cudaError_t launch_aos_to_soa(const double* src, int rows, int64_t n, R* const* dst, float* const* lo, cudaStream_t st);
template <typename R>
cudaError_t launch_soa_to_aos(R* const* src, float* const* lo, int rows, int64_t n, double* dst, cudaStream_t st);

// Observables: block partial sums (FP64) and their fixed-order total.
template <typename R>
cudaError_t launch_observables(const KParams<R>& kp, int from_fo, double cut, double width,
                               double* partials, int64_t nblocks_max, double* out, cudaStream_t st);

// Batched persistent launch (lim_batch.cu): one launch advances every listed
// (ensemble, tile) item through the chunk window [chunk_lo, chunk_lo + chunk_len),
// counted from each ensemble's first step (KParams::step_base) and cut at its last.
template <typename R>
struct BatchLaunch {
    const KParams<R>* ens;     // per-ensemble parameters (device)
    const int2* items;         // this chunk's items: (ensemble, tile of blockDim particles)
    unsigned* counter;         // this chunk's work counter, zero before the launch
    int n_items;
    int64_t chunk_lo, chunk_len;
    uint2 rk[10];              // Philox round keys of the batch's seed
};
// cap: FP32 build capped at 64 registers (four 256-thread blocks per SM).
template <typename R>
cudaError_t launch_batch(const BatchLaunch<R>& bl, int dims, int pdim, bool fo, bool cap, int grid, int block,
                         cudaStream_t st);
template <typename R>
cudaError_t batch_blocks_per_sm(int dims, int pdim, bool fo, bool cap, int block, int* out);
// The per-step records of one ensemble, steps [s0, s0 + n), into `out`.
template <typename R>
cudaError_t launch_batch_table(const KParams<R>& kp, int64_t s0, int64_t n, void* out, cudaStream_t st);

// Reverse sweep of lim_adjoint (lim_adjoint.cu).  Checkpoint k of the forward pass,
// at byte offset k * (segment bytes): x[2] (float), x_lo[2] (float), p[3] (double),
// each n long.  The tape (KParams::tape) holds kTapeFields floats per particle per
// step of one segment; lam the 2 x 5 cotangents, gacc the 2 x 3 parameter sums.
constexpr int kAdjOut = 12;      // 3 observables + 3 x 3 gradients
constexpr int kAdjCot = 2;       // cotangents: the final p_x and p_y
constexpr int kAdjBlock = 128;
struct AdjointArgs {
    float* lam;
    double* gacc;
    double cut, width;
    double* partials;            // [nblocks][kAdjOut]
};
cudaError_t launch_adjoint_seed(const KParams<float>& kp, const AdjointArgs& aa, cudaStream_t st);
cudaError_t launch_adjoint_tape(const KParams<float>& kp, int64_t s0, int64_t s1, cudaStream_t st);
cudaError_t launch_adjoint_rev(const KParams<float>& kp, const AdjointArgs& aa, int64_t s0, int64_t s1, cudaStream_t st);
cudaError_t launch_adjoint_total(const KParams<float>& kp, const AdjointArgs& aa, double* out, cudaStream_t st);

// Initial-state sampling (lim_sample.cu) from the tables of sample_particles_from_FONLL
// (utils.jl:33-172), built on the host in FP64.
struct SampleTables {
    const double* r_grid; int nr;
    const double* p_grid; int np;
    const double* cdf_r;         // nr: CDF of the r marginal (polar mode)
    const double* cdf_p;         // nr x np: row j is the CDF of |p| given r_j
    const int* p_mass;           // nr: row j has non-zero mass
    const double* n_spatial;     // nr: spatial density (Cartesian mode)
    double f_max, rmax;
    int cartesian, antithetic, with_pz, med_kind, max_trials;
    unsigned long long* failed;  // particles without an accepted trial
};
template <typename R>
cudaError_t launch_sample_fonll(const KParams<R>& kp, const SampleTables& st, cudaStream_t s);

// Snapshot reduction (lim_reduce.cu): uniform bins on [0, r_max) and [0, pt_max), each
// with one overflow entry; scale = bins / max.
struct ReduceSpec {
    int r_bins, pt_bins;
    double r_scale, pt_scale;
};
constexpr int kReduceBinsMax = 4096;
inline int64_t reduce_hist_len(const ReduceSpec& rs) { return (int64_t)rs.r_bins + 1 + 2 * ((int64_t)rs.pt_bins + 1); }
// The histograms of the state and its observable sums (obs_out, kObsNum doubles);
// partials holds reduce_grid(n) x kObsNum doubles.
int reduce_grid(int64_t n);
template <typename R>
cudaError_t launch_reduce_hist(const KParams<R>& kp, bool milne, const ReduceSpec& rs, unsigned long long* hist,
                               double cut, double width, double* partials, double* obs_out, cudaStream_t st);
// Fixed-order total of nblocks x kObsNum block partials into out.
cudaError_t launch_obs_total(const double* partials, int64_t nblocks, double* out, cudaStream_t st);

// Transport tables built on the device (lim_tables.cu).
enum { TIME_DRAG = 0, TIME_TAUN = 1, TIME_TAUR = 2 };
struct TimeSplineSpec {
    int kind, nT;
    double m, DsT, Tmin, Tmax, scale;          // scale: LV_TAUN_SCALE
    int linear, quad;                          // effective_DsT forms (transport.jl:139-156)
    double slope, offset, Tfo, Tref;
    double eta_over_s, factor;                 // TIME_TAUR: factor (eta/s) / T
};
struct JuttnerSpec {
    int dims, nT, nU, np;
    double m, Tmin, dT, quantile_cap;
};
cudaError_t launch_time_spline(const TimeSplineSpec& sp, double* vals, cudaStream_t st);
cudaError_t launch_juttner_invcdf(const JuttnerSpec& js, double* cdf_scratch, double* inv, cudaStream_t st);

// Milne (tau, r) sampling tables: the radial acceptance ratio pdf/max_pdf on nbins bin
// centers and the temperature profile on an ascending r table (linear, clamped).
struct MilneTables {
    const double* centers; const double* ratio; int nbins;
    const double* rT; const double* TT; int nT;
    double lo, hi;
    int max_trials;
    unsigned long long* failed;
};
template <typename R>
cudaError_t launch_sample_milne(const KParams<R>& kp, const MilneTables& mt, cudaStream_t s);

cudaError_t launch_philox_probe(const uint32_t* ctr_key, uint32_t* out, cudaStream_t st);

// FP32 FMA issue-rate probe: `blocks` x 256 threads, 64 FMAs per thread per iteration.
cudaError_t launch_fma_probe(float* out, int blocks, int iters, cudaStream_t st);
// XU (MUFU) issue-rate probe: `blocks` x 256 threads, 64 ex2.approx per thread per iteration.
cudaError_t launch_mufu_probe(float* out, int blocks, int iters, cudaStream_t st);

// Message returned by lim_last_error(NULL) for entry points that take no context.
void set_noctx_error(const char* msg);

}  // namespace lim

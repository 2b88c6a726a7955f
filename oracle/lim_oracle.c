/*
 * lim_oracle.c — CPU FP64 restatement of LangevInMedium.jl's per-particle
 * Langevin step.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA
 * engine and the timed CPU baseline.  Nothing in the product links or calls it.
 *
 * Parity status: the reference ships no per-trajectory golden vectors (its tests
 * are analytic and statistical), so trajectory-level parity is pinned against
 * the reference's own known-answer tests (transport identities, Bjorken
 * telescoping to 1e-9, OU/Jüttner equilibria, l=1 decay, MSD, relativistic
 * switch), which this restatement passes in tests/test_oracle_kats.py.  The restated
 * initial-state samplers (orc_sample_fonll, orc_sample_milne) are pinned by the
 * reference's p_z test and by distribution tests against utils.jl's CDF construction
 * (tests/test_sample_oracle.py).
 *
 * Every function follows the Julia source line by line (paths relative to the
 * reference project); compile with -O2 -ffp-contract=off because Julia does not
 * contract a*b+c into an FMA.
 *
 * Noise is injected: either a recorded buffer [step][slot][particle] (the
 * variates the GPU consumed, for exact parity) or regenerated from the
 * counter-based Philox-4x32-10 stream keyed by (seed, particle, step, tag),
 * which the CUDA engine draws from too.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 2.220446049250313e-16          /* Julia eps() */
#define ORC_FMGEV (1.0 / 0.197327)             /* constants.jl:13,23 */
#define ORC_NOISE_SLOTS 11

enum { C_LANGEVIN = 0, C_RTA = 1, C_LANGEVIN_RTA = 2, C_FLUID = 3 };
enum { M_RT = 0, M_BJORKEN = 1, M_GRID = 2 };
enum { TAG_MOM = 1, TAG_RTA = 2, TAG_DIFF = 4, TAG_SAMPLE_XY = 5, TAG_SAMPLE_P = 6,
       TAG_SAMPLE_PZ = 7, TAG_REJECT = 8 };

typedef struct orc_params {
    double dt, t0, m, DsT, Tfo, psi2, obs_pt_cut, obs_pt_width;
    int64_t dims, pdim, coords, collision, relativistic, bjorken_redshift,
            position_diffusion, reflecting_boundary, integrator_mode,
            freezeout_capture, freezeout_interp, precision, seed,
            particle_offset, stop_after_freezeout, block_size;
    /* with recorded noise: 1 takes the RTA decisions from the record (a particle
     * collided at a step iff its u_sample slot is non-zero) instead of uc < Pcol,
     * which holds the RTA indicators fixed under parameter changes */
    int64_t rta_replay;
} orc_params;

typedef struct orc_medium {
    int64_t kind;
    /* M_RT */
    const double *xg, *tg, *T, *V, *V2;
    int64_t nr, nt;
    /* M_BJORKEN */
    double bj_T0, bj_tau0, bj_power, bj_rmax;
    /* M_GRID: float fields [it][iy][ix] */
    const float *gT, *gux, *guy;
    int64_t gnx, gny, gnt;
    double gx0, gdx, gy0, gdy, gt0, gdt;
    /* splines (transport.jl:231-253) */
    const double *drag; int64_t n_drag; double drag_Tmin, drag_invdT;
    const double *rta;  int64_t n_rta;  double rta_Tmin, rta_invdT;
    /* Jüttner inverse CDF (kernels_gpu.jl:88-117) */
    const double *icdf; int64_t nU, nT; double ic_Tmin, ic_invdT;
    /* medium temperature scale (differentiation parameter s; 1 = reference) */
    double T_scale;
} orc_medium;

/* ------------------------------------------------------------------------- */
/* Julia scalar semantics                                                     */
/* ------------------------------------------------------------------------- */
static inline int jl_isless(double a, double b)        /* Base.isless on Float64 */
{
    if (isnan(a)) return 0;
    if (isnan(b)) return 1;
    if (a < b) return 1;
    if (a == b) return signbit(a) && !signbit(b);
    return 0;
}
static inline double jl_max(double a, double b)        /* Base.max: NaN-propagating */
{
    if (isnan(a) || isnan(b)) return NAN;
    if (a > b) return a;
    if (b > a) return b;
    return signbit(a) ? b : a;
}
static inline double jl_clamp(double x, double lo, double hi)   /* ifelse(x>hi,hi,ifelse(x<lo,lo,x)) */
{
    return x > hi ? hi : (x < lo ? lo : x);
}
static inline int64_t iclamp(int64_t i, int64_t lo, int64_t hi) { return i < lo ? lo : (i > hi ? hi : i); }
static inline int jl_isfinite(double x) { return isfinite(x); }

/* searchsortedlast(v, x): last 1-based index with v[i] <= x (0 if none). */
static int64_t searchsortedlast(const double* v, int64_t n, double x)
{
    int64_t lo = 0, hi = n + 1;
    while (lo < hi - 1) {
        int64_t m = (lo + hi) >> 1;
        if (jl_isless(x, v[m - 1])) hi = m; else lo = m;
    }
    return lo;
}

/* kernels_cpu.jl:22-51 — clamped bilinear interpolation on the (r, t) table. */
static double interp2d_clamped(const double* x, int64_t nx, const double* y, int64_t ny,
                               const double* vals, double xi, double yi)
{
    xi = jl_clamp(xi, x[0], x[nx - 1]);
    yi = jl_clamp(yi, y[0], y[ny - 1]);
    int64_t i = searchsortedlast(x, nx, xi);
    int64_t j = searchsortedlast(y, ny, yi);
    i = iclamp(i, 1, nx - 1);
    j = iclamp(j, 1, ny - 1);
    double x0 = x[i - 1], x1 = x[i];
    double y0 = y[j - 1], y1 = y[j];
    double v00 = vals[(i - 1) + nx * (j - 1)], v10 = vals[i + nx * (j - 1)];
    double v01 = vals[(i - 1) + nx * j],       v11 = vals[i + nx * j];
    double dx = (x1 - x0);
    double dy = (y1 - y0);
    double xd = fabs(dx) < ORC_EPS ? 0.0 : (xi - x0) / dx;
    double yd = fabs(dy) < ORC_EPS ? 0.0 : (yi - y0) / dy;
    double c0 = v00 * (1 - xd) + v10 * xd;
    double c1 = v01 * (1 - xd) + v11 * xd;
    return c0 * (1 - yd) + c1 * yd;
}

/* kernels_cpu_GC.jl:37-57 — the Milne variant: no query clamp, no eps guard. */
static double interp2d_unclamped(const double* x, int64_t nx, const double* y, int64_t ny,
                                 const double* vals, double xi, double yi)
{
    int64_t i = searchsortedlast(x, nx, xi);
    int64_t j = searchsortedlast(y, ny, yi);
    i = iclamp(i, 1, nx - 1);
    j = iclamp(j, 1, ny - 1);
    double x0 = x[i - 1], x1 = x[i];
    double y0 = y[j - 1], y1 = y[j];
    double v00 = vals[(i - 1) + nx * (j - 1)], v10 = vals[i + nx * (j - 1)];
    double v01 = vals[(i - 1) + nx * j],       v11 = vals[i + nx * j];
    double xd = (xi - x0) / (x1 - x0);
    double yd = (yi - y0) / (y1 - y0);
    double c0 = v00 * (1 - xd) + v10 * xd;
    double c1 = v01 * (1 - xd) + v11 * xd;
    return c0 * (1 - yd) + c1 * yd;
}

/* transport.jl:231-253 — eval_tau_n_spline. */
static double eval_spline(double T, double Tmin, double invdT, const double* vals, int64_t n)
{
    if (n < 2) return vals[0];
    double x = T;
    if (!jl_isfinite(x)) return 0.0;
    double u = (x - Tmin) * invdT;
    int64_t i = (int64_t)floor(u) + 1;
    i = iclamp(i, 1, n - 1);
    double t = u - (double)(i - 1);
    double y0 = vals[i - 1];
    double y1 = vals[i];
    return (1.0 - t) * y0 + t * y1;
}

/* kernels_gpu.jl:88-117 — bilinear lookup of the Jüttner inverse CDF, in the
 * reference's arithmetic: the fractional u-index fu = clamp(u, 0, 1) (nU - 1) computed
 * directly, its floor capped to [0, nU-2]. */
static double invcdf_lookup(const orc_medium* md, double u, double T)
{
    int64_t nU = md->nU, nT = md->nT;
    double uu = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
    double fu = uu * (double)(nU - 1);
    int64_t iu = (int64_t)floor(fu);
    iu = iu < 0 ? 0 : (iu > nU - 2 ? nU - 2 : iu);
    double tu = fu - (double)iu;
    double fT = (T - md->ic_Tmin) * md->ic_invdT;
    int64_t jT = (int64_t)floor(fT);
    jT = jT < 0 ? 0 : (jT > nT - 2 ? nT - 2 : jT);
    double tT = fT - (double)jT;
    tT = tT < 0.0 ? 0.0 : (tT > 1.0 ? 1.0 : tT);
    int64_t b0 = jT * nU, b1 = (jT + 1) * nU;
    double v00 = md->icdf[b0 + iu], v10 = md->icdf[b0 + iu + 1];
    double v01 = md->icdf[b1 + iu], v11 = md->icdf[b1 + iu + 1];
    double c0 = v00 * (1.0 - tu) + v10 * tu;
    double c1 = v01 * (1.0 - tu) + v11 * tu;
    return c0 * (1.0 - tT) + c1 * tT;
}

/* ------------------------------------------------------------------------- */
/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and the variate layout  */
/* ------------------------------------------------------------------------- */
static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform in (0,1) from one Philox word: u = (w + 1/2) 2^-32, exact in double.  Both
 * precisions of the engine consume this same value. */
static inline double u01(uint32_t w) { return ((double)w + 0.5) * 0x1p-32; }

/* Four uniforms of tag `tag` for (particle, step): one Philox-4x32-10 block with
 * counter (pid, step, tag, 0) and the 64-bit seed as key. */
static void uniforms4(const orc_params* P, int64_t pid, int64_t step, int tag, double u[4])
{
    uint32_t key[2] = { (uint32_t)(uint64_t)P->seed, (uint32_t)((uint64_t)P->seed >> 32) };
    uint32_t ctr[4] = { (uint32_t)pid, (uint32_t)step, (uint32_t)tag, 0u };
    uint32_t w[4];
    orc_philox4x32_10(ctr, key, w);
    for (int k = 0; k < 4; ++k) u[k] = u01(w[k]);
}
/* Box-Muller with the angle in (-pi, pi): (rad cos(pi(2u1-1)), rad sin(pi(2u1-1))). */
static inline void box_muller(double u0, double u1, double* z0, double* z1)
{
    double rad = sqrt(-2.0 * log(u0));
    double th = M_PI * (2.0 * u1 - 1.0);
    *z0 = rad * cos(th);
    *z1 = rad * sin(th);
}

/* Inverse standard normal CDF: P. J. Acklam's rational approximation (relative error
 * 1.15e-9) refined by two Halley steps on erfc, which brings it to double precision. */
static double norm_inv(double p)
{
    static const double a[6] = { -3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                 1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00 };
    static const double b[5] = { -5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                 6.680131188771972e+01, -1.328068155288572e+01 };
    static const double c[6] = { -7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                 -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00 };
    static const double d[4] = { 7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                 3.754408661907416e+00 };
    const double plow = 0.02425;
    /* work on the lower half: pl = min(p, 1-p) is exact for the (0,1) uniforms used here,
     * and the Halley residual Phi(x) - pl then has no cancellation */
    const int upper = p > 0.5;
    const double pl = upper ? 1.0 - p : p;
    double x;
    if (pl < plow) {
        double q = sqrt(-2.0 * log(pl));
        x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    } else {
        double q = pl - 0.5, r = q * q;
        x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
    }
    for (int it = 0; it < 2; ++it) {
        double e = 0.5 * erfc(-x / M_SQRT2) - pl;
        double u = e * sqrt(2.0 * M_PI) * exp(0.5 * x * x);
        x = x - u / (1.0 + 0.5 * x * u);
    }
    return upper ? -x : x;
}
double orc_norm_inv(double p) { return norm_inv(p); }

/* Per-step variates of one particle, slot layout shared with the engine:
 *   0..2 momentum normals, 3 u_collide, 4 u_sample, 5..7 RTA direction
 *   normals, 8..10 position-diffusion normals.
 * Group MOM: (u0,u1) -> Box-Muller (xi0, xi1); xi2 = Phi^-1(u2) when pdim = 3.  The
 * collision uniform is u3 when pdim = 3, u2 when pdim < 3, and u0 when there is no
 * Langevin kick.  Group RTA (only when a particle collides): u_sample = u0,
 * (u1,u2) -> (g0, g1), g2 = Phi^-1(u3) when pdim = 3. */
typedef struct noise_src {
    const double* rec;      /* recorded buffer or NULL (Philox) */
    int64_t rec_first, rec_steps, n;
    /* decision record or NULL: dec[(step - rec_first) * n + i] gets bit 0 when the
     * particle collides (RTA) and bit 1 when it latches at freeze-out in that step */
    uint8_t* dec;
} noise_src;

static inline double rec_at(const noise_src* ns, int64_t i, int64_t step, int slot)
{
    return ns->rec[((step - ns->rec_first) * ORC_NOISE_SLOTS + slot) * ns->n + i];
}

static void draw_step(const orc_params* P, const noise_src* ns, int64_t i, int64_t step, int kick, double xi[3],
                      double* uc)
{
    if (ns->rec) {
        for (int k = 0; k < 3; ++k) xi[k] = rec_at(ns, i, step, k);
        *uc = rec_at(ns, i, step, 3);
        return;
    }
    double u[4];
    uniforms4(P, P->particle_offset + i, step, TAG_MOM, u);
    if (!kick) { xi[0] = xi[1] = xi[2] = 0.0; *uc = u[0]; return; }
    box_muller(u[0], u[1], &xi[0], &xi[1]);
    if (P->pdim == 3) {
        xi[2] = norm_inv(u[2]);
        *uc = u[3];
    } else {
        xi[2] = 0.0;
        *uc = u[2];
    }
}
static void draw_rta_sample(const orc_params* P, const noise_src* ns, int64_t i, int64_t step, double* us, double g[3])
{
    if (ns->rec) {
        *us = rec_at(ns, i, step, 4);
        for (int k = 0; k < 3; ++k) g[k] = rec_at(ns, i, step, 5 + k);
        return;
    }
    double u[4];
    uniforms4(P, P->particle_offset + i, step, TAG_RTA, u);
    *us = u[0];
    box_muller(u[1], u[2], &g[0], &g[1]);
    g[2] = P->pdim == 3 ? norm_inv(u[3]) : 0.0;
}
static void draw_diffusion(const orc_params* P, const noise_src* ns, int64_t i, int64_t step, double d[3])
{
    if (ns->rec) {
        const double* b = ns->rec + ((step - ns->rec_first) * ORC_NOISE_SLOTS) * ns->n + i;
        for (int k = 0; k < 3; ++k) d[k] = b[(8 + k) * ns->n];
        return;
    }
    double u[4], z;
    uniforms4(P, P->particle_offset + i, step, TAG_DIFF, u);
    box_muller(u[0], u[1], &d[0], &d[1]);
    box_muller(u[2], u[3], &d[2], &z);
}

/* ------------------------------------------------------------------------- */
/* Medium lookups                                                             */
/* ------------------------------------------------------------------------- */
/* 2+1D grid (extension beyond the reference): trilinear with the query clamped
 * to the grid, as the reference clamps (r, t) queries. */
static void grid_lookup(const orc_medium* md, double x, double y, double t, double out[3])
{
    double xl = md->gx0 + (double)(md->gnx - 1) * md->gdx;
    double yl = md->gy0 + (double)(md->gny - 1) * md->gdy;
    double tl = md->gt0 + (double)(md->gnt - 1) * md->gdt;
    x = jl_clamp(x, md->gx0, xl); y = jl_clamp(y, md->gy0, yl); t = jl_clamp(t, md->gt0, tl);
    double fx = (x - md->gx0) / md->gdx, fy = (y - md->gy0) / md->gdy, ft = (t - md->gt0) / md->gdt;
    int64_t ix = iclamp((int64_t)floor(fx), 0, md->gnx - 2);
    int64_t iy = iclamp((int64_t)floor(fy), 0, md->gny - 2);
    int64_t it = iclamp((int64_t)floor(ft), 0, md->gnt - 2);
    double wx = fx - (double)ix, wy = fy - (double)iy, wt = ft - (double)it;
    const float* F[3] = { md->gT, md->gux, md->guy };
    for (int f = 0; f < 3; ++f) {
        double c[2];
        for (int k = 0; k < 2; ++k) {
            const float* s = F[f] + ((it + k) * md->gny) * md->gnx;
            double v00 = s[iy * md->gnx + ix],       v10 = s[iy * md->gnx + ix + 1];
            double v01 = s[(iy + 1) * md->gnx + ix], v11 = s[(iy + 1) * md->gnx + ix + 1];
            double c0 = v00 * (1.0 - wx) + v10 * wx;
            double c1 = v01 * (1.0 - wx) + v11 * wx;
            c[k] = c0 * (1.0 - wy) + c1 * wy;
        }
        out[f] = c[0] * (1.0 - wt) + c[1] * wt;
    }
}

static double bjorken_T(const orc_medium* md, double tau)
{
    if (!(tau > md->bj_tau0)) return md->bj_T0;
    return md->bj_T0 * pow(md->bj_tau0 / tau, md->bj_power);
}

/* Temperature at the particle (T_scale multiplies the medium temperature). */
static double medium_T(const orc_medium* md, const double* x, double r, double t)
{
    double T;
    if (md->kind == M_RT) T = interp2d_clamped(md->xg, md->nr, md->tg, md->nt, md->T, r, t);
    else if (md->kind == M_BJORKEN) T = bjorken_T(md, t);
    else { double o[3]; grid_lookup(md, x[0], x[1], t, o); T = o[0]; }
    return md->T_scale == 1.0 ? T : md->T_scale * T;
}

static double r_axis_eps_of(const orc_medium* md)
{
    if (md->kind == M_RT) return md->nr >= 2 ? jl_max(1e-12, 0.5 * fabs(md->xg[1] - md->xg[0])) : 1e-6;
    return 1e-6;
}
static double r_max_of(const orc_medium* md)
{
    if (md->kind == M_RT) return md->nr >= 1 ? md->xg[md->nr - 1] : 0.0;
    if (md->kind == M_BJORKEN) return md->bj_rmax;
    double xl = md->gx0 + (double)(md->gnx - 1) * md->gdx, yl = md->gy0 + (double)(md->gny - 1) * md->gdy;
    double a = fabs(md->gx0), b = fabs(xl), c = fabs(md->gy0), d = fabs(yl);
    double r = a; if (b < r) r = b; if (c < r) r = c; if (d < r) r = d;
    return r;
}

/* ------------------------------------------------------------------------- */
/* Frame changes                                                              */
/* ------------------------------------------------------------------------- */
/* Flow at the particle for the boosts: direction (nx, ny) and signed speed v.
 * Returns 0 when the boost is skipped (r < eps, kernels_cpu.jl:75-77). */
typedef struct flow_t { double v, nx, ny; int active; } flow_t;

static flow_t flow_at(const orc_params* P, const orc_medium* md, const double* x, double t)
{
    flow_t f = { 0.0, 0.0, 0.0, 0 };
    if (md->kind == M_GRID) {
        double o[3];
        grid_lookup(md, x[0], x[1], t, o);
        /* the grid holds the flow velocity (v^x, v^y), as the reference's (r, t) tables do */
        double u2 = o[1] * o[1] + o[2] * o[2];
        double u = sqrt(u2);
        if (u < ORC_EPS) return f;
        f.v = u; f.nx = o[1] / u; f.ny = o[2] / u; f.active = 1;
        return f;
    }
    /* kernels_cpu.jl:69-87 */
    double r2 = 0.0;
    for (int64_t d = 0; d < P->dims; ++d) r2 += x[d] * x[d];
    double r = sqrt(r2);
    if (r < ORC_EPS) return f;
    double v;
    if (md->kind == M_RT) v = interp2d_clamped(md->xg, md->nr, md->tg, md->nt, md->V, r, t);
    else v = 0.0;
    if (md->kind == M_RT && md->V2 && P->dims >= 2) {
        double v2m = interp2d_clamped(md->xg, md->nr, md->tg, md->nt, md->V2, r, t);
        double phi = atan2(x[1], x[0]);
        v *= (1.0 + 2.0 * v2m * cos(2.0 * (phi - P->psi2)));
    }
    f.v = v; f.active = 1;
    if (P->dims >= 2) { f.nx = x[0] / r; f.ny = x[1] / r; }
    return f;
}

/* kernels_cpu.jl:89-145 (sign = -1, rest frame) and :188-241 (sign = +1, lab). */
static void boost(const orc_params* P, const flow_t* f, double* p, double sign)
{
    int radial = (P->dims == 1);
    double m = P->m, v = f->v;
    double vmax = sqrt(1.0 - 1e-12);
    v = jl_clamp(v, -vmax, vmax);
    double v2 = v * v;
    double gam = 1.0 / sqrt(1.0 - v2 + 1e-10);
    double p2 = 0.0;
    for (int64_t d = 0; d < P->pdim; ++d) p2 += p[d] * p[d];
    double E = sqrt(p2 + m * m);
    if (radial) {
        p[0] = sign < 0 ? gam * (p[0] - v * E) : gam * (p[0] + v * E);
        return;
    }
    double rhatx = f->nx, rhaty = f->ny;
    double px = p[0], py = p[1];
    double p_par = px * rhatx + py * rhaty;
    double p_perp_x = px - p_par * rhatx;
    double p_perp_y = py - p_par * rhaty;
    double p_par_new = sign < 0 ? gam * (p_par - v * E) : gam * (p_par + v * E);
    p[0] = p_par_new * rhatx + p_perp_x;
    p[1] = p_par_new * rhaty + p_perp_y;
}

/* The Galilean rest-frame shift subtracts (m*v)*(x/r); write it exactly. */
static void boost_galilean(const orc_params* P, const flow_t* f, double* p, int to_lab)
{
    double m = P->m, v = f->v;
    if (P->dims == 1) { if (to_lab) p[0] += m * v; else p[0] -= m * v; return; }
    if (to_lab) { p[0] += m * v * f->nx; p[1] += m * v * f->ny; }
    else        { p[0] -= m * v * f->nx; p[1] -= m * v * f->ny; }
}

static void do_boost(const orc_params* P, const flow_t* f, double* p, int to_lab)
{
    if (!f->active) return;
    if (!P->relativistic) { boost_galilean(P, f, p, to_lab); return; }
    boost(P, f, p, to_lab ? 1.0 : -1.0);
}

/* ------------------------------------------------------------------------- */
/* One Cartesian step (simulate_cpu.jl:215-303)                                */
/* ------------------------------------------------------------------------- */
typedef struct fo_state {
    double pos[3], mom[3], tau, flag;
    double lpos[3], lmom[3], ltau, lT;
} fo_state;

/* kernels_cpu.jl:246-357 + :406-417, Cartesian and radial branches. */
static void langevin_kick(const orc_params* P, const orc_medium* md, double* p, double T, const double xi[3])
{
    double M = P->m, dt = P->dt;
    double DsT_safe = P->DsT <= 0 ? 0.0 : P->DsT;
    double tau = DsT_safe == 0.0 ? 0.0 : eval_spline(T, md->drag_Tmin, md->drag_invdT, md->drag, md->n_drag);
    double etaD  = (tau > 0.0 && jl_isfinite(tau)) ? (1.0 / tau) : 0.0;
    double kappa = (tau > 0.0 && jl_isfinite(tau)) ? ((2.0 * M * T) / tau) : 0.0;
    double kT = sqrt(kappa);
    double det[3] = { 0, 0, 0 }, sto[3] = { 0, 0, 0 };
    int64_t pd = P->pdim;
    if (P->dims == 1) {
        double ps = 0.0;
        for (int64_t d = 0; d < pd; ++d) ps += p[d] * p[d];
        double pm = sqrt(ps);
        double E = sqrt(pm * pm + M * M);
        double eff = P->relativistic ? etaD * M / E : etaD;
        for (int64_t d = 0; d < pd; ++d) {
            det[d] = -eff * p[d] * dt;
            sto[d] = kT * xi[d];       /* (kL - kT) == 0 exactly: only the diagonal survives */
        }
    } else if (P->integrator_mode == 1) {
        /* kernels_gpu.jl:361-393 (GPU-only drift-midpoint) */
        if (etaD > 0.0 && dt > 0.0) {
            double p2 = 0.0;
            for (int64_t d = 0; d < pd; ++d) p2 += p[d] * p[d];
            double E = sqrt(p2 + M * M);
            double eff = P->relativistic ? etaD * M / E : etaD;
            double a_half = exp(-eff * (0.5 * dt));
            double p2m = 0.0;
            for (int64_t d = 0; d < pd; ++d) { double pm = a_half * p[d]; p2m += pm * pm; }
            double Em = sqrt(p2m + M * M);
            eff = P->relativistic ? etaD * M / Em : etaD;
            double a = exp(-eff * dt);
            double np = kT * sqrt((1.0 - a * a) / (2.0 * eff * dt));
            for (int64_t d = 0; d < pd; ++d) { det[d] = (a - 1.0) * p[d]; sto[d] = np * xi[d]; }
        } else {
            for (int64_t d = 0; d < pd; ++d) { det[d] = 0.0; sto[d] = kT * xi[d]; }
        }
    } else if (etaD > 0) {
        double p2 = 0.0;
        for (int64_t d = 0; d < pd; ++d) p2 += p[d] * p[d];
        double E = sqrt(p2 + M * M);
        double eff = P->relativistic ? etaD * M / E : etaD;
        double a = exp(-eff * dt);
        double np = (dt > 0 && eff > 0) ? (kT * sqrt((1 - a * a) / (2 * eff * dt))) : 0.0;
        for (int64_t d = 0; d < pd; ++d) { det[d] = (a - 1) * p[d]; sto[d] = np * xi[d]; }
    } else {
        for (int64_t d = 0; d < pd; ++d) { det[d] = 0.0; sto[d] = kT * xi[d]; }
    }
    double sq = sqrt(dt);
    for (int64_t d = 0; d < pd; ++d) p[d] += det[d] + sq * sto[d];
}

/* kernels_gpu.jl:653-704 with injected uniforms (the CPU twin kernels_cpu.jl:474-508
 * draws from the global RNG and cannot be fed identical noise). */
static void rta_collide(const orc_params* P, const orc_medium* md, const noise_src* ns, int64_t i, int64_t step,
                        double* p, double T, double uc)
{
    double tn = (P->DsT > 0.0 && T > 0.0) ? eval_spline(T, md->rta_Tmin, md->rta_invdT, md->rta, md->n_rta) : 0.0;
    double Pcol = (tn > 0.0 && jl_isfinite(tn)) ? jl_clamp(P->dt / tn, 0.0, 1.0) : 1.0;
    /* rand() < Pcol with rand() in [0,1): Pcol = 1 always collides */
    int collide = uc < Pcol || Pcol >= 1.0;
    if (P->rta_replay && ns->rec) collide = rec_at(ns, i, step, 4) != 0.0;
    if (!collide) return;
    if (ns->dec) ns->dec[(step - ns->rec_first) * ns->n + i] |= 1u;
    double us, g[3];
    draw_rta_sample(P, ns, i, step, &us, g);
    double pstar = invcdf_lookup(md, us, T);
    if (P->dims == 1) { p[0] = (g[0] < 0.0 ? -1.0 : 1.0) * pstar; return; }
    double nrm2 = 0.0;
    for (int64_t d = 0; d < P->pdim; ++d) nrm2 += g[d] * g[d];
    double inv = pstar / sqrt(nrm2 > 1e-300 ? nrm2 : 1e-300);
    for (int64_t d = 0; d < P->pdim; ++d) p[d] = g[d] * inv;
}

/* kernels_cpu.jl:671-735 */
static void set_to_fluid(const orc_params* P, const orc_medium* md, const double* x, double* p, double t)
{
    double m = P->m, r, v;
    if (md->kind == M_GRID) {
        double o[3];
        grid_lookup(md, x[0], x[1], t, o);
        double u = sqrt(o[1] * o[1] + o[2] * o[2]);
        if (u < ORC_EPS) { p[0] = 0.0; p[1] = 0.0; return; }
        double vmax = sqrt(1.0 - 1e-12);
        double vc = P->relativistic ? jl_clamp(u, -vmax, vmax) : u;
        double g = P->relativistic ? 1.0 / sqrt(1.0 - vc * vc + 1e-10) : 1.0;
        p[0] = m * g * vc * (o[1] / u);
        p[1] = m * g * vc * (o[2] / u);
        return;
    }
    if (P->dims == 1) r = x[0];
    else r = sqrt(x[0] * x[0] + x[1] * x[1]);
    if (r < ORC_EPS) return;
    v = md->kind == M_RT ? interp2d_clamped(md->xg, md->nr, md->tg, md->nt, md->V, r, t) : 0.0;
    if (!P->relativistic) {
        if (P->dims == 1) p[0] = m * v;
        else { p[0] = m * v * (x[0] / r); p[1] = m * v * (x[1] / r); }
        return;
    }
    double vmax = sqrt(1.0 - 1e-12);
    v = jl_clamp(v, -vmax, vmax);
    double gam = 1.0 / sqrt(1.0 - v * v + 1e-10);
    if (P->dims == 1) p[0] = m * gam * v;
    else { p[0] = m * gam * v * (x[0] / r); p[1] = m * gam * v * (x[1] / r); }
}

/* kernels_cpu.jl:510-637 */
static void update_positions(const orc_params* P, const orc_medium* md, const noise_src* ns,
                             int64_t i, int64_t step, double* x, double* p, double t)
{
    double m = P->m, dt = P->dt;
    double r_axis_eps = r_axis_eps_of(md);
    double r_max = r_max_of(md);
    double E2 = m * m;
    for (int64_t d = 0; d < P->pdim; ++d) E2 += p[d] * p[d];
    double E = P->relativistic ? sqrt(E2) : m;
    if (P->dims == 1) {
        double r = x[0], pr = p[0];
        double r_abs = fabs(r);
        double r_safe = (r_abs < r_axis_eps) ? r_axis_eps : r_abs;
        double dr = (pr / E) * dt;
        if (P->position_diffusion) {
            double xs[1] = { r_safe };
            double T = medium_T(md, xs, r_safe, t);
            double D = (P->DsT / jl_max(T, ORC_EPS)) / ORC_FMGEV;
            if (D > 0) {
                double dn[3];
                draw_diffusion(P, ns, i, step, dn);
                dr += (D / r_safe) * dt + sqrt(2 * D * dt) * dn[0];
            }
        }
        double r_new = r + dr;
        if (r_new < 0) { r_new = -r_new; p[0] = -p[0]; }
        if (P->reflecting_boundary && r_max > 0.0 && r_new > r_max) {
            r_new = 2 * r_max - r_new;
            p[0] = -p[0];
            if (r_new < 0.0) { r_new = -r_new; p[0] = -p[0]; }
        }
        x[0] = r_new;
        return;
    }
    for (int64_t d = 0; d < P->dims; ++d) x[d] += dt * p[d] / E;
    if (P->position_diffusion) {
        double r2 = 0.0;
        for (int64_t d = 0; d < P->dims; ++d) r2 += x[d] * x[d];
        double r_now = sqrt(r2);
        double T = medium_T(md, x, r_now, t);
        double D = (P->DsT / jl_max(T, ORC_EPS)) / ORC_FMGEV;
        if (D > 0) {
            double s = sqrt(2 * D * dt), dn[3];
            draw_diffusion(P, ns, i, step, dn);
            for (int64_t d = 0; d < P->dims; ++d) x[d] += s * dn[d];
        }
    }
    if (P->reflecting_boundary && r_max > 0.0) {
        double r2 = 0.0;
        for (int64_t d = 0; d < P->dims; ++d) r2 += x[d] * x[d];
        double r_now = sqrt(r2);
        if (r_now > r_max) {
            double invr = 1.0 / jl_max(r_now, r_axis_eps);
            double ppar = 0.0;
            for (int64_t d = 0; d < P->dims; ++d) ppar += p[d] * (x[d] * invr);
            for (int64_t d = 0; d < P->dims; ++d) p[d] -= 2 * ppar * (x[d] * invr);
            double scale = (2 * r_max - r_now) * invr;
            for (int64_t d = 0; d < P->dims; ++d) x[d] *= scale;
        }
    }
}

/* kernels_gpu.jl:588-635 (the reference has no CPU twin) */
static void freezeout_latch(const orc_params* P, const orc_medium* md, const double* x, const double* p,
                            double tau, fo_state* fo)
{
    if (fo->flag != 0.0) return;
    double r;
    if (P->dims == 1) r = fabs(x[0]);
    else { double r2 = 0.0; for (int64_t d = 0; d < P->dims; ++d) r2 += x[d] * x[d]; r = sqrt(r2); }
    double T = medium_T(md, x, r, tau);
    if (T < P->Tfo) {
        double Tl = fo->lT;
        double frac = (P->freezeout_interp && Tl > P->Tfo && Tl > T) ? (Tl - P->Tfo) / (Tl - T) : 1.0;
        for (int64_t d = 0; d < P->dims; ++d) fo->pos[d] = fo->lpos[d] + frac * (x[d] - fo->lpos[d]);
        for (int64_t d = 0; d < P->pdim; ++d) fo->mom[d] = fo->lmom[d] + frac * (p[d] - fo->lmom[d]);
        fo->tau = fo->ltau + frac * (tau - fo->ltau);
        fo->flag = 1.0;
    } else {
        for (int64_t d = 0; d < P->dims; ++d) fo->lpos[d] = x[d];
        for (int64_t d = 0; d < P->pdim; ++d) fo->lmom[d] = p[d];
        fo->ltau = tau;
        fo->lT = T;
    }
}

static int nonfinite(const orc_params* P, const double* x, const double* p)
{
    for (int64_t d = 0; d < P->dims; ++d) if (!isfinite(x[d])) return 1;
    for (int64_t d = 0; d < P->pdim; ++d) if (!isfinite(p[d])) return 1;
    return 0;
}

static void cart_step(const orc_params* P, const orc_medium* md, const noise_src* ns,
                      int64_t i, int64_t step, double* x, double* p)
{
    double t = step * P->dt + P->t0;
    flow_t f = flow_at(P, md, x, t);
    /* 1. rest-frame boost */
    do_boost(P, &f, p, 0);
    /* 1b. Bjorken redshift of p_z (kernels_cpu.jl:427-435) */
    if (P->bjorken_redshift) {
        double ta = P->t0 + (step - 1) * P->dt;
        if (ta > 0) p[2] *= ta / (ta + P->dt);
    }
    if (P->collision == C_FLUID) {
        set_to_fluid(P, md, x, p, t);
    } else {
        double r2 = 0.0;
        for (int64_t d = 0; d < P->dims; ++d) r2 += x[d] * x[d];
        double r = sqrt(r2);
        double T = jl_max(medium_T(md, x, r, t), 0.0);
        const int kick = P->collision == C_LANGEVIN || P->collision == C_LANGEVIN_RTA;
        double xi[3], uc;
        draw_step(P, ns, i, step, kick, xi, &uc);
        if (kick) langevin_kick(P, md, p, T, xi);
        if (P->collision == C_RTA || P->collision == C_LANGEVIN_RTA) rta_collide(P, md, ns, i, step, p, T, uc);
        do_boost(P, &f, p, 1);
    }
    update_positions(P, md, ns, i, step, x, p, t);
}

/* ------------------------------------------------------------------------- */
/* Milne (tau, r) step (simulate_cpu_general_coords.jl:83-126)                 */
/* ------------------------------------------------------------------------- */
static void milne_step(const orc_params* P, const orc_medium* md, const noise_src* ns,
                       int64_t i, int64_t step, double* x, double* p)
{
    double t = step * P->dt + P->t0, m = P->m, dt = P->dt;
    double r = fabs(x[1]);
    /* kernels_cpu_GC.jl:64-82 */
    double v = interp2d_unclamped(md->xg, md->nr, md->tg, md->nt, md->V, r, t);
    double g = 1.0 / sqrt(1 - v * v + 1e-10);
    double pt = p[0], pr = p[1];
    p[0] = g * (pt - v * pr);
    p[1] = g * (pr - v * pt);
    /* kernels_cpu_GC.jl:110-174 (Christoffel symbols are identically zero) */
    double T = interp2d_unclamped(md->xg, md->nr, md->tg, md->nt, md->T, fabs(x[1]), t);
    if (md->T_scale != 1.0) T *= md->T_scale;
    double DsT_safe = P->DsT <= 0 ? 0.0 : P->DsT;
    double tn = DsT_safe == 0.0 ? 0.0 : eval_spline(T, md->drag_Tmin, md->drag_invdT, md->drag, md->n_drag);
    double etaD  = (tn > 0.0 && jl_isfinite(tn)) ? (1.0 / tn) : 0.0;
    double kappa = (tn > 0.0 && jl_isfinite(tn)) ? ((2.0 * m * T) / tn) : 0.0;
    double kT = sqrt(kappa);
    double p0 = sqrt(m * m + p[1] * p[1]);
    double geo = 0.0;
    for (int nu = 0; nu < 2; ++nu)
        for (int rho = 0; rho < 2; ++rho) geo += -0.0 * p[nu] * p[rho] / p0;
    geo *= dt;
    double xi[3], uc_unused;
    draw_step(P, ns, i, step, 1, xi, &uc_unused);
    double det, sto;
    if (etaD > 0.0 && dt > 0.0) {
        double a = exp(-etaD * dt);
        double np = kT * sqrt((1.0 - a * a) / (2.0 * etaD * dt));
        det = (a - 1.0) * p[1] + geo;
        sto = np * xi[0];
    } else {
        det = geo;
        sto = kT * xi[0];
    }
    /* kernels_cpu_GC.jl:244-256 */
    p[1] += det + sqrt(dt) * sto;
    p[0] = sqrt(m * m + p[1] * p[1]);
    /* kernels_cpu_GC.jl:85-102 */
    v = interp2d_unclamped(md->xg, md->nr, md->tg, md->nt, md->V, fabs(x[1]), t);
    g = 1.0 / sqrt(1 - v * v + 1e-8);
    pt = p[0]; pr = p[1];
    p[0] = g * (pt + v * pr);
    p[1] = g * (pr + v * pt);
    /* kernels_cpu_GC.jl:259-274 */
    double E = p[0];
    x[0] += dt * p[0] / E;
    x[1] += dt * p[1] / E;
}

/* ------------------------------------------------------------------------- */
/* Public oracle entry points                                                 */
/* ------------------------------------------------------------------------- */
/* Step-0 lab boost (simulate_cpu.jl:160-163); x, p column-major (rows, n). */
void orc_initial_lab_boost(const orc_params* P, const orc_medium* md, double* x, double* p, int64_t n)
{
    if (P->coords == 1) return;   /* the Milne CPU driver has none */
    for (int64_t i = 0; i < n; ++i) {
        double* xi = x + i * P->dims;
        double* pi = p + i * P->pdim;
        flow_t f = flow_at(P, md, xi, 0 * P->dt + P->t0);
        do_boost(P, &f, pi, 1);
    }
}

/*
 * Run steps first_step .. first_step+nsteps-1 on column-major x (dims, n) and
 * p (pdim, n).  Snapshots after steps with s % save_every == 0 go to slot
 * s/save_every - first_slot of hist_x/hist_p (NULL to skip).  fo (n records)
 * may be NULL.  rec: recorded noise [nsteps][slots][n] or NULL for Philox.
 * Returns the first step at which any particle is non-finite, or -1.
 * threads <= 0: use every OpenMP thread.
 */
int64_t orc_run(const orc_params* P, const orc_medium* md, double* x, double* p, int64_t n,
                int64_t first_step, int64_t nsteps, int64_t save_every, int64_t first_slot,
                double* hist_x, double* hist_p, fo_state* fo, const double* rec, int threads, uint8_t* dec)
{
    noise_src ns = { rec, first_step, nsteps, n, dec };
    int64_t first_bad = INT64_MAX;
#ifdef _OPENMP
    int nth = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nth) reduction(min:first_bad)
#endif
    for (int64_t i = 0; i < n; ++i) {
        double xs[3] = { 0, 0, 0 }, ps[3] = { 0, 0, 0 };
        for (int64_t d = 0; d < P->dims; ++d) xs[d] = x[i * P->dims + d];
        for (int64_t d = 0; d < P->pdim; ++d) ps[d] = p[i * P->pdim + d];
        int64_t bad = INT64_MAX;
        for (int64_t s = first_step; s < first_step + nsteps; ++s) {
            /* stop_after_freezeout: a latched particle is not advanced any further (its
             * outputs are the latch's), as the engine's live-list runs do */
            if (fo && P->freezeout_capture && P->stop_after_freezeout && fo[i].flag != 0.0) break;
            if (P->coords == 1) milne_step(P, md, &ns, i, s, xs, ps);
            else {
                cart_step(P, md, &ns, i, s, xs, ps);
                if (fo && P->freezeout_capture) {
                    const double was = fo[i].flag;
                    freezeout_latch(P, md, xs, ps, s * P->dt + P->t0, &fo[i]);
                    if (dec && was == 0.0 && fo[i].flag != 0.0) dec[(s - first_step) * n + i] |= 2u;
                }
            }
            if (bad == INT64_MAX && nonfinite(P, xs, ps)) bad = s;
            if (save_every > 0 && (s % save_every) == 0 && hist_x && hist_p) {
                int64_t slot = s / save_every - first_slot;
                for (int64_t d = 0; d < P->dims; ++d) hist_x[(slot * n + i) * P->dims + d] = xs[d];
                for (int64_t d = 0; d < P->pdim; ++d) hist_p[(slot * n + i) * P->pdim + d] = ps[d];
            }
        }
        for (int64_t d = 0; d < P->dims; ++d) x[i * P->dims + d] = xs[d];
        for (int64_t d = 0; d < P->pdim; ++d) p[i * P->pdim + d] = ps[d];
        if (bad < first_bad) first_bad = bad;
    }
    return first_bad == INT64_MAX ? -1 : first_bad;
}

/* kernels_cpu.jl:442-458 (_draw_juttner_pstar_lib): the CPU RTA's Juttner magnitude
 * sampler for P(p) ~ p^(d-1) exp(-(E - m)/T), by rejection under the flat envelope
 * 1.3 x the exact peak on [0, pmax), pmax = 16 sqrt(m T) + 16 T, at most 1e5 tries (then
 * the peak momentum).  Its two uniforms per try come from Philox, counter
 * (pid, try, TAG_REJECT), instead of Julia's global rand(); in the reference only the
 * GPU form (the inverse-CDF table) takes injected uniforms.  Used to compare the two
 * samplers' distributions.  tries[k]: the tries the k-th draw took. */
static double juttner_pstar_rejection(const orc_params* P, double m, double T, int64_t d, int64_t pid,
                                      int64_t* tries)
{
    *tries = 0;
    if (T <= 0.0) return 0.0;
    const double a = (double)(d - 1);
    const double E_peak = (a * T + sqrt(a * a * T * T + 4.0 * m * m)) / 2.0;
    const double p_peak = sqrt(jl_max(E_peak * E_peak - m * m, 1e-12));
    const double gpeak = pow(p_peak, a) * exp(-(E_peak - m) / T);     /* 0^0 = 1, as in Julia */
    const double wmax = 1.3 * jl_max(gpeak, 1e-300);
    const double pmax = 16.0 * sqrt(m * T) + 16.0 * T;
    for (int64_t t = 0; t < 100000; ++t) {
        double u[4];
        uniforms4(P, pid, t, TAG_REJECT, u);
        const double p = pmax * u[0];
        const double E = sqrt(m * m + p * p);
        const double w = pow(p, a) * exp(-(E - m) / T);
        *tries = t + 1;
        if (u[1] * wmax <= w) return p;
    }
    return p_peak;
}

void orc_juttner_rejection(const orc_params* P, double m, double T, int64_t d, int64_t first_pid, int64_t n,
                           double* out, int64_t* tries)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t k = 0; k < n; ++k) out[k] = juttner_pstar_rejection(P, m, T, d, first_pid + k, &tries[k]);
}

/* simulate_cpu.jl:325-404 with the legacy force kernels_cpu.jl:359-404 and the update
 * :406-417: the static-temperature momentum-only path.  kappa = 2.5 T^3,
 * eta_D = kappa / (2 T m), kL = kT = sqrt(kappa); per component det = -eta_D p dt and
 * sto = sum_j ((kL - kT) u_d u_j + kT delta_dj) xi_j, which is kT xi_d because
 * kL - kT = 0; p += det + sqrt(dt) sto.  The momentum normals are the step's (TAG_MOM).
 * |p| after every step s with s % save_every == 0 goes to hist[(s / save_every -
 * first_slot) n + i] for slots in [0, nslots). */
void orc_run_static(const orc_params* P, double T, double* p, int64_t n, int64_t first_step, int64_t nsteps,
                    int64_t save_every, int64_t first_slot, int64_t nslots, double* hist, int threads)
{
    noise_src ns = { NULL, 0, 0, 0, NULL };
    const double kappa = 2.5 * (T * T * T);
    const double etaD = kappa / (2.0 * T * P->m);
    const double kL = sqrt(kappa), kT = sqrt(kappa);
    const double sq = sqrt(P->dt);
    const int64_t pd = P->pdim;
#ifdef _OPENMP
    int nth = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nth)
#endif
    for (int64_t i = 0; i < n; ++i) {
        double ps[3] = { 0, 0, 0 };
        for (int64_t d = 0; d < pd; ++d) ps[d] = p[i * pd + d];
        for (int64_t s = first_step; s < first_step + nsteps; ++s) {
            double xi[3], uc;
            draw_step(P, &ns, i, s, 1, xi, &uc);
            double pm = 0.0;
            for (int64_t d = 0; d < pd; ++d) pm += ps[d] * ps[d];
            pm = sqrt(pm);
            double u[3];                       /* p_units: the projector term multiplies them by 0 */
            for (int64_t d = 0; d < pd; ++d) u[d] = pm < 2.220446049250313e-16 ? 0.0 : ps[d] / pm;
            double det[3], sto[3];
            for (int64_t d = 0; d < pd; ++d) {
                det[d] = -etaD * ps[d] * P->dt;
                double acc = 0.0;
                for (int64_t j = 0; j < pd; ++j)
                    acc += (kL - kT) * u[d] * u[j] * xi[j] + kT * (d == j ? 1.0 : 0.0) * xi[j];
                sto[d] = acc;
            }
            for (int64_t d = 0; d < pd; ++d) ps[d] += det[d] + sq * sto[d];
            if (save_every > 0 && hist && s % save_every == 0) {
                const int64_t slot = s / save_every - first_slot;
                if (slot >= 0 && slot < nslots) {
                    double p2 = 0.0;
                    for (int64_t d = 0; d < pd; ++d) p2 += ps[d] * ps[d];
                    hist[slot * n + i] = sqrt(p2);
                }
            }
        }
        for (int64_t d = 0; d < pd; ++d) p[i * pd + d] = ps[d];
    }
}

/* Helpers exported for tests. */
double orc_interp2d_clamped(const double* x, int64_t nx, const double* y, int64_t ny,
                            const double* vals, double xi, double yi)
{ return interp2d_clamped(x, nx, y, ny, vals, xi, yi); }
double orc_eval_spline(double T, double Tmin, double invdT, const double* vals, int64_t n)
{ return eval_spline(T, Tmin, invdT, vals, n); }
double orc_invcdf_lookup(const orc_medium* md, double u, double T) { return invcdf_lookup(md, u, T); }
void orc_uniforms4(const orc_params* P, int64_t pid, int64_t step, int tag, double u[4])
{ uniforms4(P, pid, step, tag, u); }
/* The variates the engine draws for (particle i, step) in recording-slot order,
 * as if the particle collided (slots 4..7 are drawn regardless). */
void orc_step_variates(const orc_params* P, int64_t i, int64_t step, int kick, double out[11])
{
    noise_src ns = { NULL, 0, 0, 0, NULL };
    double xi[3], uc, us, g[3], d[3];
    for (int k = 0; k < 11; ++k) out[k] = 0.0;
    draw_step(P, &ns, i, step, kick, xi, &uc);
    draw_rta_sample(P, &ns, i, step, &us, g);
    draw_diffusion(P, &ns, i, step, d);
    for (int k = 0; k < 3; ++k) { out[k] = xi[k]; out[5 + k] = g[k]; out[8 + k] = d[k]; }
    out[3] = uc; out[4] = us;
}
int64_t orc_sizeof_params(void) { return (int64_t)sizeof(orc_params); }
int64_t orc_sizeof_medium(void) { return (int64_t)sizeof(orc_medium); }
int64_t orc_sizeof_fo(void) { return (int64_t)sizeof(fo_state); }
int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* Initial-state sampling (checker of lim_sample_fonll)                       */
/* ------------------------------------------------------------------------- */
/* utils.jl:33-172 sample_particles_from_FONLL and utils.jl:499-551
 * sample_pz_conditional_juttner / append_thermal_pz, drawing from the particle's
 * counter-based stream instead of the global RNG: block (pid, trial, tag). */
static int64_t ss_last(const double* g, int64_t n, double x)   /* searchsortedlast, 0-based, capped to n-2 */
{
    int64_t lo = -1, hi = n;
    while (hi - lo > 1) { int64_t mid = (lo + hi) / 2; if (g[mid] <= x) lo = mid; else hi = mid; }
    if (lo < 0) lo = 0;
    return lo > n - 2 ? n - 2 : lo;
}
static double inv_cdf(const double* cdf, const double* grid, int64_t n, double u)
{
    if (u <= cdf[0]) return grid[0];
    if (u >= cdf[n - 1]) return grid[n - 1];
    int64_t k = ss_last(cdf, n, u);
    double w = (u - cdf[k]) / (cdf[k + 1] - cdf[k]);
    return grid[k] + w * (grid[k + 1] - grid[k]);
}
static void words(const orc_params* P, int64_t pid, int64_t draw, int tag, uint32_t w[4])
{
    uint32_t key[2] = { (uint32_t)(uint64_t)P->seed, (uint32_t)((uint64_t)P->seed >> 32) };
    uint32_t ctr[4] = { (uint32_t)pid, (uint32_t)draw, (uint32_t)tag, 0u };
    orc_philox4x32_10(ctr, key, w);
}
static double sample_pz_cond(const orc_params* P, int64_t pid, double mT, double T, int max_trials)
{
    if (!(T > 0.0 && mT > 0.0)) return 0.0;
    double a = mT / T;
    if (a > 1.05) {
        double c = a / (a - 1.0) > 2.0 ? a / (a - 1.0) : 2.0;
        double sig = sqrt(c / a);
        for (int t = 0; t < max_trials; ++t) {
            uint32_t w[4];
            double z0, z1;
            words(P, pid, t, TAG_SAMPLE_PZ, w);
            box_muller(u01(w[0]), u01(w[1]), &z0, &z1);
            double y = sig * z0, ch = cosh(y);
            double acc = ch * exp(-a * (ch - 1.0) + a * y * y / (2.0 * c));
            if (u01(w[2]) <= acc) return mT * sinh(y);
        }
        return 0.0;
    }
    double b = sqrt(2.0) * T;
    for (int t = 0; t < 10 * max_trials; ++t) {           /* 1e6 trials for the loose envelope */
        uint32_t w[4];
        words(P, pid, t, TAG_SAMPLE_PZ, w);
        double pz = -b * log(u01(w[0])) * (u01(w[1]) < 0.5 ? -1.0 : 1.0);
        double acc = exp(-(sqrt(mT * mT + pz * pz) - (mT + fabs(pz)) / sqrt(2.0)) / T);
        if (u01(w[2]) <= acc) return pz;
    }
    return 0.0;
}

/* p_z draws of particles pid = particle_offset + 0 .. n-1 at fixed (mT, T). */
void orc_sample_pz(const orc_params* P, double mT, double T, int64_t n, double* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = sample_pz_cond(P, P->particle_offset + i, mT, T, 100000);
}

/* Samples n particles into x (2, n) and p (pdim, n), column-major (Julia) layout.
 * f[ip + np*ir] = f(r_ir, p_ip).  Returns the number of particles without an accepted
 * trial, or -1 when the polar normalisation is zero. */
int64_t orc_sample_fonll(const orc_params* P, const orc_medium* md, const double* r_grid, int64_t nr,
                         const double* p_grid, int64_t np, const double* f, int64_t n, int cartesian,
                         int antithetic, int thermal_pz, double* x, double* p)
{
    const double eps = 2.220446049250313e-16;
    const int max_trials = 100000;
    double dr = 0.0, dp = 0.0;
    for (int64_t k = 1; k < nr; ++k) dr += r_grid[k] - r_grid[k - 1];
    for (int64_t k = 1; k < np; ++k) dp += p_grid[k] - p_grid[k - 1];
    dr /= (double)(nr - 1);
    dp /= (double)(np - 1);
    double* cdf_p = calloc((size_t)(nr * np), sizeof(double));
    double* nsp = calloc((size_t)nr, sizeof(double));
    double* cdf_r = calloc((size_t)nr, sizeof(double));
    int* mass = calloc((size_t)nr, sizeof(int));
    for (int64_t ir = 0; ir < nr; ++ir) {
        double tot = 0.0;
        for (int64_t ip = 0; ip < np; ++ip) tot += p_grid[ip] * f[ip + np * ir];
        nsp[ir] = tot * dp;
        if (!(tot > 0)) continue;
        mass[ir] = 1;
        double* row = cdf_p + ir * np, acc = 0.0;
        for (int64_t ip = 0; ip < np; ++ip) { acc += p_grid[ip] * f[ip + np * ir]; row[ip] = acc * dp; }
        row[0] = 0.0;
        for (int64_t k = 1; k < np; ++k) row[k] = jl_max(row[k], row[k - 1] + eps);
        double last = row[np - 1];
        for (int64_t k = 0; k < np; ++k) row[k] /= last;
        row[np - 1] = 1.0;
    }
    double fmax = 0.0;
    for (int64_t k = 0; k < nr; ++k) fmax = jl_max(fmax, nsp[k]);
    fmax += eps;
    int64_t failed = 0;
    if (!cartesian) {
        double Z = 0.0;
        for (int64_t ir = 0; ir < nr; ++ir)
            for (int64_t ip = 0; ip < np; ++ip) Z += r_grid[ir] * p_grid[ip] * f[ip + np * ir];
        Z *= dr * dp;
        if (Z == 0.0) { failed = -1; goto done; }
        double acc = 0.0;
        for (int64_t ir = 0; ir < nr; ++ir) {
            double pr = 0.0;
            for (int64_t ip = 0; ip < np; ++ip) pr += r_grid[ir] * p_grid[ip] * f[ip + np * ir] / Z;
            acc += pr * dp;
            cdf_r[ir] = acc * dr;
        }
        cdf_r[0] = 0.0;
        for (int64_t k = 1; k < nr; ++k) cdf_r[k] = jl_max(cdf_r[k], cdf_r[k - 1] + eps);
        double last = cdf_r[nr - 1];
        for (int64_t k = 0; k < nr; ++k) cdf_r[k] /= last;
        cdf_r[nr - 1] = 1.0;
    }
    {
        const double rmax = r_grid[nr - 1];
        const int64_t half = n / 2;
        for (int64_t i = 0; i < n; ++i) {
            int64_t draw = i;
            int mirror = 0;
            if (antithetic) {
                if (i < 2 * half) { draw = i / 2; mirror = (int)(i & 1); }
                else draw = half;
            }
            const int64_t pid = P->particle_offset + draw;
            double xx = 0.0, yy = 0.0, r = 0.0, pm = 0.0, php = 0.0;
            uint32_t w[4], v[4];
            if (cartesian) {
                int ok = 0;
                for (int t = 0; t < max_trials && !ok; ++t) {
                    words(P, pid, t, TAG_SAMPLE_XY, w);
                    double xt = rmax * (2.0 * u01(w[0]) - 1.0), yt = rmax * (2.0 * u01(w[1]) - 1.0);
                    double rt = sqrt(xt * xt + yt * yt);
                    if (rt > rmax) continue;
                    double nrv = 0.0;
                    if (rt >= r_grid[0] && rt <= r_grid[nr - 1]) {
                        int64_t k = ss_last(r_grid, nr, rt);
                        double wk = (rt - r_grid[k]) / (r_grid[k + 1] - r_grid[k]);
                        nrv = nsp[k] + wk * (nsp[k + 1] - nsp[k]);
                    }
                    if (u01(w[2]) * fmax > nrv) continue;
                    xx = xt; yy = yt; r = rt;
                    words(P, pid, t, TAG_SAMPLE_P, v);
                    double rc = jl_clamp(r, r_grid[0], r_grid[nr - 1]);
                    int64_t j = ss_last(r_grid, nr, rc) + (rc >= r_grid[nr - 1] ? 1 : 0);
                    pm = mass[j] ? inv_cdf(cdf_p + j * np, p_grid, np, u01(v[0])) : 0.0;
                    php = 2.0 * M_PI * u01(v[1]);
                    ok = 1;
                }
                if (!ok) ++failed;
            } else {
                words(P, pid, 0, TAG_SAMPLE_XY, w);
                r = jl_clamp(inv_cdf(cdf_r, r_grid, nr, u01(w[0])), r_grid[0], r_grid[nr - 1]);
                double phi = 2.0 * M_PI * u01(w[1]);
                xx = r * cos(phi); yy = r * sin(phi);
                int64_t j = ss_last(r_grid, nr, r) + (r >= r_grid[nr - 1] ? 1 : 0);
                pm = mass[j] ? inv_cdf(cdf_p + j * np, p_grid, np, u01(w[2])) : 0.0;
                php = 2.0 * M_PI * u01(w[3]);
            }
            double px = pm * cos(php), py = pm * sin(php), pz = 0.0;
            if (P->pdim == 3 && thermal_pz) {
                double xv[3] = { xx, yy, 0.0 };
                double T = medium_T(md, xv, sqrt(xx * xx + yy * yy), P->t0);
                T = T > 0.0 ? T : 0.0;
                double mT = sqrt(P->m * P->m + px * px + py * py);
                pz = sample_pz_cond(P, pid, mT, T, max_trials);
            }
            if (mirror) { px = -px; py = -py; pz = -pz; }
            x[2 * i] = xx; x[2 * i + 1] = yy;
            p[P->pdim * i] = px; p[P->pdim * i + 1] = py;
            if (P->pdim == 3) p[P->pdim * i + 2] = pz;
        }
    }
done:
    free(cdf_p); free(nsp); free(cdf_r); free(mass);
    return failed;
}

/* utils.jl:350-400 sample_initial_particles_milne!, with the particle's counter-based
 * draws (trial t: block (pid, t, SAMPLE_XY); p_r: block (pid, 0, SAMPLE_P)) and T(r)
 * linear on (r_T, T_r).  x (2, n) = (t0, r), p (2, n) = (p^tau, |p^r|).  Returns the
 * number of particles without an accepted trial, or -1 for a density without a
 * positive finite maximum. */
int64_t orc_sample_milne(const orc_params* P, double x_lo, double x_hi, int64_t nbins, const double* T_c,
                         const double* ur_c, const double* mu_c, const double* r_T, const double* T_r, int64_t nT,
                         int64_t n, double* x, double* p)
{
    const double m = P->m, dx = (x_hi - x_lo) / (double)nbins;
    double* centers = calloc((size_t)nbins, sizeof(double));
    double* ratio = calloc((size_t)nbins, sizeof(double));
    double sum = 0.0, pmax = 0.0;
    int64_t failed = 0;
    for (int64_t k = 0; k < nbins; ++k) {
        double e0 = x_lo + dx * (double)k, e1 = x_lo + dx * (double)(k + 1);
        centers[k] = (e0 + e1) / 2.0;
        double g = sqrt(1.0 + ur_c[k] * ur_c[k]);
        ratio[k] = pow(T_c[k], 1.5) / g * exp((mu_c[k] - m * g) / T_c[k]);
        sum += ratio[k];
    }
    for (int64_t k = 0; k < nbins; ++k) { ratio[k] = ratio[k] / sum / dx; pmax = ratio[k] > pmax ? ratio[k] : pmax; }
    if (!(pmax > 0.0) || !isfinite(pmax)) { failed = -1; goto done; }
    for (int64_t k = 0; k < nbins; ++k) ratio[k] /= pmax;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t pid = P->particle_offset + i;
        double r = 0.0;
        int ok = 0;
        for (int t = 0; t < 100000 && !ok; ++t) {
            uint32_t w[4];
            words(P, pid, t, TAG_SAMPLE_XY, w);
            double rt = x_lo + (x_hi - x_lo) * u01(w[0]);
            int64_t idx = 0;                         /* searchsortedfirst(centers, rt) */
            while (idx < nbins && centers[idx] < rt) ++idx;
            double acc = idx < nbins ? ratio[idx] : 0.0;
            if (u01(w[1]) < acc) { r = rt; ok = 1; }
        }
        if (!ok) ++failed;
        double rq = jl_clamp(r, r_T[0], r_T[nT - 1]);
        int64_t k = ss_last(r_T, nT, rq);
        double wk = (rq - r_T[k]) / (r_T[k + 1] - r_T[k]);
        double T = T_r[k] + wk * (T_r[k + 1] - T_r[k]);
        uint32_t v[4];
        double z0, z1;
        words(P, pid, 0, TAG_SAMPLE_P, v);
        box_muller(u01(v[0]), u01(v[1]), &z0, &z1);
        double pr = sqrt(m * T) * z0;
        x[2 * i] = P->t0; x[2 * i + 1] = r;
        p[2 * i] = sqrt(m * m + pr * pr); p[2 * i + 1] = fabs(pr);
    }
done:
    free(centers); free(ratio);
    return failed;
}

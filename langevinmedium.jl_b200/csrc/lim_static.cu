// lim_static.cu — the reference's static-temperature momentum-only path
// (simulate_ensemble_bulk(::CPUBackend, T::Float64), simulate.jl:89-109 ->
// simulate_cpu.jl:325-404), one thread per particle for the whole run.
//
// Its force is the legacy one of kernels_cpu.jl:359-404: kappa = 2.5 T^3,
// eta_D = kappa / (2 T m), kL = kT = sqrt(kappa), an Euler drag -eta_D p dt and the kick
// sqrt(dt) kT xi (the longitudinal-transverse projector term (kL - kT) u (u . xi) is
// identically zero), with the momentum update of kernels_cpu.jl:406-417.  There is no
// position, no medium and no frame change; the driver records |p| every save_every
// steps (simulate_cpu.jl:378-383).  The noise is the step's momentum normals, counter
// (particle, step, TAG_MOM), as in every other kernel.
#include "lim_internal.h"

namespace lim {

template <typename R, int PDIM>
__global__ void __launch_bounds__(256) k_static_T(const StaticRun sr, int64_t s0, int64_t s1)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sr.n) return;
    double p[3] = { 0.0, 0.0, 0.0 };
#pragma unroll
    for (int d = 0; d < PDIM; ++d) p[d] = sr.p[d][i];
    const double T = sr.T;
    const double kappa = 2.5 * (T * T * T);
    const double etaD = kappa / (2.0 * T * sr.m);
    const double kT = sqrt(kappa);
    const double sqdt = sqrt(sr.dt);
    const R etaR = (R)etaD, kTR = (R)kT, dtR = (R)sr.dt, sqdtR = (R)sqdt;
    const uint32_t pid = (uint32_t)(sr.pid_offset + i);
    for (int64_t s = s0; s < s1; ++s) {
        const uint4 u = philox_words(sr.rk, pid, (uint32_t)s, TAG_MOM);
        R xi[3];
        box_muller(u.x, u.y, xi[0], xi[1]);
        xi[2] = PDIM == 3 ? norm_inv(u.z, R(0)) : R(0);
#pragma unroll
        for (int d = 0; d < PDIM; ++d) {
            if (sizeof(R) == 8) {
                const double det = -etaD * p[d] * sr.dt;
                const double sto = kT * (double)xi[d];
                p[d] += det + sqdt * sto;
            } else {                     // FP32 increment added to the FP64 momentum
                const R det = -etaR * (R)p[d] * dtR;
                const R sto = kTR * xi[d];
                p[d] += (double)(det + sqdtR * sto);
            }
        }
        if (sr.save_every > 0 && s % sr.save_every == 0) {
            const int64_t slot = s / sr.save_every - sr.first_slot;
            if (slot >= 0 && slot < sr.nslots) {
                double p2 = 0.0;
#pragma unroll
                for (int d = 0; d < PDIM; ++d) p2 += p[d] * p[d];
                sr.hist[slot * sr.n + i] = sqrt(p2);
            }
        }
    }
#pragma unroll
    for (int d = 0; d < PDIM; ++d) sr.p[d][i] = p[d];
}

template <typename R>
cudaError_t launch_static_T(const StaticRun& sr, int pdim, int64_t s0, int64_t s1, cudaStream_t st)
{
    if (sr.n == 0 || s1 <= s0) return cudaSuccess;
    const unsigned g = (unsigned)((sr.n + 255) / 256);
    switch (pdim) {
    case 1: k_static_T<R, 1><<<g, 256, 0, st>>>(sr, s0, s1); break;
    case 2: k_static_T<R, 2><<<g, 256, 0, st>>>(sr, s0, s1); break;
    case 3: k_static_T<R, 3><<<g, 256, 0, st>>>(sr, s0, s1); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template cudaError_t launch_static_T<double>(const StaticRun&, int, int64_t, int64_t, cudaStream_t);
template cudaError_t launch_static_T<float>(const StaticRun&, int, int64_t, int64_t, cudaStream_t);

}  // namespace lim

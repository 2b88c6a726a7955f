"""The reference's two RTA momentum samplers draw the same Juttner magnitude
distribution P(p*) ~ p*^(d-1) exp(-(E - m)/T):

  - the CPU sampler _draw_juttner_pstar_lib (kernels_cpu.jl:442-458): rejection under a
    flat envelope on [0, pmax), pmax = 16 sqrt(m T) + 16 T, at most 1e5 tries, restated
    in the oracle with Philox uniforms;
  - the GPU sampler (kernels_gpu.jl:88-117 on build_juttner_invcdf, transport.jl:277-365):
    an inverse-CDF table bilinear in (u, T), clamped at the 1 - 1e-6 quantile; this is
    the engine's and the oracle's RTA.

Checked here: a two-sample Kolmogorov-Smirnov test between them, each against the exact
CDF by quadrature, <p*^2> against the exact moment, and the tail mass each one drops:
beyond pmax for the rejection sampler (below 1e-15 at these (m, T)), above the clamped
quantile for the table (1e-6 by construction)."""
import numpy as np
import pytest
from scipy import integrate, stats

CASES = [(1.5, 0.20, 3), (1.5, 0.40, 3), (4.75, 0.30, 3), (1.5, 0.30, 2), (1.5, 0.30, 1)]
N = 200_000


def weight(p, m, T, d):
    return p ** (d - 1) * np.exp(-(np.sqrt(m * m + p * p) - m) / T)


def exact_cdf(m, T, d):
    pmax = 16.0 * np.sqrt(m * T) + 16.0 * T
    norm = integrate.quad(weight, 0.0, np.inf, args=(m, T, d), limit=400)[0]
    grid = np.linspace(0.0, pmax, 20001)
    w = weight(grid, m, T, d)
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (w[1:] + w[:-1]) * np.diff(grid))])
    cum /= norm
    return grid, cum, norm


@pytest.mark.parametrize("m,T,d", CASES)
def test_rejection_and_inverse_cdf_agree(lmb, orc, m, T, d):
    tr = lmb.transport
    case = CASES.index((m, T, d))
    P = orc.make_params(seed=0x4C494D07 + case)
    rej, tries = orc.juttner_rejection(P, m, T, d, N)
    assert np.all(tries >= 1) and np.all(tries < 100000)
    vals, nU, nT, Tmin, invdT = tr.build_juttner_invcdf(m, d, Tmin=0.15, Tmax=0.5)
    md = orc.Medium()
    md.invcdf(vals, nU, nT, Tmin, invdT)
    u = (np.random.default_rng(11 + case).integers(0, 2 ** 32, N).astype(np.float64) + 0.5) * 2.0 ** -32
    tab = np.array([orc.invcdf_lookup(md, float(x), T) for x in u])
    grid, cum, norm = exact_cdf(m, T, d)
    cdf = lambda x: np.interp(x, grid, cum)
    ks2 = stats.ks_2samp(rej, tab)
    ks_rej = stats.kstest(rej, cdf)
    ks_tab = stats.kstest(tab, cdf)
    # tail masses: beyond pmax (rejection) and above the table's largest value (inverse CDF)
    pmax = 16.0 * np.sqrt(m * T) + 16.0 * T
    tail_rej = integrate.quad(weight, pmax, np.inf, args=(m, T, d))[0] / norm
    tail_tab = integrate.quad(weight, float(tab.max()), np.inf, args=(m, T, d))[0] / norm
    jT = int(np.clip(np.floor((T - Tmin) * invdT), 0, nT - 2))
    p_cap = max(vals[jT * nU + nU - 1], vals[(jT + 1) * nU + nU - 1])
    tail_cap = integrate.quad(weight, float(p_cap), np.inf, args=(m, T, d))[0] / norm
    p2 = integrate.quad(lambda p: p * p * weight(p, m, T, d), 0.0, np.inf, limit=400)[0] / norm
    se = np.sqrt(np.var(rej ** 2) / N)
    print(f"m={m} T={T} d={d}: KS two-sample p={ks2.pvalue:.3g}; vs exact: rejection p={ks_rej.pvalue:.3g}, "
          f"table p={ks_tab.pvalue:.3g}; <p^2> exact {p2:.5f}, rejection {np.mean(rej ** 2):.5f}, table "
          f"{np.mean(tab ** 2):.5f} (s.e. {se:.5f}); mean tries {tries.mean():.2f}; tail beyond pmax {tail_rej:.2e}, "
          f"beyond the table's cap {tail_cap:.2e}")
    assert ks2.pvalue > 1e-3 and ks_rej.pvalue > 1e-3 and ks_tab.pvalue > 1e-3
    assert abs(np.mean(rej ** 2) - p2) < 4 * se and abs(np.mean(tab ** 2) - p2) < 4 * se
    assert tail_rej < 1e-15
    assert tail_cap < 2e-6 and tail_tab < 2e-6

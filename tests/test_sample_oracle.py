"""The oracle's initial-state samplers (the checkers of lim_sample_fonll and
lim_sample_milne) against the
reference's own statements about it:

* test_momentum_dims3.jl:98-117 (S): the conditional p_z draw has the thermal <p_z^2>
  of exp(-sqrt(mT^2 + p_z^2)/T) (quadrature, rtol 0.02 at 2e5 draws), zero mean, and
  antithetic pairs mirror p_z exactly;
* utils.jl:33-172: the position density is n(r) (Cartesian mode) or the r marginal of
  r p f (polar mode), and |p| | r follows the row CDF built from p f(r, p) — checked by
  Kolmogorov–Smirnov tests against those CDFs, restated here in numpy;
* utils.jl:350-400: the Milne sampler's r follows the binned Boltzmann density (the
  first bin center >= r decides), p^r is half-normal with sigma = sqrt(m T(r)) and p^tau
  is on shell.
"""
import numpy as np
import pytest
from scipy import integrate, stats

EPS = np.finfo(np.float64).eps


def fonll_like(nr=61, np_=121, rmax=9.0, pmax=15.0):
    r = np.linspace(0.0, rmax, nr)
    p = np.linspace(0.0, pmax, np_)
    R, Pm = np.meshgrid(r, p)                      # (Np, Nr), as utils.jl expects
    f = np.exp(-R ** 2 / (2 * 2.5 ** 2)) * (1 + 0.3 * np.cos(R)) * Pm ** 0.5 * np.exp(-Pm / (1.2 + 0.1 * R))
    return r, p, f


def row_cdfs(r, p, f):
    """utils.jl:56-72: the conditional CDF of |p| given the r node."""
    dp = np.mean(np.diff(p))
    out = []
    for i in range(r.size):
        pdf = p * f[:, i]
        if not pdf.sum() > 0:
            out.append(None)
            continue
        c = np.cumsum(pdf) * dp
        c[0] = 0.0
        for k in range(1, c.size):
            c[k] = max(c[k], c[k - 1] + EPS)
        c /= c[-1]
        c[-1] = 1.0
        out.append(c)
    return out


def polar_r_cdf(r, p, f):
    """utils.jl:135-157: the r marginal of r p f, cumulated on the r grid."""
    dr, dp = np.mean(np.diff(r)), np.mean(np.diff(p))
    P = r[None, :] * p[:, None] * f
    P = P / (P.sum() * dr * dp)
    c = np.cumsum(P.sum(axis=0) * dp) * dr
    c[0] = 0.0
    for k in range(1, c.size):
        c[k] = max(c[k], c[k - 1] + EPS)
    c /= c[-1]
    c[-1] = 1.0
    return c


def pit_p(r_samples, pmag, r, p, cdfs):
    """Probability integral transform of each |p| under its r node's row CDF."""
    j = np.clip(np.searchsorted(r, r_samples, side="right") - 1, 0, r.size - 1)
    return np.array([np.interp(pm, p, cdfs[jj]) for pm, jj in zip(pmag, j)])


@pytest.mark.parametrize("mT,T", [(1.6, 0.3), (2.5, 0.45), (1.5, 0.156), (0.2, 0.3)])
def test_pz_conditional_is_thermal(orc, mT, T):
    P = orc.make_params(seed=7, dims=2, pdim=3)
    s = orc.sample_pz(P, mT, T, 200_000)
    num = integrate.quad(lambda z: z * z * np.exp(-(np.sqrt(mT * mT + z * z) - mT) / T), -np.inf, np.inf,
                         epsrel=1e-10)[0]
    den = integrate.quad(lambda z: np.exp(-(np.sqrt(mT * mT + z * z) - mT) / T), -np.inf, np.inf, epsrel=1e-10)[0]
    assert np.mean(s ** 2) == pytest.approx(num / den, rel=0.02)
    assert abs(np.mean(s)) < 4 * np.std(s) / np.sqrt(s.size)


def test_pz_degenerate_inputs(orc):
    P = orc.make_params(seed=7, dims=2, pdim=3)
    assert np.all(orc.sample_pz(P, 1.5, 0.0, 8) == 0.0)       # T = 0: no thermal p_z
    assert np.all(orc.sample_pz(P, 0.0, 0.3, 8) == 0.0)


def test_polar_sampling_follows_the_tables(orc):
    r, p, f = fonll_like()
    P = orc.make_params(seed=11, dims=2, pdim=2)
    n = 20_000
    x, pm, failed = orc.sample_fonll(P, None, r, p, f, n, cartesian=False)
    assert failed == 0
    rs = np.hypot(x[0], x[1])
    c = polar_r_cdf(r, p, f)
    assert stats.kstest(rs, lambda v: np.interp(v, r, c)).pvalue > 1e-3
    assert stats.kstest(np.arctan2(x[1], x[0]), stats.uniform(-np.pi, 2 * np.pi).cdf).pvalue > 1e-3
    u = pit_p(rs, np.hypot(pm[0], pm[1]), r, p, row_cdfs(r, p, f))
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    assert stats.kstest(np.arctan2(pm[1], pm[0]), stats.uniform(-np.pi, 2 * np.pi).cdf).pvalue > 1e-3


def test_cartesian_sampling_follows_n_of_r(orc):
    r, p, f = fonll_like()
    P = orc.make_params(seed=12, dims=2, pdim=2)
    n = 20_000
    x, pm, failed = orc.sample_fonll(P, None, r, p, f, n, cartesian=True)
    assert failed == 0
    rs = np.hypot(x[0], x[1])
    assert rs.max() <= r[-1]
    dp = np.mean(np.diff(p))
    nsp = (p[:, None] * f).sum(axis=0) * dp                 # n(r) = int p f dp (utils.jl:89)
    fine = np.linspace(0.0, r[-1], 20001)
    dens = fine * np.interp(fine, r, nsp)                   # uniform in the plane: r n(r) dr
    cdf = integrate.cumulative_trapezoid(dens, fine, initial=0.0)
    cdf /= cdf[-1]
    assert stats.kstest(rs, lambda v: np.interp(v, fine, cdf)).pvalue > 1e-3
    u = pit_p(rs, np.hypot(pm[0], pm[1]), r, p, row_cdfs(r, p, f))
    assert stats.kstest(u, "uniform").pvalue > 1e-3


def test_antithetic_pairs_and_odd_count(orc):
    r, p, f = fonll_like()
    P = orc.make_params(seed=13, dims=2, pdim=3, t0=0.6)
    md = orc.Medium().bjorken(0.4, 0.6)
    for cart in (True, False):
        x, pm, failed = orc.sample_fonll(P, md, r, p, f, 1001, cartesian=cart, antithetic=True, thermal_pz=True)
        assert failed == 0
        assert np.array_equal(x[:, 0:1000:2], x[:, 1:1000:2])
        assert np.array_equal(pm[:, 0:1000:2], -pm[:, 1:1000:2])
        assert not np.array_equal(x[:, 1000], x[:, 998])     # the odd one is its own draw
        assert np.all(pm[2] != 0.0)


def test_thermal_pz_uses_medium_at_t0(orc):
    """p_z of particle i is the conditional draw at its mT and T(x_i, t0) (utils.jl:533-551)."""
    r, p, f = fonll_like()
    P = orc.make_params(seed=14, dims=2, pdim=3, t0=0.6, m=1.5)
    md = orc.Medium().bjorken(0.4, 0.6)
    x, pm, _ = orc.sample_fonll(P, md, r, p, f, 64, cartesian=True, thermal_pz=True)
    for i in range(0, 64, 7):
        mT = np.sqrt(1.5 ** 2 + pm[0, i] ** 2 + pm[1, i] ** 2)
        Pi = orc.make_params(seed=14, dims=2, pdim=3, t0=0.6, m=1.5, particle_offset=i)
        assert orc.sample_pz(Pi, mT, 0.4, 1)[0] == pm[2, i]


def test_zero_density(orc):
    r, p, _ = fonll_like(nr=5, np_=5)
    P = orc.make_params(seed=15, dims=2, pdim=2)
    _, _, failed = orc.sample_fonll(P, None, r, p, np.zeros((5, 5)), 3, cartesian=False)
    assert failed == -1                                     # "Distribution normalization is zero."


def milne_profiles(nbins=200, x_hi=10.0):
    c = (np.arange(nbins) + 0.5) * x_hi / nbins
    T = lambda r: 0.42 * np.exp(-np.asarray(r) ** 2 / 30.0) + 0.05
    return c, T(c), 0.04 * c, 0.02 * np.sin(c), T


def test_milne_sampler_follows_the_binned_density(orc):
    """utils.jl:356-399: r by rejection against the binned n_boltz (the first bin center
    >= r decides), p^r half-normal with sigma = sqrt(m T(r)), p^tau on shell."""
    m, x_hi, n = 1.5, 10.0, 20_000
    c, Tc, urc, muc, Tf = milne_profiles(x_hi=x_hi)
    rT = np.linspace(0.0, x_hi, 1601)
    P = orc.make_params(seed=21, dims=2, pdim=2, m=m, t0=0.4)
    x, p, failed = orc.sample_milne(P, 0.0, x_hi, Tc, urc, muc, rT, Tf(rT), n)
    assert failed == 0
    assert np.all(x[0] == 0.4)
    g = np.sqrt(1 + urc ** 2)
    nb = Tc ** 1.5 / g * np.exp((muc - m * g) / Tc)
    # density of r: nb[k] on (c[k-1], c[k]] (k = 0 from x_lo), 0 beyond the last center
    edges = np.concatenate([[0.0], c])
    mass = nb * np.diff(edges)
    cdf_nodes = np.concatenate([[0.0], np.cumsum(mass)]) / mass.sum()
    assert stats.kstest(x[1], lambda v: np.interp(v, edges, cdf_nodes)).pvalue > 1e-3
    sig = np.sqrt(m * np.interp(x[1], rT, Tf(rT)))
    u = 2 * stats.norm.cdf(p[1] / sig) - 1
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    assert np.allclose(p[0], np.sqrt(m * m + p[1] ** 2), rtol=1e-15)
    assert np.all(p[1] >= 0)


def test_milne_sampler_degenerate_density(orc):
    c, Tc, urc, muc, Tf = milne_profiles(nbins=4)
    P = orc.make_params(seed=22, dims=2, pdim=2, m=1.5)
    rT = np.linspace(0, 10, 5)
    _, _, failed = orc.sample_milne(P, 0.0, 10.0, np.zeros(4), urc, muc, rT, Tf(rT), 3)
    assert failed == -1

"""ctypes wrapper of the CPU FP64 restatement (lim_oracle.c).

TEST INFRASTRUCTURE ONLY — the parity checker and the timed CPU baseline.  The
engine never imports this module.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm use it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblim_oracle.so"

NOISE_SLOTS = 11
M_RT, M_BJORKEN, M_GRID = 0, 1, 2


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("dt", "t0", "m", "DsT", "Tfo", "psi2", "obs_pt_cut", "obs_pt_width")] + \
               [(n, C.c_int64) for n in ("dims", "pdim", "coords", "collision", "relativistic", "bjorken_redshift",
                                         "position_diffusion", "reflecting_boundary", "integrator_mode",
                                         "freezeout_capture", "freezeout_interp", "precision", "seed",
                                         "particle_offset", "stop_after_freezeout", "block_size", "rta_replay")]


_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)


class OrcMedium(C.Structure):
    _fields_ = [("kind", C.c_int64),
                ("xg", _DP), ("tg", _DP), ("T", _DP), ("V", _DP), ("V2", _DP),
                ("nr", C.c_int64), ("nt", C.c_int64),
                ("bj_T0", C.c_double), ("bj_tau0", C.c_double), ("bj_power", C.c_double), ("bj_rmax", C.c_double),
                ("gT", _FP), ("gux", _FP), ("guy", _FP),
                ("gnx", C.c_int64), ("gny", C.c_int64), ("gnt", C.c_int64),
                ("gx0", C.c_double), ("gdx", C.c_double), ("gy0", C.c_double), ("gdy", C.c_double),
                ("gt0", C.c_double), ("gdt", C.c_double),
                ("drag", _DP), ("n_drag", C.c_int64), ("drag_Tmin", C.c_double), ("drag_invdT", C.c_double),
                ("rta", _DP), ("n_rta", C.c_int64), ("rta_Tmin", C.c_double), ("rta_invdT", C.c_double),
                ("icdf", _DP), ("nU", C.c_int64), ("nT", C.c_int64), ("ic_Tmin", C.c_double), ("ic_invdT", C.c_double),
                ("T_scale", C.c_double)]


FO_FIELDS = 16   # pos[3], mom[3], tau, flag, lpos[3], lmom[3], ltau, lT


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "lim_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True, capture_output=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        L.orc_run.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcMedium), _DP, _DP, C.c_int64, C.c_int64, C.c_int64,
                              C.c_int64, C.c_int64, _DP, _DP, _DP, _DP, C.c_int, C.POINTER(C.c_uint8)]
        L.orc_run.restype = C.c_int64
        L.orc_initial_lab_boost.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcMedium), _DP, _DP, C.c_int64]
        L.orc_initial_lab_boost.restype = None
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_philox4x32_10.restype = None
        L.orc_uniforms4.argtypes = [C.POINTER(OrcParams), C.c_int64, C.c_int64, C.c_int, _DP]
        L.orc_uniforms4.restype = None
        L.orc_interp2d_clamped.argtypes = [_DP, C.c_int64, _DP, C.c_int64, _DP, C.c_double, C.c_double]
        L.orc_interp2d_clamped.restype = C.c_double
        L.orc_eval_spline.argtypes = [C.c_double, C.c_double, C.c_double, _DP, C.c_int64]
        L.orc_eval_spline.restype = C.c_double
        L.orc_invcdf_lookup.argtypes = [C.POINTER(OrcMedium), C.c_double, C.c_double]
        L.orc_invcdf_lookup.restype = C.c_double
        for f in ("orc_sizeof_params", "orc_sizeof_medium", "orc_sizeof_fo"):
            getattr(L, f).restype = C.c_int64
        L.orc_max_threads.restype = C.c_int
        L.orc_step_variates.argtypes = [C.POINTER(OrcParams), C.c_int64, C.c_int64, C.c_int, _DP]
        L.orc_step_variates.restype = None
        L.orc_sample_fonll.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcMedium), _DP, C.c_int64, _DP, C.c_int64,
                                       _DP, C.c_int64, C.c_int, C.c_int, C.c_int, _DP, _DP]
        L.orc_sample_fonll.restype = C.c_int64
        L.orc_sample_milne.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_double, C.c_int64, _DP, _DP, _DP, _DP,
                                       _DP, C.c_int64, C.c_int64, _DP, _DP]
        L.orc_sample_milne.restype = C.c_int64
        L.orc_juttner_rejection.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_double, C.c_int64, C.c_int64,
                                            C.c_int64, _DP, C.POINTER(C.c_int64)]
        L.orc_juttner_rejection.restype = None
        L.orc_run_static.argtypes = [C.POINTER(OrcParams), C.c_double, _DP, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                     C.c_int64, C.c_int64, _DP, C.c_int]
        L.orc_run_static.restype = None
        L.orc_sample_pz.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_double, C.c_int64, _DP]
        L.orc_sample_pz.restype = None
        assert L.orc_sizeof_params() == C.sizeof(OrcParams)
        assert L.orc_sizeof_medium() == C.sizeof(OrcMedium)
        assert L.orc_sizeof_fo() == FO_FIELDS * 8
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_DP)


def make_params(**kw) -> OrcParams:
    P = OrcParams()
    d = dict(dt=0.001, t0=0.0, m=1.0, DsT=0.2, Tfo=0.156, psi2=0.0, obs_pt_cut=5.0, obs_pt_width=0.1, dims=3, pdim=0,
             coords=0, collision=0, relativistic=1, bjorken_redshift=0, position_diffusion=0, reflecting_boundary=0,
             integrator_mode=0, freezeout_capture=0, freezeout_interp=1, precision=0, seed=0x4C494D00,
             particle_offset=0, stop_after_freezeout=0, block_size=0, rta_replay=0)
    d.update(kw)
    if d["pdim"] <= 0:
        d["pdim"] = d["dims"]
    for k, v in d.items():
        setattr(P, k, float(v) if isinstance(getattr(P, k), float) else int(v))
    return P


class Medium:
    """Holds the arrays an OrcMedium points to (keeps them alive)."""

    def __init__(self):
        self.s = OrcMedium()
        self.s.T_scale = 1.0
        self._keep = []

    def _k(self, a, dtype=np.float64):
        a = np.ascontiguousarray(a, dtype=dtype)
        self._keep.append(a)
        return a

    def rt(self, xgrid, tgrid, T, V, V2=None):
        s = self.s
        s.kind = M_RT
        xg, tg = self._k(xgrid), self._k(tgrid)
        s.xg, s.tg = _d(xg), _d(tg)
        s.nr, s.nt = xg.size, tg.size
        s.T = _d(self._k(np.asarray(T, dtype=np.float64).ravel(order="F")))
        s.V = _d(self._k(np.asarray(V, dtype=np.float64).ravel(order="F")))
        s.V2 = None if V2 is None else _d(self._k(np.asarray(V2, dtype=np.float64).ravel(order="F")))
        return self

    def bjorken(self, T0, tau0, power=1.0 / 3.0, r_max=0.0):
        s = self.s
        s.kind = M_BJORKEN
        s.bj_T0, s.bj_tau0, s.bj_power, s.bj_rmax = T0, tau0, power, r_max
        return self

    def grid(self, T, ux, uy, x0, dx, y0, dy, tau0, dtau):
        s = self.s
        s.kind = M_GRID
        Tg, ug, vg = self._k(T, np.float32), self._k(ux, np.float32), self._k(uy, np.float32)
        s.gT, s.gux, s.guy = (a.ctypes.data_as(_FP) for a in (Tg, ug, vg))
        s.gnt, s.gny, s.gnx = Tg.shape
        s.gx0, s.gdx, s.gy0, s.gdy, s.gt0, s.gdt = x0, dx, y0, dy, tau0, dtau
        return self

    def spline(self, which, Tmin, invdT, vals):
        v = self._k(vals)
        if which == 0:
            self.s.drag, self.s.n_drag, self.s.drag_Tmin, self.s.drag_invdT = _d(v), v.size, Tmin, invdT
        elif which == 1:
            self.s.rta, self.s.n_rta, self.s.rta_Tmin, self.s.rta_invdT = _d(v), v.size, Tmin, invdT
        # the drag-derivative tables (2, 3) belong to the engine's reverse sweep only
        return self

    def invcdf(self, vals, nU, nT, Tmin, invdT):
        v = self._k(vals)
        self.s.icdf, self.s.nU, self.s.nT, self.s.ic_Tmin, self.s.ic_invdT = _d(v), nU, nT, Tmin, invdT
        return self

    def scale(self, s):
        self.s.T_scale = float(s)
        return self


def to_flat(a, rows):
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    assert a.shape[0] == rows, (a.shape, rows)
    return np.ascontiguousarray(a.T).reshape(-1).copy()


def from_flat(b, rows, n):
    return b.reshape(n, rows).T.copy()


def initial_lab_boost(P: OrcParams, md: Medium, x, p):
    n = np.asarray(x).shape[-1]
    xb, pb = to_flat(x, P.dims), to_flat(p, P.pdim)
    lib().orc_initial_lab_boost(C.byref(P), C.byref(md.s), _d(xb), _d(pb), n)
    return from_flat(xb, P.dims, n), from_flat(pb, P.pdim, n)


def run(P: OrcParams, md: Medium, x, p, first_step, nsteps, *, save_every=0, first_slot=0, nslots=0,
        fo=None, rec=None, threads=0, decisions=False):
    """Run the restatement.  Returns dict(x, p, first_bad, hist_x, hist_p, fo), and with
    decisions=True "dec": uint8 (nsteps, N), bit 0 = the particle collided (RTA) in
    that step, bit 1 = it latched at freeze-out in that step.  fo: an initial latch
    state (N * FO_FIELDS doubles, per particle pos[3], mom[3], tau, flag, lpos[3],
    lmom[3], ltau, lT), zeros when None."""
    n = np.asarray(x).shape[-1]
    xb, pb = to_flat(x, P.dims), to_flat(p, P.pdim)
    hx = hp = None
    if save_every > 0 and nslots > 0:
        hx = np.zeros(nslots * n * P.dims)
        hp = np.zeros(nslots * n * P.pdim)
    fob = None
    if P.freezeout_capture:
        fob = np.zeros(n * FO_FIELDS) if fo is None else fo
    recb = None
    if rec is not None:
        recb = np.ascontiguousarray(rec, dtype=np.float64).reshape(-1)
        assert recb.size == nsteps * NOISE_SLOTS * n
    dec = np.zeros((nsteps, n), dtype=np.uint8) if decisions else None
    bad = lib().orc_run(C.byref(P), C.byref(md.s), _d(xb), _d(pb), n, first_step, nsteps, save_every, first_slot,
                        _d(hx), _d(hp), _d(fob), _d(recb), int(threads),
                        None if dec is None else dec.ctypes.data_as(C.POINTER(C.c_uint8)))
    out = dict(x=from_flat(xb, P.dims, n), p=from_flat(pb, P.pdim, n), first_bad=int(bad), fo=fob)
    if dec is not None:
        out["dec"] = dec
    if hx is not None:
        out["hist_x"] = [from_flat(hx[k * n * P.dims:(k + 1) * n * P.dims], P.dims, n) for k in range(nslots)]
        out["hist_p"] = [from_flat(hp[k * n * P.pdim:(k + 1) * n * P.pdim], P.pdim, n) for k in range(nslots)]
    if fob is not None:
        f = fob.reshape(n, FO_FIELDS)
        out["fo_pos"] = f[:, 0:P.dims].T.copy()
        out["fo_mom"] = f[:, 3:3 + P.pdim].T.copy()
        out["fo_tau"] = f[:, 6].copy()
        out["fo_flag"] = f[:, 7].copy()
        out["fo_lpos"] = f[:, 8:8 + P.dims].T.copy()
        out["fo_lmom"] = f[:, 11:11 + P.pdim].T.copy()
        out["fo_ltau"] = f[:, 14].copy()
        out["fo_lT"] = f[:, 15].copy()
    return out


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def uniforms4(P, pid, step, tag):
    u = np.zeros(4)
    lib().orc_uniforms4(C.byref(P), pid, step, tag, _d(u))
    return u


def step_variates(P, pid, step, kick=True):
    """The 11 recording slots the engine draws for (particle, step), as if it collided."""
    out = np.zeros(NOISE_SLOTS)
    lib().orc_step_variates(C.byref(P), pid, step, int(bool(kick)), _d(out))
    return out


def max_threads() -> int:
    return int(lib().orc_max_threads())


def sample_fonll(P: OrcParams, md: Medium | None, r_grid, p_grid, f, n, *, cartesian=True, antithetic=False,
                 thermal_pz=False):
    """Restatement of the device FONLL sampler.  f has Julia's shape (Np, Nr).
    Returns (x (2, n), p (pdim, n), failed)."""
    rg = np.ascontiguousarray(r_grid, dtype=np.float64)
    pg = np.ascontiguousarray(p_grid, dtype=np.float64)
    fm = np.asarray(f, dtype=np.float64)
    assert fm.shape == (pg.size, rg.size)
    fb = np.ascontiguousarray(fm.T).reshape(-1)          # f[ip + np*ir]
    xb = np.zeros(max(2 * n, 1))
    pb = np.zeros(max(P.pdim * n, 1))
    mds = None if md is None else C.byref(md.s)
    failed = lib().orc_sample_fonll(C.byref(P), mds, _d(rg), rg.size, _d(pg), pg.size, _d(fb), int(n),
                                    int(bool(cartesian)), int(bool(antithetic)), int(bool(thermal_pz)), _d(xb), _d(pb))
    return from_flat(xb[:2 * n], 2, n), from_flat(pb[:P.pdim * n], P.pdim, n), int(failed)


def sample_pz(P: OrcParams, mT, T, n):
    """p_z draws of particles particle_offset + 0 .. n-1 at fixed (mT, T)."""
    out = np.zeros(max(int(n), 1))
    lib().orc_sample_pz(C.byref(P), float(mT), float(T), int(n), _d(out))
    return out[:int(n)]


def sample_milne(P: OrcParams, x_lo, x_hi, T_c, ur_c, mu_c, r_T, T_r, n):
    """Restatement of the device Milne sampler.  Returns (x (2, n), p (2, n), failed)."""
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (T_c, ur_c, mu_c, r_T, T_r)]
    xb = np.zeros(max(2 * n, 1))
    pb = np.zeros(max(2 * n, 1))
    failed = lib().orc_sample_milne(C.byref(P), float(x_lo), float(x_hi), a[0].size, _d(a[0]), _d(a[1]), _d(a[2]),
                                    _d(a[3]), _d(a[4]), a[3].size, int(n), _d(xb), _d(pb))
    return from_flat(xb[:2 * n], 2, n), from_flat(pb[:2 * n], 2, n), int(failed)


def juttner_rejection(P: OrcParams, m: float, T: float, d: int, n: int, first_pid: int = 0):
    """n draws of the CPU RTA's rejection sampler (kernels_cpu.jl:442-458) with Philox
    uniforms; returns (p*, tries per draw)."""
    out = np.zeros(n)
    tries = np.zeros(n, dtype=np.int64)
    lib().orc_juttner_rejection(C.byref(P), float(m), float(T), int(d), int(first_pid), int(n), _d(out),
                                tries.ctypes.data_as(C.POINTER(C.c_int64)))
    return out, tries


def invcdf_lookup(md: "Medium", u: float, T: float) -> float:
    """The inverse-CDF table lookup of the GPU RTA (kernels_gpu.jl:88-117)."""
    return float(lib().orc_invcdf_lookup(C.byref(md.s), float(u), float(T)))


def run_static(P: OrcParams, T: float, p, first_step: int, nsteps: int, *, save_every=0, first_slot=0, nslots=0,
               threads=0):
    """The static-temperature momentum-only path (simulate_cpu.jl:325-404); returns
    (p (pdim, N), |p| history (nslots, N))."""
    n = np.asarray(p).shape[-1]
    pb = to_flat(p, P.pdim)
    hist = np.zeros((max(nslots, 0), n))
    lib().orc_run_static(C.byref(P), float(T), _d(pb), n, int(first_step), int(nsteps), int(save_every),
                         int(first_slot), int(nslots), _d(hist) if nslots > 0 else None, int(threads))
    return from_flat(pb, P.pdim, n), hist

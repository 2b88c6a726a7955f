"""ctypes binding of ``liblangevin_b200.so`` (the C-ABI declared in include/langevin_b200.h).

This is the Python twin of the Julia ``ccall`` layer: plain pointers and sizes, an
``int`` status per call, and ``lim_last_error`` turned into an exception.  There is
no fallback: if the CUDA library is missing or no GPU is present, the calls fail.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "liblangevin_b200.so"
HEADER = PKG_DIR.parent / "include" / "langevin_b200.h"
DIAG_HEADER = PKG_DIR.parent / "include" / "langevin_b200_diag.h"

LIM_OK, LIM_ERR_ARG, LIM_ERR_CUDA, LIM_ERR_STATE, LIM_ERR_NONFINITE, LIM_ERR_TIMEOUT, LIM_ERR_UNSUPPORTED, LIM_ERR_NOMEM = \
    0, -1, -2, -3, -4, -5, -6, -7
LIM_FP64, LIM_FP32 = 0, 1
LIM_COORDS_CARTESIAN, LIM_COORDS_MILNE = 0, 1
LIM_COLL_LANGEVIN, LIM_COLL_RTA, LIM_COLL_LANGEVIN_RTA, LIM_COLL_FLUID = 0, 1, 2, 3
LIM_SPLINE_DRAG, LIM_SPLINE_RTA, LIM_SPLINE_DRAG_DA, LIM_SPLINE_DRAG_DB = 0, 1, 2, 3
LIM_NOISE_SLOTS = 11
OBS_NAMES = ("count", "mean_pt", "mean_cos2phi", "frac_pt_gt", "frac_pt_gt_smooth", "mean_p2", "mean_E",
             "mean_lam1_num", "mean_px", "mean_wpx", "mean_pz2", "mean_x2")
LIM_OBS_NUM = len(OBS_NAMES)


class LimParams(C.Structure):
    """lim_params: every field 8 bytes wide (same layout in C, Julia and here)."""
    _fields_ = [(n, C.c_double) for n in ("dt", "t0", "m", "DsT", "Tfo", "psi2", "obs_pt_cut", "obs_pt_width")] + \
               [(n, C.c_int64) for n in ("dims", "pdim", "coords", "collision", "relativistic", "bjorken_redshift",
                                         "position_diffusion", "reflecting_boundary", "integrator_mode",
                                         "freezeout_capture", "freezeout_interp", "precision", "seed",
                                         "particle_offset", "stop_after_freezeout", "block_size")]


class LimError(RuntimeError):
    """A non-zero status from the engine; ``code`` is the LIM_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_lib = None

_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
_U32P = C.POINTER(C.c_uint32)
_I64P = C.POINTER(C.c_int64)

class LimBatchShape(C.Structure):
    """lim_batch_shape: block, chunk_steps, blocks_per_sm, reg_cap (0 = automatic)."""
    _fields_ = [(n, C.c_int64) for n in ("block", "chunk_steps", "blocks_per_sm", "reg_cap")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class LimDsForm(C.Structure):
    _fields_ = [("linear", C.c_int64), ("slope", C.c_double), ("offset", C.c_double), ("Tfo", C.c_double),
                ("quad", C.c_int64), ("Tref", C.c_double)]


LIM_TIME_DRAG, LIM_TIME_TAUN, LIM_TIME_TAUR = 0, 1, 2


class LimReduceSpec(C.Structure):
    _fields_ = [("r_bins", C.c_int64), ("r_max", C.c_double), ("pt_bins", C.c_int64), ("pt_max", C.c_double)]


def reduce_spec(r_bins: int, r_max: float, pt_bins: int, pt_max: float) -> LimReduceSpec:
    return LimReduceSpec(int(r_bins), float(r_max), int(pt_bins), float(pt_max))


class _PinnedBlock:
    """Owner of one lim_host_alloc block; freed when the last array viewing it goes."""

    def __init__(self, lib, nbytes: int):
        self.lib, self.ptr = lib, C.c_void_p()
        rc = lib.lim_host_alloc(int(nbytes), C.byref(self.ptr))
        if rc != LIM_OK:
            raise LimError(rc, lib.lim_last_error(None).decode())

    def __del__(self):
        # at interpreter exit module globals (ctypes included) may already be gone
        ptr, self.ptr = getattr(self, "ptr", None), None
        if ptr is not None and ptr.value:
            self.lib.lim_host_free(ptr)


def pinned_empty(n: int, dtype=np.float64, lib: C.CDLL | None = None) -> np.ndarray:
    """An uninitialised 1-D array of n elements in page-locked host memory
    (lim_host_alloc): snapshot histories written into it move at the host-link rate."""
    lib = lib or load_library()
    dt = np.dtype(dtype)
    n = int(n)
    block = _PinnedBlock(lib, max(n, 1) * dt.itemsize)
    raw = (C.c_char * (max(n, 1) * dt.itemsize)).from_address(block.ptr.value)
    raw._owner = block                       # the ctypes view keeps the block alive
    return np.frombuffer(raw, dtype=dt, count=n)


def split_reduced(out: np.ndarray, spec: LimReduceSpec) -> dict:
    """(nslots, stride) doubles of lim_run_reduced / lim_reduce_state -> named arrays."""
    nr, npt = int(spec.r_bins) + 1, int(spec.pt_bins) + 1
    o = out.reshape(-1, LIM_OBS_NUM + nr + 2 * npt)
    return dict(obs=o[:, :LIM_OBS_NUM].copy(), r_counts=o[:, LIM_OBS_NUM:LIM_OBS_NUM + nr].copy(),
                pt_counts=o[:, LIM_OBS_NUM + nr:LIM_OBS_NUM + nr + npt].copy(),
                pt_cos2=o[:, LIM_OBS_NUM + nr + npt:].copy())


_SIGS = {
    "lim_abi_version": ([], C.c_int),
    "lim_create": ([C.c_int, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "lim_destroy": ([C.c_void_p], C.c_int),
    "lim_last_error": ([C.c_void_p], C.c_char_p),
    "lim_synchronize": ([C.c_void_p], C.c_int),
    "lim_device_bytes": ([C.c_void_p, _I64P], C.c_int),
    "lim_set_params": ([C.c_void_p, C.POINTER(LimParams)], C.c_int),
    "lim_set_medium_rt": ([C.c_void_p, _DP, C.c_int64, _DP, C.c_int64, _DP, _DP, _DP], C.c_int),
    "lim_set_medium_bjorken": ([C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double], C.c_int),
    "lim_set_medium_grid": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                             C.c_double, C.c_double, C.c_double, _FP, _FP, _FP], C.c_int),
    "lim_set_spline": ([C.c_void_p, C.c_int, C.c_double, C.c_double, _DP, C.c_int64], C.c_int),
    "lim_set_invcdf": ([C.c_void_p, _DP, C.c_int64, C.c_int64, C.c_double, C.c_double], C.c_int),
    "lim_upload_state": ([C.c_void_p, _DP, C.c_int64, _DP, C.c_int64, C.c_int64], C.c_int),
    "lim_download_state": ([C.c_void_p, _DP, _DP], C.c_int),
    "lim_initial_lab_boost": ([C.c_void_p], C.c_int),
    "lim_state_save": ([C.c_void_p], C.c_int),
    "lim_state_restore": ([C.c_void_p], C.c_int),
    "lim_run": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _DP, _DP], C.c_int),
    "lim_run_static_T": ([C.c_void_p, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _DP],
                         C.c_int),
    "lim_status": ([C.c_void_p, _I64P], C.c_int),
    "lim_download_freezeout": ([C.c_void_p, _DP, _DP, _DP, _DP], C.c_int),
    "lim_observables": ([C.c_void_p, C.c_int, _DP], C.c_int),
    "lim_record_noise": ([C.c_void_p, C.c_int64, C.c_int64], C.c_int),
    "lim_download_noise": ([C.c_void_p, _DP], C.c_int),
    "lim_philox_device": ([C.c_void_p, _U32P, _U32P, _U32P], C.c_int),
    "lim_last_run_stats": ([C.c_void_p, _DP, _I64P], C.c_int),
    "lim_probe_fma_rate": ([C.c_void_p, _DP, _DP], C.c_int),
    "lim_probe_mufu_rate": ([C.c_void_p, _DP, _DP], C.c_int),
    "lim_observables_noalloc": ([C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_double,
                                 C.c_double, C.c_double, C.c_void_p, C.c_void_p], C.c_int),
    "lim_set_medium_scale": ([C.c_void_p, C.c_double], C.c_int),
    "lim_rta_decisions": ([C.c_void_p, C.c_int, C.c_int64, C.c_int64], C.c_int),
    "lim_copy_rta_decisions": ([C.c_void_p, C.c_void_p], C.c_int),
    "lim_adjoint": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int64, _DP, _DP], C.c_int),
    "lim_adjoint_stats": ([C.c_void_p, _DP, _DP], C.c_int),
    "lim_build_time_spline": ([C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(LimDsForm), C.c_double,
                               C.c_double, C.c_int64, C.c_double, C.c_double, C.c_double], C.c_int),
    "lim_build_juttner_invcdf": ([C.c_void_p, C.c_double, C.c_int64, C.c_double, C.c_double, C.c_int64, C.c_int64,
                                  C.c_int64, C.c_double], C.c_int),
    "lim_get_spline": ([C.c_void_p, C.c_int, _DP, _DP, _DP, C.c_int64, _I64P], C.c_int),
    "lim_get_invcdf": ([C.c_void_p, _DP, C.c_int64, _I64P, _I64P, _DP, _DP], C.c_int),
    "lim_host_alloc": ([C.c_int64, C.POINTER(C.c_void_p)], C.c_int),
    "lim_host_free": ([C.c_void_p], C.c_int),
    "lim_reduce_stride": ([C.POINTER(LimReduceSpec)], C.c_int64),
    "lim_reduce_state": ([C.c_void_p, C.POINTER(LimReduceSpec), _DP], C.c_int),
    "lim_run_reduced": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.POINTER(LimReduceSpec),
                         _DP], C.c_int),
    "lim_sample_milne": ([C.c_void_p, C.c_double, C.c_double, C.c_int64, _DP, _DP, _DP, _DP, _DP, C.c_int64,
                          C.c_int64], C.c_int),
    "lim_sample_fonll": ([C.c_void_p, _DP, C.c_int64, _DP, C.c_int64, _DP, C.c_int64, C.c_int, C.c_int, C.c_int],
                         C.c_int),
    "lim_batch_create": ([C.c_int, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "lim_batch_destroy": ([C.c_void_p], C.c_int),
    "lim_batch_last_error": ([C.c_void_p], C.c_char_p),
    "lim_batch_add": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, _I64P], C.c_int),
    "lim_batch_set_shape": ([C.c_void_p, C.POINTER(LimBatchShape)], C.c_int),
    "lim_batch_get_shape": ([C.c_void_p, C.POINTER(LimBatchShape)], C.c_int),
    "lim_batch_run": ([C.c_void_p], C.c_int),
    "lim_batch_tune": ([C.c_void_p, C.POINTER(LimBatchShape), _DP], C.c_int),
    "lim_batch_stats": ([C.c_void_p, _DP, _I64P, _I64P], C.c_int),
}


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the engine.  Raises if the in-tree library has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with __graft_entry__.build() "
                          "(there is no CPU fallback for the engine)")
    lib = C.CDLL(str(p))
    for name, (args, res) in _SIGS.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
    if path is None:
        _lib = lib
    return lib


def _dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def julia_layout(a, rows: int) -> np.ndarray:
    """(rows, N) array -> the column-major flat buffer a Julia Matrix would hold."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    if a.shape[0] != rows:
        raise ValueError(f"expected {rows} rows, got array of shape {a.shape}")
    return np.ascontiguousarray(a.T).reshape(-1)


def from_julia_layout(buf: np.ndarray, rows: int, n: int) -> np.ndarray:
    """Flat column-major buffer -> (rows, N) array view."""
    return buf.reshape(n, rows).T


class Engine:
    """One engine context on one CUDA device (lim_create .. lim_destroy)."""

    def __init__(self, device: int = 0, stream: int | None = None, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.ctx = C.c_void_p()
        rc = self.lib.lim_create(int(device), C.c_void_p(stream) if stream else None, C.byref(self.ctx))
        if rc != LIM_OK:
            raise LimError(rc, self.lib.lim_last_error(None).decode())
        self.params = LimParams()
        self.n = 0

    # -- plumbing ------------------------------------------------------------------
    def _check(self, rc: int):
        if rc != LIM_OK:
            raise LimError(rc, self.lib.lim_last_error(self.ctx).decode())

    def close(self):
        if self.ctx:
            self.lib.lim_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration ---------------------------------------------------------------
    def set_params(self, **kw):
        P = LimParams()
        defaults = dict(dt=0.001, t0=0.0, m=1.0, DsT=0.2, Tfo=0.156, psi2=0.0, obs_pt_cut=5.0, obs_pt_width=0.1,
                        dims=3, pdim=0, coords=0, collision=0, relativistic=1, bjorken_redshift=0,
                        position_diffusion=0, reflecting_boundary=0, integrator_mode=0, freezeout_capture=0,
                        freezeout_interp=1, precision=0, seed=0x4C494D00, particle_offset=0,
                        stop_after_freezeout=0, block_size=0)
        unknown = set(kw) - set(defaults)
        if unknown:
            raise TypeError(f"unknown engine parameters: {sorted(unknown)}")
        defaults.update(kw)
        for k, v in defaults.items():
            setattr(P, k, float(v) if isinstance(getattr(P, k), float) else int(v))
        self._check(self.lib.lim_set_params(self.ctx, C.byref(P)))
        self.params = P
        if P.pdim <= 0:
            P.pdim = P.dims
        return P

    def set_medium_rt(self, xgrid, tgrid, T, V, V2=None):
        xg = np.ascontiguousarray(xgrid, dtype=np.float64)
        tg = np.ascontiguousarray(tgrid, dtype=np.float64)
        Tf = np.ascontiguousarray(np.asarray(T, dtype=np.float64).ravel(order="F"))
        Vf = np.ascontiguousarray(np.asarray(V, dtype=np.float64).ravel(order="F"))
        V2f = None if V2 is None else np.ascontiguousarray(np.asarray(V2, dtype=np.float64).ravel(order="F"))
        if Tf.size != xg.size * tg.size or Vf.size != Tf.size or (V2f is not None and V2f.size != Tf.size):
            raise ValueError("T/V/V2 must have shape (len(xgrid), len(tgrid))")
        self._check(self.lib.lim_set_medium_rt(self.ctx, _dptr(xg), xg.size, _dptr(tg), tg.size,
                                               _dptr(Tf), _dptr(Vf), _dptr(V2f)))

    def set_medium_bjorken(self, T0, tau0, power=1.0 / 3.0, r_max=0.0):
        self._check(self.lib.lim_set_medium_bjorken(self.ctx, T0, tau0, power, r_max))

    def set_medium_grid(self, T, ux, uy, x0, dx, y0, dy, tau0, dtau):
        """Fields of shape (nt, ny, nx) (x fastest)."""
        T = np.ascontiguousarray(T, dtype=np.float32)
        ux = np.ascontiguousarray(ux, dtype=np.float32)
        uy = np.ascontiguousarray(uy, dtype=np.float32)
        nt, ny, nx = T.shape
        if ux.shape != T.shape or uy.shape != T.shape:
            raise ValueError("T, ux, uy must share the shape (nt, ny, nx)")
        self._check(self.lib.lim_set_medium_grid(self.ctx, nx, ny, nt, x0, dx, y0, dy, tau0, dtau,
                                                 _fptr(T), _fptr(ux), _fptr(uy)))

    def set_spline(self, which, Tmin, invdT, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        self._check(self.lib.lim_set_spline(self.ctx, int(which), float(Tmin), float(invdT), _dptr(v), v.size))

    def build_time_spline(self, which, kind, m, DsT, *, Tmin, Tmax, nT=1024, DsT_linear=False, DsT_slope=1.765,
                          DsT_offset=-0.159, Tfo=0.156, DsT_quad=False, DsT_Tref=0.0, eta_over_s=0.16,
                          factor=5.0, scale=None):
        """A time spline built on the device (lim_build_time_spline); keywords as
        transport.build_*_spline.  scale defaults to transport.LV_TAUN_SCALE."""
        from . import transport as _tr
        form = LimDsForm(int(bool(DsT_linear)), float(DsT_slope), float(DsT_offset), float(Tfo),
                         int(bool(DsT_quad)), float(DsT_Tref))
        sc = _tr.LV_TAUN_SCALE if scale is None else float(scale)
        self._check(self.lib.lim_build_time_spline(self.ctx, int(which), int(kind), float(m), float(DsT),
                                                   C.byref(form), float(Tmin), float(Tmax), int(nT),
                                                   float(eta_over_s), float(factor), sc))

    def build_juttner_invcdf(self, m, dimensions, *, Tmin, Tmax, nT=256, nU=2048, np_=8192, quantile_cap=1.0e-6):
        self._check(self.lib.lim_build_juttner_invcdf(self.ctx, float(m), int(dimensions), float(Tmin), float(Tmax),
                                                      int(nT), int(nU), int(np_), float(quantile_cap)))

    def get_spline(self, which):
        """(Tmin, invdT, vals) of the installed spline."""
        n = C.c_int64(0)
        t0, inv = C.c_double(0), C.c_double(0)
        self._check(self.lib.lim_get_spline(self.ctx, int(which), C.byref(t0), C.byref(inv), None, 0, C.byref(n)))
        vals = np.zeros(max(n.value, 1))
        self._check(self.lib.lim_get_spline(self.ctx, int(which), None, None, _dptr(vals), vals.size, C.byref(n)))
        return t0.value, inv.value, vals[:n.value]

    def get_invcdf(self):
        """(vals, nU, nT, Tmin, invdT) of the installed inverse-CDF table."""
        nU, nT = C.c_int64(0), C.c_int64(0)
        t0, inv = C.c_double(0), C.c_double(0)
        self._check(self.lib.lim_get_invcdf(self.ctx, None, 0, C.byref(nU), C.byref(nT), C.byref(t0), C.byref(inv)))
        vals = np.zeros(max(nU.value * nT.value, 1))
        self._check(self.lib.lim_get_invcdf(self.ctx, _dptr(vals), vals.size, None, None, None, None))
        return vals[:nU.value * nT.value], nU.value, nT.value, t0.value, inv.value

    def set_invcdf(self, vals, nU, nT, Tmin, invdT):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        self._check(self.lib.lim_set_invcdf(self.ctx, _dptr(v), int(nU), int(nT), float(Tmin), float(invdT)))

    # -- state -----------------------------------------------------------------------
    def upload_state(self, x, p):
        dims, pdim = int(self.params.dims), int(self.params.pdim)
        xb = julia_layout(x, dims)
        pb = julia_layout(p, pdim)
        n = xb.size // dims
        if pb.size != n * pdim:
            raise ValueError("x and p hold different particle counts")
        self._check(self.lib.lim_upload_state(self.ctx, _dptr(xb), dims, _dptr(pb), pdim, n))
        self.n = n

    def upload_state_flat(self, xbuf: np.ndarray, pbuf: np.ndarray, n: int):
        """Upload from flat Julia-layout buffers (e.g. pinned host memory)."""
        self._check(self.lib.lim_upload_state(self.ctx, _dptr(xbuf), int(self.params.dims), _dptr(pbuf),
                                              int(self.params.pdim), int(n)))
        self.n = int(n)

    def sample_fonll(self, r_grid, p_grid, f, n: int, *, cartesian: bool = True, antithetic: bool = False,
                     thermal_pz: bool = False):
        """Sample n initial particles on the device from the density f(r, p) (Julia's
        shape (Np, Nr), as sample_particles_from_FONLL takes it) into the state."""
        rg = np.ascontiguousarray(r_grid, dtype=np.float64)
        pg = np.ascontiguousarray(p_grid, dtype=np.float64)
        fm = np.asarray(f, dtype=np.float64)
        if fm.shape != (pg.size, rg.size) and fm.shape == (rg.size, pg.size):
            fm = fm.T                                   # Nr x Np is transposed, as utils.jl:43-49 does
        if fm.shape != (pg.size, rg.size):
            raise ValueError(f"f must have shape (len(p_grid), len(r_grid)) = {(pg.size, rg.size)}, got {fm.shape}")
        fb = np.ascontiguousarray(fm.T).reshape(-1)
        self._check(self.lib.lim_sample_fonll(self.ctx, _dptr(rg), rg.size, _dptr(pg), pg.size, _dptr(fb), int(n),
                                              int(bool(cartesian)), int(bool(antithetic)), int(bool(thermal_pz))))
        self.n = int(n)

    def sample_milne(self, x_lo: float, x_hi: float, T_c, ur_c, mu_c, r_T, T_r, n: int):
        """Sample n Milne (tau, r) particles on the device (lim_sample_milne): profiles
        at the nbins bin centers of [x_lo, x_hi], T(r) on the table (r_T, T_r)."""
        Tc = np.ascontiguousarray(T_c, dtype=np.float64)
        uc = np.ascontiguousarray(ur_c, dtype=np.float64)
        mc = np.ascontiguousarray(mu_c, dtype=np.float64)
        rT = np.ascontiguousarray(r_T, dtype=np.float64)
        TT = np.ascontiguousarray(T_r, dtype=np.float64)
        if not (Tc.size == uc.size == mc.size) or rT.size != TT.size:
            raise ValueError("the bin profiles and the T(r) table must have matching lengths")
        self._check(self.lib.lim_sample_milne(self.ctx, float(x_lo), float(x_hi), Tc.size, _dptr(Tc), _dptr(uc),
                                              _dptr(mc), _dptr(rT), _dptr(TT), rT.size, int(n)))
        self.n = int(n)

    def download_state(self):
        dims, pdim, n = int(self.params.dims), int(self.params.pdim), self.n
        xb = np.empty(max(n * dims, 1))
        pb = np.empty(max(n * pdim, 1))
        self._check(self.lib.lim_download_state(self.ctx, _dptr(xb), _dptr(pb)))
        return from_julia_layout(xb[:n * dims], dims, n), from_julia_layout(pb[:n * pdim], pdim, n)

    def download_state_flat(self, xbuf: np.ndarray | None, pbuf: np.ndarray | None):
        self._check(self.lib.lim_download_state(self.ctx, _dptr(xbuf), _dptr(pbuf)))

    def state_save(self):
        self._check(self.lib.lim_state_save(self.ctx))

    def state_restore(self):
        self._check(self.lib.lim_state_restore(self.ctx))

    def initial_lab_boost(self):
        self._check(self.lib.lim_initial_lab_boost(self.ctx))

    def run(self, first_step: int, nsteps: int, save_every: int = 0, first_slot: int = 0,
            hist_x: np.ndarray | None = None, hist_p: np.ndarray | None = None):
        self._check(self.lib.lim_run(self.ctx, int(first_step), int(nsteps), int(save_every), int(first_slot),
                                     _dptr(hist_x), _dptr(hist_p)))

    def run_static_T(self, T: float, first_step: int, nsteps: int, save_every: int = 0, first_slot: int = 0,
                     hist_pmag: np.ndarray | None = None):
        """The static-temperature momentum-only path (lim_run_static_T); hist_pmag: a
        (nslots, N) array of |p| snapshots, slot s / save_every - first_slot."""
        nslots = 0 if hist_pmag is None else int(hist_pmag.shape[0])
        if hist_pmag is not None and (hist_pmag.dtype != np.float64 or not hist_pmag.flags.c_contiguous):
            raise ValueError("hist_pmag must be a C-contiguous float64 array of shape (nslots, N)")
        self._check(self.lib.lim_run_static_T(self.ctx, float(T), int(first_step), int(nsteps), int(save_every),
                                              int(first_slot), nslots, _dptr(hist_pmag)))

    def reduce_state(self, spec: LimReduceSpec) -> dict:
        """The current state reduced on the device (lim_reduce_state): one slot."""
        out = np.zeros(max(int(self.lib.lim_reduce_stride(C.byref(spec))), 1))   # an invalid spec fails below
        self._check(self.lib.lim_reduce_state(self.ctx, C.byref(spec), _dptr(out)))
        return {k: v[0] for k, v in split_reduced(out, spec).items()}

    def run_reduced(self, first_step: int, nsteps: int, save_every: int, first_slot: int, nslots: int,
                    spec: LimReduceSpec) -> dict:
        """run() with every snapshot reduced on the device (lim_run_reduced)."""
        out = np.zeros(max(nslots * int(self.lib.lim_reduce_stride(C.byref(spec))), 1))
        self._check(self.lib.lim_run_reduced(self.ctx, int(first_step), int(nsteps), int(save_every),
                                             int(first_slot), int(nslots), C.byref(spec), _dptr(out)))
        return split_reduced(out, spec)

    def status(self) -> int:
        v = C.c_int64(-1)
        self._check(self.lib.lim_status(self.ctx, C.byref(v)))
        return int(v.value)

    def download_freezeout(self):
        dims, pdim, n = int(self.params.dims), int(self.params.pdim), self.n
        fp, fm, ft, ff = np.empty(max(n * dims, 1)), np.empty(max(n * pdim, 1)), np.empty(max(n, 1)), np.empty(max(n, 1))
        self._check(self.lib.lim_download_freezeout(self.ctx, _dptr(fp), _dptr(fm), _dptr(ft), _dptr(ff)))
        return dict(pos=from_julia_layout(fp[:n * dims], dims, n), mom=from_julia_layout(fm[:n * pdim], pdim, n),
                    tau=ft[:n].copy(), flag=ff[:n].copy())

    def download_freezeout_flat(self, fo_pos, fo_mom, fo_tau, fo_flag):
        """Freeze-out outputs into caller buffers in the Julia layout (e.g. page-locked
        host memory): fo_pos (dims, n), fo_mom (pdim, n), fo_tau (n), fo_flag (n)."""
        self._check(self.lib.lim_download_freezeout(self.ctx, _dptr(fo_pos), _dptr(fo_mom), _dptr(fo_tau),
                                                    _dptr(fo_flag)))

    def observables(self, from_freezeout: bool = False) -> dict:
        out = np.zeros(LIM_OBS_NUM)
        self._check(self.lib.lim_observables(self.ctx, int(bool(from_freezeout)), _dptr(out)))
        cnt = out[0]
        res = {"count": cnt}
        for k, name in enumerate(OBS_NAMES[1:], start=1):
            res[name] = out[k] / cnt if cnt > 0 else float("nan")
        res["sums"] = out
        return res

    def record_noise(self, first_step: int, nsteps: int):
        self._check(self.lib.lim_record_noise(self.ctx, int(first_step), int(nsteps)))
        self._rec_steps = int(nsteps)

    def download_noise(self) -> np.ndarray:
        out = np.empty(self._rec_steps * LIM_NOISE_SLOTS * self.n)
        self._check(self.lib.lim_download_noise(self.ctx, _dptr(out)))
        return out.reshape(self._rec_steps, LIM_NOISE_SLOTS, self.n)

    def philox(self, ctr, key):
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        o = (C.c_uint32 * 4)()
        self._check(self.lib.lim_philox_device(self.ctx, c, k, o))
        return list(o)

    def last_run_stats(self):
        ms = C.c_double(0.0)
        nl = C.c_int64(0)
        self._check(self.lib.lim_last_run_stats(self.ctx, C.byref(ms), C.byref(nl)))
        return ms.value, int(nl.value)

    def probe_fma_rate(self):
        """(thread FMA instructions per second, probe ms) of the FP32 FMA issue probe."""
        r = C.c_double(0.0)
        ms = C.c_double(0.0)
        self._check(self.lib.lim_probe_fma_rate(self.ctx, C.byref(r), C.byref(ms)))
        return r.value, ms.value

    def probe_mufu_rate(self):
        """(thread MUFU instructions per second, probe ms) of the XU-pipe probe."""
        r = C.c_double(0.0)
        ms = C.c_double(0.0)
        self._check(self.lib.lim_probe_mufu_rate(self.ctx, C.byref(r), C.byref(ms)))
        return r.value, ms.value

    def device_bytes(self) -> int:
        v = C.c_int64(0)
        self._check(self.lib.lim_device_bytes(self.ctx, C.byref(v)))
        return int(v.value)

    def synchronize(self):
        self._check(self.lib.lim_synchronize(self.ctx))

    # -- pathwise gradients --------------------------------------------------------------
    def set_medium_scale(self, s: float):
        self._check(self.lib.lim_set_medium_scale(self.ctx, float(s)))

    def rta_decisions(self, mode: int, first_step: int = 1, nsteps: int = 1):
        """0 off, 1 record the following runs' RTA decisions, 2 replay them."""
        self._check(self.lib.lim_rta_decisions(self.ctx, int(mode), int(first_step), int(nsteps)))

    def copy_rta_decisions(self, src: "Engine"):
        self._check(self.lib.lim_copy_rta_decisions(self.ctx, src.ctx))

    def adjoint(self, first_step: int, nsteps: int, checkpoint_every: int = 64):
        """Advance like run() and return (obs[3], grad[3, 3]): <pT>, <cos 2phi>, the smoothed
        fraction above obs_pt_cut, and their derivatives w.r.t. (a, b, s)."""
        obs = np.zeros(3)
        grad = np.zeros(9)
        self._check(self.lib.lim_adjoint(self.ctx, int(first_step), int(nsteps), int(checkpoint_every),
                                         _dptr(obs), _dptr(grad)))
        return obs, grad.reshape(3, 3)

    def adjoint_stats(self):
        f = C.c_double(0.0)
        r = C.c_double(0.0)
        self._check(self.lib.lim_adjoint_stats(self.ctx, C.byref(f), C.byref(r)))
        return f.value, r.value


class Batch:
    """Many engine contexts advanced together (lim_batch_*): one persistent launch per
    chunk of steps, the chunk loop replayed as a CUDA graph.  The engines are
    referenced, not copied; keep them open while the batch lives."""

    def __init__(self, device: int = 0, stream: int | None = None, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.h = C.c_void_p()
        rc = self.lib.lim_batch_create(int(device), C.c_void_p(stream) if stream else None, C.byref(self.h))
        if rc != LIM_OK:
            raise LimError(rc, self.lib.lim_batch_last_error(None).decode())
        self.engines = []

    def _check(self, rc: int):
        if rc != LIM_OK:
            raise LimError(rc, self.lib.lim_batch_last_error(self.h).decode())

    def close(self):
        if self.h:
            self.lib.lim_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, engine: Engine, first_step: int, nsteps: int) -> int:
        idx = C.c_int64(-1)
        self._check(self.lib.lim_batch_add(self.h, engine.ctx, int(first_step), int(nsteps), C.byref(idx)))
        self.engines.append(engine)
        return int(idx.value)

    def set_shape(self, block=0, chunk_steps=0, blocks_per_sm=0, reg_cap=0):
        sh = LimBatchShape(int(block), int(chunk_steps), int(blocks_per_sm), int(reg_cap))
        self._check(self.lib.lim_batch_set_shape(self.h, C.byref(sh)))

    def shape(self) -> dict:
        sh = LimBatchShape()
        self._check(self.lib.lim_batch_get_shape(self.h, C.byref(sh)))
        return sh.as_dict()

    def run(self):
        self._check(self.lib.lim_batch_run(self.h))

    def tune(self):
        """Autotune the launch shape on this batch; returns (shape dict, best ms)."""
        sh = LimBatchShape()
        ms = C.c_double(0.0)
        self._check(self.lib.lim_batch_tune(self.h, C.byref(sh), C.byref(ms)))
        return sh.as_dict(), ms.value

    def stats(self):
        ms = C.c_double(0.0)
        nl = C.c_int64(0)
        ps = C.c_int64(0)
        self._check(self.lib.lim_batch_stats(self.h, C.byref(ms), C.byref(nl), C.byref(ps)))
        return ms.value, int(nl.value), int(ps.value)

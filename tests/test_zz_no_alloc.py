"""lim_observables_noalloc: the observables entry point for hosts that cannot
allocate device memory themselves (their memory comes from their own pool, or the
call runs where allocation is not allowed).  It must give the same sums as the
context path (lim_observables) on the same ensemble, call after call, although
every call reuses the library's one fixed scratch array.

Collected last on purpose: a run that stops at the first failure has already run
every other test.  Device buffers here come from torch, as they would from the
host's own allocator."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def context_sums(capi, x, p, m, cut, width):
    """Sums of the existing entry point on an engine context holding the same state."""
    eng = capi.Engine(0)
    dims, pdim = x.shape[0], p.shape[0]
    eng.set_params(dims=dims, pdim=pdim, m=m, DsT=0.0, obs_pt_cut=cut, obs_pt_width=width, precision=0)
    eng.set_medium_rt([0.0, 1.0], [0.0, 1.0], np.full((2, 2), 0.3), np.zeros((2, 2)))
    eng.upload_state(x, p)
    sums = eng.observables()["sums"].copy()
    eng.close()
    return sums


def noalloc_sums(capi, x, p, m, cut, width):
    """x = None: no positions (x_dev = NULL, dims = 0)."""
    lib = capi.load_library()
    pdim, n = p.shape[0], p.shape[1]
    dims = 0 if x is None else x.shape[0]
    xd = None if x is None else torch.from_numpy(capi.julia_layout(x, dims).copy()).cuda()
    pd = torch.from_numpy(capi.julia_layout(p, pdim).copy()).cuda()
    out = torch.full((capi.LIM_OBS_NUM,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.lim_observables_noalloc(0, C.c_void_p(pd.data_ptr()), pdim,
                                     None if xd is None else C.c_void_p(xd.data_ptr()), dims, n,
                                     m, cut, width, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == capi.LIM_OK, lib.lim_last_error(None)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_context_path_on_two_calls(lmb):
    capi = lmb.capi
    rng = np.random.default_rng(2026)
    m, cut, width = 1.5, 2.0, 0.25
    # first call: a large ensemble (many scratch rows); second: a small one, so stale
    # rows of the first call would show up if the entry point read them
    for n, pdim in ((700_001, 3), (5_003, 2)):
        p = rng.normal(0.0, 1.7, (pdim, n))
        x = rng.normal(0.0, 3.0, (2, n))
        ref = context_sums(capi, x, p, m, cut, width)
        got = noalloc_sums(capi, x, p, m, cut, width)
        assert got[0] == n == ref[0]
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-9)


def test_noalloc_rejects_sizes_beyond_the_scratch_limit(lmb):
    capi = lmb.capi
    lib = capi.load_library()
    out = torch.zeros(capi.LIM_OBS_NUM, dtype=torch.float64, device="cuda")
    rc = lib.lim_observables_noalloc(0, C.c_void_p(out.data_ptr()), 3, None, 0, 16_777_217, 1.5, 5.0, 0.1,
                                     C.c_void_p(out.data_ptr()), None)
    assert rc == capi.LIM_ERR_ARG
    assert b"exceeds the fixed scratch limit" in lib.lim_last_error(None)
    rc = lib.lim_observables_noalloc(0, C.c_void_p(out.data_ptr()), 4, None, 0, 10, 1.5, 5.0, 0.1,
                                     C.c_void_p(out.data_ptr()), None)
    assert rc == capi.LIM_ERR_ARG


def test_noalloc_without_positions_and_with_zero_width(lmb):
    """x_dev = NULL (dims 0) leaves the |x|^2 sum at zero and the momentum sums as the
    context path gives them; pt_width <= 0 stands for 1e-3 in both entry points."""
    capi = lmb.capi
    rng = np.random.default_rng(7)
    n, m, cut = 40_000, 4.75, 1.0
    p = rng.normal(0.0, 1.2, (3, n))
    x = rng.normal(0.0, 2.0, (2, n))
    ref = context_sums(capi, x, p, m, cut, 0.2)
    got = noalloc_sums(capi, None, p, m, cut, 0.2)
    assert got[11] == 0.0
    np.testing.assert_allclose(got[:11], ref[:11], rtol=1e-12, atol=1e-9)
    ref0 = context_sums(capi, x, p, m, cut, 0.0)
    got0 = noalloc_sums(capi, x, p, m, cut, 0.0)
    np.testing.assert_allclose(got0, ref0, rtol=1e-12, atol=1e-9)


def test_noalloc_empty_ensemble_gives_zeros(lmb):
    capi = lmb.capi
    got = noalloc_sums(capi, None, np.zeros((3, 0)), 1.5, 5.0, 0.1)
    assert np.array_equal(got, np.zeros(capi.LIM_OBS_NUM))

"""CPU-side checks of the C-ABI boundary: the library loads and exports every
symbol the public header declares, the ctypes struct matches the C layout, and
calls that need a GPU fail with a status (no crash) when none is present."""
import ctypes as C
import re

import numpy as np
import pytest
import torch


def declared_functions(header_text: str):
    body = re.sub(r"/\*.*?\*/", "", header_text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(lim_\w+)\s*\(", body, flags=re.M)))


def test_header_symbols_exported(lmb):
    lib = lmb.capi.load_library()
    names = declared_functions(lmb.capi.HEADER.read_text()) + declared_functions(lmb.capi.DIAG_HEADER.read_text())
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert not [n for n in names if n not in lmb.capi._SIGS]


def test_params_struct_layout(lmb):
    P = lmb.capi.LimParams
    assert C.sizeof(P) == 8 * 24
    assert [f[0] for f in P._fields_][:3] == ["dt", "t0", "m"]


def test_abi_version(lmb):
    assert lmb.capi.load_library().lim_abi_version() == 1


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_cleanly(lmb):
    with pytest.raises(lmb.capi.LimError):
        lmb.capi.Engine(0)
    assert lmb.capi.load_library().lim_last_error(None)


def test_oracle_header_and_product_params_agree(lmb, orc):
    """The oracle's parameter block starts with the C-ABI's layout (tests pass one to the
    other); its only addition is the checker's RTA-replay switch at the end."""
    a = [f[0] for f in lmb.capi.LimParams._fields_]
    b = [f[0] for f in orc.OrcParams._fields_]
    assert b[:len(a)] == a and b[len(a):] == ["rta_replay"]


def test_reduce_stride_on_host(lmb):
    """lim_reduce_stride is host arithmetic: the per-slot layout of lim_run_reduced."""
    capi = lmb.capi
    L = capi.load_library()
    spec = capi.reduce_spec(64, 16.0, 50, 5.0)
    assert L.lim_reduce_stride(C.byref(spec)) == capi.LIM_OBS_NUM + 65 + 2 * 51
    assert L.lim_reduce_stride(C.byref(capi.reduce_spec(0, 16.0, 50, 5.0))) == -1
    out = np.arange(2 * (capi.LIM_OBS_NUM + 65 + 102), dtype=np.float64)
    parts = capi.split_reduced(out, spec)
    assert parts["obs"].shape == (2, capi.LIM_OBS_NUM) and parts["pt_cos2"].shape == (2, 51)

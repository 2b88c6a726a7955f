"""B200-native heavy-quark Langevin engine with LangevInMedium.jl's simulate interface.

The per-particle Langevin time loop runs in hand-written CUDA (sm_100a) behind the
C-ABI of include/langevin_b200.h; this package is the host side: backend markers,
``simulate_ensemble_bulk``, the transport-table precompute and the hydro loaders.
"""
from .backends import AbstractBackend, B200Backend, B200_GCBackend
from .simulate import FreezeOut, simulate_ensemble_bulk
from .hydro import HydroRT, HydroXY
from .transport import (GevInvTofm, fmGeV, build_juttner_invcdf, build_tau_drag_spline, build_tau_R_spline,
                        build_taun_current_spline, effective_DsT, eval_tau_n_spline, tau_drag, tau_n_main3)
from .utils import append_thermal_pz, check_momentum_dims, sample_pz_conditional_juttner
from .pipeline import EnsembleStream
from . import capi, hydro, pipeline, sharding, transport, utils, workloads

__all__ = ["AbstractBackend", "B200Backend", "B200_GCBackend", "FreezeOut", "simulate_ensemble_bulk",
           "GevInvTofm", "fmGeV", "build_juttner_invcdf", "build_tau_drag_spline", "build_tau_R_spline",
           "build_taun_current_spline", "effective_DsT", "eval_tau_n_spline", "tau_drag", "tau_n_main3",
           "append_thermal_pz", "check_momentum_dims", "sample_pz_conditional_juttner", "capi", "HydroRT",
           "HydroXY", "EnsembleStream"]

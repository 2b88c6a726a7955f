"""The static work model behind the roofline fractions (langevinmedium.jl_b200/
work_model.json): every count is a non-negative number of a known instruction class,
and the per-particle-step totals are the ones the measurement notes quote (the
Bjorken Langevin+RTA step 248.5, the 2+1D grid step with the freeze-out latch 328.5),
so a change to the counts shows up here before it moves a reported fraction."""
import json
from pathlib import Path

import pytest

MODEL = Path(__file__).resolve().parents[1] / "langevinmedium.jl_b200" / "work_model.json"
CLASSES = {"fp32", "fp64", "int", "mufu", "conv", "mem", "control"}


def totals(workload):
    tot = {}
    for item in workload["items"].values():
        for k, c in item.items():
            tot[k] = tot.get(k, 0.0) + c
    return tot


@pytest.fixture(scope="module")
def model():
    return json.loads(MODEL.read_text())


def test_counts_are_known_classes(model):
    for name, w in model["workloads"].items():
        for item, counts in w["items"].items():
            assert set(counts) <= CLASSES, (name, item, counts)
            assert all(isinstance(c, (int, float)) and c >= 0 for c in counts.values()), (name, item)
        assert w["hbm_bytes_per_particle_per_launch"] > 0


@pytest.mark.parametrize("name,total,xu", [("bjorken_langevin_rta_fp32", 248.5, 34.0),
                                           ("grid2p1_langevin_rta_fo_fp32", 328.5, 48.0)])
def test_totals(model, name, total, xu):
    tot = totals(model["workloads"][name])
    assert sum(tot.values()) == pytest.approx(total)
    assert tot.get("mufu", 0) + tot.get("conv", 0) == pytest.approx(xu)   # the XU share of the per-pipe bound

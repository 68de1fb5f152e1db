"""Precision study: the FP32 GPU path against an FP64 build of the same
scheme on the same inputs, short runs.

A moist supercell state (cold rain) and a squall-line state (open x) run N
large steps on the GPU (FP32, FP64 vertical solve), in the oracle's FP32
build and in its FP64 build (tests/precision.py).  For every prognostic
field the GPU's RMS difference from FP64 (relative to the field's RMS) must
be within 3 times the FP32 oracle's own spread plus a floor of 1e-6 for
fields that stay near zero, and its water and mass budgets must agree with
the FP64 run's to 1e-4.  Run with -s to see the table (one JSON line).
The same comparison at the configurations' full run lengths is in
test_named_configs_gpu.py.
"""
import json

import pytest

import precision as P

pytestmark = pytest.mark.gpu

K, FLOOR = 3.0, 1e-6


def _check(rep):
    print(json.dumps({"precision": rep}))
    bad = [(n, f["gpu_rms_rel"], f["fp32_rms_rel"]) for n, f in rep["fields"].items()
           if not f["finite"] or f["gpu_rms_rel"] > K * f["fp32_rms_rel"] + FLOOR]
    assert not bad, bad
    assert abs(rep["water_drift_gpu"] - rep["water_drift_fp64"]) < 1e-4
    assert abs(rep["mass_drift_gpu"] - rep["mass_drift_fp64"]) < 1e-4


def test_fp32_gpu_against_fp64(cress, oracle_lib):
    from cress_b200 import cases
    nx, ny, nz, dx = 40, 40, 30, 1000.0
    case = cases.supercell_case(nx, ny, nz, dx, ztop=10000.0, seed=12, cloud=True,
                                rad=(6000.0, 6000.0, 1400.0))
    _check(P.moist_study(cress, oracle_lib, case, dx, 24, 5.0, 1.0))


def test_fp32_gpu_against_fp64_squall_open_x(cress, oracle_lib):
    """The squall-line configuration (line thermal +2 K with seeded 0.1 K
    noise, 20 m/s low-level shear, dx = 500 m, open radiation x boundaries
    with per-point phase speeds, periodic y) on a reduced grid.  With open
    boundaries water and mass leave and enter the domain, so the drifts are
    compared between the GPU and the FP64 build, not against zero."""
    from cress_b200 import cases
    nx, ny, nz, dx = 64, 24, 36, 500.0
    case = cases.squall_case(nx, ny, nz, dx, ztop=12000.0, seed=7, xrad=4000.0)
    _check(P.moist_study(cress, oracle_lib, case, dx, 30, 3.0, 0.5, obc=4, label="squall line, open x"))

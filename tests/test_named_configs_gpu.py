"""Parity at the named configurations and their run lengths: the FP32 GPU
path against the oracle's FP64 and FP32 builds, field by field.

* Dry warm bubble exactly as configured: 64x64x40, dx = dy = 500 m,
  uniform dz = 300 m, flat, periodic sides, rigid lid with a Rayleigh
  sponge above 9 km; neutral theta = 300 K, 1000 hPa, no wind or moisture;
  +2 K cos^2 bubble of radius 2 km centred at z = 1.5 km plus seeded
  +-0.01 K noise; dtbig = 2 s with nsstp = 16 acoustic substeps
  (dtsml = 0.25 s); Smagorinsky turbulence; 150 large steps = 300 s.
* Moist supercell (cold rain) for 2 h of model time: 1440 steps of 5 s
  with 10 substeps, on a reduced grid (40x40x40, dx = 1 km, stretched
  100 -> 500 m to 12 km) where the FP64 oracle is affordable.
* Squall line (line thermal, 20 m/s low-level shear, open radiation x
  boundaries with the constant phase speed gwave, wbc = ebc = 7, periodic
  y) for 1 h: 1200 steps of 3 s with 12 substeps on a reduced grid
  (128x16x36, dx = 500 m; the frame moves at 16 m/s, umove, so the line
  stays inside the 64 km domain while its convection peaks at ~30 m/s).

The reference's shipped configurations run the 1.5-order TKE closure
(tubopt=2); C1 and C2 are also run with it, from zero TKE, with the TKE
among the checked fields.

Per-field tolerance (stated here, checked on every field): the GPU's RMS
difference from the FP64 build, relative to the field's FP64 RMS, must be
within K times the FP32 oracle's own spread from FP64 plus a floor:
    gpu_rms_rel <= K * spread + FLOOR
with K = 3 for the dry bubble (a smooth flow: both FP32 builds round
differently but neither diverges) and K = 4 for the moist runs (moist
convection amplifies round-off over hours, so two FP32 builds drift apart
by amounts of the order of their distance from FP64), FLOOR = 1e-6
(fields that stay near zero).  For the dry bubble the spread is the FP32
oracle's distance from FP64; for the moist runs it is the larger of that
and the distance of a second FP32 oracle run, started from theta' one ulp
up: after hours of convection one FP32 run is a single sample of the
chaotic growth of round-off, and in the C2 supercell the ice number of
one FP32 run stayed at 0.19 of its RMS from FP64 while the run one ulp
away reached 0.70 (the two FP32 runs 0.79 apart).  Budgets: the total-water and mass drifts
over the run (relative to the initial totals) must match the FP64 build's
within 3 times the FP32 build's own drift difference plus 1e-5, and the
accumulated surface precipitation within 5% of the FP64 build's.  Each
test prints its table as one JSON line (run with -s).
"""
import json

import numpy as np
import pytest

import precision as P

pytestmark = pytest.mark.gpu


def _check_budgets(rep, keys=("water", "mass")):
    for b in keys:
        spread = abs(rep[f"{b}_drift_fp32"] - rep[f"{b}_drift_fp64"])
        assert abs(rep[f"{b}_drift_gpu"] - rep[f"{b}_drift_fp64"]) <= 3.0 * spread + 1e-5, (b, rep)


def _check_fields(rep, k, floor=1e-6):
    bad = []
    for n, f in rep["fields"].items():
        assert f["finite"], n
        spread = max(f["fp32_rms_rel"], f.get("fp32p_rms_rel", 0.0))
        if f["gpu_rms_rel"] > k * spread + floor:
            bad.append((n, f["gpu_rms_rel"], f["fp32_rms_rel"], f.get("fp32p_rms_rel")))
    assert not bad, bad


def test_c1_dry_warm_bubble_300s(cress, oracle_lib):
    from cress_b200 import cases
    dx, dz = 500.0, 300.0
    case = cases.dry_case(64, 64, 40, dx, dz, sthopt=0, seed=11, ptp0=2.0, rad=(2000.0, 2000.0, 2000.0),
                          u0=0.0, shear=0.0, vspbar=0.005, botbar=9000.0, noise=0.01, dthdz=0.0)
    rep = P.dry_study(cress, oracle_lib, case, dx, dz, 150, 2.0, 0.25, tubopt=1, sthopt=0,
                      label="dry warm bubble 64x64x40, 300 s")
    print(json.dumps({"named_config": rep}))
    assert rep["nsstp"] == 16
    _check_fields(rep, 3.0)
    _check_budgets(rep, ("mass",))


def test_c1_dry_warm_bubble_300s_tke(cress, oracle_lib):
    from cress_b200 import cases
    dx, dz = 500.0, 300.0
    case = cases.dry_case(64, 64, 40, dx, dz, sthopt=0, seed=11, ptp0=2.0, rad=(2000.0, 2000.0, 2000.0),
                          u0=0.0, shear=0.0, vspbar=0.005, botbar=9000.0, noise=0.01, dthdz=0.0)
    rep = P.dry_study(cress, oracle_lib, case, dx, dz, 150, 2.0, 0.25, tubopt=2, sthopt=0,
                      label="dry warm bubble 64x64x40, 300 s, TKE closure")
    print(json.dumps({"named_config": rep}))
    assert rep["fields"]["tke"]["fp64_rms"] > 0.0   # the closure is active
    _check_fields(rep, 3.0)
    _check_budgets(rep, ("mass",))


def test_c2_supercell_2h_tke(cress, oracle_lib):
    from cress_b200 import cases
    dx = 1000.0
    case = cases.supercell_case(40, 40, 40, dx, ztop=12000.0, seed=12, cloud=True,
                                rad=(6000.0, 6000.0, 1400.0))
    rep = P.moist_study(cress, oracle_lib, case, dx, 1440, 5.0, 1.0, tubopt=2,
                        label="supercell 40x40x40, 2 h, TKE closure")
    print(json.dumps({"named_config": rep}))
    assert rep["fields"]["tke"]["fp64_rms"] > 0.0
    _check_fields(rep, 4.0)
    assert rep["precip_rel_diff_gpu"] < 0.05
    _check_budgets(rep)


def test_c2_supercell_2h(cress, oracle_lib):
    from cress_b200 import cases
    dx = 1000.0
    case = cases.supercell_case(40, 40, 40, dx, ztop=12000.0, seed=12, cloud=True,
                                rad=(6000.0, 6000.0, 1400.0))
    rep = P.moist_study(cress, oracle_lib, case, dx, 1440, 5.0, 1.0, label="supercell 40x40x40, 2 h")
    print(json.dumps({"named_config": rep}))
    _check_fields(rep, 4.0)
    assert rep["precip_rel_diff_gpu"] < 0.05
    _check_budgets(rep)


def test_c3_squall_line_1h(cress, oracle_lib):
    from cress_b200 import cases
    dx = 500.0
    case = cases.squall_case(128, 16, 36, dx, ztop=12000.0, seed=7, xrad=4000.0, umove=16.0)
    rep = P.moist_study(cress, oracle_lib, case, dx, 1200, 3.0, 0.5, obc=7,
                        label="squall line 128x16x36, open x (wbc=ebc=7), 1 h")
    print(json.dumps({"named_config": rep}))
    assert rep["max_w_gpu"] > 5.0          # the line is convecting
    _check_fields(rep, 4.0)
    assert rep["precip_rel_diff_gpu"] < 0.05
    _check_budgets(rep)

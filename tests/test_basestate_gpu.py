"""The base state from a sounding, computed on the GPU in FP64
(cress_base_state), against the oracle's FP64 restatement of set1d,
vextlow, intrpsnd, setbase/bcbase, baserho and sndwave.

Both compute in double; the device's exp/log and the host's differ in the
last place, so every column must agree to 1e-12 relative (1e-9 absolute
for the winds).  The oracle's FP32 build (the reference's own precision)
is reported next to it.
"""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def supercell_sounding(n=121):
    """The analytic supercell sounding on n levels to 20 km: theta 300 K at
    the ground to 343 K at 12 km (z^1.25), isothermal 213 K above; relative
    humidity 100 - 75 (z/12 km)^1.25 percent (25 above); quarter-circle
    hodograph to 7 m/s over 2 km, then u to 30 m/s at 6 km."""
    z = np.linspace(0.0, 20000.0, n)
    th = np.where(z <= 12000.0, 300.0 + 43.0 * (z / 12000.0) ** 1.25,
                  343.0 * np.exp(9.8 * (z - 12000.0) / (1004.0 * 213.0)))
    rh = 100.0 * np.where(z <= 12000.0, 1.0 - 0.75 * (z / 12000.0) ** 1.25, 0.25)
    a = 0.5 * np.pi * np.clip(z / 2000.0, 0.0, 1.0)
    u = np.where(z < 2000.0, 7.0 * (1.0 - np.cos(a)), 7.0 + 23.0 * np.clip((z - 2000.0) / 4000.0, 0.0, 1.0))
    v = 7.0 * np.sin(a)
    return z, u, v, th, rh


def compare(cress, oracle_lib, nk, zph, jcb, snd, tvar, hvar, psnd0):
    z, u, v, pt, q = snd
    got = cress.base_state(nk, zph, jcb, z, u, v, pt, q, psnd0, tvar=tvar, hvar=hvar)
    r64 = oracle_lib.base_state(nk, zph, jcb, z, u, v, pt, q, psnd0, tvar=tvar, hvar=hvar, prec=64)
    r32 = oracle_lib.base_state(nk, zph, jcb, z, u, v, pt, q, psnd0, tvar=tvar, hvar=hvar, prec=32)
    rep = {}
    for name in cress.BASE_COLUMNS:
        g, r = got[name][1:], r64[name][1:]
        assert np.isfinite(g).all(), name
        scale = float(np.abs(r).max()) + 1e-300
        err = float(np.abs(g - r).max())
        rep[name] = {"gpu_fp64_vs_oracle_fp64": err / scale,
                     "oracle_fp32_vs_fp64": float(np.abs(r32[name][1:] - r).max()) / scale}
        tol = 1e-9 if name in ("ubr", "vbr") else 1e-12 * scale
        assert err <= tol, (name, err, scale)
    print(json.dumps({"base_state": rep}))
    return got


def test_supercell_sounding_stretched_grid(cress, oracle_lib):
    from cress_b200 import cases
    nk = 67
    c = cases.moist_columns(nk)
    got = compare(cress, oracle_lib, nk, c["zph"], c["jcb"].astype(np.float64), supercell_sounding(), "p", "r", 1.0e5)
    # hydrostatic: the Exner function falls with height, the air is lighter aloft
    assert np.all(np.diff(got["pibr"][1:nk]) < 0) and np.all(np.diff(got["rbr"][1:nk]) < 0)
    assert got["qvbr"][2] > got["qvbr"][20] > 0.0


def test_temperature_sounding_uniform_grid(cress, oracle_lib):
    nk, dz = 43, 300.0
    zph = np.zeros(nk + 1)
    for k in range(3, nk + 1):
        zph[k] = zph[k - 1] + dz
    zph[1] = -zph[3]
    jcb = np.ones(nk + 1)
    z = np.linspace(0.0, 15000.0, 61)
    t = np.maximum(300.0 - 0.0065 * z, 216.65)
    qv = 0.012 * np.exp(-z / 2500.0)
    compare(cress, oracle_lib, nk, zph, jcb, (z, 0.0 * z + 5.0, 0.0 * z, t, qv), "t", "q", 1.0e5)


def test_rejects_decreasing_heights(cress):
    nk = 20
    zph = np.arange(nk + 1, dtype=np.float64) * 100.0
    z = np.array([0.0, 500.0, 400.0, 1000.0])
    with pytest.raises(cress.CressError) as e:
        cress.base_state(nk, zph, np.ones(nk + 1), z, z * 0, z * 0, z * 0 + 300.0, z * 0 + 50.0, 1e5)
    assert e.value.code == 1

"""Domain diagnostics and the HE-VI autotuner on the GPU.

cress_diagnostics sums the water, precipitated water and mass budgets of a
time level in FP64 on the device; the same sums formed here in float64
from the host copies of the fields must agree to round-off (the order of
summation differs), the maxima exactly, and a planted NaN must be counted
and reported as CRESS_E_NONFINITE.  cress_autotune must pick a usable tile
shape without touching the state the next large step starts from.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def moist_solver(cress, oracle_lib, seed=4):
    from cress_b200 import cases
    dx = 1000.0
    case = cases.supercell_case(36, 30, 22, dx, ztop=8000.0, seed=seed, cloud=True,
                                rad=(6000.0, 6000.0, 1400.0))
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    s = cress.Solver(ni, nj, nk, dx, dx, case["dz"], sthopt=1, cphopt=3)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]
    for n, a in zip(NAMES, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    return s, case


def host_sums(s, case, cress, level):
    ni, nj, nk = case["dims"]
    dx, dz = 1000.0, float(np.float32(case["dz"]))   # the context holds dz as float
    sl = (slice(1, nk - 2), slice(2, nj - 1), slice(2, ni - 1))   # k = 2..nk-2, j, i interior
    rst = case["base"]["rst"].astype(np.float64)[sl]
    rcsq = case["base"]["rcsq"].astype(np.float64)[sl]
    f = {n: s.get_field(n, level).astype(np.float64) for n in NAMES}
    q = sum(f[n][sl] for n in ("qv", "qc", "qr", "qi", "qs", "qg"))
    water = float(np.sum(rst * q)) * dx * dx * dz
    mass = float(np.sum(rst * (1.0 + f["pp"][sl] / rcsq))) * dx * dx * dz
    pr = s.get_precip().astype(np.float64)
    precip = float(np.sum(pr[:, 1, 2:nj - 1, 2:ni - 1])) * 1.e3 * dx * dx
    mx = {n: float(np.abs(f[n][sl]).max()) for n in ("u", "v", "w", "ptp")}
    return water, precip, mass, mx


def test_diagnostics_match_host_sums(cress, oracle_lib):
    s, case = moist_solver(cress, oracle_lib)
    nsstp = 10
    s.large_step(0, 2.5, nsstp, 0.5)
    s.large_step(5000, 5.0, nsstp, 1.0)
    for level in (cress.PAST, cress.NOW):
        d = s.diagnostics(level)
        water, precip, mass, mx = host_sums(s, case, cress, level)
        assert d["nonfinite"] == 0
        assert d["water"] == pytest.approx(water, rel=1e-9)
        assert d["precip"] == pytest.approx(precip, rel=1e-9, abs=1e-6)
        assert d["mass"] == pytest.approx(mass, rel=1e-9)
        assert d["max_u"] == mx["u"] and d["max_v"] == mx["v"]
        assert d["max_w"] == mx["w"] and d["max_ptp"] == mx["ptp"]
    # the budget moves by round-off, clipping and advection error only
    d0 = s.diagnostics(cress.PAST)
    d1 = s.diagnostics(cress.NOW)
    drift = abs((d1["water"] + d1["precip"]) - (d0["water"] + d0["precip"])) / d0["water"]
    assert drift < 5e-2, drift
    s.close()


def test_nonfinite_value_is_reported(cress, oracle_lib):
    s, case = moist_solver(cress, oracle_lib, seed=6)
    ni, nj, nk = case["dims"]
    qc = s.get_field("qc", cress.NOW)
    qc[nk // 2, nj // 2, ni // 2] = np.nan
    s.put_field("qc", cress.NOW, qc)
    d = s.diagnostics(cress.NOW, check=False)
    assert d["nonfinite"] == 1
    with pytest.raises(cress.CressError) as e:
        s.diagnostics(cress.NOW)
    assert e.value.code == 5   # CRESS_E_NONFINITE
    assert s.diagnostics(cress.PAST)["nonfinite"] == 0
    s.close()


def test_autotune_keeps_state(cress, oracle_lib):
    s, case = moist_solver(cress, oracle_lib, seed=9)
    s.large_step(0, 2.5, 10, 0.5)
    before = [s.get_field(n, lvl) for n in NAMES for lvl in (cress.PAST, cress.NOW)]
    best, ms = s.autotune(nsstp=4, dts=1.0, reps=2)
    assert 0 <= best < cress.NTILES
    assert ms[best] > 0 and all(m == -1 or m >= ms[best] for m in ms)
    after = [s.get_field(n, lvl) for n in NAMES for lvl in (cress.PAST, cress.NOW)]
    for a, b in zip(before, after):
        assert np.array_equal(a, b, equal_nan=True)
    s.large_step(5000, 5.0, 10, 1.0)   # runs with the chosen tile
    assert s.diagnostics(cress.NOW)["nonfinite"] == 0
    s.close()

"""Checks of the GPU cold-rain microphysics that do not go through the
oracle: cases whose outcome follows from the scheme's definition by hand,
and the water budget of coldblk + fallblk.

The oracle (oracle/micro.h) and the device code restate the same reference
routines, so agreement between them cannot expose a slip made in both.
These tests derive the expected result from the process definitions and
the physical constants alone (SrcOrig/comphy.f90), on the GPU path:

* no hydrometeors in subsaturated air: s_cloudphy and s_satadjst leave
  every field unchanged, bit for bit, and no precipitation falls;
* homogeneous freezing (T <= tlow = 233.16 K, s_nuc1stc nuhci = qc): all
  cloud water becomes cloud ice in one step and theta' rises by
  qc lf / (cp pi), lf = lf0 + (cw - ci)(T - t0);
* melting of cloud ice above t0 (s_melting mlic = qi): all cloud ice
  becomes cloud water and theta' falls by qi lf / (cp pi);
* pure-vapour supersaturation (s_swadjst): the adjusted state keeps
  qv + qc and sits on the saturation curve (Tetens over water, setblk.f90)
  with the latent heat released in theta', compared with an FP64 solution
  of that balance found by bisection;
* per-column water budget of s_cloudphy on a state with every process
  active and no water near the surface or the top: the column's total
  water (vapour and the five hydrometeors, weighted by rho J dz) does not
  change beyond FP32 round-off, and no precipitation falls.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MICRO = ["ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]
# SrcOrig/comphy.f90
CP, RD, P0 = 1004.0, 287.0, 1.0e5
LV0, LF0, CW, CI, T0, TLOW = 2.50078e6, 3.34e5, 4.218e3, 2.106e3, 273.16, 233.16
ES0, EPSVA = 610.78, 0.622


def _setup(cress, nx=12, ny=10, nz=12, dz=300.0):
    from cress_b200 import cases
    dims, base, past, fut, cols = cases.micro_case(nx, ny, nz, dz, seed=9)
    ni, nj, nk = dims
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, dz, sthopt=1, cphopt=3)
    s.set_base3d(base)
    s.set_base_moist(base["pbr"], base["qvbr"])
    pp = np.zeros((nk, nj + 2, ni + 2), np.float32)
    pi = ((base["pbr"].astype(np.float64) + pp) / P0) ** (RD / CP)
    return s, dims, base, pp, pi


def _uniform_state(dims, base, pi, temp, qv_of_t=None, **q):
    """theta' giving temperature `temp` everywhere, the named mixing ratios
    and numbers (constants), everything else zero."""
    ni, nj, nk = dims
    shp = (nk, nj + 2, ni + 2)
    st = {k: np.zeros(shp, np.float32) for k in MICRO}
    st["ptp"] = (temp / pi - base["ptbr"].astype(np.float64)).astype(np.float32)
    for k, v in q.items():
        st[k][:] = v
    if qv_of_t is not None:
        st["qv"] = qv_of_t.astype(np.float32)
    return st


def _put(s, cress, st, pp, levels):
    for lvl in levels:
        for k in MICRO:
            s.put_field(k, lvl, st[k])
        s.put_field("pp", lvl, pp)


def _qvs_w(t, p):
    esw = ES0 * np.exp(17.269 * (t - T0) / (t - 35.86))
    return EPSVA * esw / (p - esw)


def _qvs_i(t, p):
    esi = ES0 * np.exp(21.875 * (t - T0) / (t - 7.66))
    return EPSVA * esi / (p - esi)


def _lv(t):
    return LV0 * (T0 / t) ** (0.167 + 3.67e-4 * t)


def _sl(dims):
    ni, nj, nk = dims
    return (slice(2, nk - 3), slice(2, nj - 1), slice(2, ni - 1))   # levels 3..nk-3, interior columns


def test_no_hydrometeors_is_identity(cress):
    s, dims, base, pp, pi = _setup(cress)
    p = base["pbr"].astype(np.float64)
    t = 265.0
    st = _uniform_state(dims, base, pi, t, qv_of_t=0.5 * np.minimum(_qvs_w(t, p), _qvs_i(t, p)))
    _put(s, cress, st, pp, (cress.PAST, cress.FUTURE, cress.NOW))
    s.put_precip(np.zeros((5, 2, dims[1] + 2, dims[0] + 2), np.float32))
    s.cloudphy(5.0)
    s.satadjst(cress.NOW)
    for k in MICRO:
        assert np.array_equal(s.get_field(k, cress.FUTURE), st[k]), k
        assert np.array_equal(s.get_field(k, cress.NOW), st[k]), k
    assert not s.get_precip().any()
    s.close()


def test_homogeneous_freezing_below_tlow(cress):
    s, dims, base, pp, pi = _setup(cress)
    t, qc0 = 228.0, 1.0e-4
    st = _uniform_state(dims, base, pi, t, qc=qc0)
    _put(s, cress, st, pp, (cress.PAST, cress.FUTURE))
    s.cloudphy(1.0)
    out = {k: s.get_field(k, cress.FUTURE) for k in MICRO}
    s.close()
    sl = _sl(dims)
    assert np.all(out["qc"][sl] == 0.0)
    assert np.allclose(out["qi"][sl], qc0, rtol=1e-4, atol=0)       # slow ice fall: 1e-4 m/s
    tpast = (base["ptbr"].astype(np.float64) + st["ptp"]) * pi
    dth = qc0 * (LF0 + (CW - CI) * (tpast - T0)) / (CP * pi)
    got = out["ptp"].astype(np.float64) - st["ptp"]
    assert np.allclose(got[sl], dth[sl], rtol=2e-3, atol=0)
    assert np.all(out["ni"][sl] > 0.0)


def test_cloud_ice_melts_above_t0(cress):
    s, dims, base, pp, pi = _setup(cress)
    p = base["pbr"].astype(np.float64)
    t, qi0 = 280.0, 1.0e-5
    st = _uniform_state(dims, base, pi, t, qv_of_t=0.5 * _qvs_w(t, p), qi=qi0, ni=qi0 / 1.0e-11)
    _put(s, cress, st, pp, (cress.PAST, cress.FUTURE))
    s.cloudphy(1.0)
    out = {k: s.get_field(k, cress.FUTURE) for k in MICRO}
    s.close()
    sl = _sl(dims)
    assert np.all(out["qi"][sl] == 0.0)
    # the new cloud water falls at 0.1 m/s: over 2 s a level keeps what it
    # gets from above to ~1e-3 (the density changes with height)
    assert np.allclose(out["qc"][sl], qi0, rtol=2e-3, atol=0)
    tpast = (base["ptbr"].astype(np.float64) + st["ptp"]) * pi
    dth = -qi0 * (LF0 + (CW - CI) * (tpast - T0)) / (CP * pi)
    got = out["ptp"].astype(np.float64) - st["ptp"]
    assert np.allclose(got[sl], dth[sl], rtol=2e-3, atol=0)
    assert np.array_equal(out["qv"], st["qv"])


def test_vapour_supersaturation_adjusts_to_saturation(cress):
    s, dims, base, pp, pi = _setup(cress)
    p = base["pbr"].astype(np.float64)
    t0 = 290.0
    qv0 = 1.08 * _qvs_w(t0, p)
    st = _uniform_state(dims, base, pi, t0, qv_of_t=qv0)
    _put(s, cress, st, pp, (cress.NOW,))
    s.satadjst(cress.NOW)
    out = {k: s.get_field(k, cress.NOW).astype(np.float64) for k in ("ptp", "qv", "qc")}
    s.close()
    sl = _sl(dims)
    qv0f = st["qv"].astype(np.float64)
    # water is conserved
    assert np.allclose((out["qv"] + out["qc"])[sl], qv0f[sl], rtol=2e-6, atol=0)
    # FP64 solution of qv0 - qc = qvs_w(T0 + lv qc / cp, p) by bisection
    tp = (base["ptbr"].astype(np.float64) + st["ptp"]) * pi
    lo, hi = np.zeros_like(qv0f), qv0f.copy()
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        f = (qv0f - mid) - _qvs_w(tp + _lv(tp) * mid / CP, p)
        lo = np.where(f > 0, mid, lo)
        hi = np.where(f > 0, hi, mid)
    qc_exact = 0.5 * (lo + hi)
    assert np.all(qc_exact[sl] > 0)
    assert np.allclose(out["qc"][sl], qc_exact[sl], rtol=5e-3, atol=0)
    dth = out["ptp"] - st["ptp"]
    assert np.allclose(dth[sl], (_lv(tp) * out["qc"] / (CP * pi))[sl], rtol=5e-3, atol=0)


def test_cloudphy_column_water_budget(cress):
    """Every process of s_coldblk moves water between vapour and the five
    hydrometeors, and s_fallblk's upwind flux form moves it between levels,
    so the column total (levels 1..nk-2, weighted by rho J dz) is conserved
    while no water reaches the surface or enters from the top ghost level.
    The state (every process active) is emptied below 1.8 km and in the top
    levels; the fall sub-steps keep the Courant number below 1, so water
    moves at most one level per sub-step and none falls out."""
    from cress_b200 import cases
    dz = 300.0
    dims, base, past, fut, cols = cases.micro_case(37, 29, 40, dz, seed=3)
    ni, nj, nk = dims
    for st in (past, fut):
        for k in ("qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"):
            st[k][:6] = 0.0
            st[k][nk - 5:] = 0.0
        st["qv"][nk - 5:] = 0.0
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, dz, sthopt=1, cphopt=3)
    s.set_base3d(base)
    s.set_base_moist(base["pbr"], base["qvbr"])
    for k in MICRO:
        s.put_field(k, cress.PAST, past[k])
        s.put_field(k, cress.FUTURE, fut[k])
    s.put_field("pp", cress.PAST, past["pp"])
    s.put_precip(np.zeros((5, 2, nj + 2, ni + 2), np.float32))
    s.cloudphy(5.0)
    out = {k: s.get_field(k, cress.FUTURE) for k in MICRO}
    prec = s.get_precip()
    s.close()
    rst = base["rst"].astype(np.float64)
    lv = slice(0, nk - 2)                     # levels 1 .. nk-2
    cs = (slice(2, nj - 1), slice(2, ni - 1))

    def column_water(f):
        q = sum(f[k].astype(np.float64) for k in ("qv", "qc", "qr", "qi", "qs", "qg"))
        return np.sum((rst * q)[lv], axis=0)[cs] * dz          # kg m^-2

    before, after = column_water(fut), column_water(out)
    moved = sum(np.abs(out[k].astype(np.float64) - fut[k])[lv].sum(axis=0)[cs]
                for k in ("qc", "qr", "qi", "qs", "qg"))
    resid = after - before
    print(f"column budget: max |residual| {np.abs(resid).max():.3e} kg/m2 of column water up to "
          f"{before.max():.3e} kg/m2")
    assert not prec.any()                     # nothing reached the surface
    assert moved.max() > 1e-4                 # the processes and the fall did change the state
    assert np.all(np.abs(resid) <= 2e-6 * before + 1e-9)

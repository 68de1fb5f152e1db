"""CPU checks of the oracle itself (no GPU).

The reference ships no tests or golden outputs, so the oracle is pinned by
properties the reference's equations must satisfy:
  * a hydrostatic rest state with zero forcing stays exactly at rest;
  * a periodic shift of the inputs shifts the outputs (bcycle wrap);
  * the FP32 and FP64 builds agree to float rounding;
  * the FP32 Thomas solve and the FP64 solve agree to float rounding.
The first three hold for both small steps, HE-VI (impopt=1) and HE-VE
(impopt=0, with a step short enough for its explicit vertical terms).
"""
import numpy as np
import pytest

import helpers as H


def cfg_for(ni, nj, nk, dx=500.0, dz=300.0, sthopt=0, impopt=1):
    return dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=sthopt, divopt=2, buyopt=1,
                weicoe=0.6, impopt=impopt)


@pytest.mark.parametrize("impopt", [1, 0])
def test_rest_state(oracle_lib, impopt):
    ni, nj, nk = H.dims(16, 12, 10)
    base = H.base3d(ni, nj, nk, 300.0)
    z = [np.zeros((nk, nj + 2, ni + 2), np.float32) for _ in range(4)]
    st = [a.copy() for a in z]
    oracle_lib.small_steps(cfg_for(ni, nj, nk, impopt=impopt), base, z, st, 4, 0.25)
    for a in st:
        assert np.all(a == 0.0)


@pytest.mark.parametrize("impopt", [1, 0])
def test_periodic_shift_equivariance(oracle_lib, impopt):
    nx, ny, nz = 16, 12, 10
    ni, nj, nk = H.dims(nx, ny, nz)
    base = H.base3d(ni, nj, nk, 300.0)
    st, frc = H.small_state(ni, nj, nk, 3, base)
    cfg = cfg_for(ni, nj, nk, impopt=impopt)
    a = [x.copy() for x in st]
    oracle_lib.small_steps(cfg, base, frc, a, 3, 0.25)

    def shift(x, stag, s):
        y = x.copy()
        # interior x-range of the periodic domain: i = 2..ni-2 (period nx)
        y[:, :, 2:ni - 1] = np.roll(x[:, :, 2:ni - 1], s, axis=2)
        if stag == "u":
            y[:, :, ni - 1] = y[:, :, 2]
        return H.bcycle(y, stag)

    stags = ["u", "v", "s", "s"]
    st2 = [shift(x, t, 5) for x, t in zip(st, stags)]
    frc2 = [shift(x, t, 5) for x, t in zip(frc, stags)]
    b = [x.copy() for x in st2]
    oracle_lib.small_steps(cfg, base, frc2, b, 3, 0.25)
    for x, y, t in zip(a, b, stags):
        m = H.interior_mask(ni, nj, nk, t)
        xs = shift(x, t, 5)
        assert np.array_equal(xs[m], y[m])


@pytest.mark.parametrize("impopt", [1, 0])
def test_fp32_vs_fp64_spread(oracle_lib, impopt):
    ni, nj, nk = H.dims(20, 16, 12)
    base = H.base3d(ni, nj, nk, 250.0, sthopt=1)
    st, frc = H.small_state(ni, nj, nk, 4, base)
    cfg = cfg_for(ni, nj, nk, dx=1000.0, dz=250.0, sthopt=1, impopt=impopt)
    dts = 0.5 if impopt else 0.1
    a = [x.copy() for x in st]
    b = [x.copy() for x in st]
    oracle_lib.small_steps(cfg, base, frc, a, 6, dts, prec=32, fp64_solve=0)
    oracle_lib.small_steps(cfg, base, frc, b, 6, dts, prec=64)
    for x, y in zip(a, b):
        scale = np.abs(y).max()
        assert np.abs(x - y).max() <= 1e-4 * scale


def test_fp64_solve_close_to_fp32_solve(oracle_lib):
    ni, nj, nk = H.dims(20, 16, 30)
    base = H.base3d(ni, nj, nk, 250.0, sthopt=1)
    st, frc = H.small_state(ni, nj, nk, 8, base)
    cfg = cfg_for(ni, nj, nk, dx=1000.0, dz=250.0, sthopt=1)
    a = [x.copy() for x in st]
    b = [x.copy() for x in st]
    oracle_lib.small_steps(cfg, base, frc, a, 2, 0.5, prec=32, fp64_solve=0)
    oracle_lib.small_steps(cfg, base, frc, b, 2, 0.5, prec=32, fp64_solve=1)
    w32, w64 = a[2], b[2]
    assert np.abs(w32 - w64).max() <= 1e-5 * np.abs(w64).max()


def test_moist_step_fp32_vs_fp64_and_water(oracle_lib):
    """The moist large step (cphopt=3) runs in both precisions and the two
    agree to a small fraction of each field's range."""
    from cress_b200 import cases
    case = cases.supercell_case(16, 14, 14, 1000.0, ztop=5000.0, seed=2, cloud=True,
                                rad=(4000.0, 4000.0, 1200.0))
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    botbar = 0.6 * zph[nk - 1]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, botbar)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=case["dz"], sthopt=1, vspbar=0.005,
               botbar=botbar)
    init = list(case["level"]) + [case["moist"][n] for n in oracle_lib.MOIST_STATE_NAMES[5:]]
    runs = []
    for bits in (32, 64):
        past = [a.copy() for a in init]
        now = [a.copy() for a in init]
        prec = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
        npstp = oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec, 2, 5.0, 1.0,
                                       prec_bits=bits)
        assert npstp >= 1
        runs.append((now, prec))
    sl = (slice(0, nk - 1), slice(2, nj - 1), slice(2, ni - 1))
    for name, a, b in zip(oracle_lib.MOIST_STATE_NAMES, runs[0][0], runs[1][0]):
        assert np.isfinite(a).all(), name
        scale = float(np.abs(b[sl]).max()) + 1e-12
        assert float(np.abs(a[sl] - b[sl]).max()) <= 2e-2 * scale, name
    assert float(np.abs(runs[0][1] - runs[1][1]).max()) <= 2e-2 * float(np.abs(runs[1][1]).max()) + 1e-9


def test_mlp_oracle_gradient_finite_differences():
    """The oracle's backward pass (exact float64 mode) against central
    differences on a sample of parameters."""
    from oracle import mlp as M
    rng = np.random.default_rng(1)
    p = rng.uniform(-0.2, 0.2, M.count())
    x = rng.standard_normal((8, 16))
    t = rng.standard_normal((8, 9))
    M.ROUND = False
    try:
        _, g = M.loss_grad(p, x, t)
        idx = rng.choice(M.count(), 40, replace=False)
        # keep to the parameters the padding does not zero out
        for i in idx:
            e = np.zeros_like(p)
            e[i] = 1e-5
            fd = (M.loss_grad(p + e, x, t)[0] - M.loss_grad(p - e, x, t)[0]) / 2e-5
            assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
    finally:
        M.ROUND = True


def test_smagorinsky_fp32_vs_fp64_and_active(oracle_lib):
    """Dry large steps with Smagorinsky turbulence (tubopt=1) in neutral
    stratification: float and double agree to a small fraction of each
    field's range, and the turbulence changes the result."""
    from cress_b200 import cases
    dx, dz = 500.0, 300.0
    case = cases.dry_case(24, 20, 16, dx, dz, sthopt=1, seed=3, vspbar=0.005, dthdz=0.0, noise=0.5)
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    out = {}
    for tub, prec in ((1, 32), (1, 64), (0, 32)):
        cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, vspbar=0.005,
                   botbar=0.6 * zph[nk - 1], tubopt=tub)
        past = [a.copy() for a in case["level"]]
        now = [a.copy() for a in case["level"]]
        oracle_lib.dry_steps(cfg, case["base"], zph, past, now, 3, 2.0, 0.25, start=True, prec=prec)
        out[(tub, prec)] = now
    sl = (slice(0, nk - 1), slice(2, nj - 1), slice(2, ni - 1))
    changed = 0.0
    for n in range(5):
        a, b, c = out[(1, 32)][n][sl], out[(1, 64)][n][sl], out[(0, 32)][n][sl]
        scale = float(np.abs(b).max()) + 1e-12
        assert np.isfinite(a).all()
        assert float(np.abs(a - b).max()) <= 1e-3 * scale
        changed = max(changed, float(np.abs(a - c).max()) / scale)
    assert changed > 1e-3


def test_tke_closure_fp32_vs_fp64_spins_up(oracle_lib):
    """Dry large steps with the 1.5-order TKE closure (tubopt=2) from zero
    TKE in neutral stratification: the minimum viscosity where shear beats
    stability gives shear production, so TKE appears within a few steps,
    stays non-negative (the clipped step), float and double agree to a
    small fraction of each field's range, and the flow differs from the
    Smagorinsky run."""
    from cress_b200 import cases
    dx, dz = 500.0, 300.0
    case = cases.dry_case(24, 20, 16, dx, dz, sthopt=1, seed=3, vspbar=0.005, dthdz=0.0, noise=0.5)
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    out = {}
    for tub, prec in ((2, 32), (2, 64), (1, 32)):
        cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, vspbar=0.005,
                   botbar=0.6 * zph[nk - 1], tubopt=tub)
        past = [a.copy() for a in case["level"]]
        now = [a.copy() for a in case["level"]]
        if tub == 2:
            past.append(np.zeros_like(past[0]))
            now.append(np.zeros_like(now[0]))
        oracle_lib.dry_steps(cfg, case["base"], zph, past, now, 6, 2.0, 0.25, start=True, prec=prec)
        out[(tub, prec)] = now
    sl = (slice(0, nk - 1), slice(2, nj - 1), slice(2, ni - 1))
    for n in range(6):
        a, b = out[(2, 32)][n][sl], out[(2, 64)][n][sl]
        scale = float(np.abs(b).max()) + 1e-30
        assert np.isfinite(a).all()
        assert float(np.abs(a - b).max()) <= 1e-3 * scale, n
    tke = out[(2, 32)][5][sl]
    assert tke.min() >= 0.0 and tke.max() > 1e-4 and (tke > 0).mean() > 0.5
    changed = max(float(np.abs(out[(2, 32)][n][sl] - out[(1, 32)][n][sl]).max()) /
                  float(np.abs(out[(1, 32)][n][sl]).max()) for n in range(5))
    assert changed > 1e-3


def test_fourth_order_vertical_advection(oracle_lib):
    """advopt=3 (advuvw.f90 / advs.f90 / advp.f90, the advopt.eq.3 branches):
    float and double agree, and the result differs from advopt=2 by a
    small amount (the vertical truncation error of the 2nd-order scheme)."""
    from cress_b200 import cases
    dx, dz = 500.0, 300.0
    case = cases.dry_case(24, 20, 16, dx, dz, sthopt=1, seed=3, vspbar=0.005, dthdz=0.0, noise=0.5)
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    out = {}
    for adv, prec in ((3, 32), (3, 64), (2, 32)):
        cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, vspbar=0.005,
                   botbar=0.6 * zph[nk - 1], advopt=adv)
        past = [a.copy() for a in case["level"]]
        now = [a.copy() for a in case["level"]]
        oracle_lib.dry_steps(cfg, case["base"], zph, past, now, 3, 2.0, 0.25, start=True, prec=prec)
        out[(adv, prec)] = now
    sl = (slice(0, nk - 1), slice(2, nj - 1), slice(2, ni - 1))
    changed = 0.0
    for n in range(5):
        a, b, c = out[(3, 32)][n][sl], out[(3, 64)][n][sl], out[(2, 32)][n][sl]
        scale = float(np.abs(b).max()) + 1e-12
        assert np.isfinite(a).all()
        assert float(np.abs(a - b).max()) <= 1e-3 * scale
        changed = max(changed, float(np.abs(a - c).max()) / scale)
    assert 1e-7 < changed < 1e-2


def test_base_state_restatement_is_hydrostatic(oracle_lib):
    """The base state from the supercell sounding (set1d ... sndwave): the
    Exner function falls with height at the rate -g / (cp theta_v) to the
    accuracy of the sounding's interpolation, and the FP32 build stays
    within 1e-5 of the FP64 build."""
    from cress_b200 import cases
    nk = 67
    c = cases.moist_columns(nk)
    z = np.linspace(0.0, 20000.0, 121)
    th = np.where(z <= 12000.0, 300.0 + 43.0 * (z / 12000.0) ** 1.25,
                  343.0 * np.exp(9.8 * (z - 12000.0) / (1004.0 * 213.0)))
    rh = 100.0 * np.where(z <= 12000.0, 1.0 - 0.75 * (z / 12000.0) ** 1.25, 0.25)
    b = oracle_lib.base_state(nk, c["zph"], c["jcb"].astype(np.float64), z, 0 * z, 0 * z, th, rh, 1e5)
    b32 = oracle_lib.base_state(nk, c["zph"], c["jcb"].astype(np.float64), z, 0 * z, 0 * z, th, rh, 1e5,
                                prec=32)
    zph = c["zph"]
    zs = 0.5 * (zph[1:nk] + zph[2:nk + 1])           # scalar levels k = 1..nk-1
    pi, ptv = b["pibr"][1:nk], b["ptvbr"][1:nk]
    slope = np.diff(pi) / np.diff(zs)
    expect = -9.8 / (1004.0 * 0.5 * (ptv[1:] + ptv[:-1]))
    assert np.allclose(slope[1:-1], expect[1:-1], rtol=2e-3)
    for name in ("pbr", "ptbr", "rbr", "rcsq"):
        r = b[name][1:]
        assert np.abs(b32[name][1:] - r).max() <= 1e-5 * np.abs(r).max(), name

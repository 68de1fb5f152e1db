"""GPU parity of whole large steps with the 1.5-order TKE closure (tubopt=2)
against the CPU oracle.

The eddy viscosity is the Deardorff form from the past TKE, the winds,
theta' and the moist species mix with it, and the TKE itself is stepped:
advection, shear production, smoothing, dissipation, transport with twice
the momentum diffusivity, Rayleigh damping, buoyancy production, the
clipped leapfrog and the doubled Asselin filter (SrcOrig/forcetke.f90:
269-354, eddyvis.f90:448-481, steps.f90:999-1014, timeflt.f90:866-884).

Cases: a dry warm bubble in neutral stratification starting from a seeded
TKE field (every term active from the first step) and from zero TKE (the
minimum viscosity where shear exceeds stability starts it); a moist
supercell with a seeded TKE field.  Tolerances as the Smagorinsky runs of
the same cases: dry max|gpu - oracle| <= 1e-4 max|oracle| + 1e-6 per field
and level; moist 99.9% of cells within 1e-4 of the field's maximum and
every cell within 1e-2, precipitation within 1e-3.
"""
import numpy as np
import pytest

import helpers as H
import test_large_gpu as LG
import test_moist_gpu as MG

pytestmark = pytest.mark.gpu


def seeded_tke(shape, seed, amp=0.4):
    """A smooth positive TKE field (m^2/s^2) with periodic ghosts and the
    zero-gradient levels 1 and nk-1 of s_vbcs."""
    rng = np.random.default_rng(seed)
    t = np.abs(H.smooth_noise(rng, shape, amp)).astype(np.float32) + np.float32(0.01)
    t[0] = t[1]
    t[-2] = t[-3]
    return H.bcycle(t, "s")


def run_dry(cress, oracle_lib, nx, ny, nz, nsteps, seed, tke0, advopt=2):
    from cress_b200 import cases
    dx, dz, dtbig, dtsml = 500.0, 300.0, 2.0, 0.25
    case = cases.dry_case(nx, ny, nz, dx, dz, sthopt=1, seed=seed, vspbar=0.005, dthdz=0.0, noise=0.5)
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    botbar = 0.6 * zph[nk - 1]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, botbar)
    shape = (nk, nj + 2, ni + 2)
    tke = seeded_tke(shape, seed + 100) if tke0 else np.zeros(shape, np.float32)
    init = list(case["level"]) + [tke]
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, smtopt=3, vspopt=2, coropt=0,
               vspbar=0.005, botbar=botbar, tubopt=2, advopt=advopt)
    past = [a.copy() for a in init]
    now = [a.copy() for a in init]
    oracle_lib.dry_steps(cfg, case["base"], zph, past, now, nsteps, dtbig, dtsml, start=True)

    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1, tubopt=2, advopt=advopt)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    names = LG.NAMES + ["tke"]
    for n, a in zip(names, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    nsstp = 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))
    for step in range(nsteps):
        first = step == 0
        s.large_step(round(step * dtbig * 1000), 0.5 * dtbig if first else dtbig, nsstp,
                     0.5 * dtsml if first else dtsml)
    got = [[s.get_field(n, lvl) for n in names] for lvl in (cress.PAST, cress.NOW)]
    s.close()
    return (ni, nj, nk), (past, now), got


def check_dry(dims, ref, got, rtol=1e-4):
    ni, nj, nk = dims
    for lvl in range(2):
        for name, r, g in zip(LG.NAMES + ["tke"], ref[lvl], got[lvl]):
            m = LG.region(name if name != "tke" else "ptp", ni, nj, nk)
            scale = float(np.abs(r[m]).max())
            err = float(np.abs(g[m] - r[m]).max())
            assert np.isfinite(g[m]).all(), name
            assert err <= rtol * scale + 1e-6, f"level {lvl} {name}: err {err:.3e} scale {scale:.3e}"
    tke = got[1][5][LG.region("ptp", ni, nj, nk)]
    assert tke.min() >= 0.0 and tke.max() > 0.0


def test_dry_large_steps_tke_seeded(cress, oracle_lib):
    dims, ref, got = run_dry(cress, oracle_lib, 40, 32, 24, 4, seed=5, tke0=True)
    check_dry(dims, ref, got)


def test_dry_large_steps_tke_from_zero_ragged(cress, oracle_lib):
    dims, ref, got = run_dry(cress, oracle_lib, 37, 29, 20, 5, seed=9, tke0=False)
    check_dry(dims, ref, got)


def test_dry_large_steps_tke_4th_order_vertical_advection(cress, oracle_lib):
    # advopt=3 in the TKE equation's advection as well
    dims, ref, got = run_dry(cress, oracle_lib, 40, 32, 24, 4, seed=6, tke0=True, advopt=3)
    check_dry(dims, ref, got)


def test_moist_large_steps_tke(cress, oracle_lib):
    from cress_b200 import cases
    nx, ny, nz, nsteps, seed = 36, 30, 22, 3, 11
    dx, dtbig, dtsml = 1000.0, 5.0, 1.0
    case = cases.supercell_case(nx, ny, nz, dx, ztop=8000.0, seed=seed, cloud=True, rad=(6000.0, 6000.0, 1400.0))
    ni, nj, nk = case["dims"]
    dz, zph = case["dz"], case["zph"]
    vspbar, botbar = 0.005, 0.6 * zph[nk - 1]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, vspbar, botbar)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, smtopt=3, vspopt=2, coropt=0,
               vspbar=vspbar, botbar=botbar, thresq=1e-12, tubopt=2)
    tke = seeded_tke((nk, nj + 2, ni + 2), seed + 100)
    init = list(case["level"]) + [case["moist"][n] for n in MG.NAMES[5:]] + [tke]
    past = [a.copy() for a in init]
    now = [a.copy() for a in init]
    prec_ref = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
    oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec_ref, nsteps, dtbig, dtsml, start=True)

    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1, cphopt=3, thresq=1e-12, tubopt=2)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    names = MG.NAMES + ["tke"]
    for n, a in zip(names, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    nsstp = 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))
    for step in range(nsteps):
        first = step == 0
        s.large_step(round(step * dtbig * 1000), 0.5 * dtbig if first else dtbig, nsstp,
                     0.5 * dtsml if first else dtsml)
    gp = [s.get_field(n, cress.PAST) for n in names]
    gn = [s.get_field(n, cress.NOW) for n in names]
    prec = s.get_precip()
    s.close()
    # the 14 prognostic fields and the precipitation as the moist test checks them
    MG.check((ni, nj, nk), (past[:14], now[:14], prec_ref), (gp[:14], gn[:14], prec))
    m = MG.region("ptp", ni, nj, nk)
    for r, g in ((past[14], gp[14]), (now[14], gn[14])):
        scale = float(np.abs(r[m]).max())
        err = np.abs(g[m] - r[m])
        assert np.isfinite(g[m]).all() and g[m].min() >= 0.0
        assert float((err <= 1e-4 * scale).mean()) >= 0.999 and float(err.max()) <= 1e-2 * scale

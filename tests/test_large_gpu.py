"""GPU parity of whole dry large steps (s_intgdrv) against the CPU oracle.

A warm bubble in a sheared flow on a stretched grid, with 4th-order
smoothing, Rayleigh damping aloft and (optionally) Coriolis, is advanced
a few leapfrog steps by cress_large_step and by the oracle's restatement;
both time levels (t-dt and t) must agree field by field.  Tolerance:
max|gpu - oracle| <= 1e-4 * max|oracle| + 1e-6 per field, set by float
rounding differences (FMA contraction, reciprocal multiplies) that the
leapfrog steps carry forward.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "pp", "ptp"]
STAG = {"u": "u", "v": "v", "w": "s", "pp": "s", "ptp": "s"}


def region(name, ni, nj, nk):
    m = np.zeros((nk, nj + 2, ni + 2), bool)
    ih = ni + 1 if STAG[name] == "u" else ni
    jh = nj + 1 if STAG[name] == "v" else nj
    k0, k1 = (1, nk) if name == "w" else (1, nk - 1)
    m[k0 - 1:k1, 0:jh + 1, 0:ih + 1] = True
    return m


def run_case(cress, oracle_lib, nx, ny, nz, nsteps, coropt=0, seed=3, tubopt=0, dthdz=0.003, noise=0.01,
             impopt=1, advopt=2):
    from cress_b200 import cases
    dx, dz, dtbig, dtsml = 500.0, 300.0, 2.0, 0.25
    case = cases.dry_case(nx, ny, nz, dx, dz, sthopt=1, seed=seed, vspbar=0.005, dthdz=dthdz, noise=noise)
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    botbar = 0.6 * zph[nk - 1]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, botbar)
    fc = 0.5 * 7.292e-5 * np.sin(np.deg2rad(35.0)) if coropt else 0.0
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, smtopt=3, vspopt=2,
               coropt=coropt, vspbar=0.005, botbar=botbar, fc=fc, tubopt=tubopt, impopt=impopt, advopt=advopt)
    past = [a.copy() for a in case["level"]]
    now = [a.copy() for a in case["level"]]
    oracle_lib.dry_steps(cfg, case["base"], zph, past, now, nsteps, dtbig, dtsml, start=True)

    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1, coropt=coropt, fc=fc, tubopt=tubopt, impopt=impopt,
                     advopt=advopt)
    s.set_base3d(case["base"])
    rb3 = cases.expand(rbct, ni, nj, nk)
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], rb3, ksp0)
    for n, a in zip(NAMES, case["level"]):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    nsstp = 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))
    for step in range(nsteps):
        first = step == 0
        s.large_step(round(step * dtbig * 1000), 0.5 * dtbig if first else dtbig, nsstp,
                     0.5 * dtsml if first else dtsml)
    gp = [s.get_field(n, cress.PAST) for n in NAMES]
    gn = [s.get_field(n, cress.NOW) for n in NAMES]
    s.close()
    return (ni, nj, nk), (past, now), (gp, gn)


def check(dims, ref, got, rtol=1e-4):
    ni, nj, nk = dims
    for lvl in range(2):
        for name, r, g in zip(NAMES, ref[lvl], got[lvl]):
            m = region(name, ni, nj, nk)
            scale = float(np.abs(r[m]).max())
            err = float(np.abs(g[m] - r[m]).max())
            assert np.isfinite(g[m]).all(), name
            assert err <= rtol * scale + 1e-6, f"level {lvl} {name}: err {err:.3e} scale {scale:.3e}"


def test_dry_large_steps(cress, oracle_lib):
    dims, ref, got = run_case(cress, oracle_lib, 40, 32, 24, 3)
    check(dims, ref, got)


def test_dry_large_steps_coriolis_ragged(cress, oracle_lib):
    dims, ref, got = run_case(cress, oracle_lib, 37, 29, 20, 2, coropt=1, seed=9)
    check(dims, ref, got)


def test_dry_large_steps_smagorinsky(cress, oracle_lib):
    # neutral stratification and noise so the eddy viscosity is active
    dims, ref, got = run_case(cress, oracle_lib, 40, 32, 24, 4, seed=5, tubopt=1, dthdz=0.0, noise=0.5)
    check(dims, ref, got)


def test_dry_large_steps_4th_order_vertical_advection(cress, oracle_lib):
    # advopt=3: 4th-order vertical advection of u, v, w and theta' on
    # levels 3..nk-3 (w: 3..nk-2), 2nd order next to the boundaries
    dims, ref, got = run_case(cress, oracle_lib, 37, 29, 20, 3, seed=4, dthdz=0.0, noise=0.5, advopt=3)
    check(dims, ref, got)


def test_dry_large_steps_heve(cress, oracle_lib):
    # the explicit small step (impopt=0) inside whole large steps
    dims, ref, got = run_case(cress, oracle_lib, 40, 32, 24, 3, seed=7, impopt=0)
    check(dims, ref, got)

"""Precision study: the FP32 GPU path against an FP64 build of the same
scheme on the same inputs.

A moist supercell state (cold rain) runs N large steps on the GPU (FP32,
FP64 vertical solve), in the oracle's FP32 build and in its FP64 build.
For every prognostic field and the accumulated precipitation the test
reports the RMS (relative to the field's RMS) and the maximum difference
of GPU - FP64 next to the oracle's own FP32 - FP64 spread, and the drift
of the total water (vapour + hydrometeors + precipitated) and of the mass.
The GPU's error must be of the order of the FP32 build's own (within a
factor 20 in RMS, plus a floor for fields that stay near zero), and its
budgets must agree with the FP64 run's to 1e-4.  Run with -s to see the
table (one JSON line).
"""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def budgets(case, fields, prec, dx, dz, i0=2):
    ni, nj, nk = case["dims"]
    sl = (slice(1, nk - 2), slice(2, nj - 1), slice(i0, ni - 1))
    rst = case["base"]["rst"].astype(np.float64)[sl]
    rcsq = case["base"]["rcsq"].astype(np.float64)[sl]
    f = {n: a.astype(np.float64) for n, a in zip(NAMES, fields)}
    q = sum(f[n][sl] for n in ("qv", "qc", "qr", "qi", "qs", "qg"))
    water = float(np.sum(rst * q)) * dx * dx * dz
    precip = float(np.sum(prec.astype(np.float64)[:, 1, 2:nj - 1, i0:ni - 1])) * 1.e3 * dx * dx
    mass = float(np.sum(rst * (1.0 + f["pp"][sl] / rcsq))) * dx * dx * dz
    return water + precip, mass


def _study(cress, oracle_lib, case, dx, nsteps, dtbig, dtsml, obc=0, label="supercell"):
    ni, nj, nk = case["dims"]
    dz, zph = case["dz"], case["zph"]
    vspbar, botbar = 0.005, 0.6 * zph[nk - 1]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, vspbar, botbar)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, smtopt=3, vspopt=2, coropt=0,
               vspbar=vspbar, botbar=botbar, thresq=1e-12, obc=obc, gwave=20.0)
    init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]

    runs = {}
    for bits in (64, 32):
        past = [a.copy() for a in init]
        now = [a.copy() for a in init]
        prec = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
        oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec, nsteps, dtbig, dtsml, start=True,
                               prec_bits=bits, omp=True)
        runs[bits] = (now, prec)

    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1, cphopt=3, thresq=1e-12, obc=obc, gwave=20.0)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases_expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    for n, a in zip(NAMES, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    nsstp = 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))
    for step in range(nsteps):
        first = step == 0
        s.large_step(round(step * dtbig * 1000), 0.5 * dtbig if first else dtbig, nsstp,
                     0.5 * dtsml if first else dtsml)
    gpu = ([s.get_field(n, cress.NOW) for n in NAMES], s.get_precip())
    s.close()

    i0 = 1 if obc else 2   # open x: the boundary columns are prognostic too
    sl = (slice(1, nk - 2), slice(2, nj - 1), slice(i0, ni - 1))
    ref, ref_prec = runs[64]
    o32, o32_prec = runs[32]
    report = {"case": label, "grid": [ni - 3, nj - 3, nk - 3], "open_x": obc, "steps": nsteps,
              "simulated_s": (nsteps - 0.5) * dtbig, "fields": {}}

    def stats(a, b):
        d = (a.astype(np.float64) - b.astype(np.float64))[sl] if a.ndim == 3 else (a - b)
        r = b.astype(np.float64)[sl] if b.ndim == 3 else b.astype(np.float64)
        rms_ref = float(np.sqrt(np.mean(r * r))) + 1e-30
        return float(np.sqrt(np.mean(d * d))) / rms_ref, float(np.abs(d).max()), rms_ref

    for n, g, r, o in zip(NAMES, gpu[0], ref, o32):
        eg, mg, rms = stats(g, r)
        eo, mo, _ = stats(o, r)
        report["fields"][n] = {"gpu_rms_rel": eg, "gpu_max": mg, "fp32_oracle_rms_rel": eo,
                               "fp32_oracle_max": mo, "fp64_rms": rms}
        assert np.isfinite(g[sl]).all(), n
        # near-zero fields (an absent species) get an absolute floor
        assert eg <= 20.0 * eo + 1e-6 or mg <= 1e-9, (n, eg, eo)
    pg = gpu[1][:, 1, 2:nj - 1, i0:ni - 1].astype(np.float64)
    pr = ref_prec[:, 1, 2:nj - 1, i0:ni - 1].astype(np.float64)
    report["precip_accum_rel_diff"] = abs(pg.sum() - pr.sum()) / (abs(pr.sum()) + 1e-30)

    dzf = float(np.float32(dz))
    w0, m0 = budgets(case, init, np.zeros_like(ref_prec), dx, dzf, i0)
    wg, mg_ = budgets(case, gpu[0], gpu[1], dx, dzf, i0)
    wr, mr = budgets(case, ref, ref_prec, dx, dzf, i0)
    report["water_drift_gpu"] = (wg - w0) / w0
    report["water_drift_fp64"] = (wr - w0) / w0
    report["mass_drift_gpu"] = (mg_ - m0) / m0
    report["mass_drift_fp64"] = (mr - m0) / m0
    print(json.dumps({"precision": report}))
    assert abs(report["water_drift_gpu"] - report["water_drift_fp64"]) < 1e-4
    assert abs(report["mass_drift_gpu"] - report["mass_drift_fp64"]) < 1e-4


def cases_expand(col, ni, nj, nk):
    from cress_b200 import cases
    return cases.expand(col, ni, nj, nk)


def test_fp32_gpu_against_fp64(cress, oracle_lib):
    from cress_b200 import cases
    nx, ny, nz, dx = 40, 40, 30, 1000.0
    case = cases.supercell_case(nx, ny, nz, dx, ztop=10000.0, seed=12, cloud=True,
                                rad=(6000.0, 6000.0, 1400.0))
    _study(cress, oracle_lib, case, dx, 24, 5.0, 1.0)


def test_fp32_gpu_against_fp64_squall_open_x(cress, oracle_lib):
    """The squall-line configuration (line thermal +2 K with seeded 0.1 K
    noise, 20 m/s low-level shear, dx = 500 m, open radiation x boundaries
    with per-point phase speeds, periodic y) on a reduced grid.  With open
    boundaries water and mass leave and enter the domain, so the drifts are
    compared between the GPU and the FP64 build, not against zero."""
    from cress_b200 import cases
    nx, ny, nz, dx = 64, 24, 36, 500.0
    case = cases.squall_case(nx, ny, nz, dx, ztop=12000.0, seed=7, xrad=4000.0)
    _study(cress, oracle_lib, case, dx, 30, 3.0, 0.5, obc=4, label="squall line, open x")

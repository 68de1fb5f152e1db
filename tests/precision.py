"""Precision studies shared by the parity tests: one configuration run on the
GPU (FP32, FP64 vertical solve) and in the oracle's FP32 and FP64 builds
from the same initial state, with per-field statistics against the FP64
run and the water / dry-mass budgets.

Statistics per prognostic field over the interior (levels 2..nk-2):
  gpu_rms_rel      RMS(GPU - FP64) / RMS(FP64)
  gpu_max          max |GPU - FP64|
  fp32_rms_rel     RMS(FP32 oracle - FP64) / RMS(FP64)   (the FP32 spread)
  fp32_max         max |FP32 oracle - FP64|
  gpu_fp32_rms_rel RMS(GPU - FP32 oracle) / RMS(FP64)
  fp32p_rms_rel    RMS(FP32 oracle from theta' one ulp up - FP64) / RMS(FP64)
                   (moist runs: a second FP32 realization of the same run)
"""
import numpy as np

MOIST = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]
DRY = ["u", "v", "w", "pp", "ptp"]


def nsstp_of(dtbig, dtsml):
    """SrcOrig/slvstep.f90:176."""
    return 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))


def interior(ni, nj, nk, i0=2):
    return (slice(1, nk - 2), slice(2, nj - 1), slice(i0, ni - 1))


def moist_budgets(case, fields, prec, dx, dz, i0=2):
    """Total water (vapour + hydrometeors + accumulated precipitation, kg)
    and dry-air-plus-vapour mass (kg) of the interior, in FP64."""
    ni, nj, nk = case["dims"]
    sl = interior(ni, nj, nk, i0)
    rst = case["base"]["rst"].astype(np.float64)[sl]
    rcsq = case["base"]["rcsq"].astype(np.float64)[sl]
    f = {n: a.astype(np.float64) for n, a in zip(MOIST, fields)}
    q = sum(f[n][sl] for n in ("qv", "qc", "qr", "qi", "qs", "qg"))
    water = float(np.sum(rst * q)) * dx * dx * dz
    precip = float(np.sum(prec.astype(np.float64)[:, 1, 2:nj - 1, i0:ni - 1])) * 1.e3 * dx * dx
    mass = float(np.sum(rst * (1.0 + f["pp"][sl] / rcsq))) * dx * dx * dz
    return water + precip, mass


def dry_mass(case, fields, dx, dz):
    ni, nj, nk = case["dims"]
    sl = interior(ni, nj, nk)
    rst = case["base"]["rst"].astype(np.float64)[sl]
    rcsq = case["base"]["rcsq"].astype(np.float64)[sl]
    pp = fields[3].astype(np.float64)[sl]
    return float(np.sum(rst * (1.0 + pp / rcsq))) * dx * dx * dz


def field_stats(names, gpu, o64, o32, sl):
    out = {}
    for n, g, r, o in zip(names, gpu, o64, o32):
        r64 = r.astype(np.float64)[sl]
        rms_ref = float(np.sqrt(np.mean(r64 * r64))) + 1e-30
        dg = g.astype(np.float64)[sl] - r64
        do = o.astype(np.float64)[sl] - r64
        dgo = g.astype(np.float64)[sl] - o.astype(np.float64)[sl]
        out[n] = {"gpu_rms_rel": float(np.sqrt(np.mean(dg * dg))) / rms_ref,
                  "gpu_max": float(np.abs(dg).max()),
                  "fp32_rms_rel": float(np.sqrt(np.mean(do * do))) / rms_ref,
                  "fp32_max": float(np.abs(do).max()),
                  "gpu_fp32_rms_rel": float(np.sqrt(np.mean(dgo * dgo))) / rms_ref,
                  "fp64_rms": rms_ref,
                  "finite": bool(np.isfinite(g[sl]).all())}
    return out


def _vsp(oracle_lib, nk, zph, vspbar, botbar):
    return oracle_lib.vspdmp(nk, zph, vspbar, botbar)


def _run_gpu(cress, case, names, init, s, nsteps, dtbig, dtsml, rbct, ksp0, moist):
    from cress_b200 import cases
    ni, nj, nk = case["dims"]
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    if moist:
        s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    for n, a in zip(names, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    nsstp = nsstp_of(dtbig, dtsml)
    for step in range(nsteps):
        first = step == 0
        s.large_step(round(step * dtbig * 1000), 0.5 * dtbig if first else dtbig, nsstp,
                     0.5 * dtsml if first else dtsml)
    out = [s.get_field(n, cress.NOW) for n in names]
    prec = s.get_precip() if moist else None
    diag = s.diagnostics(cress.NOW, check=False)
    s.close()
    return out, prec, diag


def _tke0(case):
    """Zero TKE (a fresh start of the TKE closure)."""
    ni, nj, nk = case["dims"]
    return np.zeros((nk, nj + 2, ni + 2), np.float32)


def moist_study(cress, oracle_lib, case, dx, nsteps, dtbig, dtsml, obc=0, label="supercell", tubopt=0):
    """Cold-rain (cphopt=3) run of `nsteps` large steps; returns the report.
    tubopt=2 adds the TKE closure, starting from zero TKE, and the TKE to
    the report's fields."""
    ni, nj, nk = case["dims"]
    dz, zph = case["dz"], case["zph"]
    vspbar, botbar = 0.005, 0.6 * zph[nk - 1]
    rbct, ksp0 = _vsp(oracle_lib, nk, zph, vspbar, botbar)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, smtopt=3, vspopt=2, coropt=0,
               vspbar=vspbar, botbar=botbar, thresq=1e-12, obc=obc, gwave=20.0, tubopt=tubopt)
    names = MOIST + (["tke"] if tubopt == 2 else [])
    init = list(case["level"]) + [case["moist"][n] for n in MOIST[5:]] + ([_tke0(case)] if tubopt == 2 else [])
    runs = {}
    # FP64, FP32, and FP32 again from an initial theta' one ulp up: over
    # hours of moist convection one FP32 realization is a single sample of
    # the chaotic growth of round-off, and sparse threshold-driven fields
    # (the ice number above all) can stay close to FP64 in one realization
    # and not in another
    for key, bits in ((64, 64), (32, 32), ("32p", 32)):
        st = [a.copy() for a in init]
        if key == "32p":
            st[4] = np.nextafter(st[4], np.float32(np.inf)).astype(np.float32)
        past = [a.copy() for a in st]
        now = [a.copy() for a in st]
        prec = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
        oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec, nsteps, dtbig, dtsml, start=True,
                               prec_bits=bits, omp=True)
        runs[key] = (now, prec)
    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1, cphopt=3, thresq=1e-12, obc=obc, gwave=20.0, tubopt=tubopt)
    gpu, gprec, diag = _run_gpu(cress, case, names, init, s, nsteps, dtbig, dtsml, rbct, ksp0, True)

    i0 = 1 if obc else 2   # open x: the boundary columns are prognostic too
    sl = interior(ni, nj, nk, i0)
    ref, ref_prec = runs[64]
    o32, o32_prec = runs[32]
    rep = {"case": label, "grid": [ni - 3, nj - 3, nk - 3], "dx_m": dx, "open_x": obc, "steps": nsteps,
           "dtbig_s": dtbig, "simulated_s": nsteps * dtbig,
           "tubopt": tubopt, "fields": field_stats(names, gpu, ref, o32, sl), "max_w_gpu": diag["max_w"]}
    for n, r, o in zip(names, ref, runs["32p"][0]):
        r64 = r.astype(np.float64)[sl]
        d = o.astype(np.float64)[sl] - r64
        rep["fields"][n]["fp32p_rms_rel"] = float(np.sqrt(np.mean(d * d))) / rep["fields"][n]["fp64_rms"]
    acc = {k: float(v[:, 1, 2:nj - 1, i0:ni - 1].astype(np.float64).sum())
           for k, v in (("gpu", gprec), ("fp64", ref_prec), ("fp32", o32_prec))}
    rep["precip_accum_kg_m2"] = acc
    rep["precip_rel_diff_gpu"] = abs(acc["gpu"] - acc["fp64"]) / (abs(acc["fp64"]) + 1e-30)
    rep["precip_rel_diff_fp32"] = abs(acc["fp32"] - acc["fp64"]) / (abs(acc["fp64"]) + 1e-30)
    dzf = float(np.float32(dz))
    w0, m0 = moist_budgets(case, init, np.zeros_like(ref_prec), dx, dzf, i0)
    for key, f, p in (("gpu", gpu, gprec), ("fp64", ref, ref_prec), ("fp32", o32, o32_prec)):
        w, m = moist_budgets(case, f, p, dx, dzf, i0)
        rep[f"water_drift_{key}"] = (w - w0) / w0
        rep[f"mass_drift_{key}"] = (m - m0) / m0
    return rep


def dry_study(cress, oracle_lib, case, dx, dz, nsteps, dtbig, dtsml, tubopt=1, sthopt=0, label="dry"):
    """Dry (cphopt=0) run of `nsteps` large steps; returns the report.
    tubopt=2 (the TKE closure) starts from zero TKE and reports the TKE."""
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = _vsp(oracle_lib, nk, zph, case["vspbar"], case["botbar"])
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=sthopt, smtopt=3, vspopt=2, coropt=0,
               vspbar=case["vspbar"], botbar=case["botbar"], tubopt=tubopt, impopt=1)
    names = DRY + (["tke"] if tubopt == 2 else [])
    init = list(case["level"]) + ([_tke0(case)] if tubopt == 2 else [])
    runs = {}
    for bits in (64, 32):
        past = [a.copy() for a in init]
        now = [a.copy() for a in init]
        oracle_lib.dry_steps(cfg, case["base"], zph, past, now, nsteps, dtbig, dtsml, start=True, prec=bits,
                             omp=True)
        runs[bits] = now
    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=sthopt, tubopt=tubopt)
    gpu, _, diag = _run_gpu(cress, case, names, init, s, nsteps, dtbig, dtsml, rbct, ksp0, False)
    sl = interior(ni, nj, nk)
    rep = {"case": label, "grid": [ni - 3, nj - 3, nk - 3], "dx_m": dx, "dz_m": dz, "steps": nsteps,
           "dtbig_s": dtbig, "nsstp": nsstp_of(dtbig, dtsml), "simulated_s": nsteps * dtbig,
           "tubopt": tubopt, "fields": field_stats(names, gpu, runs[64], runs[32], sl), "max_w_gpu": diag["max_w"]}
    m0 = dry_mass(case, case["level"], dx, dz)
    for key, f in (("gpu", gpu), ("fp64", runs[64]), ("fp32", runs[32])):
        rep[f"mass_drift_{key}"] = (dry_mass(case, f, dx, dz) - m0) / m0
    return rep

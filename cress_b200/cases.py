"""Synthetic idealized cases: base state columns and initial perturbations.

The reference builds its base state on the host during s_inivar
(SrcOrig/inivar.f90:611-850): sounding -> hydrostatic 1-D profile (set1d)
-> 3-D base arrays (setbase, baserho, sndwave) and passes them to the
solver.  The C-ABI receives those arrays; this module produces them for
standalone runs and benchmarks, horizontally uniform (flat terrain), in the
reference layout a(0:ni+1, 0:nj+1, 1:nk) = numpy (nk, nj+2, ni+2).

Rules followed:
  rst = |jcb| * rbr                       SrcOrig/baserho.f90:160
  rst8w(k) = .5*(rst(k-1)+rst(k)), bc8w   SrcOrig/var8uvw.f90:190-196, SrcOrig/bc8w.f90:130-184
  rcsq = cp/cv * pbr                      SrcOrig/sndwave.f90:119
  rbr = pbr / (rd * ptvbr * pibr)         SrcOrig/setbase.f90:177-182
"""
import numpy as np

G, CP, CV, RD, RV, P0 = 9.8, 1004.0, 717.0, 287.0, 461.0, 1.0e5
BASE_NAMES = ["jcb", "jcb8u", "jcb8v", "jcb8w", "rbr", "ptbr", "rst", "rst8u", "rst8v",
              "rst8w", "rcsq"]


def dims(nx, ny, nz):
    """Array dims of an nx x ny x nz interior (SrcOrig/setdim.f90:196-199)."""
    return nx + 3, ny + 3, nz + 3


def stretched_jcb(nk, dz, dzmin):
    """Jacobian jcb(k) = dz_k/dz of a tanh-stretched grid with the lowest
    layer dzmin and mean spacing dz (top = dz*(nk-3))."""
    k = np.arange(nk + 1, dtype=np.float64)
    n = nk - 3
    s = np.linspace(0.0, 1.0, n)
    w = dzmin / dz + (2.0 - 2.0 * dzmin / dz) * s  # linear ramp, mean 1
    jcb = np.ones(nk + 1)
    jcb[2:2 + n] = w
    jcb[1] = jcb[2]
    jcb[nk - 1:] = jcb[nk - 2]
    return jcb


def base_columns(nk, dz, sthopt=0, dzmin=None, theta_sfc=300.0, dthdz=0.0, qv_sfc=0.0):
    """1-D base columns (index k = 1..nk) of a hydrostatic profile integrated
    in FP64 (Exner form) with theta(z) = theta_sfc + dthdz*z."""
    if sthopt:
        jcb = stretched_jcb(nk, dz, dzmin if dzmin else 0.4 * dz)
    else:
        jcb = np.ones(nk + 1)
    zw = np.zeros(nk + 1)
    for k in range(3, nk + 1):
        zw[k] = zw[k - 1] + jcb[k - 1] * dz
    zw[2] = 0.0
    zs = np.zeros(nk + 1)
    zs[1:nk] = 0.5 * (zw[1:nk] + zw[2:nk + 1])
    zs[1] = -zs[2]
    zs[nk] = zs[nk - 1] + jcb[nk - 1] * dz
    theta = theta_sfc + dthdz * zs
    # Exner integration d(pi)/dz = -g/(cp*theta), FP64 trapezoid from the surface
    pi = np.ones(nk + 1)
    pi_s = 1.0
    for k in range(1, nk + 1):
        pi[k] = pi_s - G * zs[k] / (CP * 0.5 * (theta_sfc + theta[k])) if dthdz else \
            pi_s - G * zs[k] / (CP * theta_sfc)
    pbr = P0 * pi ** (CP / RD)
    ptv = theta
    rbr = pbr / (RD * ptv * pi)
    f32 = lambda a: np.asarray(a, np.float32)
    c = {"jcb": f32(jcb), "ptbr": f32(theta), "pbr": f32(pbr), "rbr": f32(rbr),
         "zs": zs}
    return _derived_columns(c, nk)


def _derived_columns(c, nk):
    """rst, rcsq and the u/v/w-point averages of jcb and rst."""
    c["rst"] = (np.abs(c["jcb"]) * c["rbr"]).astype(np.float32)
    c["rcsq"] = (np.float32(CP / CV) * c["pbr"]).astype(np.float32)
    for name in ("jcb", "rst"):
        v8w = np.zeros(nk + 1, np.float32)
        for k in range(2, nk):
            v8w[k] = np.float32(0.5) * (c[name][k - 1] + c[name][k])
        v8w[1] = v8w[3]
        v8w[nk] = v8w[nk - 2]
        c[name + "8w"] = v8w
        c[name + "8u"] = (np.float32(0.5) * (c[name] + c[name])).astype(np.float32)
        c[name + "8v"] = c[name + "8u"].copy()
    return c


def power_stretched_jcb(nk, ztop, dzmin, dzmax):
    """Jacobian of a grid whose layer thickness grows from dzmin at the
    ground to dzmax at the lid as dz(s) = dzmin + (dzmax-dzmin)*s**p,
    s = 0..1 over the nz = nk-3 layers, p chosen so the layers sum to ztop.
    Returns (jcb(k), mean spacing dz = ztop/nz)."""
    n = nk - 3
    dz = ztop / n
    if not dzmin < dz < dzmax:
        raise ValueError(f"{n} layers of {dzmin}..{dzmax} m cannot reach {ztop} m")
    s = np.linspace(0.0, 1.0, n)
    lo, hi = 0.01, 20.0
    for _ in range(200):
        p = 0.5 * (lo + hi)
        tot = np.sum(dzmin + (dzmax - dzmin) * s ** p)
        lo, hi = (p, hi) if tot > ztop else (lo, p)
    jcb = np.ones(nk + 1)
    jcb[2:2 + n] = (dzmin + (dzmax - dzmin) * s ** p) * (ztop / tot) / dz
    jcb[1] = jcb[2]
    jcb[nk - 1:] = jcb[nk - 2]
    return jcb, dz


EPSVA = RD / RV


def moist_columns(nk, ztop=18000.0, dzmin=100.0, dzmax=500.0, theta_sfc=300.0, theta_tr=343.0,
                  z_tr=12000.0, t_tr=213.0, qv_max=0.014, p_sfc=1.0e5):
    """1-D base columns of the analytic supercell sounding on a stretched
    grid: theta = theta_sfc + (theta_tr-theta_sfc)*(z/z_tr)**1.25 below the
    tropopause z_tr, theta_tr*exp(g*(z-z_tr)/(cp*t_tr)) above; relative
    humidity 1 - 0.75*(z/z_tr)**1.25 (0.25 above z_tr); qv capped at qv_max.
    Hydrostatic in the virtual potential temperature, integrated in FP64
    (Exner form, midpoint rule, qv iterated with p).  The base density
    follows rbr = pbr/(rd*ptvbr*pibr), ptvbr = ptbr*(1+qvbr/epsva)/(1+qvbr)
    (SrcOrig/setbase.f90:153-189)."""
    jcb, dz = power_stretched_jcb(nk, ztop, dzmin, dzmax)
    zw = np.zeros(nk + 1)
    for k in range(3, nk + 1):
        zw[k] = zw[k - 1] + jcb[k - 1] * dz
    zs = np.zeros(nk + 1)
    zs[1:nk] = 0.5 * (zw[1:nk] + zw[2:nk + 1])
    zs[1] = -zs[2]
    zs[nk] = zs[nk - 1] + jcb[nk - 1] * dz

    def theta_of(z):
        z = np.asarray(z, np.float64)
        zc = np.clip(z, 0.0, None)
        below = theta_sfc + (theta_tr - theta_sfc) * (np.minimum(zc, z_tr) / z_tr) ** 1.25
        above = theta_tr * np.exp(G * (zc - z_tr) / (CP * t_tr))
        return np.where(zc <= z_tr, below, above)

    def rh_of(z):
        zc = np.clip(np.asarray(z, np.float64), 0.0, z_tr)
        return 1.0 - 0.75 * (zc / z_tr) ** 1.25

    def qv_of(z, pi):
        p = P0 * pi ** (CP / RD)
        t = theta_of(z) * pi
        return np.minimum(rh_of(z) * qvs_water(t, p), qv_max)

    thv = lambda th, qv: th * (1.0 + qv / EPSVA) / (1.0 + qv)
    pi = np.empty(nk + 1)
    pi_s = (p_sfc / P0) ** (RD / CP)
    # integrate from the ground (z = 0) to each scalar level
    order = np.argsort(zs[1:]) + 1
    z_prev, pi_prev = 0.0, pi_s
    for k in [k for k in order if zs[k] >= 0.0]:
        z0, z1 = z_prev, zs[k]
        guess = pi_prev
        for _ in range(8):
            zm, pm = 0.5 * (z0 + z1), 0.5 * (pi_prev + guess)
            guess = pi_prev - G * (z1 - z0) / (CP * thv(theta_of(zm), qv_of(zm, pm)))
        pi[k] = guess
        z_prev, pi_prev = z1, guess
    k1 = 1   # the level below the ground, mirrored
    guess = pi_s
    for _ in range(8):
        zm, pm = 0.5 * zs[k1], 0.5 * (pi_s + guess)
        guess = pi_s - G * zs[k1] / (CP * thv(theta_of(zm), qv_of(zm, pm)))
    pi[k1] = guess
    pi[0] = pi[1]
    theta = theta_of(zs)
    qv = qv_of(zs, pi)
    pbr = P0 * pi ** (CP / RD)
    rbr = pbr / (RD * thv(theta, qv) * pi)
    f32 = lambda a: np.asarray(a, np.float32)
    c = {"jcb": f32(jcb), "ptbr": f32(theta), "pbr": f32(pbr), "rbr": f32(rbr), "qvbr": f32(qv),
         "zs": zs, "zph": np.where(np.arange(nk + 1) == 1, -zw[3], zw), "dz": dz}
    return _derived_columns(c, nk)


def expand(colk, ni, nj, nk):
    a = np.empty((nk, nj + 2, ni + 2), np.float32)
    a[:] = np.asarray(colk, np.float32)[1:nk + 1, None, None]
    return a


def base3d(ni, nj, nk, dz, **kw):
    c = base_columns(nk, dz, **kw)
    return {n: expand(c[n], ni, nj, nk) for n in BASE_NAMES + ["pbr"]}, c


def bcycle(a, stag):
    """Periodic wrap of SrcOrig/bcycle.f90:159-225 (plus the identity of the
    duplicated face u(ni-1)=u(2), v(nj-1)=v(2) of a periodic domain)."""
    nk, nj2, ni2 = a.shape
    ni, nj = ni2 - 2, nj2 - 2
    if stag == "u":
        a[:, :, ni - 1] = a[:, :, 2]
        a[:, :, 1] = a[:, :, ni - 2]
        a[:, :, ni] = a[:, :, 3]
    else:
        a[:, :, 1] = a[:, :, ni - 2]
        a[:, :, ni - 1] = a[:, :, 2]
    if stag == "v":
        a[:, nj - 1, :] = a[:, 2, :]
        a[:, 1, :] = a[:, nj - 2, :]
        a[:, nj, :] = a[:, 3, :]
    else:
        a[:, 1, :] = a[:, nj - 2, :]
        a[:, nj - 1, :] = a[:, 2, :]
    return a


def _wrap_index(n, stag_axis):
    """Source index of every position along one axis under the periodic wrap
    of both ghost layers (bcycle + shift2nd planes): interior 2..n-2, period
    n-3; the staggered axis also wraps n-1 (the duplicated face) and n+1."""
    P = n - 3
    src = np.arange(n + 2)
    ghosts = [0, 1, n, n + 1, n - 1] if stag_axis else [0, 1, n - 1, n]
    for g_ in ghosts:
        src[g_] = 2 + (g_ - 2) % P
    return src


def periodic_fill(a, stag):
    """Fill both periodic ghost layers of a (nk, nj+2, ni+2) array."""
    nk, nj2, ni2 = a.shape
    ni, nj = ni2 - 2, nj2 - 2
    sx = _wrap_index(ni, stag == "u")
    sy = _wrap_index(nj, stag == "v")
    a[:] = a[:, sy][:, :, sx]
    return a


def dry_case(nx, ny, nz, dx, dz, sthopt=1, seed=0, ptp0=2.0, rad=None, u0=5.0, shear=10.0,
             vspbar=0.0, botbar=1e9, noise=0.01, dthdz=0.003):
    """Dry warm-bubble state for whole large steps.

    Base wind ubr = u0 + shear * z/ztop (v = 0), theta'(bubble) = ptp0*cos^2 inside
    the ellipsoid of radius `rad` (m, x/y/z) centred at mid-domain, z = 1.5 km,
    plus seeded uniform +-noise K.  Returns a dict with dims, base (3-D
    arrays incl. ubr, vbr), zph (w-level heights, index k), rbct/ksp0 left
    for the caller (see oracle.vspdmp) and the initial level (past = now)."""
    ni, nj, nk = dims(nx, ny, nz)
    base, cols = base3d(ni, nj, nk, dz, sthopt=sthopt, dthdz=dthdz)
    jcb = cols["jcb"].astype(np.float64)
    zph = np.zeros(nk + 1)
    for k in range(3, nk + 1):
        zph[k] = zph[k - 1] + jcb[k - 1] * dz
    zph[1] = -zph[3]
    ztop = zph[nk - 1]
    zs = cols["zs"]
    ubr_col = (u0 + shear * np.clip(zs / ztop, 0.0, 1.0)).astype(np.float32)
    base["ubr"] = expand(ubr_col, ni, nj, nk)
    base["vbr"] = np.zeros_like(base["ubr"])
    rng = np.random.default_rng(seed)
    shp = (nk, nj + 2, ni + 2)
    if rad is None:
        rad = (min(nx, ny) * dx / 6.0, min(nx, ny) * dx / 6.0, 1500.0)
    x = (np.arange(ni + 2) - 0.5 * (ni + 1)) * dx
    y = (np.arange(nj + 2) - 0.5 * (nj + 1)) * dx
    z = zs[1:nk + 1]
    r = np.sqrt((x[None, None, :] / rad[0]) ** 2 + (y[None, :, None] / rad[1]) ** 2 +
                ((z[:, None, None] - 1500.0) / rad[2]) ** 2)
    ptp = np.where(r < 1.0, ptp0 * np.cos(0.5 * np.pi * r) ** 2, 0.0)
    ptp = (ptp + rng.uniform(-noise, noise, shp)).astype(np.float32)
    u = base["ubr"].copy()
    v = np.zeros(shp, np.float32)
    w = np.zeros(shp, np.float32)
    pp = np.zeros(shp, np.float32)
    level = [periodic_fill(u, "u"), periodic_fill(v, "v"), periodic_fill(w, "s"),
             periodic_fill(pp, "s"), periodic_fill(ptp, "s")]
    return dict(dims=(ni, nj, nk), base=base, cols=cols, zph=zph, level=level,
                vspbar=vspbar, botbar=botbar)


MOIST_NAMES = ["qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def supercell_case(nx, ny, nz, dx, ztop=18000.0, dzmin=100.0, dzmax=500.0, seed=0, ptp0=3.0,
                   rad=(10000.0, 10000.0, 1400.0), zc=1400.0, shear=30.0, rcirc=7.0,
                   noise=0.0, cloud=False, center=(0.0, 0.0)):
    """Moist supercell state (cold-rain microphysics, cphopt=3).

    Base state: the analytic sounding of moist_columns on a grid stretched
    from dzmin to dzmax up to ztop; quarter-circle hodograph of radius rcirc
    over 0-2 km continuing straight to `shear` m/s of u at 6 km (constant
    above).  Perturbation: +ptp0 K cos^2 ellipsoidal bubble of radii `rad`
    centred at mid-domain shifted by `center` (m), height zc, plus seeded
    uniform +-noise K.  With
    cloud=True a seeded field of cloud, rain, ice, snow and graupel (with
    ice numbers) and supersaturated pockets is added so every microphysical
    process acts from the first step.  Returns a dict with dims, base (3-D,
    incl. ubr, vbr, pbr, qvbr), cols, zph, dz (mean spacing), level (u, v,
    w, pp, ptp) and moist (qv ... ng), past = present."""
    ni, nj, nk = dims(nx, ny, nz)
    cols = moist_columns(nk, ztop, dzmin, dzmax)
    base = {n: expand(cols[n], ni, nj, nk) for n in BASE_NAMES + ["pbr", "qvbr"]}
    zs = cols["zs"]
    th = 0.5 * np.pi * np.clip(zs / 2000.0, 0.0, 1.0)
    u = np.where(zs < 2000.0, rcirc * (1.0 - np.cos(th)),
                 rcirc + (shear - rcirc) * np.clip((zs - 2000.0) / 4000.0, 0.0, 1.0))
    v = rcirc * np.sin(th)
    base["ubr"] = expand(u.astype(np.float32), ni, nj, nk)
    base["vbr"] = expand(v.astype(np.float32), ni, nj, nk)
    rng = np.random.default_rng(seed)
    shp = (nk, nj + 2, ni + 2)
    x = (np.arange(ni + 2) - 0.5 * (ni + 1)) * dx - center[0]
    y = (np.arange(nj + 2) - 0.5 * (nj + 1)) * dx - center[1]
    z = zs[1:nk + 1]
    r = np.sqrt((x[None, None, :] / rad[0]) ** 2 + (y[None, :, None] / rad[1]) ** 2 +
                ((z[:, None, None] - zc) / rad[2]) ** 2)
    ptp = np.where(r < 1.0, ptp0 * np.cos(0.5 * np.pi * r) ** 2, 0.0)
    if noise:
        ptp = ptp + rng.uniform(-noise, noise, shp)
    level = [base["ubr"].copy(), base["vbr"].copy(), np.zeros(shp, np.float32),
             np.zeros(shp, np.float32), ptp.astype(np.float32)]
    moist = {n: np.zeros(shp, np.float32) for n in MOIST_NAMES}
    moist["qv"] = base["qvbr"].copy()
    if cloud:
        zz = z[:, None, None]
        pbr = base["pbr"].astype(np.float64)
        t = (base["ptbr"] * (pbr / P0) ** (RD / CP)).astype(np.float64)

        def blob(lo, hi, zlo, zhi, amp):
            b = np.clip((_noise(rng, shp, 1.0) - lo) / (hi - lo), 0.0, 1.0)
            return amp * b * ((zz > zlo) & (zz < zhi))

        moist["qv"] = np.minimum((0.8 + 0.3 * _noise(rng, shp, 1.0)) * qvs_water(t, pbr), 0.02)
        moist["qc"] = blob(0.0, 0.6, 500.0, 9000.0, 1.5e-3)
        moist["qr"] = blob(0.1, 0.8, 0.0, 6000.0, 2.0e-3)
        moist["qi"] = blob(0.0, 0.7, 6000.0, 14000.0, 3.0e-4)
        moist["qs"] = blob(0.0, 0.7, 4500.0, 12000.0, 1.0e-3)
        moist["qg"] = blob(0.1, 0.8, 3000.0, 10000.0, 1.5e-3)
        moist["ni"] = moist["qi"] / 1.0e-11 * (0.5 + rng.random(shp))
        moist["ns"] = moist["qs"] / 5.0e-9 * (0.5 + rng.random(shp))
        moist["ng"] = moist["qg"] / 5.0e-8 * (0.5 + rng.random(shp))
    stag = ["u", "v", "s", "s", "s"]
    level = [periodic_fill(np.asarray(a, np.float32), s) for a, s in zip(level, stag)]
    moist = {n: periodic_fill(np.asarray(a, np.float32), "s") for n, a in moist.items()}
    return dict(dims=(ni, nj, nk), base=base, cols=cols, zph=cols["zph"], dz=cols["dz"],
                level=level, moist=moist)


def squall_case(nx, ny, nz, dx=500.0, ztop=18000.0, dzmin=100.0, dzmax=500.0, seed=0, ptp0=2.0,
                shear=20.0, zshear=2500.0, xrad=5000.0, zrad=1400.0, zc=1400.0, noise=0.1,
                x0=0.0, umove=0.0):
    """Squall-line state (cold-rain microphysics, open x, periodic y).

    Base state: the analytic sounding of moist_columns; unidirectional
    low-level shear, u = shear * min(z / zshear, 1) - umove, v = 0 (umove,
    a domain translation, keeps the line inside a reduced domain without
    changing the shear).  Perturbation:
    a line thermal along y of +ptp0 K, cos^2 in x (half width xrad, centred
    x0 m from mid-domain) and z (half depth zrad at height zc), plus seeded
    uniform +-noise K inside it.  Moisture: qv at the base value, no
    hydrometeors.  Same dict layout as supercell_case."""
    ni, nj, nk = dims(nx, ny, nz)
    cols = moist_columns(nk, ztop, dzmin, dzmax)
    base = {n: expand(cols[n], ni, nj, nk) for n in BASE_NAMES + ["pbr", "qvbr"]}
    zs = cols["zs"]
    u = shear * np.clip(zs / zshear, 0.0, 1.0) - umove
    base["ubr"] = expand(u.astype(np.float32), ni, nj, nk)
    base["vbr"] = expand(np.zeros_like(u, dtype=np.float32), ni, nj, nk)
    rng = np.random.default_rng(seed)
    shp = (nk, nj + 2, ni + 2)
    x = (np.arange(ni + 2, dtype=np.float64) - 0.5 * (ni + 1)) * dx - x0
    z = zs[1:nk + 1]
    r = np.sqrt((x[None, :] / xrad) ** 2 + ((z[:, None] - zc) / zrad) ** 2)   # (nk, ni+2)
    line = np.where(r < 1.0, ptp0 * np.cos(0.5 * np.pi * r) ** 2, 0.0).astype(np.float32)
    ptp = np.broadcast_to(line[:, None, :], shp).copy()
    if noise:
        inside = np.broadcast_to((r < 1.0)[:, None, :], shp)
        ptp += np.where(inside, rng.uniform(-noise, noise, shp).astype(np.float32), np.float32(0))
    level = [base["ubr"].copy(), base["vbr"].copy(), np.zeros(shp, np.float32),
             np.zeros(shp, np.float32), ptp]
    moist = {n: np.zeros(shp, np.float32) for n in MOIST_NAMES}
    moist["qv"] = base["qvbr"].copy()
    stag = ["u", "v", "s", "s", "s"]
    level = [periodic_fill(np.asarray(a, np.float32), s) for a, s in zip(level, stag)]
    moist = {n: periodic_fill(np.asarray(a, np.float32), "s") for n, a in moist.items()}
    return dict(dims=(ni, nj, nk), base=base, cols=cols, zph=cols["zph"], dz=cols["dz"],
                level=level, moist=moist)


def qvs_water(t, p):
    """Saturation mixing ratio over water, Tetens form of SrcOrig/setblk.f90:333,338."""
    esw = 610.78 * np.exp(17.269 * (t - 273.16) / (t - 35.86))
    return 0.622 * esw / (p - esw)


def micro_case(nx, ny, nz, dz, seed=0, sthopt=1):
    """A moist, cloudy state for the cold-rain microphysics: past and future
    levels of theta', qv, qc, qr, qi, qs, qg, ni, ns, ng (plus the past p')
    spanning warm rain below the melting level, mixed phase above it and
    cold ice aloft, sub- and super-saturated air.  Seeded; fields are
    periodic-consistent.  Returns dims, base (ptbr, rbr, pbr, jcb, rst),
    past, fut dicts."""
    ni, nj, nk = dims(nx, ny, nz)
    b3, cols = base3d(ni, nj, nk, dz, sthopt=sthopt, dthdz=0.004)
    rng = np.random.default_rng(seed)
    shp = (nk, nj + 2, ni + 2)
    zs = cols["zs"][1:nk + 1][:, None, None]
    pbr = b3["pbr"].astype(np.float64)
    pi = (pbr / 1.0e5) ** (287.0 / 1004.0)
    t = b3["ptbr"] * pi

    def field(lo, hi, zlo, zhi, amp):
        x = _noise(rng, shp, 1.0)
        blob = np.clip((x - lo) / (hi - lo), 0.0, 1.0)
        band = ((zs > zlo) & (zs < zhi)).astype(np.float64)
        return amp * blob * band

    rh = 0.75 + 0.35 * _noise(rng, shp, 1.0)
    qv = np.minimum(rh * qvs_water(t, pbr), 0.02)
    qc = field(0.0, 0.6, 500.0, 9000.0, 2.0e-3)
    qr = field(0.1, 0.8, 0.0, 6000.0, 3.0e-3)
    qi = field(0.0, 0.7, 6000.0, 14000.0, 5.0e-4)
    qs = field(0.0, 0.7, 4500.0, 12000.0, 1.5e-3)
    qg = field(0.1, 0.8, 3000.0, 10000.0, 2.5e-3)
    rbr = b3["rbr"].astype(np.float64)
    ni_ = qi / 1.0e-11 * (0.5 + rng.random(shp))
    ns_ = qs / 5.0e-9 * (0.5 + rng.random(shp))
    ng_ = qg / 5.0e-8 * (0.5 + rng.random(shp))
    ptp = 0.5 * _noise(rng, shp, 1.0)
    pp = 30.0 * _noise(rng, shp, 1.0)
    past = dict(ptp=ptp, qv=qv, qc=qc, qr=qr, qi=qi, qs=qs, qg=qg, ni=ni_, ns=ns_, ng=ng_, pp=pp)
    past = {k: periodic_fill(np.asarray(v, np.float32), "s") for k, v in past.items()}
    fut = {}
    for k in ("ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"):
        v = past[k].astype(np.float64)
        if k == "ptp":
            v = v + 0.1 * _noise(rng, shp, 1.0)
        else:
            v = np.maximum(v * (1.0 + 0.1 * _noise(rng, shp, 1.0)), 0.0)
        fut[k] = periodic_fill(np.asarray(v, np.float32), "s")
    base = dict(b3)
    base["qvbr"] = np.zeros_like(b3["pbr"])
    return (ni, nj, nk), base, past, fut, cols


def _noise(rng, shape, amp):
    x = rng.standard_normal(shape)
    for ax in (1, 2):
        x = (x + np.roll(x, 1, ax) + np.roll(x, -1, ax)) / 3.0
    return (amp * x / (np.abs(x).max() + 1e-30)).astype(np.float32)


def acoustic_case(nx, ny, nz, dx, dz, seed=0, sthopt=1):
    """A perturbed dry state for the small step: past-level u, v, w, p' and
    the large-step forcings ufrc, vfrc, wfrc, pfrc (seeded, periodic)."""
    ni, nj, nk = dims(nx, ny, nz)
    base, cols = base3d(ni, nj, nk, dz, sthopt=sthopt, dthdz=0.003)
    rng = np.random.default_rng(seed)
    shp = (nk, nj + 2, ni + 2)
    u = _noise(rng, shp, 6.0) + np.float32(8.0)
    v = _noise(rng, shp, 6.0) - np.float32(2.0)
    w = _noise(rng, shp, 1.5)
    pp = _noise(rng, shp, 40.0)
    w[1] = 0.0
    w[nk - 2] = 0.0
    rst = base["rst"]
    frc = [_noise(rng, shp, 2e-3) * rst, _noise(rng, shp, 2e-3) * rst,
           _noise(rng, shp, 4e-3) * rst, _noise(rng, shp, 0.3)]
    st = [u, v, w, pp]
    for a, t in zip(st + frc, ["u", "v", "s", "s", "u", "v", "s", "s"]):
        bcycle(a, t)
    return (ni, nj, nk), base, st, frc

"""Shared test helpers: seeded synthetic base states and perturbation fields.

Arrays follow the reference layout a(0:ni+1, 0:nj+1, 1:nk): numpy shape
(nk, nj+2, ni+2), x fastest.  Base states are horizontally uniform (flat
terrain, idealized soundings) and built with the interpolation rules of
SrcOrig/var8uvw.f90:166-202 and SrcOrig/bc8w.f90:130-184 so the 3-D arrays
look like the reference's after s_baserho.
"""
import numpy as np

G, CP, CV, RD, P0 = 9.8, 1004.0, 717.0, 287.0, 1.0e5


def dims(nx, ny, nz):
    return nx + 3, ny + 3, nz + 3


def columns(nk, dz, sthopt=0, theta0=300.0, stretch=0.35):
    """1-D base columns (index k = 1..nk at position k, position 0 unused)."""
    k = np.arange(nk + 1, dtype=np.float64)
    if sthopt:
        # a smooth stretching: jcb = dz_k/dz varies between 1-stretch and 1+stretch
        jcb = 1.0 + stretch * np.tanh((k - nk / 2.0) / (nk / 4.0))
    else:
        jcb = np.ones(nk + 1)
    # heights of scalar levels: z = cumulative sum of jcb*dz, level 2 at 0.5*jcb*dz
    zs = np.zeros(nk + 1)
    for kk in range(2, nk + 1):
        zs[kk] = zs[kk - 1] + 0.5 * (jcb[kk - 1] + jcb[kk]) * dz if kk > 2 else 0.5 * jcb[2] * dz
    zs[1] = -zs[2]
    theta = theta0 + 0.003 * zs                    # mildly stable
    pi = 1.0 - G * zs / (CP * theta0)
    pbr = P0 * pi ** (CP / RD)
    rbr = pbr / (RD * theta * pi)
    c = {}
    f32 = lambda a: a.astype(np.float32)
    c["jcb"] = f32(jcb)
    c["ptbr"] = f32(theta)
    c["pbr"] = f32(pbr)
    c["rbr"] = f32(rbr)
    c["rst"] = (np.abs(c["jcb"]) * c["rbr"]).astype(np.float32)           # baserho.f90:160
    c["rcsq"] = (np.float32(CP / CV) * c["pbr"]).astype(np.float32)        # sndwave.f90:119
    for name in ("jcb", "rst"):
        v8w = np.zeros(nk + 1, np.float32)
        for kk in range(2, nk):                                            # var8uvw.f90:190-196
            v8w[kk] = np.float32(0.5) * (c[name][kk - 1] + c[name][kk])
        v8w[1] = v8w[3]                                                    # bc8w.f90:136
        v8w[nk] = v8w[nk - 2]                                              # bc8w.f90:166
        c[name + "8w"] = v8w
        c[name + "8u"] = (np.float32(0.5) * (c[name] + c[name])).astype(np.float32)
        c[name + "8v"] = c[name + "8u"].copy()
    return c


def expand(colk, ni, nj, nk):
    """1-D column (index k) -> horizontally uniform 3-D array."""
    a = np.empty((nk, nj + 2, ni + 2), np.float32)
    a[:] = colk[1:nk + 1, None, None]
    return a


def base3d(ni, nj, nk, dz, sthopt=0):
    c = columns(nk, dz, sthopt)
    return {n: expand(c[n], ni, nj, nk) for n in
            ("jcb", "jcb8u", "jcb8v", "jcb8w", "rbr", "ptbr", "rst", "rst8u", "rst8v", "rst8w",
             "rcsq", "pbr")}


def bcycle(a, stag):
    """Periodic wrap of SrcOrig/bcycle.f90:159-225 on a (nk, nj+2, ni+2) array."""
    nk, nj2, ni2 = a.shape
    ni, nj = ni2 - 2, nj2 - 2
    if stag == "u":
        iw, ir, ie, ier = 3, 1, ni - 2, ni
    else:
        iw, ir, ie, ier = 2, 1, ni - 2, ni - 1
    if stag == "v":
        js, jr, jn, jnr = 3, 1, nj - 2, nj
    else:
        js, jr, jn, jnr = 2, 1, nj - 2, nj - 1
    # On a periodic domain the face u(ni-1) is the face u(2) (and v(nj-1) is
    # v(2)); the reference keeps them equal because both are updated by the
    # same formula from wrapped inputs.  Enforce it on synthetic inputs.
    if stag == "u":
        a[:, :, ni - 1] = a[:, :, 2]
    if stag == "v":
        a[:, nj - 1, :] = a[:, 2, :]
    a[:, :, ir] = a[:, :, ie]
    a[:, :, ier] = a[:, :, iw]
    a[:, jr, :] = a[:, jn, :]
    a[:, jnr, :] = a[:, js, :]
    return a


def smooth_noise(rng, shape, amp, scale=3):
    """Random field with some spatial smoothness (box-filtered white noise)."""
    x = rng.standard_normal(shape)
    for ax in (1, 2):
        y = x.copy()
        for s in range(1, scale):
            y += np.roll(x, s, axis=ax) + np.roll(x, -s, axis=ax)
        x = y / (2 * scale - 1)
    return (amp * x / (np.abs(x).max() + 1e-30)).astype(np.float32)


def small_state(ni, nj, nk, seed=0, base=None):
    """Past-level u, v, w, p' and the four forcings of a perturbed state.

    Ghosts are periodic-consistent (as the reference's are after bcycle) and
    the rigid-lid levels of w are zero."""
    rng = np.random.default_rng(seed)
    shp = (nk, nj + 2, ni + 2)
    u = smooth_noise(rng, shp, 8.0) + np.float32(5.0)
    v = smooth_noise(rng, shp, 8.0) - np.float32(3.0)
    w = smooth_noise(rng, shp, 2.0)
    pp = smooth_noise(rng, shp, 60.0)
    w[1] = 0.0            # k = 2 (bottom, rigid)
    w[nk - 2] = 0.0       # k = nk-1 (top, rigid)
    rst = base["rst"] if base is not None else np.ones(shp, np.float32)
    ufrc = smooth_noise(rng, shp, 2e-3) * rst
    vfrc = smooth_noise(rng, shp, 2e-3) * rst
    wfrc = smooth_noise(rng, shp, 5e-3) * rst
    pfrc = smooth_noise(rng, shp, 0.5)
    for a, st in ((u, "u"), (v, "v"), (w, "s"), (pp, "s"), (ufrc, "u"), (vfrc, "v"),
                  (wfrc, "s"), (pfrc, "s")):
        bcycle(a, st)
    return [u, v, w, pp], [ufrc, vfrc, wfrc, pfrc]


def interior_mask(ni, nj, nk, stag):
    """Region of a small-step output that the reference defines: layer-1
    ghosts included, layer-2 ghosts (i=0, ni+1, ...) excluded."""
    m = np.zeros((nk, nj + 2, ni + 2), bool)
    ih = ni if stag == "u" else ni - 1
    jh = nj if stag == "v" else nj - 1
    m[:, 1:jh + 1, 1:ih + 1] = True
    return m

"""GPU parity of open (radiation) west and east boundaries against the CPU
oracle: wbc = ebc = 7 (constant phase speed gwave), 4 (phase speed per
point from three time levels) and 5 (its column average), periodic y.

A moist supercell state is advanced a few leapfrog steps by
cress_large_step and by the oracle's restatement (s_rbcu/v/w/ss in every
acoustic substep, s_rbcpt/qv/q/s in the leapfrog step, s_phasev after the
Asselin filter, the 4th-order stencils narrowed at the boundary columns).
Both time levels of all 14 fields must agree on the interior and on the
boundary columns (u: i = 1 and ni; the rest: i = 1 and ni-1), with the
tolerance of the periodic moist parity test (FP32 with FMA contraction
and the CUDA math library against glibc without contraction):
99.9% of cells within 1e-4 of the field's maximum, every cell within 1e-2.
"""
import numpy as np
import pytest

from test_moist_gpu import FLOOR, NAMES

pytestmark = pytest.mark.gpu


def region(name, ni, nj, nk):
    m = np.zeros((nk, nj + 2, ni + 2), bool)
    i1 = ni if name == "u" else ni - 1
    j1 = nj - 1 if name == "v" else nj - 2
    k1 = nk if name == "w" else nk - 1
    m[0:k1, 2:j1 + 1, 1:i1 + 1] = True
    return m


def run_case(cress, oracle_lib, obc, nx=40, ny=24, nz=22, nsteps=5, seed=5, dtbig=5.0, dtsml=1.0, dry=False,
             tile=0):
    from cress_b200 import cases
    dx = 1000.0
    case = cases.supercell_case(nx, ny, nz, dx, ztop=8000.0, seed=seed, cloud=not dry,
                                rad=(5000.0, 5000.0, 1400.0))
    ni, nj, nk = case["dims"]
    dz, zph = case["dz"], case["zph"]
    vspbar, botbar = 0.005, 0.6 * zph[nk - 1]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, vspbar, botbar)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=1, smtopt=3, vspopt=2, coropt=0,
               vspbar=vspbar, botbar=botbar, thresq=1e-12, obc=obc, gwave=20.0)
    names = NAMES[:5] if dry else NAMES
    init = list(case["level"]) + ([] if dry else [case["moist"][n] for n in NAMES[5:]])
    past = [a.copy() for a in init]
    now = [a.copy() for a in init]
    prec_ref = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
    if dry:
        oracle_lib.dry_steps(cfg, case["base"], zph, past, now, nsteps, dtbig, dtsml, start=True)
    else:
        oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec_ref, nsteps, dtbig, dtsml, start=True)

    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1, cphopt=0 if dry else 3, thresq=1e-12, obc=obc,
                     gwave=20.0, tile=tile)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    if not dry:
        s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
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
    prec = None if dry else s.get_precip()
    s.close()
    return (ni, nj, nk), names, (past, now, prec_ref), (gp, gn, prec)


def check(dims, names, ref, got):
    ni, nj, nk = dims
    for lvl in range(2):
        for name, r, g in zip(names, ref[lvl], got[lvl]):
            m = region(name, ni, nj, nk)
            floor = FLOOR.get(name, 0.0)
            scale = float(np.abs(r[m]).max()) + 1e-30
            err = np.maximum(np.abs(g[m] - r[m]) - floor, 0.0)
            assert np.isfinite(g[m]).all(), (lvl, name)
            frac = float((err <= 1e-4 * scale).mean())
            emax = float(err.max()) / (scale + floor)
            assert frac >= 0.999, f"level {lvl} {name}: only {frac:.4f} within 1e-4 (max rel {emax:.2e})"
            assert emax <= 1e-2, f"level {lvl} {name}: max rel err {emax:.2e}"
            # the boundary columns themselves (u: 1 and ni; the rest: 1 and ni-1)
            ie = ni if name == "u" else ni - 1
            for i in (1, ie):
                bc = np.abs(g[:nk - 1, 2:nj - 1, i] - r[:nk - 1, 2:nj - 1, i]) - floor
                assert float(bc.max()) <= 1e-2 * (scale + floor), (lvl, name, i)
    if got[2] is not None:
        sl = (slice(None), 1, slice(2, nj - 1), slice(1, ni))
        pr, pg = ref[2][sl], got[2][sl]
        assert np.isfinite(pg).all()
        assert float(np.abs(pg - pr).max()) <= 1e-3 * float(np.abs(pr).max()) + 1e-9


@pytest.mark.parametrize("obc,tile", [(7, 0), (4, 0), (5, 0), (4, 11), (4, 12), (4, 13)])
def test_open_x_moist_steps(cress, oracle_lib, obc, tile):
    # tile 11: the HE-VI variant with the level table in global memory;
    # tile 12: the column kept on chip
    dims, names, ref, got = run_case(cress, oracle_lib, obc, tile=tile)
    check(dims, names, ref, got)


def test_open_x_dry_steps_ragged(cress, oracle_lib):
    # nx not a multiple of the 32-column tiles: the east boundary falls inside a tile
    dims, names, ref, got = run_case(cress, oracle_lib, 4, nx=45, ny=19, nz=20, nsteps=6, dry=True)
    check(dims, names, ref, got)


def test_open_x_differs_from_periodic(cress, oracle_lib):
    """The open run is not the periodic one: its boundary columns carry
    radiated values (the outflow side loses the bubble's signal)."""
    _, _, _, open_ = run_case(cress, oracle_lib, 7, nsteps=4)
    dims, _, _, per = run_case(cress, oracle_lib, 0, nsteps=4)
    ni = dims[0]
    d = np.abs(open_[1][0][:, :, 1:ni] - per[1][0][:, :, 1:ni]).max()
    assert d > 1e-3


def test_phase_speeds_option7_and_restart_round_trip(cress, oracle_lib):
    """With wbc = ebc = 7 the phase speeds after a step are the constant
    gwave*dtb/dx, clipped at 1, scaled by dts/dtb for u, v, w, p' (phvuvw /
    phvs), float for float; cress_put_phase / cress_get_phase round-trip the
    reference's ucpx(1:nj,1:nk,1:2) layout."""
    from cress_b200 import cases
    case = cases.squall_case(40, 16, 20, 500.0, ztop=8000.0, seed=3)
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    s = cress.Solver(ni, nj, nk, 500.0, 500.0, case["dz"], sthopt=1, cphopt=3, obc=7, gwave=30.0)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    for n, a in zip(NAMES, list(case["level"]) + [case["moist"][m] for m in NAMES[5:]]):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    assert not s.get_phase("u").any()   # zero on a fresh start
    dtb, dts = np.float32(3.0), np.float32(0.5)
    s.large_step(0, 1.5, 12, 0.25)
    s.large_step(3000, float(dtb), 12, float(dts))
    gw = np.float32(30.0) * dtb * (np.float32(1.0) / np.float32(500.0))
    west, east = np.maximum(-gw, np.float32(-1.0)), np.minimum(gw, np.float32(1.0))
    for name, sml, kend in (("u", True, nk - 2), ("w", True, nk - 1), ("pp", True, nk - 2), ("ptp", False, nk - 2),
                            ("qr", False, nk - 2)):
        c = s.get_phase(name)   # (side, k-1, j-1)
        scale = dts / dtb if sml else np.float32(1.0)
        wv, ev = (west * scale, east * scale) if sml else (west, east)
        assert np.all(c[0, 1:kend, 0:nj - 1] == wv), name
        assert np.all(c[1, 1:kend, 0:nj - 1] == ev), name
    rng = np.random.default_rng(0)
    x = rng.uniform(-0.3, 0.3, (2, nk, nj)).astype(np.float32)
    s.put_phase("v", x)
    assert np.array_equal(s.get_phase("v"), x)
    s.close()


def test_open_x_rejects_other_tiles(cress):
    from cress_b200 import cases
    case = cases.dry_case(40, 30, 20, 1000.0, 300.0, sthopt=1, seed=1)
    ni, nj, nk = case["dims"]
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, 300.0, sthopt=1, obc=7, tile=3)
    s.set_base3d(case["base"])
    with pytest.raises(cress.CressError) as e:
        s.small_steps(2, 0.5)
    assert e.value.code == 2 and "tiles 0, 11, 12 and 13" in str(e.value)
    s.close()

"""GPU parity of the fused HE-VI small step against the CPU oracle.

Tolerance: the GPU path computes in FP32 with fused multiply-adds and
solves the w tridiagonal in FP64; the oracle restates the reference in FP32
(fp64_solve=1 matches the GPU's solve).  Per-substep agreement is then set
by float rounding; after n substeps we allow
    max |gpu - oracle| <= 2e-5 * (n + 1) * max|oracle| (per field),
and require the FP32-vs-FP64 oracle spread to be of the same order.
"""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

STAG = {"u": "u", "v": "v", "w": "s", "pp": "s"}


def run_pair(cress, oracle_lib, nx, ny, nz, nsstp, sthopt=0, seed=1, dts=0.5, tile=0, dx=1000.0,
             dz=250.0, impopt=1, divopt=2):
    ni, nj, nk = H.dims(nx, ny, nz)
    base = H.base3d(ni, nj, nk, dz, sthopt)
    st, frc = H.small_state(ni, nj, nk, seed, base)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=sthopt, divopt=divopt, buyopt=1,
               weicoe=0.6, impopt=impopt)
    ref = [a.copy() for a in st]
    oracle_lib.small_steps(cfg, base, frc, ref, nsstp, dts, prec=32, fp64_solve=1)
    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=sthopt, tile=tile, impopt=impopt, divopt=divopt)
    s.set_base3d(base)
    out = s.smalldrv(nsstp, dts, *st, *frc)
    s.close()
    return ni, nj, nk, ref, out


def check(ni, nj, nk, ref, out, nsstp, rtol=2e-5):
    for name, r, g in zip(("u", "v", "w", "pp"), ref, out):
        m = H.interior_mask(ni, nj, nk, STAG[name])
        scale = float(np.abs(r[m]).max()) + 1e-30
        err = float(np.abs(g[m] - r[m]).max())
        assert np.isfinite(g[m]).all(), name
        assert err <= rtol * (nsstp + 1) * scale, f"{name}: max err {err:.3e} scale {scale:.3e}"


@pytest.mark.parametrize("sthopt", [0, 1])
def test_one_substep(cress, oracle_lib, sthopt):
    ni, nj, nk, ref, out = run_pair(cress, oracle_lib, 64, 48, 40, 1, sthopt=sthopt)
    check(ni, nj, nk, ref, out, 1)


@pytest.mark.parametrize("tile", list(range(14)))
def test_ragged_domain_tiles(cress, oracle_lib, tile):
    # nx, ny not multiples of the tile: partial edge tiles on both axes
    ni, nj, nk, ref, out = run_pair(cress, oracle_lib, 45, 37, 21, 3, tile=tile, seed=5)
    check(ni, nj, nk, ref, out, 3)


@pytest.mark.parametrize("tile", [12, 13])
@pytest.mark.parametrize("divopt,sthopt", [(2, 1), (1, 1), (0, 0)])
def test_onchip_tile_interior_blocks(cress, oracle_lib, divopt, sthopt, tile):
    # tile 12 (the column kept on chip): 4 x 5 tiles, so interior blocks
    # (plain stores) and edge blocks (periodic images, partial tiles) both run
    ni, nj, nk, ref, out = run_pair(cress, oracle_lib, 100, 37, 30, 4, sthopt=sthopt, tile=tile, seed=9,
                                    divopt=divopt)
    check(ni, nj, nk, ref, out, 4)


def test_sixteen_substeps(cress, oracle_lib):
    ni, nj, nk, ref, out = run_pair(cress, oracle_lib, 64, 64, 40, 16, sthopt=1, seed=7, dts=0.25,
                                    dx=500.0, dz=300.0)
    check(ni, nj, nk, ref, out, 16)


def test_rest_state_stays_at_rest(cress):
    nx, ny, nz = 40, 40, 24
    ni, nj, nk = H.dims(nx, ny, nz)
    base = H.base3d(ni, nj, nk, 300.0)
    z = np.zeros((nk, nj + 2, ni + 2), np.float32)
    s = cress.Solver(ni, nj, nk, 500.0, 500.0, 300.0)
    s.set_base3d(base)
    out = s.smalldrv(8, 0.25, z, z, z, z, z, z, z, z)
    s.close()
    for a in out:
        assert np.all(a == 0.0)


def test_nonuniform_base_rejected(cress):
    ni, nj, nk = H.dims(24, 24, 16)
    base = H.base3d(ni, nj, nk, 300.0)
    base["rbr"][5, 10, 10] *= 1.01
    s = cress.Solver(ni, nj, nk, 500.0, 500.0, 300.0)
    with pytest.raises(cress.CressError) as e:
        s.set_base3d(base)
    assert e.value.code == 4
    s.close()


# HE-VE (impopt=0): the explicit small step, with a step short enough for
# its vertical terms (dts < dz / c_s).
@pytest.mark.parametrize("sthopt", [0, 1])
def test_heve_substeps(cress, oracle_lib, sthopt):
    ni, nj, nk, ref, out = run_pair(cress, oracle_lib, 64, 48, 40, 6, sthopt=sthopt, seed=3, dts=0.2,
                                    impopt=0)
    check(ni, nj, nk, ref, out, 6)


@pytest.mark.parametrize("divopt", [0, 1])
def test_heve_ragged_divopt(cress, oracle_lib, divopt):
    ni, nj, nk, ref, out = run_pair(cress, oracle_lib, 45, 37, 21, 4, seed=9, dts=0.2, impopt=0,
                                    divopt=divopt)
    check(ni, nj, nk, ref, out, 4)

"""The bounded-wait failure path of the HE-VI kernel, without a GPU fault.

Every ring wait in the kernels is bounded; when one gives up, the kernel
records it in the context's device error word, stops issuing copies, waits
(with the full limit) for the copies already in flight and returns, and the
host reports CRESS_E_TIMEOUT.  The test hook cress_set_spin_limit(0) makes
the level loop's first wait give up at once, so every block takes that
path; nothing is left waiting and no copy outlives its block.  The same
context must then run normally again and match the oracle.
"""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

STAG = {"u": "u", "v": "v", "w": "s", "pp": "s"}


def test_wait_gives_up_reports_timeout_and_context_recovers(cress, oracle_lib):
    nx, ny, nz, nsstp, dts = 40, 24, 20, 2, 0.5
    ni, nj, nk = H.dims(nx, ny, nz)
    base = H.base3d(ni, nj, nk, 250.0, 1)
    st, frc = H.small_state(ni, nj, nk, 3, base)
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, 250.0, sthopt=1, tile=0)
    s.set_base3d(base)

    s.set_spin_limit(0)
    with pytest.raises(cress.CressError) as e:
        s.smalldrv(nsstp, dts, *st, *frc)
    assert e.value.code == 6, str(e.value)          # CRESS_E_TIMEOUT
    assert "bounded device-side wait" in str(e.value)

    s.set_spin_limit(-1)                             # the default limit again
    out = s.smalldrv(nsstp, dts, *st, *frc)
    s.sync()                                         # no error left behind
    s.close()

    cfg = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=250.0, sthopt=1, divopt=2, buyopt=1,
               weicoe=0.6)
    ref = oracle_lib.small_steps(cfg, base, frc, [a.copy() for a in st], nsstp, dts, prec=32,
                                 fp64_solve=1)
    for name, r, g in zip(("u", "v", "w", "pp"), ref, out):
        m = H.interior_mask(ni, nj, nk, STAG[name])
        scale = float(np.abs(r[m]).max()) + 1e-30
        assert np.isfinite(g[m]).all(), name
        assert float(np.abs(g[m] - r[m]).max()) <= 2e-5 * (nsstp + 1) * scale, name

"""The oracle's open radiation x boundaries (CPU only): runs with each
supported option (4, 5, 7) stay finite and differ from the periodic run."""
import numpy as np

NAMES = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def _case(nx=24, ny=12, nz=16, seed=4, cloud=True):
    from cress_b200 import cases
    return cases.supercell_case(nx, ny, nz, 1000.0, ztop=6000.0, seed=seed, cloud=cloud,
                                rad=(4000.0, 4000.0, 1200.0))


def _run(oracle_lib, case, obc, nsteps, init=None):
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=case["dz"], sthopt=1, smtopt=3, vspopt=2,
               vspbar=0.005, botbar=0.6 * zph[nk - 1], obc=obc, gwave=20.0)
    if init is None:
        init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]
    past = [a.copy() for a in init]
    now = [a.copy() for a in init]
    prec = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
    oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec, nsteps, 5.0, 1.0, start=True)
    return past, now


def test_open_runs_finite_and_boundary_driven(oracle_lib):
    case = _case()
    ni, nj, nk = case["dims"]
    _, per = _run(oracle_lib, case, 0, 4)
    for obc in (4, 5, 7):
        _, opn = _run(oracle_lib, case, obc, 4)
        for n, a in zip(NAMES, opn):
            assert np.isfinite(a[:, 2:nj - 1, 1:ni]).all(), (obc, n)
        d = float(np.abs(opn[3][:nk - 1, 2:nj - 1, 1:ni] - per[3][:nk - 1, 2:nj - 1, 1:ni]).max())
        assert d > 0.0, obc

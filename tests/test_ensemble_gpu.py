"""Ensembles: members of uneven sizes stepped together (one acoustic launch
per substep over every member's tiles, the rest on each member's stream,
eagerly or replayed from CUDA graphs) give bitwise the same states as the
same members stepped one by one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def member(cress, oracle_lib, nx, ny, nz, seed):
    from cress_b200 import cases
    case = cases.supercell_case(nx, ny, nz, 1000.0, ztop=8000.0, seed=seed, cloud=True,
                                rad=(5000.0, 5000.0, 1400.0))
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, case["dz"], sthopt=1, cphopt=3)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]
    for n, a in zip(NAMES, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    return s


SIZES = [(40, 33, 22, 1), (29, 45, 22, 2), (64, 20, 22, 3)]


def run(cress, oracle_lib, together, nsteps=3, graphs=False):
    sols = [member(cress, oracle_lib, *sz) for sz in SIZES]
    ens = cress.Ensemble(sols, graphs=graphs) if together else None
    for step in range(nsteps):
        first = step == 0
        args = (step * 5000, 2.5 if first else 5.0, 10, 0.5 if first else 1.0)
        if together:
            ens.large_step(*args)
        else:
            for s in sols:
                s.large_step(*args)
    out = [[s.get_field(n, cress.NOW) for n in NAMES] + [s.get_precip()] for s in sols]
    if ens:
        ens.close()
    for s in sols:
        s.close()
    return out


@pytest.mark.parametrize("graphs,nsteps", [(False, 3), (True, 9)])
def test_ensemble_matches_members_one_by_one(cress, oracle_lib, graphs, nsteps):
    a = run(cress, oracle_lib, False, nsteps)
    b = run(cress, oracle_lib, True, nsteps, graphs)
    for m, (x, y) in enumerate(zip(a, b)):
        for n, p, q in zip(NAMES + ["precip"], x, y):
            assert np.isfinite(q).all(), (m, n)
            assert np.array_equal(p, q), (m, n)

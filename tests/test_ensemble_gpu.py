"""Ensembles: members of uneven sizes stepped together (one acoustic launch
per substep over every member's tiles with tile 0's or tile 13's kernel,
the rest on each member's stream, eagerly or replayed from CUDA graphs).

With tile 0 the states equal the same members stepped one by one, bit for
bit.  Tile 13's batched kernel is a separate compilation of the same
substep code, in which the compiler may fuse multiply-adds differently,
so there the states agree with the one-by-one run to 1e-4 of each field's
maximum (1e-3 for the precipitation), and each member is checked against
the oracle with the moist tolerance.  The ensemble autotuner leaves the
members' state alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def member(cress, oracle_lib, nx, ny, nz, seed, tile=0):
    from cress_b200 import cases
    case = cases.supercell_case(nx, ny, nz, 1000.0, ztop=8000.0, seed=seed, cloud=True,
                                rad=(5000.0, 5000.0, 1400.0))
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, case["dz"], sthopt=1, cphopt=3, tile=tile)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]
    for n, a in zip(NAMES, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    return s


SIZES = [(40, 33, 22, 1), (29, 45, 22, 2), (64, 20, 22, 3)]


def run(cress, oracle_lib, together, nsteps=3, graphs=False, tile=0):
    sols = [member(cress, oracle_lib, *sz, tile=tile) for sz in SIZES]
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


@pytest.mark.parametrize("graphs,nsteps,tile", [(False, 3, 0), (True, 9, 0), (False, 3, 13), (True, 9, 13)])
def test_ensemble_matches_members_one_by_one(cress, oracle_lib, graphs, nsteps, tile):
    a = run(cress, oracle_lib, False, nsteps, tile=tile)
    b = run(cress, oracle_lib, True, nsteps, graphs, tile=tile)
    for m, (x, y) in enumerate(zip(a, b)):
        for n, p, q in zip(NAMES + ["precip"], x, y):
            assert np.isfinite(q).all(), (m, n)
            if tile == 0:
                assert np.array_equal(p, q), (m, n)
            else:
                tol = (1e-3 if n == "precip" else 1e-4) * float(np.abs(p).max()) + 1e-9
                assert float(np.abs(p - q).max()) <= tol, (m, n, float(np.abs(p - q).max()), tol)


def test_ensemble_autotune_keeps_state(cress, oracle_lib):
    sols = [member(cress, oracle_lib, *sz) for sz in SIZES]
    ens = cress.Ensemble(sols)
    ens.large_step(0, 2.5, 10, 0.5)
    before = [[s.get_field(n, lvl) for n in NAMES] for s in sols for lvl in (cress.PAST, cress.NOW)]
    tile, ms = ens.autotune(10, 1.0, reps=2)
    assert tile in (0, 13) and ms[0] > 0 and ms[13] > 0, (tile, ms)
    assert ms[tile] == min(ms.values())
    after = [[s.get_field(n, lvl) for n in NAMES] for s in sols for lvl in (cress.PAST, cress.NOW)]
    for x, y in zip(before, after):
        for p, q in zip(x, y):
            assert np.array_equal(p, q)
    ens.large_step(5000, 5.0, 10, 1.0)
    for s in sols:
        assert np.isfinite(s.get_field("w", cress.NOW)).all()
    ens.close()
    for s in sols:
        s.close()


def test_ensemble_tile13_matches_oracle(cress, oracle_lib):
    """Every member of a tile-13 ensemble, three moist large steps, against
    the oracle's moist steps from the same state (the moist parity bar:
    99.9% of cells within 1e-4 of the field's maximum, all within 1e-2,
    precipitation within 1e-3)."""
    from cress_b200 import cases
    import test_moist_gpu as MG
    sizes = SIZES
    sols = [member(cress, oracle_lib, *sz, tile=13) for sz in sizes]
    ens = cress.Ensemble(sols, graphs=False)
    nsteps = 3
    for step in range(nsteps):
        first = step == 0
        ens.large_step(step * 5000, 2.5 if first else 5.0, 10, 0.5 if first else 1.0)
    got = [([s.get_field(n, cress.PAST) for n in NAMES], [s.get_field(n, cress.NOW) for n in NAMES],
            s.get_precip()) for s in sols]
    ens.close()
    for s in sols:
        s.close()
    for (nx, ny, nz, seed), (gp, gn, gprec) in zip(sizes, got):
        case = cases.supercell_case(nx, ny, nz, 1000.0, ztop=8000.0, seed=seed, cloud=True,
                                    rad=(5000.0, 5000.0, 1400.0))
        ni, nj, nk = case["dims"]
        zph = case["zph"]
        cfg = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=case["dz"], sthopt=1, smtopt=3, vspopt=2,
                   coropt=0, vspbar=0.005, botbar=0.6 * zph[nk - 1], thresq=1e-12, tubopt=0)
        init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]
        past = [a.copy() for a in init]
        now = [a.copy() for a in init]
        prec = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
        oracle_lib.moist_steps(cfg, case["base"], zph, past, now, prec, nsteps, 5.0, 1.0, start=True)
        MG.check((ni, nj, nk), (past, now, prec), (gp, gn, gprec))

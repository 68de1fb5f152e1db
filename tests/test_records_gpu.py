"""GPU checks of the device-side dump and restart writers against the
oracle's restatement of the reference's records (oracle/records.py), bit
for bit (the records are copies and float32 averages of the state, so no
tolerance applies):

* cress_dump_3d after moist steps with the TKE closure, for dmpvar
  selecting every supported variable ('o') and the totals ('-');
* cress_restart_write for the same state (cold rain, TKE) and for an open-x
  squall line (phase speeds in the file);
* a restart round trip: a fresh context restored by cress_restart_read
  continues exactly as the original does;
* a stream with a corrupted record length is refused.
"""
import numpy as np
import pytest

from oracle import records as R

pytestmark = pytest.mark.gpu

MOIST = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def _solver(cress, case, tubopt=0, obc=0):
    from cress_b200 import cases
    import oracle
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    s = cress.Solver(ni, nj, nk, case["dx"], case["dx"], case["dz"], sthopt=1, cphopt=3, thresq=1e-12,
                     tubopt=tubopt, obc=obc, gwave=20.0)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    return s


def _start(cress, s, case, tubopt):
    init = list(case["level"]) + [case["moist"][n] for n in MOIST[5:]]
    names = MOIST + (["tke"] if tubopt == 2 else [])
    if tubopt == 2:
        rng = np.random.default_rng(4)
        init.append(np.abs(rng.standard_normal(init[0].shape)).astype(np.float32) * np.float32(0.2))
    for n, a in zip(names, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    return names


def _steps(s, n, first=True, dtbig=5.0, dtsml=1.0, t0=0):
    nsstp = 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))
    for step in range(n):
        f = first and step == 0
        s.large_step(round((t0 + step) * dtbig * 1000), 0.5 * dtbig if f else dtbig, nsstp,
                     0.5 * dtsml if f else dtsml)


@pytest.fixture(scope="module")
def supercell():
    from cress_b200 import cases
    case = cases.supercell_case(36, 30, 22, 1000.0, ztop=8000.0, seed=11, cloud=True, rad=(6000.0, 6000.0, 1400.0))
    case["dx"] = 1000.0
    return case


def test_dump_records_match_oracle(cress, supercell):
    s = _solver(cress, supercell, tubopt=2)
    names = _start(cress, s, supercell, 2)
    _steps(s, 3)
    fields = {n: s.get_field(n, cress.NOW) for n in names}
    for dmpvar in ("ooooooooxxxo", "--x--x", "xxo-oo-o"):
        got, gnames = s.dump_3d(dmpvar)
        ref, rnames = R.dump_3d(fields, supercell["base"], dmpvar, cphopt=3, tubopt=2)
        assert gnames == rnames, dmpvar
        assert got.shape == ref.shape and np.array_equal(got.view(np.uint32), ref.view(np.uint32)), dmpvar
    with pytest.raises(cress.CressError) as e:
        s.dump_3d("xxxxxxxxxxx+")   # the maximum wind is not kept
    assert e.value.code == 2
    s.close()


def test_restart_records_match_oracle_and_round_trip(cress, supercell):
    s = _solver(cress, supercell, tubopt=2)
    names = _start(cress, s, supercell, 2)
    _steps(s, 3)
    data = s.restart_write()
    now = {n: s.get_field(n, cress.NOW) for n in names}
    past = {n: s.get_field(n, cress.PAST) for n in names}
    ref = R.restart_records(past, now, s.get_precip(), None, cphopt=3, tubopt=2)
    assert data.nbytes == len(ref) and data.tobytes() == ref

    # a fresh context restored from the records holds the same two levels
    # and continues as the original: every point the model computes (the
    # interior; its ghosts are copies) agrees bit for bit.  Points no step
    # writes -- level nk above the lid, the outermost ghost row of a face
    # field -- keep whatever their buffers held, here as in the reference,
    # and a restart does not carry the future buffers' stale values there.
    s2 = _solver(cress, supercell, tubopt=2)
    s2.restart_read(data)
    for n in names:
        for lvl in (cress.PAST, cress.NOW):
            assert np.array_equal(s.get_field(n, lvl), s2.get_field(n, lvl)), (n, lvl)
    _steps(s, 2, first=False, t0=3)
    _steps(s2, 2, first=False, t0=3)
    ni, nj, nk = supercell["dims"]
    for n in names:
        i1 = ni - 1 if n == "u" else ni - 2
        j1 = nj - 1 if n == "v" else nj - 2
        k1 = nk if n == "w" else nk - 1
        sl = (slice(0, k1), slice(2, j1 + 1), slice(2, i1 + 1))
        for lvl in (cress.PAST, cress.NOW):
            assert np.array_equal(s.get_field(n, lvl)[sl], s2.get_field(n, lvl)[sl]), (n, lvl)
    assert np.array_equal(s.get_precip(), s2.get_precip())

    bad = data.copy()
    bad[0] ^= 1   # the first record's leading length
    with pytest.raises(cress.CressError) as e:
        s2.restart_read(bad)
    assert e.value.code == 1
    s.close()
    s2.close()


def test_restart_records_open_x(cress):
    from cress_b200 import cases
    case = cases.squall_case(64, 16, 24, 500.0, ztop=10000.0, seed=7, xrad=4000.0)
    case["dx"] = 500.0
    s = _solver(cress, case, obc=4)
    _start(cress, s, case, 0)
    _steps(s, 3, dtbig=3.0, dtsml=0.5)
    data = s.restart_write()
    now = {n: s.get_field(n, cress.NOW) for n in MOIST}
    past = {n: s.get_field(n, cress.PAST) for n in MOIST}
    phase = {n: s.get_phase(n) for n in MOIST}
    assert any(np.abs(p).max() > 0 for p in phase.values())   # the boundaries radiate
    ref = R.restart_records(past, now, s.get_precip(), phase, cphopt=3)
    assert data.tobytes() == ref
    s2 = _solver(cress, case, obc=4)
    s2.restart_read(data)
    for n in MOIST:
        assert np.array_equal(s2.get_phase(n), phase[n]), n
    s.close()
    s2.close()

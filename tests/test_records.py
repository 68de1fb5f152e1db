"""CPU checks of the oracle's restatement of the dump and restart records
(oracle/records.py), which the device writers are compared with bit for bit.

* dump: the variable order of s_outdmp for a full dmpvar, the averaging of
  staggered variables to scalar points on an index-valued field, the
  totals of dmpvar '-';
* restart: every record framed by its 4-byte length on both sides, the
  payload sizes of the full-shape arrays, the precipitation planes and the
  zero y phase speeds, read back unchanged.
"""
import numpy as np

from oracle import records as R


def _level(ni, nj, nk, names, seed):
    rng = np.random.default_rng(seed)
    return {n: rng.standard_normal((nk, nj + 2, ni + 2)).astype(np.float32) for n in names}


MOIST = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng", "tke"]


def test_dump_order_averaging_and_totals():
    ni, nj, nk = 9, 8, 7
    f = _level(ni, nj, nk, MOIST, 1)
    f["u"][:] = np.arange(ni + 2, dtype=np.float32)[None, None, :]   # u(i) = i
    base = _level(ni, nj, nk, ["ubr", "vbr", "pbr", "ptbr", "qvbr"], 2)
    rec, names = R.dump_3d(f, base, "ooooooooxxxo", cphopt=3, tubopt=2)
    assert names == ["ubar", "u", "vbar", "v", "w", "pbar", "pp", "ptbar", "ptp", "qvbar", "qv",
                     "qc", "qr", "qi", "qs", "qg", "nci", "ncs", "ncg", "tke"]
    nx, ny, nz = ni - 3, nj - 3, nk - 3
    assert rec.shape == (len(names), nz, ny, nx) and rec.dtype == np.float32
    # u averaged to scalar points: i = 2..ni-2 -> i + 0.5
    assert np.array_equal(rec[1], np.broadcast_to(np.arange(2, ni - 1, dtype=np.float32) + 0.5, (nz, ny, nx)))
    # w averaged in k: records k = 2..nk-2
    w = f["w"]
    assert np.array_equal(rec[4], (np.float32(.5) * (w[1:nk - 2] + w[2:nk - 1]))[:, 2:nj - 1, 2:ni - 1])
    rec2, names2 = R.dump_3d(f, base, "--x--", cphopt=0)
    assert names2 == ["u", "v", "p", "pt"]
    assert np.array_equal(rec2[2], (base["pbr"] + f["pp"])[1:nk - 2, 2:nj - 1, 2:ni - 1])


def test_restart_framing_sizes_and_round_trip():
    ni, nj, nk = 9, 8, 7
    now, past = _level(ni, nj, nk, MOIST, 3), _level(ni, nj, nk, MOIST, 4)
    prec = np.random.default_rng(5).standard_normal((5, 2, nj + 2, ni + 2)).astype(np.float32)
    phase = {n: np.full((2, nk, nj), i, np.float32) for i, n in enumerate(MOIST[:14])}
    full = 4 * (ni + 2) * (nj + 2) * nk
    plane = 4 * (ni + 2) * (nj + 2)
    for cph, tub, ph in ((0, 0, None), (3, 2, None), (3, 0, phase)):
        data = R.restart_records(past, now, prec, ph, cphopt=cph, tubopt=tub)
        recs = R.split_records(data)
        sizes = [len(r) for r in recs]
        expect = [full] * 10
        cpx, cpy = 4 * 2 * nk * nj, 4 * 2 * nk * ni
        if ph is not None:
            expect += [cpx, cpy] * 5
        if cph == 3:
            expect += [full, full] + ([cpx, cpy] if ph is not None else []) + [2 * full, 2 * full]
            expect += [2 * cpx, 2 * cpy] if ph is not None else []
            expect += [3 * full] * 4 + ([3 * cpx, 3 * cpy, 3 * cpx, 3 * cpy] if ph is not None else [])
            expect += [2 * plane, 2 * plane, 3 * plane, 3 * plane]
        if tub == 2:
            expect += [full, full]
        assert sizes == expect, (cph, tub, ph is not None)
        assert np.array_equal(np.frombuffer(recs[0], np.float32).reshape(nk, nj + 2, ni + 2), now["u"])
        assert np.array_equal(np.frombuffer(recs[9], np.float32).reshape(nk, nj + 2, ni + 2), past["ptp"])
        if ph is not None:
            assert not np.frombuffer(recs[11], np.float32).any()    # ucpy: periodic y

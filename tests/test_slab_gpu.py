"""GPU checks of the y-slab decomposition (cress_slab_*): one periodic
domain split into y slabs, each a context of its own stepped by its own
host thread, exchanging ghost rows (after every acoustic substep and at the
end of each step) and the sedimentation sub-step minimum through the
in-process link, must compute what the single domain computes.

The single-domain run on the GPU is the reference here (its parity with
the oracle is the large-step tests'); every interior point of every field
of both time levels must agree bit for bit: the slabs run the same kernels
on the same values, the ghost rows they receive are the rows the periodic
wrap copies.  Cases: the moist supercell with the TKE closure split 2 ways
(uneven) and 3 ways, one rank alone (its own neighbour: the periodic wrap),
and a rank whose partner never steps (the bounded barrier gives up with
CRESS_E_TIMEOUT and leaves the GPU usable).
"""
import concurrent.futures as cf

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MOIST = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]
NAMES = MOIST + ["tke"]
DTB, DTS = 5.0, 1.0


def _periodic(a, stag):
    """Both ghost layers in x and y from the periodic images (the rule of the
    end-of-step halo: ghost g <- interior 2 + (g-2) mod (n-3); u ghosts are
    columns 0, 1, ni, ni+1, v ghosts rows 0, 1, nj, nj+1, else 0, 1, n-1, n),
    so that the single domain and the slabs start from the same state."""
    a = a.copy()
    nk, nj2, ni2 = a.shape
    ni, nj = ni2 - 2, nj2 - 2
    img = lambda n, g: 2 + (g - 2) % (n - 3)
    for x in ([0, 1, ni, ni + 1] if stag == "u" else [0, 1, ni - 1, ni]):
        a[:, :, x] = a[:, :, img(ni, x)]
    for y in ([0, 1, nj, nj + 1] if stag == "v" else [0, 1, nj - 1, nj]):
        a[:, y, :] = a[:, img(nj, y), :]
    return a


def _case():
    from cress_b200 import cases
    case = cases.supercell_case(40, 36, 22, 1000.0, ztop=8000.0, seed=13, cloud=True, rad=(6000.0, 6000.0, 1400.0))
    rng = np.random.default_rng(17)
    init = list(case["level"]) + [case["moist"][n] for n in MOIST[5:]]
    init.append(np.abs(rng.standard_normal(init[0].shape)).astype(np.float32) * np.float32(0.2))
    case["init"] = [_periodic(a, {"u": "u", "v": "v"}.get(n, "s")) for n, a in zip(NAMES, init)]
    return case


def _solver(cress, case, nj=None, rows=None):
    """A context on the whole domain, or on the slab whose local rows are
    the global rows `rows` (the periodic images for the ghost rows)."""
    from cress_b200 import cases
    import oracle
    ni, njg, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    cut = (lambda a: a) if rows is None else (lambda a: np.ascontiguousarray(a[:, rows, :]))
    nj = njg if nj is None else nj
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, case["dz"], sthopt=1, cphopt=3, thresq=1e-12, tubopt=2)
    s.set_base3d({k: cut(v) for k, v in case["base"].items()})
    s.set_base_large(cut(case["base"]["ubr"]), cut(case["base"]["vbr"]), cut(cases.expand(rbct, ni, njg, nk)), ksp0)
    s.set_base_moist(cut(case["base"]["pbr"]), cut(case["base"]["qvbr"]))
    for n, a in zip(NAMES, case["init"]):
        s.put_field(n, cress.PAST, cut(a))
        s.put_field(n, cress.NOW, cut(a))
    return s


def _slab_rows(njg, sizes):
    """Global row indices of each slab's local rows 0..nj+1 (nj = its
    interior rows + 3), periodic over the global interior rows 2..njg-2."""
    P = njg - 3
    assert sum(sizes) == P
    out, off = [], 0
    for n in sizes:
        loc = np.arange(n + 5)                       # local rows 0 .. nj+1
        out.append(2 + (loc - 2 + off) % P)
        off += n
    return out


def _step(s, n, t0=0):
    nsstp = 20 * int(1.e2 * (DTB + .001)) // int(1.e3 * (DTS + .0001))
    for q in range(n):
        first = t0 == 0 and q == 0
        s.large_step(round((t0 + q) * DTB * 1000), 0.5 * DTB if first else DTB, nsstp,
                     0.5 * DTS if first else DTS)


def _run_slabs(cress, case, sizes, nsteps):
    ni, njg, nk = case["dims"]
    rows = _slab_rows(njg, sizes)
    solvers = [_solver(cress, case, nj=n + 3, rows=r) for n, r in zip(sizes, rows)]
    grp = cress.SlabGroup(len(sizes))
    for r, s in enumerate(solvers):
        s.slab_attach(grp, r)
    with cf.ThreadPoolExecutor(len(solvers)) as ex:
        list(ex.map(lambda s: _step(s, nsteps), solvers))
    got = {}
    for n in NAMES:
        for lvl in (cress.PAST, cress.NOW):
            # each slab's interior rows 2..nj-2, in global order
            got[(n, lvl)] = np.concatenate([s.get_field(n, lvl)[:, 2:sz + 2, :] for s, sz in zip(solvers, sizes)],
                                           axis=1)
    precip = np.concatenate([s.get_precip()[:, :, 2:sz + 2, :] for s, sz in zip(solvers, sizes)], axis=2)
    for s in solvers:
        s.close()
    grp.close()
    return got, precip


def _run_single(cress, case, nsteps):
    s = _solver(cress, case)
    _step(s, nsteps)
    njg = case["dims"][1]
    got = {(n, lvl): s.get_field(n, lvl)[:, 2:njg - 1, :] for n in NAMES for lvl in (cress.PAST, cress.NOW)}
    precip = s.get_precip()[:, :, 2:njg - 1, :]
    s.close()
    return got, precip


@pytest.fixture(scope="module")
def single(cress):
    case = _case()
    return case, _run_single(cress, case, 4)


def _compare(case, ref, got):
    ni, njg, nk = case["dims"]
    (rf, rp), (gf, gp) = ref, got
    for (n, lvl), r in rf.items():
        g = gf[(n, lvl)]
        i1 = ni - 1 if n == "u" else ni - 2
        k1 = nk if n == "w" else nk - 1
        sl = (slice(0, k1), slice(None), slice(2, i1 + 1))
        assert np.isfinite(g[sl]).all(), (n, lvl)
        assert np.array_equal(g[sl], r[sl]), (n, lvl, float(np.abs(g[sl] - r[sl]).max()))
    assert np.array_equal(gp[:, :, :, 2:ni - 1], rp[:, :, :, 2:ni - 1])


@pytest.mark.parametrize("sizes", [(20, 16), (11, 12, 13)])
def test_slabs_match_single_domain(cress, single, sizes):
    case, ref = single
    _compare(case, ref, _run_slabs(cress, case, list(sizes), 4))


def test_one_rank_is_the_periodic_domain(cress, single):
    case, ref = single
    _compare(case, ref, _run_slabs(cress, case, [case["dims"][1] - 3], 4))


def test_nccl_single_rank_is_the_periodic_domain(cress, single):
    """The NCCL link on one GPU: a single rank is its own northern and
    southern neighbour, so its rows go out with ncclSend and come back with
    ncclRecv (and the sub-step word through ncclAllReduce) as the periodic
    wrap; the result must be the single domain's."""
    case, ref = single
    njg = case["dims"][1]
    s = _solver(cress, case)
    s.slab_attach_nccl(0, 1, cress.slab_nccl_id())
    _step(s, 4)
    got = {(n, lvl): s.get_field(n, lvl)[:, 2:njg - 1, :] for n in NAMES for lvl in (cress.PAST, cress.NOW)}
    precip = s.get_precip()[:, :, 2:njg - 1, :]
    s.slab_detach()
    s.close()
    _compare(case, ref, (got, precip))


def test_missing_rank_times_out(cress, single):
    case, _ = single
    ni, njg, nk = case["dims"]
    rows = _slab_rows(njg, [18, 18])
    s0 = _solver(cress, case, nj=21, rows=rows[0])
    s1 = _solver(cress, case, nj=21, rows=rows[1])
    grp = cress.SlabGroup(2, timeout_ms=500)
    s0.slab_attach(grp, 0)
    s1.slab_attach(grp, 1)
    with pytest.raises(cress.CressError) as e:
        _step(s0, 1)                      # rank 1 never steps
    assert e.value.code == 6, str(e.value)   # CRESS_E_TIMEOUT
    # the group is broken for the other rank too, and the GPU stays usable
    with pytest.raises(cress.CressError) as e:
        _step(s1, 1)
    assert e.value.code == 7
    s0.slab_detach()
    s1.slab_detach()
    s0.sync()
    s1.sync()
    s0.close()
    s1.close()
    grp.close()

"""Large steps replayed from CUDA graphs give bitwise the same state as the
eager path (same kernels, same arguments), for the dry and the moist step,
with periodic and with open radiation x boundaries, and count the same
kernel launches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def make(cress, oracle_lib, graphs, cphopt, obc=0):
    from cress_b200 import cases
    case = cases.supercell_case(36, 28, 20, 1000.0, ztop=7000.0, seed=6, cloud=True,
                                rad=(5000.0, 5000.0, 1200.0))
    ni, nj, nk = case["dims"]
    zph = case["zph"]
    rbct, ksp0 = oracle_lib.vspdmp(nk, zph, 0.005, 0.6 * zph[nk - 1])
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, case["dz"], sthopt=1, cphopt=cphopt, obc=obc)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    names = NAMES if cphopt else NAMES[:5]
    if cphopt:
        s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in NAMES[5:]]
    for n, a in zip(names, init):
        s.put_field(n, cress.PAST, a)
        s.put_field(n, cress.NOW, a)
    s.set_graphs(graphs)
    return s, names


@pytest.mark.parametrize("cphopt,obc", [(0, 0), (3, 0), (3, 4)])
def test_graph_replay_is_bitwise_identical(cress, oracle_lib, cphopt, obc):
    out = []
    for graphs in (False, True):
        s, names = make(cress, oracle_lib, graphs, cphopt, obc)
        s.large_step(0, 2.5, 10, 0.5)
        for n in range(1, 8):
            s.large_step(n * 5000, 5.0, 10, 1.0)
        out.append(([s.get_field(n, cress.NOW) for n in names] +
                    [s.get_field(n, cress.PAST) for n in names], s.launch_count()))
        s.close()
    (a, la), (b, lb) = out
    assert la == lb
    for x, y in zip(a, b):
        assert np.array_equal(x, y)

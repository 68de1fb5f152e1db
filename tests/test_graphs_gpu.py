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


def test_async_readback_matches_sync(cress, oracle_lib):
    """cress_get_fields_async captures each step's fields at the point of the
    call and copies them on a second stream while later steps run: after
    cress_wait_fields every step's host copy equals a synchronous read of
    the same step, bit for bit, with the read-backs of consecutive steps in
    flight over the next step's host->device copies."""
    import torch
    s, names = make(cress, oracle_lib, True, 3)
    ref = make(cress, oracle_lib, True, 3)[0]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    shape = ref.shape
    bufs = [[pin(np.zeros(shape, np.float32)) for _ in names] for _ in range(2)]
    want = []
    for n in range(5):
        ctime, dtb, dts = (0, 2.5, 0.5) if n == 0 else (n * 5000, 5.0, 1.0)
        ref.large_step(ctime, dtb, 10, dts)
        want.append([ref.get_field(f, cress.NOW) for f in names])
        # the asynchronous context re-reads its inputs from the host each step
        if n > 0:
            for f, a in zip(names, inputs):
                s.put_field(f, cress.NOW, a)
        s.large_step(ctime, dtb, 10, dts)
        if n > 0:
            s.wait_fields()
            got = bufs[(n - 1) % 2]
            for f, g, w in zip(names, got, want[n - 1]):
                assert np.array_equal(g, w), (n - 1, f)
        s.get_fields_async(cress.NOW, names, bufs[n % 2])
        inputs = [a.copy() for a in want[n]]
    s.wait_fields()
    for f, g, w in zip(names, bufs[4 % 2], want[4]):
        assert np.array_equal(g, w), (4, f)
    s.close()
    ref.close()


def test_async_input_matches_put_field(cress, oracle_lib):
    """cress_put_fields_async: every step's past and present levels go in
    from host arrays on the input stream, queued behind the previous step,
    whose compute and read-back are still in flight, and the host waits
    for a step's result only after the next step is queued (two read-backs
    in flight); each step's result equals the same step fed through
    cress_put_field, bit for bit, with inputs that differ from step to step
    (states of a third run)."""
    import torch
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    src, names = make(cress, oracle_lib, True, 3)
    states = []
    src.large_step(0, 2.5, 10, 0.5)
    for n in range(1, 5):
        src.large_step(n * 5000, 5.0, 10, 1.0)
        states.append(([pin(src.get_field(f, cress.PAST)) for f in names],
                       [pin(src.get_field(f, cress.NOW)) for f in names]))
    src.close()
    ref, _ = make(cress, oracle_lib, True, 3)
    want = []
    for n, (past, now) in enumerate(states):
        for f, a, b in zip(names, past, now):
            ref.put_field(f, cress.PAST, a)
            ref.put_field(f, cress.NOW, b)
        ref.large_step(50000 + n * 5000, 5.0, 10, 1.0)
        want.append([ref.get_field(f, cress.NOW) for f in names])
    ref.close()
    s, _ = make(cress, oracle_lib, True, 3)
    bufs = [[pin(np.zeros(s.shape, np.float32)) for _ in names] for _ in range(2)]
    s.put_fields_async(cress.PAST, names, states[0][0])
    s.put_fields_async(cress.NOW, names, states[0][1])
    for n in range(len(states)):
        s.large_step(50000 + n * 5000, 5.0, 10, 1.0)
        s.get_fields_async(cress.NOW, names, bufs[n % 2])
        if n + 1 < len(states):   # the next inputs, queued before the host waits
            s.put_fields_async(cress.PAST, names, states[n + 1][0])
            s.put_fields_async(cress.NOW, names, states[n + 1][1])
        s.wait_fields(in_flight=1)
        if n > 0:
            for f, g, w in zip(names, bufs[(n - 1) % 2], want[n - 1]):
                assert np.array_equal(g, w), (n - 1, f)
    s.wait_fields()
    for f, g, w in zip(names, bufs[(len(states) - 1) % 2], want[-1]):
        assert np.array_equal(g, w), (len(states) - 1, f)
    s.close()

"""Replica driver (one domain per rank, no data-path collective) on CPU
ranks over gloo, world size 2.

Each rank builds its own dry acoustic domain seeded by its rank, steps it
with the CPU oracle's small-step loop inside `timed_steps` (barriers on
both sides, max over ranks of the timed seconds), and reports a checksum.
Checked: the rank bookkeeping, that the max-over-ranks time is the largest
rank's own time, that each rank's result equals a single-process run of the
same seed (no cross-talk between replicas), and that the replicas differ.
A second test starts two ranks through `relaunch_under_torchrun`, the path
`bench.py --gpus N` takes when run directly.
"""
import os
import re
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _domain(seed):
    from cress_b200 import cases
    (ni, nj, nk), base, st, frc = cases.acoustic_case(16, 12, 10, 1000.0, 250.0, seed=seed, sthopt=1)
    cfg = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=250.0, sthopt=1, divopt=2, buyopt=1,
               weicoe=0.6)
    return cfg, base, st, frc


def _checksum(st):
    return [float(np.sum(a, dtype=np.float64)) for a in st]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world), OMP_NUM_THREADS="1")
    sys.path.insert(0, ROOT)
    import time
    import oracle
    from cress_b200.replicas import Replicas, WallTimer, timed_steps
    try:
        rep = Replicas("gloo", timeout_s=60)
        cfg, base, st, frc = _domain(rep.seed(100))

        def step():
            oracle.small_steps(cfg, base, frc, st, 1, 0.5)
            time.sleep(0.05 * (rep.rank + 1))   # ranks of unequal speed

        own = []

        class T(WallTimer):
            def stop(self):
                t = super().stop()
                own.append(t)
                return t

        tmax = timed_steps(rep, step, 3, 1, T())
        times = rep.gather([own[0]])
        q.put((rep.rank, rep.world, own[0], tmax, [t[0] for t in times], _checksum(st)))
        rep.close()
    except Exception as e:   # report instead of hanging the parent
        q.put(("error", repr(e)))


def test_replicas_gloo_world2(oracle_lib):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(r[0] != "error" for r in res), res
    res.sort()
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    own = [r[2] for r in res]
    for r in res:
        assert r[3] == pytest.approx(max(own), rel=1e-12)   # every rank sees the slowest rank's time
        assert r[4] == pytest.approx(own, rel=1e-12)
    assert own[1] > own[0]                                  # rank 1 sleeps longer per step
    # each replica equals a single-process run of its own seed
    for rank, r in enumerate(res):
        cfg, base, st, frc = _domain(100 + rank)
        for _ in range(4):   # 1 warm-up + 3 timed steps
            oracle_lib.small_steps(cfg, base, frc, st, 1, 0.5)
        assert r[5] == _checksum(st)
    assert res[0][5] != res[1][5]


def test_relaunch_under_torchrun(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {ROOT!r})
        from cress_b200.replicas import Replicas
        rep = Replicas("gloo", timeout_s=60)
        m = rep.max(10.0 + rep.rank)
        print(f"rank {{rep.rank}} of {{rep.world}} max {{m}}", flush=True)
        rep.close()
    """))
    out = subprocess.run([sys.executable, "-c", textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {ROOT!r})
        from cress_b200.replicas import relaunch_under_torchrun
        sys.exit(relaunch_under_torchrun(2, {str(script)!r}, [], timeout_s=240))
    """)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    # the two ranks share one stdout, so their lines may interleave
    found = sorted(re.findall(r"rank (\d) of (\d) max ([0-9.]+)", out.stdout))
    assert found == [("0", "2", "11.0"), ("1", "2", "11.0")], out.stdout

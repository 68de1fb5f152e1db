"""Independent replicas across GPUs: one domain per rank, no data-path
collective.

The reference decomposes one domain over MPI ranks (SrcOrig/sethalo.f90:
485-505 sets up the halo neighbours of each subdomain).  Here the first
multi-GPU mode is the ensemble's: every rank (one process per GPU) owns a
whole domain of its own, seeded by its rank, and steps it alone.  The only
collectives are the barriers around a timed region and the max over ranks
of its duration, so the aggregate throughput is (units all ranks
processed) / (slowest rank's time): weak scaling.

Ranks come from the torchrun environment (RANK, LOCAL_RANK, WORLD_SIZE,
MASTER_ADDR, MASTER_PORT); `relaunch_under_torchrun` starts N such ranks
when a program was run directly with N > 1.
"""
import datetime
import os
import socket
import subprocess
import sys
import time


class Replicas:
    """Rank bookkeeping and the two collectives of a replica run.

    backend: "nccl" (one GPU per rank) or "gloo" (CPU ranks).  With
    WORLD_SIZE 1 no process group is made and every collective is local."""

    def __init__(self, backend="nccl", timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def seed(self, base):
        """Seed of this rank's domain: every rank a different one."""
        return int(base) + self.rank

    def _tensor(self, values, dtype):
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor(values, dtype=dtype, device=dev)

    def barrier(self):
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x):
        """Max over ranks of a float (every rank gets it)."""
        if self._dist is None:
            return float(x)
        import torch
        t = self._tensor([float(x)], torch.float64)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if self._dist is None:
            return float(x)
        import torch
        t = self._tensor([float(x)], torch.float64)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, values):
        """Every rank's list of floats (same length on every rank), as a
        list of lists indexed by rank."""
        if self._dist is None:
            return [list(map(float, values))]
        import torch
        t = self._tensor([float(v) for v in values], torch.float64)
        out = [torch.zeros_like(t) for _ in range(self.world)]
        self._dist.all_gather(out, t)
        return [[float(v) for v in o.cpu().tolist()] for o in out]

    def close(self):
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


class WallTimer:
    """Host wall clock (the caller synchronizes any device work in `stop`)."""

    def __init__(self, sync=None):
        self._sync = sync
        self._t0 = 0.0

    def start(self):
        self._t0 = time.perf_counter()

    def stop(self):
        if self._sync is not None:
            self._sync()
        return time.perf_counter() - self._t0


class CudaEventTimer:
    """CUDA events recorded on the stream the timed work is launched on."""

    def __init__(self, stream):
        import torch
        self.stream = stream
        self._e0 = torch.cuda.Event(enable_timing=True)
        self._e1 = torch.cuda.Event(enable_timing=True)

    def start(self):
        self._e0.record(self.stream)

    def stop(self):
        self._e1.record(self.stream)
        self._e1.synchronize()
        return self._e0.elapsed_time(self._e1) * 1e-3


def timed_steps(rep, step, steps, warmup, timer, sync=None, inside=None):
    """`warmup` untimed calls of step(), then `steps` timed ones bracketed by
    a barrier and a synchronize on both sides.  Returns the max over ranks
    of the timed seconds.  `inside` is an optional context manager entered
    around the timed region (e.g. a clock sampler)."""
    import contextlib
    for _ in range(warmup):
        step()
    if sync is not None:
        sync()
    rep.barrier()
    with (inside if inside is not None else contextlib.nullcontext()):
        timer.start()
        for _ in range(steps):
            step()
        secs = timer.stop()
        if sync is not None:
            sync()
        rep.barrier()
    return rep.max(secs)


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch_under_torchrun(nproc, script, argv, timeout_s=None):
    """Run `script argv` as nproc ranks on this node (torchrun, rendezvous on
    127.0.0.1) and return its exit code; the ranks' output goes to this
    process's stdout/stderr."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), script] + list(argv)
    return subprocess.run(cmd, timeout=timeout_s).returncode

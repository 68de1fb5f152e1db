"""Benchmark: CReSS solver time integration on B200.

Prints ONE JSON line (rank 0).  See the argparse help for the workload
options.  Timing: CUDA events on the library's stream (shared with torch's
current stream), barrier + synchronize around the timed region, max over
ranks.  Multi-GPU runs are independent replicas (one domain per GPU, no
data-path collective): "scaling": "weak".
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_BYTES_PER_CELL_SUBSTEP = 48  # u,v,w,p' read+write, 4 forcings read (float32)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 2 + i and r[2 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_baseline_small(args, cfg, base, st, frc, threads):
    """Oracle (C++ restatement, OpenMP) on a bounded sample of the workload:
    the same nz and substep count on a horizontally reduced domain."""
    import oracle
    from cress_b200 import cases
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sx, sy = args.cpu_nx, args.cpu_ny
    (ni, nj, nk), b2, st2, frc2 = cases.acoustic_case(sx, sy, args.nz, args.dx, args.dz, seed=3,
                                                      sthopt=1)
    c2 = dict(cfg, ni=ni, nj=nj, nk=nk)
    oracle.build()
    s = [a.copy() for a in st2]
    t0 = time.perf_counter()
    oracle.small_steps(c2, b2, frc2, s, args.nsstp, args.dts, prec=32, fp64_solve=1, omp=True)
    dt = time.perf_counter() - t0
    cells = sx * sy * args.nz
    return {"value": cells / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{sx}x{sy}x{args.nz} domain, one small-step loop of {args.nsstp} HE-VI "
                      f"substeps (C++ oracle, OpenMP {threads} threads), {dt:.2f} s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nz", type=int, default=64)
    ap.add_argument("--dx", type=float, default=1000.0)
    ap.add_argument("--dz", type=float, default=281.25)
    ap.add_argument("--nsstp", type=int, default=20)
    ap.add_argument("--dts", type=float, default=0.5)
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--cpu-nx", type=int, default=128)
    ap.add_argument("--cpu-ny", type=int, default=128)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cfg_json = {"workload": f"hevi small-step loop, {args.nx}x{args.ny}x{args.nz} moist-supercell "
                            f"grid shape (stretched dz), {args.nsstp} substeps of dts={args.dts}",
                "nx": args.nx, "ny": args.ny, "nz": args.nz, "nsstp": args.nsstp,
                "l2": "inputs larger than L2 (8 x 72 MB fields per step)",
                "parallelism": f"replicas{world}"}
    metric = "cell-updates/s on 1 B200: plain vs learned-microphysics form at stated error"

    if args.impl == "reference":
        if rank != 0:
            return
        from cress_b200 import cases
        cfg = dict(dx=args.dx, dy=args.dx, dz=args.dz, sthopt=1, divopt=2, buyopt=1, weicoe=0.6)
        threads = os.cpu_count() or 1
        times = []
        res = None
        for _ in range(args.warmup + args.steps):
            res = cpu_baseline_small(args, cfg, None, None, None, threads)
            times.append(res["value"])
        v = float(np.median(times[args.warmup:]))
        res["value"] = v
        print(json.dumps({"metric": metric, "value": v, "unit": "cell-updates/s", "n_gpus": 0,
                          "steps": args.steps, "warmup": args.warmup, "impl": "reference",
                          "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                          "config": cfg_json, "cpu_baseline": res,
                          "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    import torch.distributed as dist
    import cress_b200
    from cress_b200 import cases

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    (ni, nj, nk), base, st, frc = cases.acoustic_case(args.nx, args.ny, args.nz, args.dx, args.dz,
                                                      seed=100 + rank, sthopt=1)
    s = cress_b200.Solver(ni, nj, nk, args.dx, args.dx, args.dz, sthopt=1, tile=args.tile,
                          device=local)
    # A dedicated (non-default) stream shared by the library and torch's
    # events, so the events bracket exactly the library's kernels.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    s.set_stream(stream.cuda_stream)
    s.set_base3d(base)
    for name, a in zip(("u", "v", "w", "pp"), st):
        s.put_field(name, cress_b200.PAST, a)
    for name, a in zip(("u", "v", "w", "pp"), frc):
        s.put_field(name, cress_b200.FORCING, a)
    s.sync()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        s.small_steps(args.nsstp, args.dts)
    barrier()
    l0 = s.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            s.small_steps(args.nsstp, args.dts)
        e1.record(stream)
        barrier()
    launches = s.launch_count() - l0
    ms = max_over_ranks(e0.elapsed_time(e1))
    cells = args.nx * args.ny * args.nz
    value = world * cells * args.steps / (ms * 1e-3)
    per_launch_s = ms * 1e-3 / (args.steps * args.nsstp)
    peak, peak_kind = measured_peaks()
    achieved = HBM_BYTES_PER_CELL_SUBSTEP * cells / per_launch_s / 1e9

    # End to end through the public host-array entry point (s_smalldrv's
    # interface): H2D of u,v,w,p' (past) and the 4 forcings from pinned host
    # memory, the substeps, D2H of the 4 future fields, every step.
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    ins = [pin(a) for a in st + frc]
    outs = [pin(np.empty_like(st[0])) for _ in range(4)]
    for _ in range(args.warmup):
        s.smalldrv(args.nsstp, args.dts, *ins, out=outs)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.smalldrv(args.nsstp, args.dts, *ins, out=outs)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": int(sum(a.nbytes for a in ins)),
           "d2h_bytes_per_step": int(sum(a.nbytes for a in outs))}
    s.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cfg = dict(dx=args.dx, dy=args.dx, dz=args.dz, sthopt=1, divopt=2, buyopt=1, weicoe=0.6)
        cpu = cpu_baseline_small(args, cfg, None, None, None, os.cpu_count() or 1)

    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg_json,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": peak_kind,
                         "kernel": "k_hevi_substep", "bytes_per_launch": HBM_BYTES_PER_CELL_SUBSTEP * cells,
                         "ms_per_launch": per_launch_s * 1e3},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clk.summary(),
            "cpu_baseline": cpu}))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

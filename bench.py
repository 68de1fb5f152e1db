"""Benchmark: CReSS solver time integration on B200.

Workload (default): the moist supercell, 512x512x64 (dx = 1 km, dz
stretched from 100 m to 500 m up to 18 km), cold-rain bulk microphysics
(cphopt=3: qv, qc, qr, qi, qs, qg, ni, ns, ng), dtbig = 5 s with 10 HE-VI
acoustic substeps.  One step = one leapfrog large step of s_intgdrv:
forcing (advection, 4th-order smoothing, Rayleigh sponge, moist buoyancy),
10 HE-VI substeps, theta' and the nine moist scalars' steps, s_cloudphy
(process rates + sedimentation), the Asselin filter, saturation adjustment
on t and t+dt, periodic ghost planes.  The state starts from a seeded
cloudy field so the microphysics is active in a large share of the cells.
Metric: cell-updates/s (interior cells x large steps / s).

Prints ONE JSON line (rank 0).  Timing: CUDA events on the library's stream
(a dedicated torch stream that the library is told to use), barrier +
synchronize around the timed region, max over ranks.  Multi-GPU runs are
independent replicas (one domain per GPU, no data-path collective):
"scaling": "weak".  --impl reference times the CPU restatement (OpenMP) of
the same step on the host cores.
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

HEVI_BYTES_PER_CELL = 48  # u,v,w,p' read + write and 4 forcings read, float32
# DRAM bytes per cell of one HE-VI launch measured by ncu on a 384x384x64
# domain (dram__bytes_read.sum + dram__bytes_write.sum over 384*384*63
# cells); the traffic grows with the cells.  Tile 0 (k_hevi2) parks the
# eliminated right-hand sides in HBM: 632.6 MB; tile 13 (k_hevi4) keeps
# them on chip: 349.7 + 121.0 MB.
HEVI_TRAFFIC_PER_CELL = {0: 632.6e6 / (384 * 384 * 63), 13: (349.68e6 + 120.99e6) / (384 * 384 * 63)}
HEVI_KERNEL = {0: "k_hevi2", 11: "k_hevi2", 12: "k_hevi3", 13: "k_hevi4"}
METRIC = "cell-updates/s on 1 B200: plain vs learned-microphysics form at stated error"
MOIST = ["qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]
NAMES = ["u", "v", "w", "pp", "ptp"] + MOIST
VSPBAR = 0.005
CTIME = 1000   # any non-zero model time (ms): a step after the first


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
        self._p = None
        self._t = None
        self._first = threading.Event()

    def _read(self):
        for line in self._p.stdout:
            if line.strip():
                self.rows.append([x.strip() for x in line.split(",")])
                self._first.set()

    def __enter__(self):
        # one nvidia-smi in its own sampling loop (every 50 ms) for the
        # whole timed region; its start-up (NVML initialisation) can hold
        # up CUDA calls for a second or more, so the timed region starts
        # only once it has delivered its first sample
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                        "--format=csv,noheader,nounits", "-lms", "50"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._p = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(timeout=20)
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._p.terminate()
        try:
            self._p.wait(timeout=10)
        except Exception:
            self._p.kill()
            self._p.wait()
        if self._t is not None:
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


def make_case(nx, ny, nz, dx, seed):
    from cress_b200 import cases
    case = cases.supercell_case(nx, ny, nz, dx, seed=seed, cloud=True)
    nk = case["dims"][2]
    case["botbar"] = 0.6 * case["zph"][nk - 1]
    return case


def vspdmp_columns(nk, zph, vspbar, botbar):
    """rbct(k), ksp0 of s_vspdmp (vspopt=2, vspdmp.f90:222-292), float32."""
    rbct = np.zeros(nk + 1, np.float32)
    ksp0 = 2
    for k in range(3, nk + 1):
        if np.float32(zph[k]) > np.float32(botbar):
            ksp0 = k - 1
            break
    cc = np.float32(3.141592)
    for k in range(2, nk):
        z = np.float32(zph[k])
        if z > np.float32(botbar):
            rbct[k] = np.float32(0.5) * np.float32(vspbar) * (
                np.float32(1) - np.cos(cc * (z - np.float32(botbar)) /
                                       (np.float32(zph[nk - 1]) - np.float32(botbar))))
    return rbct, ksp0


def nsstp_of(dtbig, dtsml):
    """slvstep.f90:176."""
    return 20 * int(1.e2 * (dtbig + .001)) // int(1.e3 * (dtsml + .0001))


class CpuMoist:
    """The oracle (C++ restatement, OpenMP on `threads` host threads) on an
    nx x ny x nz moist supercell domain, built once; step(n) runs n moist
    large steps and returns the seconds they took."""

    def __init__(self, args, threads, nx, ny):
        import oracle
        os.environ["OMP_NUM_THREADS"] = str(threads)
        oracle.build()
        self.oracle = oracle
        self.args = args
        self.cells = nx * ny * args.nz
        case = make_case(nx, ny, args.nz, args.dx, 3)
        ni, nj, nk = case["dims"]
        self.cfg = dict(ni=ni, nj=nj, nk=nk, dx=args.dx, dy=args.dx, dz=case["dz"], sthopt=1, smtopt=3,
                        vspopt=2, coropt=0, vspbar=VSPBAR, botbar=case["botbar"], tubopt=args.tubopt)
        init = list(case["level"]) + [case["moist"][n] for n in MOIST]
        if args.tubopt == 2:
            init.append(np.zeros_like(init[0]))   # TKE from zero
        self.past = [a.copy() for a in init]
        self.now = [a.copy() for a in init]
        self.base, self.zph = case["base"], case["zph"]
        self.prec = np.zeros((5, 2, nj + 2, ni + 2), np.float32)

    def step(self, n=1):
        t0 = time.perf_counter()
        self.oracle.moist_steps(self.cfg, self.base, self.zph, self.past, self.now, self.prec, n,
                                self.args.dtbig, self.args.dtsml, start=False, omp=True)
        return time.perf_counter() - t0


def learned_leg(args, s, stream, nsstp, cells, plain_ms, barrier, max_over_ranks, rank=0):
    """The learned-microphysics form on the same domain.  Training tuples
    come from other storms: `train_storms` supercell runs of the same size
    with new seeds (bubble amplitude, position and shear varied), each
    sampled every 60 s of model time (12 large steps) by the plain GPU
    scheme; the MLP is trained on the device; then the bench's own storm,
    which the network never saw, runs the same `eval_steps` large steps
    from one saved state with the plain and the learned process rates.
    Reports the learned form's throughput (CUDA events) and its error
    against the plain form on that held-out storm (accumulated surface
    precipitation, hydrometeor RMS)."""
    import torch
    import cress_b200
    from cress_b200 import cases
    m = cress_b200.Mlp(device=torch.cuda.current_device(), seed=7)
    m.reserve(args.train_tuples)
    rng = np.random.default_rng(500 + rank)
    seeds = []
    t_sample = time.perf_counter()
    for storm in range(args.train_storms):
        seed = int(rng.integers(1 << 30))
        seeds.append(seed)
        case = cases.supercell_case(args.nx, args.ny, args.nz, args.dx, seed=seed, cloud=True,
                                    ptp0=float(rng.uniform(2.0, 4.0)), shear=float(rng.uniform(20.0, 35.0)),
                                    center=(float(rng.uniform(-60e3, 60e3)), float(rng.uniform(-60e3, 60e3))))
        ni, nj, nk = case["dims"]
        rbct, ksp0 = vspdmp_columns(nk, case["zph"], VSPBAR, 0.6 * case["zph"][nk - 1])
        t = cress_b200.Solver(ni, nj, nk, args.dx, args.dx, case["dz"], sthopt=1, cphopt=3,
                              tile=s.cfg.tile, device=torch.cuda.current_device())
        t.set_base3d(case["base"])
        t.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
        t.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
        for n, a in zip(NAMES, list(case["level"]) + [case["moist"][q] for q in MOIST]):
            t.put_field(n, cress_b200.PAST, a)
            t.put_field(n, cress_b200.NOW, a)
        del case
        t.large_step(0, 0.5 * args.dtbig, nsstp, 0.5 * args.dtsml)
        for step in range(1, 12 * args.train_samples + 1):
            sample = step % 12 == 0 and m.tuple_count() < args.train_tuples
            if sample:
                t.set_tuple_sampling(m, stride=args.train_stride, keep_zero=0.05, seed=seed + step)
            t.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
            if sample:
                t.set_tuple_sampling(None)
        t.close()
    sample_s = time.perf_counter() - t_sample
    ntup = m.tuple_count()
    m.fit_norm()
    t0 = time.perf_counter()
    losses = m.train(args.train_steps, batch=8192, lr=1e-3, seed=5)
    train_s = time.perf_counter() - t0
    saved = [s.get_field(n, lvl) for n in NAMES for lvl in (cress_b200.PAST, cress_b200.NOW)]
    prec0 = s.get_precip()

    def restore():
        it = iter(saved)
        for n in NAMES:
            for lvl in (cress_b200.PAST, cress_b200.NOW):
                s.put_field(n, lvl, next(it))
        s.put_precip(prec0)

    def run(learned_on, chunk=0):
        restore()
        s.set_learned_micro(m if learned_on else None, chunk=chunk, resid_tol=0.5)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.eval_steps):
            s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
        e1.record(stream)
        barrier()
        t = max_over_ranks(e0.elapsed_time(e1)) / args.eval_steps
        out = {n: s.get_field(n, cress_b200.NOW) for n in MOIST[1:6]}
        stats = s.learned_stats() if learned_on else None
        return t, out, s.get_precip(), stats

    tp, qp, pp, _ = run(False)
    tc, _, _, _ = run(True, chunk=1 << 20)
    tl, ql, pl, (ncl, nfb) = run(True)
    s.set_learned_micro(None)
    m.close()
    sl = (slice(0, args.nz + 2), slice(2, args.ny + 2), slice(2, args.nx + 2))
    rms = {n: float(np.sqrt(np.mean((ql[n][sl] - qp[n][sl]) ** 2)) /
                    (np.sqrt(np.mean(qp[n][sl] ** 2)) + 1e-30)) for n in qp}
    acc_p = float(pp[:, 1].sum())
    acc_l = float(pl[:, 1].sum())
    return {"value": cells / (tl * 1e-3), "unit": "cell-updates/s", "ms_per_step": tl,
            "plain_ms_per_step_same_steps": tp, "speedup_vs_plain": tp / tl,
            "inference": "fused", "chunked_ms_per_step": tc,
            "mlp_cells": ncl, "fallback_cells": nfb,
            "precip_accum_rel_diff": abs(acc_l - acc_p) / (abs(acc_p) + 1e-30),
            "hydrometeor_rms_rel": rms,
            "train": {"tuples": int(ntup), "storms": seeds, "sampled_every_s": 12 * args.dtbig,
                      "samples_per_storm": args.train_samples, "stride": args.train_stride,
                      "sampling_seconds": sample_s, "steps": args.train_steps, "batch": 8192,
                      "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-50:])),
                      "seconds": train_s},
            "eval": "held-out storm: the timed domain, never sampled for training",
            "eval_steps": args.eval_steps, "plain_ms_per_step_timed": plain_ms}


def squall_leg(args, rank):
    """The squall-line configuration at full size: 1024 x 512 x 80, dx =
    500 m, line thermal +2 K with seeded 0.1 K noise, 20 m/s low-level
    shear, cold rain, open radiation x boundaries with per-point phase
    speeds (wbc = ebc = 4), periodic y; dtbig 3 s, dtsml 0.5 s.  Steps
    replayed from CUDA graphs, CUDA-event time on the library's stream."""
    import torch
    import cress_b200
    from cress_b200 import cases
    nx, ny, nz, dx, dtbig, dtsml = args.squall_nx, args.squall_ny, 80, 500.0, 3.0, 0.5
    case = cases.squall_case(nx, ny, nz, dx, seed=21 + rank)
    ni, nj, nk = case["dims"]
    rbct, ksp0 = vspdmp_columns(nk, case["zph"], VSPBAR, 0.6 * case["zph"][nk - 1])
    s = cress_b200.Solver(ni, nj, nk, dx, dx, case["dz"], sthopt=1, cphopt=3, obc=4, gwave=20.0,
                          device=torch.cuda.current_device())
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in MOIST]
    for n, a in zip(NAMES, init):
        s.put_field(n, cress_b200.PAST, a)
        s.put_field(n, cress_b200.NOW, a)
    del case, init
    nsstp = nsstp_of(dtbig, dtsml)
    s.set_graphs(True)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    s.large_step(0, 0.5 * dtbig, nsstp, 0.5 * dtsml)
    step = 1
    for _ in range(13):   # an eager step and a capture per pointer state, then replays
        s.large_step(round(step * dtbig * 1000), dtbig, nsstp, dtsml)
        step += 1
    s.sync()
    k = args.steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        s.large_step(round(step * dtbig * 1000), dtbig, nsstp, dtsml)
        step += 1
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / k
    diag = s.diagnostics(cress_b200.NOW, check=True)
    s.set_stream(0)
    s.close()
    cells = nx * ny * nz
    return {"grid": [nx, ny, nz], "dx_m": dx, "boundaries": "open x (wbc=ebc=4), periodic y",
            "dtbig_s": dtbig, "nsstp": nsstp, "steps": k, "ms_per_step": ms,
            "cell_updates_per_s": cells / (ms * 1e-3), "simulated_s_per_s": dtbig / (ms * 1e-3),
            "max_w_after": diag["max_w"], "timing": "CUDA events on the library stream, graph replay"}


def tke_leg(args, rank, plain_ms):
    """The supercell workload with the 1.5-order TKE closure (tubopt=2, the
    turbulence option of the reference's shipped configurations): the same
    512 x 512 x 64 cold-rain domain, TKE starting from zero and spun up by
    the warm-up steps; steps replayed from CUDA graphs, CUDA-event time on
    the library's stream.  Reported beside the plain workload's step."""
    import torch
    import cress_b200
    from cress_b200 import cases
    nsstp = nsstp_of(args.dtbig, args.dtsml)
    case = make_case(args.nx, args.ny, args.nz, args.dx, 100 + rank)
    ni, nj, nk = case["dims"]
    rbct, ksp0 = vspdmp_columns(nk, case["zph"], VSPBAR, case["botbar"])
    s = cress_b200.Solver(ni, nj, nk, args.dx, args.dx, case["dz"], sthopt=1, tile=max(args.tile, 13),
                          device=torch.cuda.current_device(), cphopt=3, tubopt=2)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in MOIST]
    for n, a in zip(NAMES, init):
        s.put_field(n, cress_b200.PAST, a)
        s.put_field(n, cress_b200.NOW, a)
    del case, init
    s.large_step(0, 0.5 * args.dtbig, nsstp, 0.5 * args.dtsml)
    s.set_graphs(True)
    for _ in range(12 + args.warmup):   # an eager step and a capture per pointer state, then replays
        s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    s.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    tke = s.get_field("tke", cress_b200.NOW)[1:nk - 1, 2:nj - 1, 2:ni - 1]
    diag = s.diagnostics(cress_b200.NOW, check=True)
    s.set_stream(0)
    s.close()
    cells = args.nx * args.ny * args.nz
    return {"grid": [args.nx, args.ny, args.nz], "tubopt": 2, "steps": args.steps, "ms_per_step": ms,
            "cell_updates_per_s": cells / (ms * 1e-3), "plain_ms_per_step": plain_ms,
            "tke_cost_ms": ms - plain_ms, "tke_max_m2s2": float(tke.max()),
            "tke_active_frac": float((tke > 0).mean()), "max_w_after": diag["max_w"],
            "timing": "CUDA events on the library stream, graph replay"}


def records_leg(s, stream, names):
    """Dump and restart records of the workload's state: the device writers
    (cress_dump_3d for every variable s_outdmp dumps with dmpvar
    'ooooooooxxxo', cress_restart_write) into page-locked host buffers,
    against reading the 14 prognostic fields back one by one and cutting
    their dump region on the host (the path without the device writers).
    Wall time around each synchronous call, median of 3."""
    import torch
    import cress_b200
    n = s.restart_size()
    rst = torch.empty(n, dtype=torch.uint8).pin_memory().numpy()

    def med(fn):
        t = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            t.append(time.perf_counter() - t0)
        return float(np.median(t))

    recs, probe_names = s.dump_3d("ooooooooxxxo")
    dmp = torch.empty(recs.shape, dtype=torch.float32).pin_memory().numpy()
    t_dump = med(lambda: s.dump_3d("ooooooooxxxo", out=dmp))
    t_rst = med(lambda: s.restart_write(out=rst))

    def host_path():
        # the same bytes formed on the host from fields read back one by one
        f = {q: s.get_field(q, cress_b200.NOW) for q in names}
        nk = f["u"].shape[0]
        parts = [(np.float32(.5) * (f["u"][1:nk - 2, 2:-3, 2:-3] + f["u"][1:nk - 2, 2:-3, 3:-2]))]
        for q in names[1:]:
            parts.append(f[q][1:nk - 2, 2:-3, 2:-3])
        return np.stack(parts)
    t_host = med(host_path)
    return {"dump": {"variables": probe_names, "bytes": int(dmp.nbytes), "ms": t_dump * 1e3,
                     "gb_per_s": dmp.nbytes / t_dump / 1e9},
            "restart": {"bytes": int(n), "ms": t_rst * 1e3, "gb_per_s": n / t_rst / 1e9},
            "host_readback_and_pack_ms": t_host * 1e3,
            "timing": "wall clock around each synchronous call (page-locked host buffers), median of 3"}


def ensemble_leg(args, rank):
    """Batched ensemble: `members` supercell domains of uneven size (nx, ny
    drawn from 96-192, nz = 48, dx = 1 km) with seeded bubble amplitude
    (1-3 K), position and shear (10-30 m/s).  Three ways to step them:
    member after member; concurrently (each member replays its CUDA graph
    on its own stream); batched (cress_ensemble_large_step: the acoustic
    substeps of all members in one launch per substep, one CUDA graph per
    ensemble step).  Wall time between device synchronizations; reports
    aggregate cell-updates/s of each."""
    import torch
    import cress_b200
    from cress_b200 import cases
    rng = np.random.default_rng(1000 + rank)
    nz, ksteps = 48, 10
    members, total = [], 0
    for mbr in range(args.members):
        nx, ny = int(rng.integers(96, 193)), int(rng.integers(96, 193))
        case = cases.supercell_case(nx, ny, nz, 1000.0, seed=int(rng.integers(1 << 30)),
                                    ptp0=float(rng.uniform(1.0, 3.0)), shear=float(rng.uniform(10.0, 30.0)),
                                    center=(float(rng.uniform(-20e3, 20e3)), float(rng.uniform(-20e3, 20e3))),
                                    rad=(8000.0, 8000.0, 1400.0))
        ni, nj, nk = case["dims"]
        rbct, ksp0 = vspdmp_columns(nk, case["zph"], VSPBAR, 0.6 * case["zph"][nk - 1])
        s = cress_b200.Solver(ni, nj, nk, 1000.0, 1000.0, case["dz"], sthopt=1, cphopt=3, tile=13,
                              device=torch.cuda.current_device())
        s.set_base3d(case["base"])
        s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
        s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
        init = list(case["level"]) + [case["moist"][n] for n in MOIST]
        for n, a in zip(NAMES, init):
            s.put_field(n, cress_b200.PAST, a)
            s.put_field(n, cress_b200.NOW, a)
        s.set_graphs(True)
        s.large_step(0, 0.5 * args.dtbig, nsstp_of(args.dtbig, args.dtsml), 0.5 * args.dtsml)
        members.append(s)
        total += nx * ny * nz
    nsstp = nsstp_of(args.dtbig, args.dtsml)
    for _ in range(13):   # per pointer state (6): an eager step, a capture, then replays
        for s in members:
            s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    torch.cuda.synchronize()

    def timed(concurrent):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if concurrent:
            for _ in range(ksteps):
                for s in members:
                    s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
            for s in members:
                s.sync()
        else:
            for s in members:
                for _ in range(ksteps):
                    s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
                s.sync()
        return time.perf_counter() - t0

    t_seq = timed(False)
    t_con = timed(True)
    # the same members as one ensemble: the acoustic substeps of all members
    # in one launch per substep, the rest on each member's stream, the whole
    # step replayed from one CUDA graph
    ens = cress_b200.Ensemble(members)
    ens.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    tile, tile_ms = ens.autotune(nsstp, args.dtsml, reps=3)   # the batched kernel: tile 0 or 13
    for _ in range(7):
        ens.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ksteps):
        ens.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    ens.sync()
    t_ens = time.perf_counter() - t0
    ens.close()
    for s in members:
        s.close()
    return {"members": args.members, "nz": nz, "cells": total, "steps": ksteps,
            "concurrent_cell_updates_per_s": total * ksteps / t_con,
            "sequential_cell_updates_per_s": total * ksteps / t_seq,
            "batched_cell_updates_per_s": total * ksteps / t_ens,
            "speedup": t_seq / t_con, "batched_speedup": t_seq / t_ens,
            "member_tile": 13, "batched_tile": tile,
            "batched_ms_per_substep": {"tile0": tile_ms[0], "tile13": tile_ms[13]},
            "timing": "wall clock between device synchronizations",
            "launch": "concurrent: one CUDA-graph launch per member per large step, one stream per member; "
                      "batched: cress_ensemble_large_step, one acoustic launch per substep for all members, "
                      "one CUDA graph per step"}


def slab_main(args, rep, cfg_json, nsstp):
    """`--decomp slab`: ONE supercell domain of nx x ny x nz split into y
    slabs over the ranks (one per GPU), the ghost rows and the sedimentation
    sub-step minimum exchanged over NCCL (cress_slab_attach_nccl); total
    work fixed as N grows (strong scaling).  Eager launches (no graphs in
    slab mode); value = all cells x steps / the slowest rank's CUDA-event
    time."""
    import torch
    import cress_b200
    from cress_b200 import cases
    from cress_b200.replicas import CudaEventTimer, timed_steps
    world, rank = rep.world, rep.rank
    case = make_case(args.nx, args.ny, args.nz, args.dx, 100)    # the same domain on every rank
    ni, njg, nk = case["dims"]
    P = njg - 3
    sizes = [P // world + (1 if r < P % world else 0) for r in range(world)]
    off = sum(sizes[:rank])
    rows = 2 + (np.arange(sizes[rank] + 5) - 2 + off) % P          # local rows 0..nj+1 -> global rows
    cut = lambda a: np.ascontiguousarray(a[:, rows, :])
    rbct, ksp0 = vspdmp_columns(nk, case["zph"], VSPBAR, case["botbar"])
    s = cress_b200.Solver(ni, sizes[rank] + 3, nk, args.dx, args.dx, case["dz"], sthopt=1, tile=max(args.tile, 13),
                          device=torch.cuda.current_device(), cphopt=3, tubopt=args.tubopt)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    s.set_base3d({k: cut(v) for k, v in case["base"].items()})
    s.set_base_large(cut(case["base"]["ubr"]), cut(case["base"]["vbr"]), cut(cases.expand(rbct, ni, njg, nk)), ksp0)
    s.set_base_moist(cut(case["base"]["pbr"]), cut(case["base"]["qvbr"]))
    init = list(case["level"]) + [case["moist"][n] for n in MOIST]
    names = NAMES + (["tke"] if args.tubopt == 2 else [])
    if args.tubopt == 2:
        init.append(np.zeros_like(init[0]))
    for n, a in zip(names, init):
        s.put_field(n, cress_b200.PAST, cut(a))
        s.put_field(n, cress_b200.NOW, cut(a))
    del case, init
    uid = [cress_b200.slab_nccl_id() if rank == 0 else None]
    if world > 1:
        import torch.distributed as dist
        dist.broadcast_object_list(uid, src=0)
    s.slab_attach_nccl(rank, world, uid[0])
    s.large_step(0, 0.5 * args.dtbig, nsstp, 0.5 * args.dtsml)
    for _ in range(args.warmup - 1):
        s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    clk = ClockSampler(torch.cuda.current_device())
    secs = timed_steps(rep, lambda: s.large_step(CTIME, args.dtbig, nsstp, args.dtsml), args.steps, 0,
                       CudaEventTimer(stream), sync=torch.cuda.synchronize, inside=clk)
    diag = s.diagnostics(cress_b200.NOW)
    water = rep.sum(diag["water"] + diag["precip"])
    s.slab_detach()
    s.close()
    cells = args.nx * args.ny * args.nz
    if rank == 0:
        cfg = dict(cfg_json, parallelism=f"yslab{world}", slab_rows=sizes)
        print(json.dumps({"metric": METRIC, "value": cells * args.steps / secs, "unit": "cell-updates/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
                          "launch": "eager launches, y-slab ghost rows over NCCL after every substep",
                          "clocks": clk.summary(), "water_plus_precip_kg": water}))
    rep.close()


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
    ap.add_argument("--dtbig", type=float, default=5.0)
    ap.add_argument("--dtsml", type=float, default=1.0)
    ap.add_argument("--impopt", type=int, default=1, choices=[0, 1],
                    help="small step: 1 HE-VI (the configuration's), 0 HE-VE (needs --dtsml short enough)")
    ap.add_argument("--tile", type=int, default=-1,
                    help="HE-VI tile shape; -1 (default): chosen by the autotuner on the live state")
    ap.add_argument("--cpu-steps", type=int, default=2,
                    help="moist large steps of the oracle timed for cpu_baseline (same domain)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-squall", action="store_true")
    ap.add_argument("--no-tke", action="store_true")
    ap.add_argument("--no-records", action="store_true")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="multi-GPU mode: independent domains per GPU (weak scaling) or one domain in y slabs")
    ap.add_argument("--tubopt", type=int, default=0, choices=[0, 1, 2],
                    help="turbulence of the main workload: 0 none, 1 Smagorinsky, 2 TKE closure")
    ap.add_argument("--squall-nx", type=int, default=1024)
    ap.add_argument("--squall-ny", type=int, default=512)
    ap.add_argument("--members", type=int, default=32)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--train-storms", type=int, default=2,
                    help="learned leg: supercell storms of new seeds that supply the training tuples")
    ap.add_argument("--train-samples", type=int, default=3, help="sampled large steps per training storm")
    ap.add_argument("--train-stride", type=int, default=2, help="1 cell in stride sampled")
    ap.add_argument("--train-tuples", type=int, default=50_000_000, help="tuple store capacity")
    ap.add_argument("--eval-steps", type=int, default=6)
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "ours":
        # one process per GPU: start the ranks (torchrun on this node)
        from cress_b200.replicas import relaunch_under_torchrun
        sys.exit(relaunch_under_torchrun(args.gpus, os.path.abspath(__file__), sys.argv[1:]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nsstp = nsstp_of(args.dtbig, args.dtsml)
    # the workload: identical in both arms' lines
    cfg_json = {"workload": f"moist supercell large step (cold-rain bulk cphopt=3; forcing + "
                            f"{nsstp} HE-VI substeps + 10 scalar steps + cloud physics + Asselin "
                            f"filter + saturation adjustment + periodic halos), "
                            f"{args.nx}x{args.ny}x{args.nz}, dx={args.dx:g} m, dz 100->500 m to "
                            f"18 km, dtbig={args.dtbig:g} s, dtsml={args.dtsml:g} s; analytic "
                            f"sounding, quarter-circle hodograph, +3 K bubble, seeded cloud field",
                "nx": args.nx, "ny": args.ny, "nz": args.nz, "nsstp": nsstp,
                "microphysics": "plain (cold-rain bulk)", "tubopt": args.tubopt,
                "l2": "inputs larger than L2 (each field 72 MB at 512x512x64)",
                "parallelism": f"replicas{max(world, args.gpus)}"}
    cells = args.nx * args.ny * args.nz

    if args.impl == "reference":
        # the reference's CPU path (the oracle port) on the same domain, one
        # moist large step per timed step, on rank 0's host cores
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        cpu_run = CpuMoist(args, threads, args.nx, args.ny)
        secs = [cpu_run.step(1) for _ in range(args.warmup + args.steps)]
        t = float(np.median(secs[args.warmup:]))
        v = cells / t
        cpu = {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
               "sample": f"{args.nx}x{args.ny}x{args.nz} supercell domain (the workload itself), one moist "
                         f"large step of the C++ oracle (OpenMP, {threads} threads) per timed step, "
                         f"median of {args.steps} after {args.warmup} warm-up steps"}
        # n_gpus echoes the launch's N so the line pairs with our arm's; the
        # work runs on the host cores (cpu_baseline.cores) of rank 0 alone
        print(json.dumps({"metric": METRIC, "value": v, "unit": "cell-updates/s",
                          "n_gpus": max(world, args.gpus), "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": t * 1e3, "impl": "reference",
                          "hardware": f"host CPU, {threads} threads",
                          "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
                          "config": cfg_json, "cpu_baseline": cpu,
                          "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    import cress_b200
    from cress_b200 import cases
    from cress_b200.replicas import CudaEventTimer, Replicas, timed_steps

    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    if args.decomp == "slab":
        return slab_main(args, rep, cfg_json, nsstp)
    case = make_case(args.nx, args.ny, args.nz, args.dx, 100 + rank)
    ni, nj, nk = case["dims"]
    rbct, ksp0 = vspdmp_columns(nk, case["zph"], VSPBAR, case["botbar"])
    s = cress_b200.Solver(ni, nj, nk, args.dx, args.dx, case["dz"], sthopt=1, tile=max(args.tile, 0), impopt=args.impopt,
                          device=local, cphopt=3, tubopt=args.tubopt)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s.set_stream(stream.cuda_stream)
    s.set_base3d(case["base"])
    s.set_base_large(case["base"]["ubr"], case["base"]["vbr"], cases.expand(rbct, ni, nj, nk), ksp0)
    s.set_base_moist(case["base"]["pbr"], case["base"]["qvbr"])
    init = list(case["level"]) + [case["moist"][n] for n in MOIST]
    names = NAMES
    if args.tubopt == 2:   # the TKE from zero, a prognostic field like the others
        init.append(np.zeros_like(init[0]))
        names = NAMES + ["tke"]
    for n, a in zip(names, init):
        s.put_field(n, cress_b200.PAST, a)
        s.put_field(n, cress_b200.NOW, a)
    s.sync()

    def barrier():
        torch.cuda.synchronize()
        rep.barrier()
        torch.cuda.synchronize()

    max_over_ranks = rep.max

    s.large_step(0, 0.5 * args.dtbig, nsstp, 0.5 * args.dtsml)   # the first (half) step, ctime=0
    tune = None
    if args.tile < 0 and args.impopt == 1:
        best, tms = s.autotune(nsstp=nsstp, dts=args.dtsml, reps=2)
        tune = {"tile": best, "ms_per_substep": [round(t, 4) for t in tms]}
    hevi_tile = tune["tile"] if tune else max(args.tile, 0)
    if not args.no_graphs:
        # capture the CUDA graphs of the time-level rotation's 6 pointer
        # states (an eager step and a capture each) before the warm-up
        s.set_graphs(True)
        for _ in range(12):
            s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    for _ in range(args.warmup - 1):
        s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
    barrier()
    d0 = s.diagnostics(cress_b200.NOW)
    l0 = s.launch_count()
    clk = ClockSampler(local)
    secs = timed_steps(rep, lambda: s.large_step(CTIME, args.dtbig, nsstp, args.dtsml), args.steps, 0,
                       CudaEventTimer(stream), sync=torch.cuda.synchronize, inside=clk)
    launches = s.launch_count() - l0
    d1 = s.diagnostics(cress_b200.NOW)
    budget = {"water_kg": [d0["water"], d1["water"]], "precip_kg": [d0["precip"], d1["precip"]],
              "mass_kg": [d0["mass"], d1["mass"]],
              "water_drift_rel": ((d1["water"] + d1["precip"]) - (d0["water"] + d0["precip"])) / d0["water"],
              "mass_drift_rel": (d1["mass"] - d0["mass"]) / d0["mass"], "max_w": d1["max_w"],
              "nonfinite": int(d1["nonfinite"]), "over": f"{args.steps} timed steps (FP64 sums on the device)"}
    ms = secs * 1e3
    value = world * cells * args.steps / secs

    # Dominant kernel (HE-VI substep): timed alone on the same state.
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(2, args.steps // 2)
    s.small_steps(nsstp, args.dtsml)
    barrier()
    h0.record(stream)
    for _ in range(reps):
        s.small_steps(nsstp, args.dtsml)
    h1.record(stream)
    barrier()
    hevi_ms = max_over_ranks(h0.elapsed_time(h1)) / (reps * nsstp)
    peak, peak_kind = measured_peaks()
    achieved = HEVI_BYTES_PER_CELL * cells / (hevi_ms * 1e-3) / 1e9

    learned = None if args.no_learned else learned_leg(args, s, stream, nsstp, cells, ms / args.steps,
                                                        barrier, max_over_ranks, rank)
    ensemble = None if args.no_ensemble else ensemble_leg(args, rank)
    squall = None if args.no_squall else squall_leg(args, rank)
    tke = None if args.no_tke else tke_leg(args, rank, ms / args.steps)

    # End to end through the public API with host buffers: every step the
    # past and present levels (14 fields each) go host->device from pinned
    # memory, one large step runs, the new present level (14 fields) comes
    # back.  The inputs of step n+1 are queued on their own stream before
    # the host waits, so they cross while step n computes; the read-back of
    # step n runs on a third stream (the link is full duplex); the host
    # waits for step n-1's result while step n's is in flight (results
    # double-buffered).
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    past_h = [pin(a) for a in init]
    now_h = [pin(a) for a in init]
    out_h = [[pin(np.empty_like(a)) for a in init] for _ in range(2)]

    def e2e_run(nsteps):
        s.put_fields_async(cress_b200.PAST, names, past_h)
        s.put_fields_async(cress_b200.NOW, names, now_h)
        for i in range(nsteps):
            s.large_step(CTIME, args.dtbig, nsstp, args.dtsml)
            s.get_fields_async(cress_b200.NOW, names, out_h[i % 2])
            if i + 1 < nsteps:   # the next step's inputs
                s.put_fields_async(cress_b200.PAST, names, past_h)
                s.put_fields_async(cress_b200.NOW, names, now_h)
            s.wait_fields(in_flight=1)   # step i-1's result is on the host
        s.wait_fields()

    e2e_run(args.warmup)
    barrier()
    t0 = time.perf_counter()
    e2e_run(args.steps)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": int(sum(a.nbytes for a in past_h + now_h)),
           "d2h_bytes_per_step": int(sum(a.nbytes for a in out_h[0])),
           "overlap": "host->device copies of step n+1 on their own stream during step n's compute; "
                      "device->host read-back of step n on a third stream during step n+1's host->device copies; "
                      "the host waits for step n-1's result while step n's is in flight"}
    io = None if args.no_records else records_leg(s, stream, names)
    s.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cpu_run = CpuMoist(args, threads, args.nx, args.ny)
        dt = cpu_run.step(args.cpu_steps)
        cpu = {"value": cells * args.cpu_steps / dt, "unit": "cell-updates/s", "cores": threads,
               "kind": "port",
               "sample": f"{args.nx}x{args.ny}x{args.nz} supercell domain (the workload's), {args.cpu_steps} "
                         f"moist large steps of the C++ oracle (OpenMP, {threads} threads), {dt:.2f} s"}
        del cpu_run

    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg_json,
            "launch": "CUDA-graph replay per large step" if not args.no_graphs else "eager launches",
            "small_step": "HE-VI (impopt=1)" if args.impopt == 1 else "HE-VE (impopt=0)",
            "hevi_tile": hevi_tile,
            "sim_s_per_wall_s": args.dtbig / (ms / args.steps * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (HEVI_TRAFFIC_PER_CELL[hevi_tile] * cells
                                     if hevi_tile in HEVI_TRAFFIC_PER_CELL and args.impopt == 1 else None),
                         "traffic_source": "ncu dram bytes per cell at 384x384x64 scaled to this grid",
                         "peak_source": peak_kind,
                         "kernel": ("k_heve" if args.impopt == 0 else
                                    HEVI_KERNEL.get(hevi_tile, "k_hevi_substep")),
                         "bytes_per_launch": HEVI_BYTES_PER_CELL * cells,
                         "ms_per_launch": hevi_ms},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clk.summary(),
            "cpu_baseline": cpu, "learned": learned, "ensemble": ensemble, "squall_line": squall,
            "tke_closure": tke, "records": io,
            "budget": budget, "autotune": tune}))
    rep.close()


if __name__ == "__main__":
    main()

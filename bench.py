"""Benchmark of the RK4 time-stepping path on B200.

Workload (the configuration the headline metric is quoted on): FD scheme
(central FD4 + KO3), periodic z in [-3000, 3000] with nz = 32768, nvz = 256,
mu = 1, omega = 1e-3, normal ordering, theta = 1e-6 deg, CFL 0.4, FP64,
seeded synthetic initial condition (sigma_nu 0.6, sigma_nubar 0.5,
alpha 0.9, +-1e-6 ex).  A "step" is one RK4 step over the whole grid; the
metric is cell-updates/s = nz * nvz * steps / time.

  value  device-resident: K steps timed with CUDA events on the stream the
         kernels run on (per stage, so the dominant kernel's duration is
         measured in the same region); the state (537 MB per buffer) is far
         larger than L2, so no flush is needed between steps.
  e2e    through the public API with host buffers: pinned host state ->
         upload -> K steps with on-device analysis every 40 steps (the
         reference driver's ANAL_EVERY for this run) and after the last
         step -> download.
  cpu_baseline / --impl reference: the reference's own CPU build
         (oracle/_ref, compiled from its sources with its --mcore flags)
         on a z-subset of the same grid, all host threads.

Multi-GPU (torchrun): every rank evolves its own instance (different seed),
no data-path collective; value = all ranks' cell-updates / max-over-ranks
time ("weak" scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s (nz*nvz*RK4 steps), FP64"
UNIT = "cell-updates/s"
# c2: FD at scale (the headline); c1: FV WENO7 on the small 1024 x 64 grid; c3: FV
# at 65536 x 512 (FP32-bulk form, FP64 for comparison)
WORKLOADS = {
    "c2": dict(nz=32768, nvz=256, gz=2, z0=-3000.0, z1=3000.0, v0=-1.0, v1=1.0, cfl=0.4,
               pmo=1.0, omega=1e-3, theta_deg=1e-6, mu=1.0, scheme="fd"),
    "c1": dict(nz=1024, nvz=64, gz=4, z0=-600.0, z1=600.0, v0=-1.0, v1=1.0, cfl=0.4,
               pmo=1.0, omega=0.0, theta_deg=0.0, mu=1.0, scheme="fv"),
    "c3": dict(nz=65536, nvz=512, gz=4, z0=-600.0, z1=600.0, v0=-1.0, v1=1.0, cfl=0.4,
               pmo=1.0, omega=0.0, theta_deg=0.0, mu=1.0, scheme="fv"),
}
WORKLOAD_NAMES = {
    "c2": "FD (central FD4 + KO3) RK4, nz 32768 x nvz 256, periodic, mu 1, omega 1e-3, "
          "theta 1e-6 deg",
    "c1": "FV WENO7 RK4, nz 1024 x nvz 64, periodic, mu 1, omega 0",
    "c3": "FV WENO7 RK4, nz 65536 x nvz 512, periodic, mu 1, omega 0",
}
WORKLOAD = dict(WORKLOADS["c2"])
IC = dict(sig_nu=0.6, sig_nubar=0.5, alpha=0.9, amp=1e-6)
SEED = 20240601
ANAL_EVERY = 40  # manage.py: N_ITER = 4000 steps, n_analyze = 100
# algorithmic bytes per cell of stages 1..4 (64 B per FP64 state pass).  FP64:
# stage 1 reads Y, writes U; stage 2 reads U, Y, writes U'; stage 3 reads U',
# Y and U, writes U'' and A; stage 4 reads U'', A, writes Y (832 B per
# cell-update).  FP32-bulk (FP64 Y, FP32 increments D, 32 B per pass): stage 1
# reads Y, writes D1; stage 2 reads Y, D1, writes D2; stage 3 reads Y, D2,
# writes D3; stage 4 reads Y, D3, D1, D2, writes the new Y (576 B).
STAGE_BYTES = {"fp64": (128, 192, 320, 192), "fp32": (96, 128, 128, 224)}
FALLBACK_HBM_GBS = 6650.0


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profile():
    """Per-launch DRAM bytes of the stage-2 FD kernel from the committed ncu
    summary (scaled to the full grid there), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(p))
    except Exception:
        return None


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    FIELDS = ("clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) != len(self.FIELDS):
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[3:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def dist_setup(ngpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != ngpus and world > 1:
        raise SystemExit(f"--gpus {ngpus} but WORLD_SIZE {world}")
    return rank, world, local


def run_ours(args):
    import datetime

    import numpy as np
    import torch

    from cosenu_b200 import NuOsc

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sim = NuOsc(device=local, precision=args.precision, **WORKLOAD)
    sim.set_stream(stream.cuda_stream)
    cells = WORKLOAD["nz"] * WORKLOAD["nvz"]
    sim.init_seeded(SEED + rank, **IC)
    for _ in range(args.warmup):
        sim.step_rk4()
    sim.prepare_graphs()  # no graph capture inside the timed region
    barrier()

    # ---- device-resident timed region: K steps through the stepping API
    # (cosenu_step: four stage kernels per step, replayed from CUDA graphs),
    # events on the launching stream; then the same K steps once more with one
    # launch per stage and events between the stages, for the per-kernel
    # durations of the roofline
    K = args.steps
    e_run0, e_run1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4 * K + 1)]
    with ClockSampler(local) as clk:
        barrier()
        e_run0.record(stream)
        sim.evolve(K)
        e_run1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ev[0].record(stream)
        for k in range(K):
            for s in range(4):
                sim.step_stage(s)
                ev[4 * k + s + 1].record(stream)
        torch.cuda.synchronize()
    barrier()
    total_ms = e_run0.elapsed_time(e_run1)
    stagewise_ms = ev[0].elapsed_time(ev[-1])
    stage_ms = [0.0] * 4
    for k in range(K):
        for s in range(4):
            stage_ms[s] += ev[4 * k + s].elapsed_time(ev[4 * k + s + 1])
    stage_ms = [t / K for t in stage_ms]
    if dist:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = cells * K * world / (total_ms / 1e3)
    diag = sim.analyse()
    if not math.isfinite(diag["M0"]):
        raise SystemExit("non-finite state after the timed region")

    # ---- end to end through the public API with pinned host buffers
    host0 = sim.download()
    pinned = torch.from_numpy(host0).pin_memory()
    hbuf = pinned.numpy()
    out_pinned = torch.empty_like(pinned).pin_memory()
    obuf = out_pinned.numpy()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_anal = 0
    e0.record(stream)
    sim.upload(hbuf)
    sim.mark_state0()
    done = 0
    while done < K:
        n = min(ANAL_EVERY, K - done)
        sim.evolve(n)
        done += n
        # the reference driver's cadence, plus the end of the run (so the
        # leg analyses at least once whatever K is)
        if done % ANAL_EVERY == 0 or done == K:
            sim.analyse()
            n_anal += 1
    from cosenu_b200.nuosc import _ptrs
    sim._check(sim.lib.cosenu_download(sim.h, _ptrs(obuf), sim.gz))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = cells * K * world / (e2e_ms / 1e3)
    state_bytes = 8 * WORKLOAD["nvz"] * (WORKLOAD["nz"] + 2 * WORKLOAD["gz"]) * 8
    h2d = state_bytes / K
    d2h = (state_bytes + n_anal * 13 * 8) / K

    tz, tv = sim.tile()
    result = None
    if rank == 0:
        peak, peak_src = peak_hbm()
        sb = STAGE_BYTES[args.precision]
        # the slowest of the stages moving the most bytes
        dom = max((i for i in range(4) if sb[i] == max(sb)), key=lambda i: stage_ms[i])
        algo_bytes = sb[dom] * cells
        achieved = algo_bytes / (stage_ms[dom] / 1e3) / 1e9
        tr = traffic_from_profile()
        key = f"{args.workload}_{args.precision}_stage{dom + 1}_bytes_per_launch"
        traffic = tr.get(key) if (tr and WORKLOAD["nz"] == WORKLOADS[args.workload]["nz"]) else None
        cpu = cpu_baseline(args) if (world == 1 and not args.no_cpu_baseline) else None
        buf_mb = 8 * WORKLOAD["nvz"] * (WORKLOAD["nz"] + 32) * 8 / 1e6
        sch = WORKLOAD["scheme"].upper()
        result = {
            "metric": METRIC if args.precision == "fp64" else METRIC.replace("FP64", "FP32-bulk"),
            "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": total_ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 (FP64 moments/accumulator/base)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_NAMES[args.workload], "name": args.workload,
                       "nz": WORKLOAD["nz"], "nvz": WORKLOAD["nvz"], "scheme": sch,
                       "precision": args.precision.upper(), "tile": [tz, tv],
                       "l2": f"inputs larger than L2 ({buf_mb:.0f} MB per state buffer)"
                             if buf_mb > 126 else "inputs fit in L2 (small case)",
                       "instances_per_gpu": 1},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "n_anal": n_anal,
                    "note": f"upload once, {K} steps, on-device analysis every {ANAL_EVERY} "
                            f"steps and after the last ({n_anal} in all), download once"},
            "gpu_launches": 4 * K,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": f"rk4_stage_tma_kernel<{sch}, stage {dom + 1}> "
                                   f"({sb[dom] // 64 if args.precision == 'fp64' else sb[dom]} "
                                   f"{'state passes' if args.precision == 'fp64' else 'B/cell'})",
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "avg_launch_ms": stage_ms[dom], "peak_source": peak_src},
            "stage_ms": stage_ms,
            "stage_ms_note": f"per-launch CUDA-event durations from a second pass of the same {K} "
                             f"steps launched stage by stage ({stagewise_ms / K:.4f} ms per step "
                             f"that way); value and ms_per_step time the graph-launched steps",
            "gpu_launches_note": "the four stage kernels of each step, from CUDA graphs",
            "step_hbm_frac": (sum(sb) * cells / (total_ms / K / 1e3) / 1e9) / peak,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(result), flush=True)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


# ---------------------------------------------------------------------------
def _ref_exe():
    from oracle.build import ref_binary
    exe = ref_binary(WORKLOAD["scheme"])
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    return exe


def _ref_run(nz_sample: int, nsteps: int, threads: int):
    """Reference FD binary on a z-subset of the workload grid (same dz, nvz,
    physics), through its --ff path; returns the loop seconds (time.txt)."""
    from oracle.oracle import Case, Oracle, run_reference
    w = WORKLOAD
    dz = (w["z1"] - w["z0"]) / w["nz"]
    case = Case(nz=nz_sample, nvz=w["nvz"], gz=w["gz"], z0=-0.5 * nz_sample * dz,
                z1=0.5 * nz_sample * dz, cfl=w["cfl"], pmo=w["pmo"], omega=w["omega"],
                theta_deg=w["theta_deg"], mu=w["mu"], scheme=w["scheme"])
    o = Oracle()
    G, bG, st0 = o.init_seeded(case, seed=SEED, **IC)
    n_iter = max(nsteps + 1, 10)
    r = run_reference(case, G, bG, st0, n_iter=n_iter, anal_every=n_iter + 1, n_dump_rho=0,
                      nthreads=threads)
    return r["loop_seconds"], n_iter - 1


def cpu_baseline(args, budget_s: float = 20.0):
    """~10-30 s of the reference's own CPU path on this host's cores."""
    try:
        _ref_exe()
    except FileNotFoundError:
        return None
    threads = os.cpu_count() or 1
    nvz = WORKLOAD["nvz"]
    t, n = _ref_run(64, 9, threads)  # calibration
    per_cell_step = t / (64 * nvz * n)
    nz = 64
    while nz * 2 <= WORKLOAD["nz"] and per_cell_step * nz * 2 * nvz * 9 <= budget_s:
        nz *= 2
    t, n = _ref_run(nz, 9, threads)
    return {"value": nz * nvz * n / t, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"reference {WORKLOAD['scheme'].upper()} build (g++ -O3 -fopenmp, "
                      f"OMP_NUM_THREADS={threads}), "
                      f"{n} RK4 steps on a z-subset nz={nz} of the workload grid "
                      f"(same dz, nvz={nvz}, physics), loop time from its time.txt"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    try:
        _ref_exe()
    except FileNotFoundError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference build missing: {e}"}))
        return
    threads = os.cpu_count() or 1
    nvz = WORKLOAD["nvz"]
    # size the z-subset so that warm-up + K steps take about 90 s (the
    # reference driver needs N_ITER >= 10, i.e. at least 9 steps per run)
    t, n = _ref_run(512, 9, threads)
    per_cell_step = t / (512 * nvz * n)
    K, W = max(args.steps, 9), args.warmup
    W_run = max(W, 9) if W > 0 else 0
    nz = 64
    while nz * 2 <= WORKLOAD["nz"] and per_cell_step * nz * 2 * nvz * (K + W_run) <= 90.0:
        nz *= 2
    if W_run:
        _ref_run(nz, W_run, threads)
    t, n = _ref_run(nz, K, threads)
    value = nz * nvz * n / t
    sample = (f"reference {WORKLOAD['scheme'].upper()} build (g++ -O3 -fopenmp, "
              f"OMP_NUM_THREADS={threads}), {n} RK4 "
              f"steps on a z-subset nz={nz} of the workload grid (same dz, nvz={nvz}, physics); "
              "loop time from its time.txt")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": n, "warmup": W, "ms_per_step": t / n * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAMES[args.workload], "name": args.workload,
                   "sample_nz": nz},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_ensemble(args):
    """The ensemble workload: 256 uneven FV instances to t = 1000/mu.  On N
    GPUs (torchrun) every rank runs its balanced share as one batched ensemble
    (autotuned kernel family and tiles) and only the results are gathered;
    the time is the slowest rank's.  At N = 1 the plain single-instance FP64
    path is also timed, on a stratified subset (every 8th instance, full step
    counts) scaled by work, and the batched results are held to it."""
    import datetime

    import torch

    from cosenu_b200 import NuOsc
    from cosenu_b200.distributed import run_ensemble_sharded
    from cosenu_b200.ensemble import ensemble_instances

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    xs = ensemble_instances(args.instances, t_factor=args.t_factor)
    work = [x.cells * x.nsteps for x in xs]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    cfg = {}

    def runner(chunk, **kw):
        from cosenu_b200.ensemble import run_on_gpu
        res, secs, c = run_on_gpu(chunk, **kw)
        cfg.update(c)
        return res, secs

    with ClockSampler(local) as clk:
        results, t_batch, share = run_ensemble_sharded(
            xs, dist, runner=runner, reduce_device=torch.device("cuda", local),
            precision=args.precision, device=local, stream=stream)
    pee = [r["Pee"] for r in results]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    n = len(xs)
    line = {
        "metric": "instances/s (256-instance FV ensemble to t = 1000/mu)", "value": n / t_batch,
        "unit": "instances/s", "n_gpus": world, "instances": n,
        "cell_updates_per_s": sum(work) / t_batch, "seconds": t_batch,
        "higher_is_better": True, "scaling": "strong", "precision": args.precision.upper(),
        "data": "synthetic",
        "config": {"workload": "256 FV WENO7 instances, nz logU[512,8192]/256, nvz {32..256}, "
                               "alpha U[.6,1.2], sigma U[.4,.8]/U[.3,.7], mu U[.5,2], "
                               "t = 1000/mu", "t_factor": args.t_factor,
                   "sharding": f"{world} ranks, members partitioned by nz*nvz*steps, results "
                               "gathered, time max over ranks",
                   "kernel (rank 0)": {k: v for k, v in cfg.items() if k != "autotune"},
                   "rank0_members": len(share)},
        "autotune (rank 0)": cfg.get("autotune", []), "clocks": clk.summary(),
    }
    if world == 1:
        # plain path: every 8th instance alone, FP64, default kernel choice
        sub = list(range(0, n, 8))
        t_sub = 0.0
        pee_err = 0.0
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for i in sub:
            x = xs[i]
            sim = NuOsc(nz=x.nz, nvz=x.nvz, gz=4, z0=x.z0, z1=x.z1, cfl=x.cfl, omega=0.0,
                        mu=x.mu, scheme="fv")
            sim.set_stream(stream.cuda_stream)
            sim.init_seeded(x.seed, instance=x.index, sig_nu=x.sig_nu, sig_nubar=x.sig_nubar,
                            alpha=x.alpha)
            torch.cuda.synchronize()
            ev0.record(stream)
            sim.evolve(x.nsteps)
            ev1.record(stream)
            torch.cuda.synchronize()
            t_sub += ev0.elapsed_time(ev1) / 1e3
            d = abs(sim.analyse()["Pee"] - pee[i])
            if args.precision == "fp64" and d > 1e-9:
                raise SystemExit(f"ensemble member {i} differs from the plain path: {d}")
            pee_err = max(pee_err, d)
            sim.close()
        w_sub = sum(work[i] for i in sub)
        t_plain = t_sub * sum(work) / w_sub
        line.update({
            "plain_fp64_instances_per_s": n / t_plain,
            "plain_fp64_note": f"{len(sub)} of {n} instances run alone ({t_sub:.1f} s), "
                               "scaled by work",
            "speedup_vs_plain": t_plain / t_batch,
            "max_abs_err_final_Pee_vs_plain_fp64": pee_err,
            "err_subset": f"the {len(sub)} instances run alone"})
    print(json.dumps(line), flush=True)


def run_divergence_study(args):
    """Where in time the ensemble's final-P_ee difference comes from: for every
    32nd member of the ensemble workload, three runs of the same seeded set-up
    to t = 1000/mu -- FP64 (default kernel), FP64 with a different velocity-moment
    summation order (register-tiled kernel, 16 x 8 tiles: the same arithmetic up
    to rounding), and FP32-bulk -- with <P_ee> every 1/200 of the run.  Reports the
    saturation time (first |1 - <P_ee>| > 1e-2) and the first time each
    difference from the FP64 run exceeds 1e-6."""
    import torch

    from cosenu_b200 import NuOsc
    from cosenu_b200.ensemble import ensemble_instances

    torch.cuda.set_device(0)
    xs = ensemble_instances(args.instances, t_factor=args.t_factor)
    out = []
    for i in range(0, len(xs), 32):
        x = xs[i]
        runs = {}
        for name, kw in (("fp64", {}), ("fp64_reordered", {"tile_z": 16, "tile_v": 8}),
                         ("fp32_bulk", {"precision": "fp32"})):
            sim = NuOsc(nz=x.nz, nvz=x.nvz, gz=4, z0=x.z0, z1=x.z1, cfl=x.cfl, omega=0.0,
                        mu=x.mu, scheme="fv", **kw)
            sim.init_seeded(x.seed, instance=x.index, sig_nu=x.sig_nu, sig_nubar=x.sig_nubar,
                            alpha=x.alpha)
            k = max(1, x.nsteps // 200)
            t, done, pee = [], 0, []
            while done < x.nsteps:
                n = min(k, x.nsteps - done)
                sim.evolve(n)
                done += n
                t.append(done * sim.dt)
                pee.append(sim.analyse()["Pee"])
            sim.close()
            runs[name] = (t, pee)
        t, p64 = runs["fp64"]
        t_sat = next((tt for tt, p in zip(t, p64) if abs(1.0 - p) > 1e-2), None)
        rec = {"member": i, "nz": x.nz, "nvz": x.nvz, "mu": x.mu, "t_end": t[-1],
               "t_saturation": t_sat, "final_Pee_fp64": p64[-1]}
        for name in ("fp64_reordered", "fp32_bulk"):
            d = [abs(a - b) for a, b in zip(runs[name][1], p64)]
            rec[f"{name}_final_diff"] = d[-1]
            rec[f"{name}_max_diff"] = max(d)
            rec[f"{name}_t_diff_gt_1e-6"] = next((tt for tt, e in zip(t, d) if e > 1e-6), None)
            rec[f"{name}_max_diff_before_saturation"] = max(
                [e for tt, e in zip(t, d) if t_sat is None or tt < t_sat] or [0.0])
        out.append(rec)
        print(json.dumps(rec), flush=True)
    print(json.dumps({"study": "P_ee divergence in the ensemble workload", "members": out}),
          flush=True)


def run_fp32_study(args):
    """FV at 65536 x 512: the FP32-bulk form against the FP64 form on the same seeded
    input: max-abs error per component at the end, <Pee>(t) error, trace and
    ELN drift of both, and the throughput of each (timed separately)."""
    import numpy as np
    import torch

    from cosenu_b200 import NuOsc

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    n, every = args.study_steps, max(1, args.study_steps // 20)
    out = {}
    sims = {}
    for prec in ("fp64", "fp32"):
        sim = NuOsc(precision=prec, **WORKLOAD)
        sim.set_stream(stream.cuda_stream)
        sim.init_seeded(SEED, **IC)
        sims[prec] = sim
    hist = {"fp64": [], "fp32": []}
    times = {"fp64": 0.0, "fp32": 0.0}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0 = {p: sims[p].analyse() for p in sims}
    done = 0
    while done < n:
        k = min(every, n - done)
        for prec, sim in sims.items():
            e0.record(stream)
            sim.evolve(k)
            e1.record(stream)
            torch.cuda.synchronize()
            times[prec] += e0.elapsed_time(e1) / 1e3
            hist[prec].append(sim.analyse())
        done += k
    st = {p: sims[p].download() for p in sims}
    gz = WORKLOAD["gz"]
    err = np.abs(st["fp32"][:, :, gz:-gz] - st["fp64"][:, :, gz:-gz]).reshape(8, -1).max(axis=1)
    dpee = max(abs(a["Pee"] - b["Pee"]) for a, b in zip(hist["fp32"], hist["fp64"]))
    dpbee = max(abs(a["Pbee"] - b["Pbee"]) for a, b in zip(hist["fp32"], hist["fp64"]))
    drift = {p: {"trace": abs(hist[p][-1]["trace"] - a0[p]["trace"]) / abs(a0[p]["trace"]),
                 "btrace": abs(hist[p][-1]["btrace"] - a0[p]["btrace"]) / abs(a0[p]["btrace"]),
                 "eln": abs(hist[p][-1]["eln"] - a0[p]["eln"]) / abs(a0[p]["eln"])}
             for p in sims}
    cells = WORKLOAD["nz"] * WORKLOAD["nvz"]
    print(json.dumps({
        "study": "FP32-bulk vs FP64", "workload": WORKLOAD_NAMES[args.workload],
        "steps": n, "t_end": n * sims["fp64"].dt,
        "max_abs_err_per_component": dict(zip(("ee", "xx", "ex_re", "ex_im", "bee", "bxx",
                                                "bex_re", "bex_im"), err.tolist())),
        "max_abs_err_Pee_t": dpee, "max_abs_err_Pbee_t": dpbee,
        "final_Pee": {p: hist[p][-1]["Pee"] for p in sims},
        "relative_drift": drift,
        "cell_updates_per_s": {p: cells * n / times[p] for p in sims},
        "speedup_fp32_over_fp64": times["fp64"] / times["fp32"],
    }), flush=True)
    for s_ in sims.values():
        s_.close()


def run_surrogate(args):
    """The surrogate workload (nz fixed at 512 by default to fit the training
    set in the run time; --sur-nz 0 draws it log-uniform in [512, 8192] as
    the ensemble distribution does): solver targets for a training and a
    held-out set, a committee of networks trained on the GPU, held-out error
    against the solver with and without the disagreement fallback, and the
    time of both routes."""
    import numpy as np
    import torch

    from cosenu_b200.surrogate import (Surrogate, features, reseeded, solve_pee,
                                       surrogate_instances)

    torch.cuda.set_device(0)
    sur_nz = args.sur_nz or None  # 0: log-uniform in [512, 8192]
    train = surrogate_instances(args.train, seed=21, nz=sur_nz, t_factor=args.t_factor)
    test = surrogate_instances(args.test, seed=22, nz=sur_nz, t_factor=args.t_factor)
    t0 = time.perf_counter()
    y_train = solve_pee(train)
    t_train_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    y_test = solve_pee(test)
    torch.cuda.synchronize()
    t_solver = time.perf_counter() - t0
    # the solver's own seed-to-seed spread on the first 128 held-out set-ups
    y_reseed = solve_pee(reseeded(test[:128]))
    noise = float(np.abs(y_reseed - y_test[:128]).mean())
    x_train = np.stack([features(i) for i in train])
    x_test = np.stack([features(i) for i in test])
    sur = Surrogate(n_models=4)
    t0 = time.perf_counter()
    losses = sur.fit(x_train, y_train, epochs=args.epochs, batch=64, lr=2e-3)
    t_fit = time.perf_counter() - t0
    # device time per kernel class: one more training epoch of the committee
    # and one committee inference over the held-out set, with CUDA events
    sur.set_timing(True)
    for k, m in enumerate(sur.models):
        m.train(epochs=1, batch=64, lr=1e-5, seed=9000 + k)
    train_ms = sur.timing()
    sur.set_timing(True)
    sur.committee(x_test)
    infer_ms = sur.timing()
    sur.set_timing(False)
    sur.committee(x_test)  # warm-up at the timed batch size (activation buffers sized)
    t0 = time.perf_counter()
    mean, spread = sur.committee(x_test)
    t_net = time.perf_counter() - t0
    err = np.abs(mean - y_test)
    fb = spread > args.threshold
    final = mean.copy()
    final[fb] = y_test[fb]  # the solver's own answer where the committee falls back
    t_with_fb = t_net + t_solver * fb.mean()
    err_fb = np.abs(final - y_test)
    # generalisation beyond the training resolution: held-out instances with
    # nz log-uniform in [512, 8192] (the ensemble workload's distribution), solver
    # targets at their own nz
    gen = {}
    if args.gen_test > 0:
        gtest = surrogate_instances(args.gen_test, seed=23, nz=None, t_factor=args.t_factor)
        t0 = time.perf_counter()
        y_gen = solve_pee(gtest)
        t_gen_solver = time.perf_counter() - t0
        x_gen = np.stack([features(i) for i in gtest])
        g_mean, g_spread = sur.committee(x_gen)
        g_err = np.abs(g_mean - y_gen)
        g_fb = g_spread > args.threshold
        g_final = g_mean.copy()
        g_final[g_fb] = y_gen[g_fb]
        nzs = np.array([i.nz for i in gtest])
        gen = {"instances": len(gtest), "nz_range": [int(nzs.min()), int(nzs.max())],
               "mean_abs_err": float(g_err.mean()),
               "mean_abs_err_nz_le_1024": float(g_err[nzs <= 1024].mean()) if (nzs <= 1024).any() else None,
               "mean_abs_err_nz_gt_2048": float(g_err[nzs > 2048].mean()) if (nzs > 2048).any() else None,
               "fallback_fraction": float(g_fb.mean()),
               "mean_abs_err_with_fallback": float(np.abs(g_final - y_gen).mean()),
               "solver_seconds": t_gen_solver}
    tot = lambda d: sum(d.values())  # noqa: E731
    print(json.dumps({
        "metric": "surrogate vs solver on held-out instances", "train": len(train),
        "test": len(test), "nz": args.sur_nz or "log-uniform [512, 8192]", "nvz": 128, "t_factor": args.t_factor,
        "mean_abs_err": float(err.mean()), "rms_err": float(np.sqrt((err ** 2).mean())),
        "p95_instance_max_err": float(np.percentile(err.max(axis=1), 95)),
        "fallback_threshold": args.threshold, "fallback_fraction": float(fb.mean()),
        "mean_abs_err_with_fallback": float(err_fb.mean()),
        "solver_seed_to_seed_mean_abs_diff": noise,
        "baseline_mean_abs_err_train_average": float(np.abs(y_train.mean(0) - y_test).mean()),
        "baseline_mean_abs_err_no_conversion": float(np.abs(1.0 - y_test).mean()),
        "solver_seconds_test": t_solver, "surrogate_seconds_test": t_net,
        "speedup_surrogate_only": t_solver / t_net,
        "speedup_with_fallback": t_solver / t_with_fb,
        "train_data_seconds": t_train_data, "train_seconds": t_fit,
        "final_train_loss": [float(ls[-1]) for ls in losses],
        "device_ms_per_kernel_class": {
            "training_one_epoch_committee": train_ms,
            "training_gemm_share": train_ms["gemm"] / tot(train_ms),
            "inference_committee": infer_ms,
            "inference_gemm_share": infer_ms["gemm"] / tot(infer_ms)},
        "held_out_nz_loguniform": gen,
    }), flush=True)
    sur.close()


def run_surrogate_gemm_study(args):
    """Device time of the surrogate network's kernels with each GEMM kernel
    (tcgen05 with the accumulator in tensor memory, and the warp-level
    mma.sync kernel, COSENU_MLP_GEMM=mma): a committee of 4 networks
    258 -> 3 x 512 -> 128 on synthetic features and targets of the workload's
    shapes; one training epoch over 4096 rows (batches of 64) and one
    committee inference over 2048 rows, CUDA events around every launch."""
    import numpy as np
    import torch

    from cosenu_b200.surrogate import Surrogate

    torch.cuda.set_device(0)
    rng = np.random.default_rng(5)
    x_train = rng.normal(size=(4096, 258)).astype(np.float32)
    y_train = rng.uniform(0.2, 1.0, (4096, 128)).astype(np.float32)
    x_test = rng.normal(size=(2048, 258)).astype(np.float32)
    widths = [(272, 512), (512, 512), (512, 512), (512, 128)]  # input padded to 272
    flop_fwd_row = 2 * sum(a * b for a, b in widths)
    out = {}
    prev = os.environ.get("COSENU_MLP_GEMM")
    try:
        for gemm in ("tcgen05", "mma"):
            os.environ["COSENU_MLP_GEMM"] = gemm
            sur = Surrogate(n_models=4)
            sur.fit(x_train, y_train, epochs=2, batch=64, lr=1e-4)  # warm-up, buffers sized
            sur.committee(x_test)
            sur.set_timing(True)
            for k, m in enumerate(sur.models):
                m.train(epochs=1, batch=64, lr=1e-5, seed=7000 + k)
            train_ms = sur.timing()
            sur.set_timing(True)
            mean, _ = sur.committee(x_test)
            infer_ms = sur.timing()
            sur.set_timing(False)
            t0 = time.perf_counter()
            sur.committee(x_test)
            wall = time.perf_counter() - t0
            flops = 4 * flop_fwd_row * x_test.shape[0]
            out[gemm] = {"training_one_epoch_committee_ms": train_ms,
                         "inference_committee_ms": infer_ms,
                         "inference_gemm_tflops": flops / (infer_ms["gemm"] * 1e-3) / 1e12,
                         "inference_wall_s": wall, "pred": mean}
            sur.close()
    finally:
        if prev is None:
            os.environ.pop("COSENU_MLP_GEMM", None)
        else:
            os.environ["COSENU_MLP_GEMM"] = prev
    diff = float(np.abs(out["tcgen05"].pop("pred") - out["mma"].pop("pred")).max())
    try:
        bf16_peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
    except Exception:
        bf16_peak = 1590.0  # fallback
    print(json.dumps({
        "metric": "surrogate network device time by GEMM kernel",
        "network": "258 -> 3 x 512 (GELU) -> 128, BF16 operands, FP32 accumulate, committee of 4",
        "data": "synthetic features / targets", "training_rows": 4096, "batch": 64,
        "inference_rows": 2048, **out,
        "gemm_speedup_inference": out["mma"]["inference_committee_ms"]["gemm"] /
        out["tcgen05"]["inference_committee_ms"]["gemm"],
        "gemm_speedup_training": out["mma"]["training_one_epoch_committee_ms"]["gemm"] /
        out["tcgen05"]["training_one_epoch_committee_ms"]["gemm"],
        "bf16_peak_tflops": bf16_peak,
        "max_abs_diff_committee_mean": diff,
    }), flush=True)


def run_snapshot_study(args):
    """Cost of writing snapshots while the run continues.  The reference stops
    the run at every dump and reads the whole state on the host
    (src/snaps.hpp:187-218).  Three timings of the same K steps on the device
    timeline: no output; a cosenu_snapshot every N steps (device copy, then the
    pinned host copy on a side stream, waited for by a host thread as the
    rho_<t>.dat formatter does); a blocking download every N steps (the
    reference's pattern)."""
    import ctypes as C
    import threading

    import torch

    from cosenu_b200 import NuOsc

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sim = NuOsc(device=0, precision=args.precision, **WORKLOAD)
    sim.set_stream(stream.cuda_stream)
    sim.init_seeded(SEED, **IC)
    sim.evolve(max(args.warmup, 3))
    sim.snapshot()  # the first snapshot allocates its device and pinned host buffers
    sim.snapshot_wait()
    torch.cuda.synchronize()
    K, N = args.steps, args.snapshot_every

    def timed(mode):
        threads = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(0, K, N):
            sim.evolve(min(N, K - k))
            if mode == "snapshot":
                for t in threads:
                    t.join()  # the host buffer is reused by the next snapshot
                threads = []
                sim.snapshot()
                p = C.POINTER(C.c_double)()
                t = threading.Thread(target=sim.lib.cosenu_snapshot_wait, args=(sim.h, C.byref(p)))
                t.start()
                threads.append(t)
            elif mode == "download":
                sim.download()
        e1.record(stream)
        torch.cuda.synchronize()
        for t in threads:
            t.join()
        return e0.elapsed_time(e1) / K

    timed("none")  # warm-up
    ms = {m: timed(m) for m in ("none", "snapshot", "download")}
    state_bytes = 8 * 8 * WORKLOAD["nz"] * WORKLOAD["nvz"]
    print(json.dumps({
        "study": "snapshots while stepping", "workload": WORKLOAD_NAMES[args.workload],
        "steps": K, "snapshot_every": N, "state_bytes": state_bytes,
        "ms_per_step": ms,
        "overhead_per_snapshot_ms": {"snapshot": (ms["snapshot"] - ms["none"]) * N,
                                     "blocking_download": (ms["download"] - ms["none"]) * N},
        "precision": args.precision.upper(),
    }), flush=True)
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--instances", type=int, default=256, help="c4: ensemble size")
    ap.add_argument("--train", type=int, default=4096, help="c5: training instances")
    ap.add_argument("--test", type=int, default=512, help="c5: held-out instances")
    ap.add_argument("--sur-nz", type=int, default=512,
                    help="c5: nz of the solver runs (0: log-uniform in [512, 8192])")
    ap.add_argument("--epochs", type=int, default=300, help="c5: training epochs")
    ap.add_argument("--threshold", type=float, default=1e-2, help="c5: fallback threshold")
    ap.add_argument("--gemm-study", action="store_true",
                    help="c5: device time of the network with each GEMM kernel")
    ap.add_argument("--gen-test", type=int, default=64,
                    help="c5: held-out instances with nz log-uniform in [512, 8192]")
    ap.add_argument("--fp32-study", action="store_true",
                    help="FP32-bulk vs FP64 error study on the chosen workload")
    ap.add_argument("--study-steps", type=int, default=8000)
    ap.add_argument("--snapshot-study", action="store_true",
                    help="cost of a snapshot every --snapshot-every steps, asynchronous vs "
                         "blocking, on the chosen workload")
    ap.add_argument("--snapshot-every", type=int, default=100)
    ap.add_argument("--divergence-study", action="store_true",
                    help="c4: <P_ee>(t) of FP64, reordered FP64 and FP32-bulk runs of "
                         "every 32nd member")
    ap.add_argument("--t-factor", type=float, default=1000.0, help="c4: run to t_factor/mu")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["c4", "c5"], default="c2",
                    help="c2 (default, the headline): FD 32768 x 256; c1: FV 1024 x 64; "
                         "c3: FV 65536 x 512")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--nz", type=int, default=None,
                    help="smaller z extent at the same dz (profiling cases only; the headline "
                         "workload is nz = 32768)")
    args = ap.parse_args()
    if args.workload == "c4":
        if args.divergence_study:
            run_divergence_study(args)
        else:
            run_ensemble(args)
        return
    if args.workload == "c5":
        if args.gemm_study:
            run_surrogate_gemm_study(args)
        else:
            run_surrogate(args)
        return
    WORKLOAD.clear()
    WORKLOAD.update(WORKLOADS[args.workload])
    if args.nz is None:
        args.nz = WORKLOAD["nz"]
    if args.nz != WORKLOAD["nz"]:
        dz = (WORKLOAD["z1"] - WORKLOAD["z0"]) / WORKLOAD["nz"]
        WORKLOAD.update(nz=args.nz, z0=-0.5 * args.nz * dz, z1=0.5 * args.nz * dz)
    if args.fp32_study:
        run_fp32_study(args)
        return
    if args.snapshot_study:
        run_snapshot_study(args)
        return
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

"""Benchmark of the headline path: multi-seed LM IK with collision penalty.

Workload (one "step"): 256 IK problems x 128 seeds of the 7-DOF revolute
chain, 30 LM iterations (lambda 1e-2, x0.1 on accept, x10 on reject), 56
robot spheres against 100 obstacle spheres plus 200 self-collision sphere
pairs (hinge^2, margin 0.02 m, weight 1e4), then FP64 re-verification of
every problem's winning seed (success = position < 1 mm and rotation
< 0.01 rad).  Seeded synthetic data (pyroffi_b200.workloads.ik, seed 1002).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  ``value`` is problems solved per second over all
ranks with the inputs resident in HBM; ``e2e`` is the same through the
public solver API from pinned host buffers (H2D of seeds + targets, D2H of
winners / errors / success flags inside the timed region).  ``--impl
reference`` times the CPU port of the reference LM loop (oracle/cpu, FP32,
OpenMP over all host threads) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "IK solves/s @1mm/0.01rad (problems/s, solved or not; 256 targets x 128 seeds x 30 LM iters)"
UNIT = "problems/s"
P_PER_GPU, SEEDS, ITERS = 256, 128, 30
# algorithmic FLOP per seed-iteration: 6 error evaluations of
# (FK 130*7 + residual 60 + sphere transforms 33*56 + world pairs 12*56*100 + self pairs 12*200)
# + Jacobian 45*7 + normal equations and Cholesky ~800
FLOP_PER_SEED_ITER = 6 * (130 * 7 + 60 + 33 * 56 + 12 * 56 * 100 + 12 * 200) + 45 * 7 + 800
L2_FLUSH_BYTES = 256 << 20
# From one ncu capture of one launch of the LM kernel on this workload (python -m
# pyroffi_b200.profile_cases lm): DRAM bytes read + written (the ~1 MB of outputs were still in L2
# when the launch ended), and the FP32 work the kernel executed, 2 FLOP per FFMA, 1 per FADD / FMUL,
# twice that for the packed FFMA2 / FADD2 / FMUL2, summed over threads; the FMA pipe's active share.
LM_DRAM_BYTES_PER_LAUNCH = 1087744 + 256
LM_EXECUTED_FLOP_PER_LAUNCH = 29031424050
LM_FMA_PIPE_PCT = 15.5
# The same counts for the trajectory kernel's fused forward + backward launch on the 512 x 64 x 7 workload
# (python -m pyroffi_b200.profile_cases traj) and for the fused FK + collision kernel on the sweep robot's
# per-link rows (python -m pyroffi_b200.profile_cases fkc5, 4,096 configurations; per configuration).
TRAJ_EXECUTED_FLOP_PER_LAUNCH = 1339234465
TRAJ_FMA_PIPE_PCT = 29.9
SWEEP_EXECUTED_FLOP_PER_CONFIG = 27802706944 / 4096
SWEEP_FMA_PIPE_PCT = 60.4


def r4(x):
    """x rounded to 4 significant digits (keeps the JSON line short)."""
    if x is None:
        return None
    return float(f"{x:.4g}")


def ik_config():
    """The workload's config block, the same on both arms."""
    return {"workload": "ik_lm_collision", "problems_per_gpu": P_PER_GPU, "seeds": SEEDS, "iters": ITERS,
            "robot": "7-DOF chain, 56 spheres", "obstacles": 100, "self_pairs": 200, "lambda": "1e-2 x0.1/x10",
            "l2": "flushed between steps"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-sample", type=int, default=64, help="problems per CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the configs 1, 3, 4, 5 measurements")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# CPU port (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------

def cpu_port_lib():
    from oracle import cpu_port

    return cpu_port.load()


def cpu_solve(lib, w, p0, n_prob, n_threads):
    """Run the CPU port on problems [p0, p0+n_prob); returns (seconds, cfgs, errs)."""
    from oracle import cpu_port

    return cpu_port.ls_ik(lib, w, p0, n_prob, n_threads)


def cpu_success(w, p0, cfgs, errs):
    from oracle import cpu_port

    return float(np.mean(cpu_port.success(w, p0, cfgs, errs)))


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from pyroffi_b200 import workloads as W

    w = W.ik(P=P_PER_GPU, Sd=SEEDS)
    lib = cpu_port_lib()
    threads = lib.pk_cpu_max_threads()
    n = args.cpu_sample
    for i in range(args.warmup):
        cpu_solve(lib, w, (i * n) % P_PER_GPU, min(n, 2), threads)
    times, succ = [], []
    for i in range(args.steps):
        p0 = (i * n) % P_PER_GPU
        dt, cfgs, errs = cpu_solve(lib, w, p0, n, threads)
        times.append(dt)
        succ.append(cpu_success(w, p0, cfgs, errs))
    total = sum(times)
    value = n * args.steps / total
    sample = f"{n} of the 256 problems per step (all 128 seeds, 30 iterations), problems rotated across steps"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": ik_config(),
        "success_rate": float(np.mean(succ)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path is JAX (not installed); timed arm is the C port of the reference LM loop",
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def _lines(self) -> int:
        try:
            return sum(1 for r in Path(self.file.name).read_text().splitlines() if r.strip())
        except Exception:
            return 0

    def __enter__(self):
        self.n0 = 0
        self.after = False
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
            # the sampler is up (its first line written) before the timed region starts
            t0 = time.time()
            while self._lines() == 0 and time.time() - t0 < 3.0:
                time.sleep(0.01)
            self.n0 = self._lines()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            # a timed region shorter than the 100 ms period may hold no sample:
            # then the first sample after it (clocks still at their load values)
            if self._lines() <= self.n0:
                self.after = True
                t0 = time.time()
                while self._lines() <= self.n0 and time.time() - t0 < 1.0:
                    time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        rows = rows[self.n0:]                      # samples from the timed region on
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
               "reasons": sorted(reasons), "samples": len(sm)}
        if self.after:
            out["window"] = "first sample after the timed region (the region is shorter than the 100 ms period)"
        return out


def fp32_peak_tflops(torch, lib_call, stream_ptr):
    """Measured FP32 FMA roof (TFLOP/s) on this GPU."""
    out = torch.empty(148 * 8, dtype=torch.float32, device="cuda")
    blocks, iters = 148 * 8, 20000
    for _ in range(2):
        lib_call("pk_fp32_fma_peak", stream_ptr(), out.data_ptr(), iters, blocks)
    torch.cuda.synchronize()
    best = None
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        lib_call("pk_fp32_fma_peak", stream_ptr(), out.data_ptr(), iters, blocks)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    return 4096.0 * iters * blocks / (best * 1e-3) / 1e12


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))

    from pyroffi_b200 import _lib, workloads as W
    from pyroffi_b200.dist import max_over_ranks
    from pyroffi_b200.ik import BatchIkSolver

    _lib.load()
    # each rank solves its own 256 problems (weak scaling; seed offset by rank)
    w = W.ik(P=P_PER_GPU, Sd=SEEDS, seed=1002)
    if rank > 0:
        rng = np.random.default_rng(1002 + rank)
        w.seeds = rng.uniform(w.model.lower, w.model.upper, size=w.seeds.shape).astype(np.float32)
    solver = BatchIkSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, self_pairs=w.self_pairs,
                           max_iter=w.max_iter, lambda_init=w.lambda_init, lambda_down=w.lambda_down,
                           lambda_up=w.lambda_up, pos_weight=w.pos_weight, ori_weight=w.ori_weight,
                           collision_weight=w.collision_weight, collision_margin=w.collision_margin,
                           pos_tol=w.pos_tol, rot_tol=w.rot_tol, device=dev)
    seeds_d = torch.as_tensor(w.seeds, device=dev)
    tgt_d = torch.as_tensor(w.target_T, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # --- device-resident timing -------------------------------------------
    for _ in range(args.warmup):
        res = solver.solve(tgt_d, seeds_d)
    barrier()
    lm_ms, step_ms = [], []
    with ClockSampler(local) as clocks:
        barrier()
        for _ in range(args.steps):
            flush.fill_(1.0)                       # evict L2 between steps (outside the timed events)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            cfgs, errs = solver.run_lm(tgt_d, seeds_d)
            e1.record(stream)
            res_w = solver.verify_select(cfgs, errs, tgt_d)
            e2.record(stream)
            e2.synchronize()
            lm_ms.append(e0.elapsed_time(e1))
            step_ms.append(e0.elapsed_time(e2))
        barrier()
    clock_summary = clocks.summary()
    success = float(res_w[3].float().mean().item())
    t_local = sum(step_ms) / 1e3
    t_max = max_over_ranks(t_local, dev)
    value = world * P_PER_GPU * args.steps / t_max

    # --- end to end through the public API, host buffers ------------------
    seeds_h = torch.as_tensor(w.seeds).pin_memory()
    tgt_h = torch.as_tensor(w.target_T).pin_memory()
    win_h = torch.empty((P_PER_GPU, w.model.n_act), dtype=torch.float32).pin_memory()
    ok_h = torch.empty(P_PER_GPU, dtype=torch.int32).pin_memory()
    pos_h = torch.empty(P_PER_GPU, dtype=torch.float64).pin_memory()
    rot_h = torch.empty(P_PER_GPU, dtype=torch.float64).pin_memory()
    h2d = seeds_h.numel() * 4 + tgt_h.numel() * 4
    d2h = win_h.numel() * 4 + ok_h.numel() * 4 + pos_h.numel() * 8 + rot_h.numel() * 8

    def e2e_step():
        s = seeds_h.to(dev, non_blocking=True)
        t = tgt_h.to(dev, non_blocking=True)
        r = solver.solve(t, s)
        win_h.copy_(r.winner_cfg, non_blocking=True)
        ok_h.copy_(r.success, non_blocking=True)
        pos_h.copy_(r.pos_err, non_blocking=True)
        rot_h.copy_(r.rot_err, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    barrier()
    t_e2e = max_over_ranks(sum(e2e_ms) / 1e3, dev)
    e2e_value = world * P_PER_GPU * args.steps / t_e2e

    line = None
    if rank == 0:
        lm_avg_s = statistics.mean(lm_ms) / 1e3
        flops = FLOP_PER_SEED_ITER * P_PER_GPU * SEEDS * ITERS
        achieved = flops / lm_avg_s / 1e12
        peak = fp32_peak_tflops(torch, _lib.call, lambda: stream.cuda_stream)
        ok_gpu = res_w[3].cpu().numpy().astype(bool)
        cpu = None
        if not args.no_cpu_baseline:
            lib = cpu_port_lib()
            threads = lib.pk_cpu_max_threads()
            cpu_solve(lib, w, 0, 1, threads)
            dt, cfgs_c, errs_c = cpu_solve(lib, w, 0, args.cpu_sample, threads)
            cpu = {"value": r4(args.cpu_sample / dt), "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"problems 0-{args.cpu_sample - 1}, all seeds (C port, OpenMP)",
                   "success_rate": cpu_success(w, 0, cfgs_c, errs_c),
                   "gpu_success_rate_same_problems": float(ok_gpu[:args.cpu_sample].mean())}
        executed = None
        if LM_EXECUTED_FLOP_PER_LAUNCH:
            ex = LM_EXECUTED_FLOP_PER_LAUNCH / lm_avg_s / 1e12
            executed = {"achieved": r4(ex), "frac": r4(ex / peak), "fma_pipe_pct": LM_FMA_PIPE_PCT,
                        "basis": "ncu SASS counts"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": ik_config(),
            "success_rate": success,
            "successful_solves_per_s": value * success,
            "gpu_launches": 2 * args.steps,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "successful_solves_per_s": e2e_value * success},
            "roofline": {"bound": "fp32", "achieved": r4(achieved), "peak": r4(peak), "unit": "TFLOP/s",
                         "frac": r4(achieved / peak), "traffic": LM_DRAM_BYTES_PER_LAUNCH,
                         "kernel": "lm_kernel<8,1,1,2>",
                         "basis": f"dense-eq {FLOP_PER_SEED_ITER} FLOP/seed-iter; peak: FMA microbenchmark",
                         "executed": executed},
            "kernel_ms": {"lm": r4(statistics.mean(lm_ms)),
                          "verify_select": r4(statistics.mean(step_ms) - statistics.mean(lm_ms))},
            "clocks": clock_summary,
            "cpu_baseline": cpu,
        }
        if not args.no_secondary:
            line["secondary"] = secondary_metrics(torch, dev, peak, cpu=not args.no_cpu_baseline)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Secondary workloads (configs 1, 3, 4 and 5), one GPU, device-timed
# ---------------------------------------------------------------------------

def _timed_ms(torch, fn, flush, reps=5, warm=3):
    """Median CUDA-event time of fn() on the current stream, L2 flushed before each rep."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def _cpu_rate(fn, units):
    """Units per second of the oracle call fn() on the host (one run after a warm-up)."""
    fn()
    t0 = time.perf_counter()
    fn()
    return units / (time.perf_counter() - t0)


def secondary_metrics(torch, dev, fp32_peak, cpu=True):
    """Configs 1 (FK + sphere collision), 3 (trajectory cost + adjoint, CHOMP,
    SCO), HJCD / SQP on config 2's problems, 4 (mixed persistent batch IK) and
    5 (FK + collision bandwidth sweep), each against its roofline, as numbers
    only (units in the key names; workloads are described in the design
    notes).  Seeded synthetic inputs, resident in HBM; L2 flushed between reps."""
    from pyroffi_b200 import workloads as W
    from pyroffi_b200.batch_ik import MixedIkBatch
    from pyroffi_b200.collision import FkCollisionResult, fk_sphere_collision
    from pyroffi_b200.device import DeviceRobot, DeviceSpheres, DeviceWorld
    from pyroffi_b200.ik import BatchIkSolver
    from pyroffi_b200.trajopt import TrajectoryCost

    hbm = _measured_hbm()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    out = {}

    # config 1: 7-DOF chain, 8 spheres per link, 64 obstacle spheres
    w = W.fk_collision(B=65536)
    R, S, Wd = DeviceRobot.upload(w.model, dev), DeviceSpheres.upload(w.spheres, dev), DeviceWorld.upload(w.world, dev)
    N, Sp = w.spheres.n_links, w.spheres.S
    K, M = N * Sp, sum(Wd.counts())
    cfg = torch.as_tensor(w.cfg, device=dev)
    c1 = cfg[:1024].contiguous()
    r1 = fk_sphere_collision(R, S, Wd, c1)
    ms_1024 = _timed_ms(torch, lambda: fk_sphere_collision(R, S, Wd, c1, out=r1), flush)
    r2 = fk_sphere_collision(R, S, Wd, cfg, per_sphere=True)
    ms_bkm = _timed_ms(torch, lambda: fk_sphere_collision(R, S, Wd, cfg, per_sphere=True, out=r2), flush)
    n_valid = int((w.spheres.radii >= 0).sum())
    # bytes per configuration: cfg in, min + 7-float poses of the N links out, and the [K, M] rows;
    # K counts the base link's 8 padded rows (the output layout), K56 only the 56 real spheres
    bytes_cfg = 4 * w.model.n_act + 4 + 4 * 7 * N + 4 * K * M
    bytes_k56 = 4 * w.model.n_act + 4 + 4 * 7 * N + 4 * n_valid * M
    flop_cfg = 130 * w.model.n_act + 33 * n_valid + 12 * n_valid * M
    gbs = 65536 * bytes_cfg / (ms_bkm * 1e-3) / 1e9
    gbs56 = 65536 * bytes_k56 / (ms_bkm * 1e-3) / 1e9
    out["c1"] = {
        "us_B1024": r4(1e3 * ms_1024), "configs_per_s_B1024": r4(1024 / (ms_1024 * 1e-3)),
        "ms_B65536_bkm": r4(ms_bkm), "configs_per_s_B65536": r4(65536 / (ms_bkm * 1e-3)),
        "roofline": {"bound": "hbm", "achieved": r4(gbs), "peak": hbm, "unit": "GB/s", "frac": r4(gbs / hbm),
                     "bytes_per_config": bytes_cfg, f"K{K}": K,
                     "frac_K56": r4(gbs56 / hbm), "bytes_per_config_K56": bytes_k56,
                     "fp32_tflops": r4(65536 * flop_cfg / (ms_bkm * 1e-3) / 1e12)},
    }
    del r2
    if cpu:
        from oracle import collision as ocoll
        from oracle import kinematics as okin
        cs = w.cfg[:256].astype(np.float64)

        def fkc_oracle():
            links = okin.forward_kinematics(cs, w.model.as_dict())
            cen = ocoll.transform_points(links[:, :, None, :], w.spheres.centers.astype(np.float64)[None])
            d = ocoll.point_vs_world(cen, np.broadcast_to(w.spheres.radii, cen.shape[:-1]), *w.world.arrays())
            return np.where(w.spheres.radii[None, :, :, None] < 0, np.inf, d).reshape(len(cs), -1).min(axis=1)
        out["c1"]["cpu_baseline"] = {"value": r4(_cpu_rate(fkc_oracle, len(cs))), "unit": "configs/s",
                                     "cores": 1, "kind": "port", "sample": "256 configs, FP64 oracle"}

    # config 3: 512 trajectories x 64 waypoints x 7 DOF, 256 spheres + 32 boxes
    wt = W.trajectories()
    tc = TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=wt.margin, device=dev)
    x = torch.as_tensor(wt.traj, device=dev)
    ms_f = _timed_ms(torch, lambda: tc.cost(x), flush)
    ms_b = _timed_ms(torch, lambda: tc.grad(x), flush)
    ms_fb = _timed_ms(torch, lambda: tc.cost_and_grad(x), flush)
    Bt, T = wt.traj.shape[:2]
    f_bwd = 459326
    tf = Bt * T * f_bwd / (ms_fb * 1e-3) / 1e12
    out["c3"] = {
        "ms_fwd": r4(ms_f), "ms_bwd_recompute": r4(ms_b), "ms_fused_fwd_bwd": r4(ms_fb),
        "fwd_bwd_traj_per_s": r4(Bt / (ms_fb * 1e-3)),
        "roofline": {"bound": "fp32", "achieved": r4(tf), "peak": r4(fp32_peak), "unit": "TFLOP/s",
                     "frac": r4(tf / fp32_peak), "basis": "dense-eq",
                     "executed": {"achieved": r4(TRAJ_EXECUTED_FLOP_PER_LAUNCH / (ms_fb * 1e-3) / 1e12),
                                  "frac": r4(TRAJ_EXECUTED_FLOP_PER_LAUNCH / (ms_fb * 1e-3) / 1e12 / fp32_peak),
                                  "fma_pipe_pct": TRAJ_FMA_PIPE_PCT}},
    }
    if cpu:
        from oracle import traj as otraj
        md = wt.model.as_dict()

        def traj_oracle():
            for b in range(2):
                otraj.total_cost(wt.traj[b], md, wt.spheres.centers, wt.spheres.radii, wt.link_pairs,
                                 wt.world.arrays(), margin=wt.margin, w_smooth=1.0, w_acc=0.5, w_jerk=0.1,
                                 w_limits=1.0, w_coll=3.0, lower=wt.model.lower, upper=wt.model.upper)
        out["c3"]["cpu_baseline"] = {"value": r4(_cpu_rate(traj_oracle, 2)), "unit": "traj costs/s (fwd)",
                                     "cores": 1, "kind": "port", "sample": "2 traj, FP64 oracle"}

    # CHOMP optimiser on the adjoint: the config-3 trajectories, 100 iterations, one CUDA graph
    from pyroffi_b200.chomp import ChompConfig, ChompOptimizer
    ccfg = ChompConfig()
    tcc = TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=ccfg.collision_margin, device=dev)
    opt = ChompOptimizer(tcc, ccfg)
    s0, g0 = x[0, 0].clone(), x[0, -1].clone()
    opt.run(x, s0, g0, graph=True)
    ms_chomp = _timed_ms(torch, lambda: opt.run(x, s0, g0, graph=True), flush, reps=3, warm=1)
    out["chomp"] = {"ms_100_iters": r4(ms_chomp), "traj_iters_per_s": r4(Bt * ccfg.n_iters / (ms_chomp * 1e-3))}

    # SCO optimiser: 10 outer x 30 inner L-BFGS iterations, one CUDA graph
    from pyroffi_b200.sco import ScoConfig, ScoOptimizer
    scfg = ScoConfig()
    sco = ScoOptimizer(wt.model, wt.spheres, wt.world, wt.link_pairs, scfg, device=dev)
    sco.run(x, s0, g0, graph=True)
    ms_sco = _timed_ms(torch, lambda: sco.run(x, s0, g0, graph=True), flush, reps=3, warm=1)
    out["sco"] = {"ms_per_run": r4(ms_sco), "traj_per_s": r4(Bt / (ms_sco * 1e-3))}

    # HJCD-IK and SQP-IK on config 2's problems (collision on), the reference benchmark's settings
    from pyroffi_b200.hjcd import HjcdSolver
    from pyroffi_b200.sqp import SqpSolver
    wi = W.ik()
    hj = HjcdSolver(wi.model, wi.target_link, spheres=wi.spheres, world=wi.world, enable_collision=True, device=dev)
    vs = BatchIkSolver(wi.model, wi.target_link, device=dev)
    tgt_h = torch.as_tensor(wi.target_T, device=dev)
    prev_h = torch.as_tensor(wi.seeds[:, 0], device=dev)
    gen_h = torch.Generator(device=dev)
    hkw = dict(num_seeds=32, coarse_max_iter=20, lm_max_iter=40, lambda_init=1e-3, limit_prior_weight=1e-4,
               kick_scale=0.02, generator=gen_h)
    gen_h.manual_seed(0)
    hj.solve(tgt_h, prev_h, **hkw)
    ms_hj = _timed_ms(torch, lambda: hj.solve(tgt_h, prev_h, **hkw), flush, reps=5, warm=1)
    gen_h.manual_seed(0)
    _, _, parts_h = hj.solve(tgt_h, prev_h, return_all=True, **hkw)
    _, _, _, ok_h = vs.verify_select(parts_h[5], parts_h[6], tgt_h)
    P_h = wi.target_T.shape[0]
    out["hjcd"] = {"ms": r4(ms_hj), "problems_per_s": r4(P_h / (ms_hj * 1e-3)),
                   "success_rate": float(ok_h.float().mean())}
    sq = SqpSolver(wi.model, wi.target_link, spheres=wi.spheres, world=wi.world, enable_collision=True, device=dev)
    skw = dict(num_seeds=32, max_iter=60, n_inner_iters=2, pos_weight=50.0, ori_weight=10.0, lambda_init=5e-3,
               generator=gen_h)
    gen_h.manual_seed(0)
    sq.solve(tgt_h, prev_h, **skw)
    ms_sq = _timed_ms(torch, lambda: sq.solve(tgt_h, prev_h, **skw), flush, reps=5, warm=1)
    gen_h.manual_seed(0)
    _, _, parts_s = sq.solve(tgt_h, prev_h, return_all=True, **skw)
    _, _, _, ok_s = vs.verify_select(parts_s[1], parts_s[2], tgt_h)
    out["sqp"] = {"ms": r4(ms_sq), "problems_per_s": r4(P_h / (ms_sq * 1e-3)),
                  "success_rate": float(ok_s.float().mean())}

    # config 4: 4096 mixed IK problems in one persistent batch (CUDA graph), against the same kernels
    # called per class (problems padded to the class's largest seed count) and per problem
    wm = W.mixed_ik()
    o = dict(max_iter=wm.max_iter, lambda_init=wm.lambda_init, lambda_down=wm.lambda_down, lambda_up=wm.lambda_up,
             collision_weight=wm.collision_weight, collision_margin=wm.collision_margin, pos_tol=wm.pos_tol,
             rot_tol=wm.rot_tol)
    b = MixedIkBatch(wm.classes, wm.world, device=dev, **o)
    b.prepare(wm.problem_class, wm.n_seeds)
    b.load(wm.target_T, wm.seeds)
    b.capture()
    ms_batch = _timed_ms(torch, b.solve, flush, reps=3, warm=1)
    res = b.solve()
    torch.cuda.synchronize()
    n_p = len(wm.problem_class)
    succ = sum(int(r.success.sum()) for r in res) / n_p
    plain, per_problem, ok_pp = 0.0, 0.0, 0
    for c, cl in enumerate(wm.classes):
        s_c = BatchIkSolver(cl.model, cl.target_links, spheres=cl.spheres, world=wm.world, device=dev, **o)
        tg, sd = torch.as_tensor(wm.target_T[c], device=dev), torch.as_tensor(wm.seeds[c], device=dev)
        plain += _timed_ms(torch, lambda: s_c.solve(tg, sd), flush, reps=2, warm=1)
        # per problem: one solve call per problem with its own seed count (the plain drop-in pattern)
        idx = np.nonzero(wm.problem_class == c)[0]
        ns = [int(wm.n_seeds[i]) for i in idx]
        views = [(tg[j:j + 1], sd[j:j + 1, :ns[j]].contiguous()) for j in range(len(idx))]
        s_c.solve(*views[0])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(1.0)
        e0.record()
        rs = [s_c.solve(t_, s_) for t_, s_ in views]
        e1.record()
        e1.synchronize()
        per_problem += e0.elapsed_time(e1)
        ok_pp += sum(int(r_.success.sum()) for r_ in rs)
    out["c4"] = {
        "ms_batch": r4(ms_batch), "problems_per_s": r4(n_p / (ms_batch * 1e-3)), "success_rate": succ,
        "success_per_class": [round(float(r.success.float().mean()), 4) for r in res],
        "ms_per_class_padded": r4(plain), "speedup_vs_per_class": r4(plain / ms_batch),
        "ms_per_problem_calls": r4(per_problem), "success_rate_per_problem_calls": ok_pp / n_p,
        "speedup_vs_per_problem_calls": r4(per_problem / ms_batch),
        "launches_per_batch": b.launches_per_solve(),
    }
    del b

    # config 5: 16 spheres/link vs 4096 spheres + 256 oriented boxes, B = 1024 ... 262144, [B, N, M] rows
    ws = W.sweep(B=262144)
    R5, S5, W5 = DeviceRobot.upload(ws.model, dev), DeviceSpheres.upload(ws.spheres, dev), DeviceWorld.upload(ws.world, dev)
    N5, M5 = ws.spheres.n_links, sum(W5.counts())
    n_valid5 = int((ws.spheres.radii >= 0).sum())
    Ms5, Mb5 = W5.counts()[0], W5.counts()[2]
    flop5 = 130 * ws.model.n_act + 33 * n_valid5 + n_valid5 * (12 * Ms5 + 41 * Mb5)
    bytes5 = 4 * ws.model.n_act + 4 + 4 * N5 * M5
    cfg5 = torch.as_tensor(ws.cfg, device=dev)
    bnm = torch.empty((262144, N5, M5), dtype=torch.float32, device=dev)
    mind = torch.empty(262144, dtype=torch.float32, device=dev)
    sweep = {}
    for B in (1024, 16384, 65536, 262144):
        cb = cfg5[:B]
        rb = FkCollisionResult(mind[:B], None, None, bnm[:B])
        ms = _timed_ms(torch, lambda: fk_sphere_collision(R5, S5, W5, cb, link_poses=False, per_link=True, out=rb),
                       flush, reps=3)
        sweep[str(B)] = [r4(ms), r4(B / (ms * 1e-3)), r4(B * bytes5 / (ms * 1e-3) / 1e9),
                         r4(B * flop5 / (ms * 1e-3) / 1e12 / fp32_peak)]
    del bnm
    pairs5 = W.active_link_pairs(ws.model, ws.spheres)
    tc5 = TrajectoryCost(ws.model, ws.spheres, ws.world, pairs5, device=dev)
    x5 = cfg5[:65536].reshape(1024, 64, -1).contiguous()
    ms_fb5 = _timed_ms(torch, lambda: tc5.cost_and_grad(x5), flush, reps=3)
    t262 = 262144 * flop5 / (sweep["262144"][0] * 1e-3) / 1e12
    out["c5"] = {
        "by_batch_ms_cfgps_gbs_fp32frac": sweep,
        "roofline": {"bound": "fp32", "achieved": r4(t262), "peak": r4(fp32_peak), "unit": "TFLOP/s",
                     "frac": r4(t262 / fp32_peak), "B": 262144,
                     "executed": {"achieved": r4(262144 * SWEEP_EXECUTED_FLOP_PER_CONFIG / (sweep["262144"][0] * 1e-3)
                                                 / 1e12),
                                  "frac": r4(262144 * SWEEP_EXECUTED_FLOP_PER_CONFIG / (sweep["262144"][0] * 1e-3)
                                             / 1e12 / fp32_peak),
                                  "fma_pipe_pct": SWEEP_FMA_PIPE_PCT}},
        "ms_fwd_bwd_65536": r4(ms_fb5),
    }
    return out


def _measured_hbm():
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except Exception:
        return 6650.0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

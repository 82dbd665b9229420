"""Small, self-contained cases of each hot kernel for profiling (e.g. under
``ncu``): every case builds its seeded synthetic input, runs its kernel
three times and synchronises, so a profiler can skip the first launches and
capture one warm launch.

    python -m pyroffi_b200.profile_cases lm          # seed-group LM, 256 x 128 seeds, 30 iterations
    python -m pyroffi_b200.profile_cases lm 1 128    # the same with 1 lane per seed, 128 seeds per block
    python -m pyroffi_b200.profile_cases fkc1        # fused FK + collision, 65,536 configs, [B, K, M] output
    python -m pyroffi_b200.profile_cases fkc5        # fused FK + collision, 4,096 configs of the sweep robot, [B, N, M]
    python -m pyroffi_b200.profile_cases wide        # warp-per-seed LM, 15-DOF bimanual, 64 problems x 64 seeds
    python -m pyroffi_b200.profile_cases traj        # trajectory cost + adjoint, 512 x 64 x 7
    python -m pyroffi_b200.profile_cases batch       # persistent mixed batch, 512 problems
    python -m pyroffi_b200.profile_cases scolin      # SCO linearisation, 512 x 64 x 7 waypoints
    python -m pyroffi_b200.profile_cases scoinner    # SCO inner L-BFGS solve, 512 trajectories
    python -m pyroffi_b200.profile_cases sco         # whole SCO run (10 x 30 iterations), 512 x 64 x 7
    python -m pyroffi_b200.profile_cases hjcd        # HJCD-IK solve, 256 problems, collision on
    python -m pyroffi_b200.profile_cases sqp         # SQP-IK solve, 256 problems, collision on
    python -m pyroffi_b200.profile_cases chomp       # CHOMP, 512 x 64 x 7 trajectories, 5 iterations (eager)
"""

from __future__ import annotations

import sys

import torch

from . import workloads as W


def _lm(tps=0, spb=0):
    from .ik import BatchIkSolver
    w = W.ik(P=256, Sd=128)
    dev = torch.device("cuda:0")
    s = BatchIkSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, self_pairs=w.self_pairs,
                      max_iter=w.max_iter, lambda_init=w.lambda_init, lambda_down=w.lambda_down,
                      lambda_up=w.lambda_up, collision_weight=w.collision_weight,
                      collision_margin=w.collision_margin, threads_per_seed=tps, seeds_per_block=spb,
                      device=dev)
    tg, sd = torch.as_tensor(w.target_T, device=dev), torch.as_tensor(w.seeds, device=dev)
    return lambda: s.run_lm(tg, sd)


def _fkc(B, sweep):
    from .collision import fk_sphere_collision
    from .device import DeviceRobot, DeviceSpheres, DeviceWorld
    w = W.sweep(B=B) if sweep else W.fk_collision(B=B)
    dev = torch.device("cuda:0")
    R, S, Wd = DeviceRobot.upload(w.model, dev), DeviceSpheres.upload(w.spheres, dev), DeviceWorld.upload(w.world, dev)
    c = torch.as_tensor(w.cfg, device=dev)
    return lambda: fk_sphere_collision(R, S, Wd, c, per_sphere=not sweep, per_link=sweep, link_poses=not sweep)


def _wide():
    from .ik import BatchIkSolver
    w = W.mixed_ik(n_problems=1024)
    c = 2
    cl = w.classes[c]
    dev = torch.device("cuda:0")
    s = BatchIkSolver(cl.model, cl.target_links, spheres=cl.spheres, world=w.world, threads_per_seed=16,
                      max_iter=w.max_iter, lambda_init=w.lambda_init, lambda_down=w.lambda_down,
                      lambda_up=w.lambda_up, collision_weight=w.collision_weight,
                      collision_margin=w.collision_margin, device=dev)
    tg = torch.as_tensor(w.target_T[c][:64], device=dev)
    sd = torch.as_tensor(w.seeds[c][:64, :64], device=dev)
    return lambda: s.run_lm(tg, sd)


def _traj():
    from .trajopt import TrajectoryCost
    wt = W.trajectories()
    dev = torch.device("cuda:0")
    tc = TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=wt.margin, device=dev)
    x = torch.as_tensor(wt.traj, device=dev)
    return lambda: tc.cost_and_grad(x)


def _batch():
    from .batch_ik import MixedIkBatch
    w = W.mixed_ik(n_problems=512)
    b = MixedIkBatch(w.classes, w.world, device="cuda:0", max_iter=w.max_iter, lambda_init=w.lambda_init,
                     lambda_down=w.lambda_down, lambda_up=w.lambda_up, collision_weight=w.collision_weight,
                     collision_margin=w.collision_margin)
    b.prepare(w.problem_class, w.n_seeds)
    b.load(w.target_T, w.seeds)
    return b.run_lm


def _sco(stage):
    from .sco import ScoConfig, ScoOptimizer
    wt = W.trajectories()
    dev = torch.device("cuda:0")
    opt = ScoOptimizer(wt.model, wt.spheres, wt.world, wt.link_pairs, ScoConfig(), device=dev)
    x = torch.as_tensor(wt.traj, device=dev)
    if stage == "lin":
        return lambda: opt.linearize(x)
    if stage == "run":
        return lambda: opt.run(x, x[0, 0], x[0, -1])
    d, J, _ = opt.linearize(x)
    return lambda: opt.inner(x, d, J, 1.0, x[0, 0], x[0, -1])


def _hjcd():
    from .hjcd import HjcdSolver
    w = W.ik()
    dev = torch.device("cuda:0")
    s = HjcdSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, enable_collision=True, device=dev)
    tg, prev = torch.as_tensor(w.target_T, device=dev), torch.as_tensor(w.seeds[:, 0], device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    return lambda: s.solve(tg, prev, num_seeds=32, lambda_init=1e-3, limit_prior_weight=1e-4, kick_scale=0.02,
                           generator=g)


def _sqp():
    from .sqp import SqpSolver
    w = W.ik()
    dev = torch.device("cuda:0")
    s = SqpSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, enable_collision=True, device=dev)
    tg, prev = torch.as_tensor(w.target_T, device=dev), torch.as_tensor(w.seeds[:, 0], device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    return lambda: s.solve(tg, prev, num_seeds=32, generator=g)


def _chomp():
    from .chomp import ChompConfig, ChompOptimizer
    from .trajopt import TrajectoryCost
    wt = W.trajectories()
    dev = torch.device("cuda:0")
    cfg = ChompConfig(n_iters=5)
    tc = TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=cfg.collision_margin, device=dev)
    opt = ChompOptimizer(tc, cfg)
    x = torch.as_tensor(wt.traj, device=dev)
    return lambda: opt.run(x, x[0, 0], x[0, -1])


CASES = {"lm": _lm, "fkc1": lambda: _fkc(65536, False), "fkc5": lambda: _fkc(4096, True), "wide": _wide,
         "traj": _traj, "batch": _batch, "scolin": lambda: _sco("lin"), "scoinner": lambda: _sco("inner"),
         "sco": lambda: _sco("run"), "hjcd": _hjcd, "sqp": _sqp, "chomp": _chomp}


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] not in CASES or (len(argv) > 1 and argv[0] != "lm") or len(argv) > 3:
        print(__doc__)
        return 2
    fn = CASES[argv[0]](*map(int, argv[1:]))
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    print("ok", argv[0])
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Generate ``tests/golden/ref_helpers.npz`` from the reference's own helper code.

The reference's CUDA helper headers (``src/pyroffi/cuda_kernels/_fk_cuda_helpers.cuh``,
``_ik_cuda_helpers.cuh``, ``_collision_cuda_helpers.cuh``) are compiled for
the host from the reference tree by ``oracle/Makefile`` (target ``ref``) into
``oracle/_ref/libref_helpers.so``.  This script feeds them seeded inputs and
stores inputs and outputs, so the tests can pin the FP64 oracle to the
reference without the reference tree present:

    make -C oracle ref && python tests/golden/make_golden.py

Cases: SE(3) exp / compose; FK (``fk_single``) on a 7-DOF chain, a 15-DOF
bimanual tree, a 29-DOF humanoid tree and a small out-of-order tree with a
prismatic, a fixed, a mimic and a fixed-with-offset joint; stacked residual +
Jacobian (``compute_multi_ee_residual_and_jacobian``) for 1 and 2 EEs; FP64
Cholesky (``chol_solve``); every signed-distance primitive and
``colldist_from_sdf``.
"""

from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import kinematics as okin  # noqa: E402
from pyroffi_b200 import robot as R  # noqa: E402

LIB = ROOT / "oracle" / "_ref" / "libref_helpers.so"
OUT = Path(__file__).resolve().parent / "ref_helpers.npz"


def load():
    if not LIB.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    return C.CDLL(str(LIB))


def fp(a):
    return a.ctypes.data_as(C.c_void_p)


def odd_tree():
    """6 joints listed out of topological order; joint kinds: revolute (act 0),
    prismatic (act 1), fixed, mimic of act 0 (x-0.5 + 0.1), revolute (act 2),
    fixed joint with a mimic offset (no source, offset 0.3 -> rotates 0.3 rad)."""
    rng = np.random.default_rng(77)
    parent = np.array([2, -1, 1, 0, 2, 3], np.int32)
    tw = np.zeros((6, 6), np.float32)
    ax = rng.normal(size=(6, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    tw[0, 3:] = ax[0]          # revolute, act 0
    tw[1, :3] = ax[1]          # prismatic, act 1
    tw[3, 3:] = ax[3]          # mimic revolute
    tw[4, 3:] = ax[4]          # revolute, act 2
    tw[5, 3:] = ax[5]          # offset-only revolute
    ptf = np.zeros((6, 7), np.float32)
    q = rng.normal(size=(6, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    ptf[:, :4] = q
    ptf[:, 4:] = rng.uniform(-0.3, 0.3, size=(6, 3))
    act = np.array([0, 1, -1, -1, 2, -1], np.int32)
    mact = np.array([-1, -1, -1, 0, -1, -1], np.int32)
    mul = np.array([1, 1, 1, -0.5, 1, 1], np.float32)
    off = np.array([0, 0, 0, 0.1, 0, 0.3], np.float32)
    return dict(twists=tw, parent_tf=ptf, parent_idx=parent, act_idx=act, mimic_mul=mul,
                mimic_off=off, mimic_act_idx=mact, n_act=3, lower=-np.ones(3, np.float32) * 2,
                upper=np.ones(3, np.float32) * 2)


def model_dict(m: R.RobotModel):
    return dict(twists=m.twists, parent_tf=m.parent_tf, parent_idx=m.parent_idx, act_idx=m.act_idx,
                mimic_mul=m.mimic_mul, mimic_off=m.mimic_off, mimic_act_idx=m.mimic_act_idx,
                n_act=m.n_act, lower=m.lower, upper=m.upper)


def main():
    lib = load()
    lib.ref_sphere_sphere.restype = C.c_float
    for name in ("ref_sphere_capsule", "ref_sphere_box", "ref_sphere_halfspace", "ref_capsule_capsule",
                 "ref_capsule_box", "ref_capsule_halfspace"):
        getattr(lib, name).restype = C.c_float
    lib.ref_colldist_from_sdf.restype = C.c_float
    lib.ref_colldist_from_sdf.argtypes = [C.c_float, C.c_float]
    lib.ref_chol_solve_f64.restype = C.c_int
    rng = np.random.default_rng(2024)
    out: dict[str, np.ndarray] = {}

    # SE(3)
    tang = rng.normal(size=(64, 6)).astype(np.float32)
    tang[:16, :3] = 0.0             # revolute motions (v = 0)
    tang[16:24, 3:] = 0.0           # prismatic motions (omega = 0)
    tang[24:32, :3] = 0.0           # small revolute angles
    tang[24:32, 3:] *= 1e-3
    # rows 32..63: screw motions (v and omega both non-zero)
    exp_out = np.zeros((64, 7), np.float32)
    for i in range(64):
        lib.ref_se3_exp(fp(tang[i]), fp(exp_out[i]))
    out["se3_exp_in"], out["se3_exp_out"] = tang, exp_out
    A = exp_out.copy()
    B = exp_out[::-1].copy()
    comp = np.zeros_like(A)
    for i in range(64):
        lib.ref_se3_compose(fp(A[i]), fp(B[i]), fp(comp[i]))
    out["se3_compose_a"], out["se3_compose_b"], out["se3_compose_out"] = A, B, comp

    # FK on robots
    robots = {
        "chain7": model_dict(R.serial_chain(7, np.random.default_rng(1001))),
        "bimanual15": model_dict(R.bimanual_tree(np.random.default_rng(1004))),
        "humanoid29": model_dict(R.humanoid_tree(np.random.default_rng(1004))),
        "odd6": odd_tree(),
    }
    for name, md in robots.items():
        topo = okin.topo_sort(md["parent_idx"])
        nj, na = md["twists"].shape[0], md["n_act"]
        cfg = rng.uniform(md["lower"], md["upper"], size=(16, na)).astype(np.float32)
        Tw = np.zeros((16, nj, 7), np.float32)
        for b in range(16):
            lib.ref_fk_single(fp(cfg[b]), fp(md["twists"]), fp(md["parent_tf"]), fp(md["parent_idx"]),
                              fp(md["act_idx"]), fp(md["mimic_mul"]), fp(md["mimic_off"]),
                              fp(md["mimic_act_idx"]), fp(topo), fp(Tw[b]), nj, na)
        for k in ("twists", "parent_tf", "parent_idx", "act_idx", "mimic_mul", "mimic_off", "mimic_act_idx",
                  "lower", "upper"):
            out[f"fk_{name}_{k}"] = np.asarray(md[k])
        out[f"fk_{name}_topo_inv"] = topo
        out[f"fk_{name}_cfg"] = cfg
        out[f"fk_{name}_out"] = Tw

    # residual + Jacobian
    for name, ee_joints in (("chain7", [6]), ("bimanual15", [9, 15]), ("odd6", [5, 4])):
        md = robots[name]
        topo = out[f"fk_{name}_topo_inv"]
        nj, na = md["twists"].shape[0], md["n_act"]
        ne = len(ee_joints)
        tj = np.asarray(ee_joints, np.int32)
        anc = np.stack([okin.ancestor_mask(j, md["parent_idx"]) for j in tj]).astype(np.int32)
        cfg = rng.uniform(md["lower"], md["upper"], size=(16, na)).astype(np.float32)
        tq = rng.normal(size=(16, ne, 4))
        tq /= np.linalg.norm(tq, axis=-1, keepdims=True)
        tgt = np.concatenate([tq, rng.uniform(-1, 1, size=(16, ne, 3))], -1).astype(np.float32)
        tgt[:4] = 0
        # first 4 targets: pose of a nearby configuration (small residuals)
        for b in range(4):
            Tw = np.zeros((nj, 7), np.float32)
            c2 = (cfg[b] + 0.01 * rng.normal(size=na)).astype(np.float32)
            lib.ref_fk_single(fp(c2), fp(md["twists"]), fp(md["parent_tf"]), fp(md["parent_idx"]),
                              fp(md["act_idx"]), fp(md["mimic_mul"]), fp(md["mimic_off"]),
                              fp(md["mimic_act_idx"]), fp(topo), fp(Tw), nj, na)
            tgt[b] = Tw[tj]
        r = np.zeros((16, 6 * ne), np.float32)
        J = np.zeros((16, 6 * ne, na), np.float32)
        Tw = np.zeros((nj, 7), np.float32)
        for b in range(16):
            lib.ref_multi_ee_residual_and_jacobian(
                fp(cfg[b]), fp(Tw), fp(md["twists"]), fp(md["parent_tf"]), fp(md["parent_idx"]),
                fp(md["act_idx"]), fp(md["mimic_mul"]), fp(md["mimic_off"]), fp(md["mimic_act_idx"]),
                fp(topo), fp(tj), fp(anc), fp(tgt[b]), nj, na, ne, fp(r[b]), fp(J[b]))
        out[f"resjac_{name}_cfg"], out[f"resjac_{name}_target_jnts"] = cfg, tj
        out[f"resjac_{name}_ancestor_masks"], out[f"resjac_{name}_target"] = anc, tgt
        out[f"resjac_{name}_r"], out[f"resjac_{name}_J"] = r, J

    # Cholesky (FP64)
    for n in (7, 15):
        As, bs, xs, oks = [], [], [], []
        for k in range(8):
            M = rng.normal(size=(6, n))
            A = M.T @ M + (10.0 ** rng.uniform(-6, 0)) * np.eye(n)
            if k == 7:
                A = -np.eye(n)          # non-positive pivot -> zero solution
            b = rng.normal(size=n)
            Ac, bc = A.copy(), b.copy()
            ok = lib.ref_chol_solve_f64(fp(Ac), fp(bc), n)
            As.append(A), bs.append(b), xs.append(bc), oks.append(ok)
        out[f"chol{n}_A"], out[f"chol{n}_b"] = np.asarray(As), np.asarray(bs)
        out[f"chol{n}_x"], out[f"chol{n}_ok"] = np.asarray(xs), np.asarray(oks, np.int32)

    # distance primitives
    n = 256
    sph = np.concatenate([rng.uniform(-1, 1, (n, 3)), rng.uniform(0.01, 0.3, (n, 1))], 1).astype(np.float32)
    sph2 = np.concatenate([rng.uniform(-1, 1, (n, 3)), rng.uniform(0.01, 0.3, (n, 1))], 1).astype(np.float32)
    cap = np.concatenate([rng.uniform(-1, 1, (n, 6)), rng.uniform(0.01, 0.2, (n, 1))], 1).astype(np.float32)
    cap[:8, 3:6] = cap[:8, 0:3]                      # degenerate segments
    cap2 = np.concatenate([rng.uniform(-1, 1, (n, 6)), rng.uniform(0.01, 0.2, (n, 1))], 1).astype(np.float32)
    cap2[8:16, 3:6] = cap2[8:16, 0:3] + (cap[8:16, 3:6] - cap[8:16, 0:3])  # parallel
    box = np.zeros((n, 15), np.float32)
    box[:, :3] = rng.uniform(-1, 1, (n, 3))
    for i in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        Rm = np.array([[1 - 2 * (q[2] ** 2 + q[3] ** 2), 2 * (q[1] * q[2] - q[0] * q[3]), 2 * (q[1] * q[3] + q[0] * q[2])],
                       [2 * (q[1] * q[2] + q[0] * q[3]), 1 - 2 * (q[1] ** 2 + q[3] ** 2), 2 * (q[2] * q[3] - q[0] * q[1])],
                       [2 * (q[1] * q[3] - q[0] * q[2]), 2 * (q[2] * q[3] + q[0] * q[1]), 1 - 2 * (q[1] ** 2 + q[2] ** 2)]])
        box[i, 3:6], box[i, 6:9], box[i, 9:12] = Rm[:, 0], Rm[:, 1], Rm[:, 2]
    box[:, 12:15] = rng.uniform(0.05, 0.4, (n, 3))
    box[:16, :3] = sph[:16, :3] + 0.01 * rng.normal(size=(16, 3))   # centres inside boxes
    hn = rng.normal(size=(n, 3))
    hn /= np.linalg.norm(hn, axis=1, keepdims=True)
    hs = np.concatenate([hn, rng.uniform(-1, 1, (n, 3))], 1).astype(np.float32)
    res = {k: np.zeros(n, np.float32) for k in ("ss", "sc", "sb", "sh", "cc", "cb", "ch")}
    for i in range(n):
        res["ss"][i] = lib.ref_sphere_sphere(fp(sph[i]), fp(sph2[i]))
        res["sc"][i] = lib.ref_sphere_capsule(fp(sph[i]), fp(cap[i]))
        res["sb"][i] = lib.ref_sphere_box(fp(sph[i]), fp(box[i]))
        res["sh"][i] = lib.ref_sphere_halfspace(fp(sph[i]), fp(hs[i]))
        res["cc"][i] = lib.ref_capsule_capsule(fp(cap[i]), fp(cap2[i]))
        res["cb"][i] = lib.ref_capsule_box(fp(cap[i]), fp(box[i]))
        res["ch"][i] = lib.ref_capsule_halfspace(fp(cap[i]), fp(hs[i]))
    d = rng.uniform(-0.1, 0.1, 64).astype(np.float32)
    cd = np.asarray([lib.ref_colldist_from_sdf(float(x), 0.02) for x in d], np.float32)
    out.update(dist_sph=sph, dist_sph2=sph2, dist_cap=cap, dist_cap2=cap2, dist_box=box, dist_hs=hs,
               colldist_in=d, colldist_out=cd)
    for k, v in res.items():
        out[f"dist_{k}"] = v
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()

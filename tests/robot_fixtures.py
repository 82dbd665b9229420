"""Robot models from the committed fixtures of ``tests/golden/robots``."""

from pathlib import Path

import numpy as np

from pyroffi_b200.robot import RobotModel, RobotSpheres, depth_schedule

GOLDEN = Path(__file__).resolve().parent / "golden" / "robots"


def load_robot(name: str):
    """-> (RobotModel, RobotSpheres, active link pairs [P, 2], EE link index)."""
    z = np.load(GOLDEN / f"{name}.npz")
    m = RobotModel(twists=z["twists"], parent_tf=z["parent_tf"], parent_idx=z["parent_idx"], act_idx=z["act_idx"],
                   mimic_mul=z["mimic_mul"], mimic_off=z["mimic_off"], mimic_act_idx=z["mimic_act_idx"],
                   parent_joint_indices=z["parent_joint_indices"], lower=z["lower"], upper=z["upper"], name=name)
    m.topo_inv = np.asarray(z["topo_inv"], np.int32)
    m.fk_level_starts, m.fk_level_joints = depth_schedule(m.parent_idx, m.topo_inv)
    return m, RobotSpheres(centers=z["sphere_centers"], radii=z["sphere_radii"]), z["active_pairs"], int(z["ee_link"])

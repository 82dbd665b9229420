"""Parse the reference's spherized Panda (URDF + SRDF, from the reference
checkout's resources/panda) with ``pyroffi_b200.urdf.load_urdf`` and store
the kernels' robot arrays as ``robots/panda.npz``, so the GPU tests can run
the kernels on a shipped robot without the reference tree.

    python tests/golden/make_robot_fixtures.py [path/to/reference]
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from pyroffi_b200.urdf import load_urdf  # noqa: E402
from oracle.refpath import reference_root  # noqa: E402

FIELDS = ("twists", "parent_tf", "parent_idx", "act_idx", "mimic_mul", "mimic_off", "mimic_act_idx",
          "parent_joint_indices", "lower", "upper", "topo_inv")


def panda_arrays(ref: Path) -> dict:
    res = ref / "resources" / "panda"
    r = load_urdf(str(res / "panda_spherized.urdf"), srdf=str(res / "panda.srdf"))
    out = {k: getattr(r.model, k) for k in FIELDS}
    out["sphere_centers"] = r.spheres.centers
    out["sphere_radii"] = r.spheres.radii
    out["active_pairs"] = r.active_pairs
    out["link_names"] = np.array(r.link_names)
    out["ee_link"] = np.int32(r.link_index("panda_hand"))
    return out


def main(argv) -> int:
    ref = Path(argv[1]) if len(argv) > 1 else reference_root()
    if ref is None:
        print("reference checkout not found: pass its root or set PYROFFI_REF", file=sys.stderr)
        return 1
    np.savez_compressed(HERE / "robots" / "panda.npz", **panda_arrays(ref))
    print("wrote", HERE / "robots" / "panda.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))

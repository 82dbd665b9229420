"""Where the reference checkout lives -- TEST INFRASTRUCTURE ONLY.

The location comes from the environment variable ``PYROFFI_REF`` (the
reference project's root directory).  Without it, the default is the one
``oracle/Makefile`` states as ``REF_ROOT``, so the recipe that compiles the
reference's helper headers and the Python scripts that read the reference's
resources agree on a single setting.  Nothing on a GPU run reads the
reference: its outputs travel as the fixtures under ``tests/golden/``.
"""

from __future__ import annotations

import os
import re
from pathlib import Path

_MAKEFILE = Path(__file__).resolve().parent / "Makefile"


def reference_root() -> Path | None:
    """The reference project's root, or None when no such directory exists."""
    env = os.environ.get("PYROFFI_REF")
    if env:
        p = Path(env)
    else:
        m = re.search(r"^REF_ROOT\s*\?=\s*(\S+)\s*$", _MAKEFILE.read_text(), re.M)
        if not m:
            return None
        p = Path(m.group(1))
    return p if p.is_dir() else None

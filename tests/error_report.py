"""Measured errors against the FP64 oracle, per quantity (test helper).

GPU parity tests call ``record(quantity, error, case)`` with the largest
error they observed; the session keeps the maximum per quantity.  When the
environment variable ``PK_ERROR_REPORT`` names a file, the conftest hook
writes the table there as JSON at the end of the session, so a GPU run of
the suite states its errors (FK position and rotation, sphere centres,
signed distances, IK residual, trajectory cost and gradient) as numbers
rather than only as passed tolerances."""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

_ERRORS: dict[str, dict] = {}


def record(quantity: str, error, case: str = "", unit: str = "") -> None:
    e = float(np.max(error)) if np.size(error) else 0.0
    prev = _ERRORS.get(quantity)
    if prev is None or e > prev["max"]:
        _ERRORS[quantity] = {"max": e, "case": case, "unit": unit}


def write_if_requested() -> None:
    path = os.environ.get("PK_ERROR_REPORT")
    if path and _ERRORS:
        Path(path).write_text(json.dumps(_ERRORS, indent=1, sort_keys=True) + "\n")


def assert_distances(out, ref, atol=1e-5, quantity="signed distance", case=""):
    """|out - ref| <= atol on every real distance (|ref| < 1e6); entries of
    padded spheres (the 1e9-scale sentinels) only need to stay that large."""
    out = np.asarray(out, np.float64)
    ref = np.asarray(ref, np.float64)
    assert out.shape == ref.shape
    real = np.abs(ref) < 1e6
    err = np.abs(out - ref)[real]
    record(quantity, err, case, "m")
    assert err.size == 0 or err.max() <= atol, (float(err.max()), atol)
    assert np.all(np.abs(out[~real]) >= 1e6)

"""The C-ABI library loads, exports every symbol include/pyroffi_b200.h
declares, and rejects bad arguments before touching the GPU (these calls
return from host-side validation, so they run without a device)."""

import ctypes as C
import subprocess

import pytest

from pyroffi_b200 import _lib


def test_header_declares_expected_entry_points():
    names = _lib.declared_symbols()
    for n in ("pk_fk_cuda", "pk_collision_world_sphere", "pk_collision_world_sphere_reduced",
              "pk_collision_world_capsule", "pk_collision_self_sphere", "pk_collision_self_capsule",
              "pk_ls_ik_cuda", "pk_ls_ik_ex", "pk_ik_verify_select", "pk_fk_sphere_collision",
              "pk_last_error", "pk_version", "pk_status_string"):
        assert n in names, n


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in _lib.declared_symbols() if n not in exported]
    assert not missing, missing
    for n in _lib.declared_symbols():
        assert getattr(lib, n) is not None


def test_python_signatures_cover_compute_entry_points():
    compute = [n for n in _lib.declared_symbols() if n not in ("pk_last_error", "pk_version", "pk_status_string")]
    assert sorted(compute) == sorted(_lib.SIGNATURES)


def test_version_and_status_strings(lib):
    assert b"sm_100a" in lib.pk_version()
    assert lib.pk_status_string(_lib.PK_ERR_CAPACITY) == b"capacity exceeded"


def _fk_call(batch, n_act, n_joints, n_levels):
    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: validation fails first
    return lib.pk_fk_cuda(None, *([dummy] * 12), batch, n_act, n_joints, n_levels)


def test_fk_rejects_bad_extents(lib):
    assert _fk_call(-1, 7, 7, 7) == _lib.PK_ERR_INVALID
    assert b"negative" in lib.pk_last_error()
    assert _fk_call(4, 7, 65, 7) == _lib.PK_ERR_CAPACITY
    assert b"n_joints" in lib.pk_last_error()
    assert _fk_call(0, 7, 7, 7) == _lib.PK_OK        # empty batch: nothing to do


def test_lm_rejects_dof_beyond_capacity(lib):
    opt = _lib.LmOptions(30, 50, 10, 1e-2, 0.5, 3, 1e-8, 1e-8, 0, 0, 0.02, 0, 0)
    d = C.c_void_p(16)
    st = lib.pk_ls_ik_ex(None, C.byref(opt), *([d] * 25), 4, 8, 40, 40, 1, 0, 0, 0, 0, 0, 0)
    assert st == _lib.PK_ERR_CAPACITY
    assert b"n_act" in lib.pk_last_error()
    st = lib.pk_ls_ik_ex(None, C.byref(opt), *([d] * 25), 4, 8, 7, 7, 0, 0, 0, 0, 0, 0, 0)
    assert st == _lib.PK_ERR_INVALID                  # no end-effector


def test_self_sphere_rejects_negative(lib):
    d = C.c_void_p(16)
    assert lib.pk_collision_self_sphere(None, d, d, d, d, d, 4, -1, 8, 3) == _lib.PK_ERR_INVALID


def test_world_reduced_requires_k_multiple_of_n(lib):
    d = C.c_void_p(16)
    st = lib.pk_collision_world_sphere_reduced(None, d, d, d, None, None, None, d, 2, 10, 3, 0, 0, 0, 4)
    assert st == _lib.PK_ERR_INVALID


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()

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


def _seed_ik_call(name, P=4, S=8, n_act=7, n_joints=7, n_ee=1, extra=()):
    """HJCD coarse / SQP entry with dummy pointers: 21 buffers, the scalar
    attributes `extra`, two outputs, then the extents."""
    lib = _lib.load()
    d = C.c_void_p(16)
    return getattr(lib, name)(None, *([d] * 21), *extra, d, d, P, S, n_act, n_joints, n_ee, 0, 0, 0, 0, 0)


_HJCD_COARSE = (20, 0, 1e4, 0.02)
_SQP = (60, 2, 50.0, 10.0, 5e-3, 1e-8, 1e-8, 0, 1e4, 0.02)


@pytest.mark.parametrize("name,extra", [("pk_hjcd_ik_coarse_cuda", _HJCD_COARSE), ("pk_sqp_ik_cuda", _SQP)])
def test_seed_ik_entries_validate_on_the_host(lib, name, extra):
    assert _seed_ik_call(name, P=-1, extra=extra) == _lib.PK_ERR_INVALID
    assert b"negative" in lib.pk_last_error()
    assert _seed_ik_call(name, n_act=17, n_joints=17, extra=extra) == _lib.PK_ERR_CAPACITY
    assert b"16 actuated" in lib.pk_last_error()
    assert _seed_ik_call(name, n_ee=0, extra=extra) == _lib.PK_ERR_CAPACITY
    assert _seed_ik_call(name, n_ee=5, extra=extra) == _lib.PK_ERR_CAPACITY
    assert _seed_ik_call(name, n_joints=65, extra=extra) == _lib.PK_ERR_CAPACITY
    assert _seed_ik_call(name, P=0, extra=extra) == _lib.PK_OK          # no problems: nothing to do


def test_hjcd_refinement_validates_on_the_host(lib):
    d = C.c_void_p(16)
    args = (20, 6, 1e-3, 1e-4, 0.02, 1e-8, 1e-8, 0, 1e4, 0.02)

    def call(P, S, n_act, n_ee=1, noise=d):
        return lib.pk_hjcd_ik_lm_cuda(None, d, noise, *([d] * 20), *args, d, d, d, P, S, n_act, n_act, n_ee,
                                      0, 0, 0, 0, 0)
    assert call(-2, 8, 7) == _lib.PK_ERR_INVALID
    assert call(4, 8, 20) == _lib.PK_ERR_CAPACITY
    assert call(4, 8, 7, noise=None) == _lib.PK_ERR_INVALID               # kicks need the noise buffer
    assert b"noise" in lib.pk_last_error()
    assert call(0, 8, 7) == _lib.PK_OK


def test_chomp_direction_validates_on_the_host(lib):
    d = C.c_void_p(16)
    assert lib.pk_chomp_direction(None, d, d, -1, 64, 7, 24, 10.0, 1.0, 1e-6, 1, None) == _lib.PK_ERR_INVALID
    assert lib.pk_chomp_direction(None, d, d, 4, 131, 7, 24, 10.0, 1.0, 1e-6, 1, None) == _lib.PK_ERR_CAPACITY
    assert lib.pk_chomp_direction(None, d, d, 0, 64, 7, 24, 10.0, 1.0, 1e-6, 1, None) == _lib.PK_OK
    assert lib.pk_chomp_direction(None, None, None, 4, 64, 7, 24, 10.0, 1.0, 1e-6, 1, None) == _lib.PK_ERR_INVALID


def test_trajectory_cost_validates_on_the_host(lib):
    d = C.c_void_p(16)
    opt = _lib.TrajOptions(0.01, 1.0, 0.5, 0.1, 1.0, 3.0)

    def call(B, T, S, o=C.byref(opt)):
        return lib.pk_traj_cost_grad(None, o, *([d] * 22), B, T, 7, 7, 8, S, 0, 4, 0, 0, 0)
    assert call(4, 64, 33) == _lib.PK_ERR_CAPACITY                      # 32 spheres per link at most
    assert call(4, 4, 8) == _lib.PK_ERR_INVALID                         # the jerk stencil needs 5 waypoints
    assert call(-1, 64, 8) == _lib.PK_ERR_INVALID
    assert call(4, 64, 8, o=None) == _lib.PK_ERR_INVALID
    assert call(0, 64, 8) == _lib.PK_OK


def test_stage_wait_counter_rejects_null(lib):
    assert lib.pk_stage_wait_timeouts(None) == _lib.PK_ERR_INVALID
    assert b"null" in lib.pk_last_error()
    assert lib.pk_stage_wait_configure(2, 0) == _lib.PK_ERR_INVALID
    assert b"force_timeout" in lib.pk_last_error()


def test_every_declaration_cites_the_reference_or_says_it_has_none():
    """Each entry point in the header carries a comment that names the
    reference interface it replaces (file:line) or states that it has no
    reference counterpart."""
    import re
    from pathlib import Path
    text = (Path(__file__).resolve().parents[1] / "include" / "pyroffi_b200.h").read_text()
    missing = []
    for m in re.finditer(r"\n(?:int|const char\*|size_t|void)\s+(pk_\w+)\(", text):
        before = text[:m.start()]
        end = before.rfind("*/")
        comment = before[before.rfind("/*", 0, end):end]
        between = before[end + 2:]
        # the comment covers this declaration and any declarations right after it
        if re.search(r"\n\s*\n", between.strip("\n")) or not re.search(r"\.(cu|cuh|py):\d|counterpart|new target",
                                                                        comment):
            missing.append(m.group(1))
    assert not missing, missing


def test_fp64_solve_is_rejected_where_it_is_not_offered(lib):
    """fp64_solve runs in the seed-group kernel only: the batched entry and the
    other lane mappings refuse it on the host, before any launch."""
    d = C.c_void_p(16)
    opt = _lib.LmOptions(30, 50.0, 10.0, 1e-2, 0.1, 10.0, 1e-8, 1e-8, 0, 1e4, 0.02, 0, 0, 0, 1)
    cls = _lib.IkClass()
    st = lib.pk_ik_batch(None, C.byref(opt), C.byref(cls), 1, None, None, None, None, 0, 0, 0, 0, d, 1, d, 0)
    assert st == _lib.PK_ERR_INVALID and b"fp64_solve" in lib.pk_last_error()
    opt.threads_per_seed = 2
    st = lib.pk_ls_ik_ex(None, C.byref(opt), *([d] * 25), 1, 8, 7, 7, 1, 0, 0, 0, 0, 0, 0)
    assert st == _lib.PK_ERR_INVALID and b"fp64_solve" in lib.pk_last_error()


def test_nvtx_ranges_wrap_calls_when_asked(monkeypatch):
    """PK_NVTX=1 wraps each entry-point call in an NVTX range named after it
    (here with torch's NVTX calls recorded instead of sent)."""
    import torch
    pushed = []
    monkeypatch.setattr(_lib, "_NVTX", True)
    monkeypatch.setattr(torch.cuda.nvtx, "range_push", lambda name: pushed.append(name))
    monkeypatch.setattr(torch.cuda.nvtx, "range_pop", lambda: pushed.append("pop"))
    _lib.call("pk_chomp_line_select", None, None, None, None, None, None, None, 1, 0.0, 1, 0, 4, 7)
    assert pushed == ["pk_chomp_line_select", "pop"]

"""The allocation-free batched IK entry point, ``pk_ik_batch_static``.

It exists for callers that cannot allocate device memory when they solve
(for example a handler inside a runtime that owns all device memory and
gives the call no workspace, or a control loop that must not allocate once
it runs): its only scratch, the work-queue counters, sits in a fixed array
inside the library.  This test calls it through the C-ABI twice in a row on
the same inputs and checks both results against the regular entry point
``pk_ik_batch`` (which takes the counters from the caller); the second call
shows that the shared counters are cleared between calls.  It runs the same
way alone in a fresh process and after the other tests.
"""

import ctypes

import numpy as np
import pytest
import torch

from pyroffi_b200 import _lib
from pyroffi_b200 import workloads as W
from pyroffi_b200._tensors import ptr, stream_ptr
from pyroffi_b200.batch_ik import MixedIkBatch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _call(b, entry):
    Ms, Mc, Mb, Mh = b.world.counts()
    desc = ctypes.cast(b._descriptors(), ctypes.c_void_p)
    args = [stream_ptr(b.device), ctypes.byref(b.opt), desc, len(b.classes), *[ptr(t) for t in b.world.arrays()],
            Ms, Mc, Mb, Mh, ptr(b.items), b.n_items]
    if entry == "pk_ik_batch":
        args += [ptr(b.queue), 0]
    else:
        args += [0]
    _lib.call(entry, *args)


def _reset(b):
    for c in range(len(b.classes)):
        b.out_cfg[c].zero_()
        b.out_err[c].fill_(float("inf"))


def test_static_scratch_entry_matches_regular_entry_twice():
    w = W.mixed_ik(n_problems=40, seeds_range=(8, 48))
    b = MixedIkBatch(w.classes, w.world, device=DEV, max_iter=w.max_iter, lambda_init=w.lambda_init,
                     lambda_down=w.lambda_down, lambda_up=w.lambda_up, collision_weight=w.collision_weight,
                     collision_margin=w.collision_margin)
    b.prepare(w.problem_class, w.n_seeds)
    b.load(w.target_T, w.seeds)
    _reset(b)
    _call(b, "pk_ik_batch")
    torch.cuda.synchronize()
    ref_cfg = [t.clone() for t in b.out_cfg]
    ref_err = [t.clone() for t in b.out_err]
    assert all(torch.isfinite(e).any() for e, n in zip(ref_err, b.counts) if n)
    for _ in range(2):
        _reset(b)
        _call(b, "pk_ik_batch_static")
        torch.cuda.synchronize()
        for c in range(len(b.classes)):
            torch.testing.assert_close(b.out_cfg[c], ref_cfg[c], rtol=0, atol=0)
            torch.testing.assert_close(b.out_err[c], ref_err[c], rtol=0, atol=0)


def test_static_scratch_entry_forwards_argument_checks():
    """The entry validates its arguments as pk_ik_batch does: 9 classes (more
    than the batch supports) is refused before any launch, and the outputs
    stay untouched."""
    w = W.mixed_ik(n_problems=8, seeds_range=(4, 8))
    b = MixedIkBatch(w.classes, w.world, device=DEV)
    b.prepare(w.problem_class, w.n_seeds)
    Ms, Mc, Mb, Mh = b.world.counts()
    desc = ctypes.cast(b._descriptors(), ctypes.c_void_p)
    with pytest.raises(_lib.PkError) as e:
        _lib.call("pk_ik_batch_static", stream_ptr(b.device), ctypes.byref(b.opt), desc, 9,
                  *[ptr(t) for t in b.world.arrays()], Ms, Mc, Mb, Mh, ptr(b.items), b.n_items, 0)
    assert e.value.status == _lib.PK_ERR_CAPACITY
    np.testing.assert_array_equal(b.out_err[0].cpu().numpy(), np.inf)

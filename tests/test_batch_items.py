"""Host logic of the persistent batch (no GPU): the work items cover every
(problem, seed) exactly once, respect the per-body item size and come
longest first; the mixed workload has the configured class mix."""

import numpy as np

from pyroffi_b200 import workloads as W
from pyroffi_b200.batch_ik import BODY_SEED_GROUP, BODY_SEED_GROUP16, BODY_WARP, MixedIkBatch


def test_mixed_workload_shape():
    w = W.mixed_ik(n_problems=200, seeds_range=(32, 256))
    assert [c.model.n_act for c in w.classes] == [7, 6, 15, 29]
    assert [len(c.target_links) for c in w.classes] == [1, 1, 2, 2]
    counts = np.bincount(w.problem_class, minlength=4)
    assert counts.sum() == 200 and abs(counts[0] - 80) <= 2 and counts[3] == 20
    assert w.n_seeds.min() >= 32 and w.n_seeds.max() <= 256
    assert w.world.spheres.shape == (500, 4)
    for c in range(4):
        assert w.target_T[c].shape == (counts[c], len(w.classes[c].target_links), 7)
        assert w.seeds[c].shape[1] == w.n_seeds[w.problem_class == c].max()


def test_items_cover_every_seed_once():
    w = W.mixed_ik(n_problems=60, seeds_range=(1, 150))
    b = MixedIkBatch(w.classes, w.world, device="cpu")
    assert b.bodies == [BODY_SEED_GROUP, BODY_SEED_GROUP, BODY_SEED_GROUP16, BODY_WARP]
    b.prepare(w.problem_class, w.n_seeds)
    items = b.items.numpy()
    seen = {c: np.zeros((b.counts[c], b.strides[c]), int) for c in range(4)}
    for c, p, first, cnt in items:
        assert 0 < cnt <= b._chunk(c)
        seen[c][p, first:first + cnt] += 1
    for p in range(len(w.problem_class)):
        c, i = w.problem_class[p], b.index_in_class[p]
        assert np.all(seen[c][i, : w.n_seeds[p]] == 1)
        assert np.all(seen[c][i, w.n_seeds[p]:] == 0)
    cost = [b._cost_per_seed(c) * cnt for c, _, _, cnt in items]
    assert all(cost[i] >= cost[i + 1] for i in range(len(cost) - 1))
    assert items.dtype == np.int32 and items.shape[1] == 4

"""Multi-rank host logic on CPU: world_size-2 gloo process groups.

Covers the data-parallel split (contiguous ranges, no collective on the data
path), the result all-gather and the max-over-ranks timing reduction that a
multi-GPU run of the path uses, and the FK oracle evaluated per shard and
gathered back against the unsharded result.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyroffi_b200 import dist as pdist


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, n_items, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world_size,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import oracle.kinematics as okin
        from pyroffi_b200 import robot as R

        rng = np.random.default_rng(11)
        model = R.serial_chain(7, rng)
        cfg = model.random_cfgs(rng, n_items).astype(np.float64)
        local = pdist.shard(torch.as_tensor(cfg))
        a, b = pdist.shard_range(n_items, rank, world_size)
        assert torch.equal(local, torch.as_tensor(cfg[a:b]))
        T = okin.forward_kinematics(local.numpy(), model.as_dict())
        full = pdist.gather_shards(torch.as_tensor(T), n_items)
        t = pdist.max_over_ranks(0.25 * (rank + 1))
        np.save(os.path.join(out_dir, f"r{rank}.npy"), full.numpy())
        np.save(os.path.join(out_dir, f"t{rank}.npy"), np.array([t]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_items", [37, 2])
def test_gloo_two_ranks_shard_gather(tmp_path, n_items):
    ws = 2
    mp.start_processes(_worker, args=(ws, _free_port(), n_items, str(tmp_path)), nprocs=ws,
                       start_method="spawn", join=True)
    import oracle.kinematics as okin
    from pyroffi_b200 import robot as R

    rng = np.random.default_rng(11)
    model = R.serial_chain(7, rng)
    cfg = model.random_cfgs(rng, n_items).astype(np.float64)
    want = okin.forward_kinematics(cfg, model.as_dict())
    for r in range(ws):
        np.testing.assert_array_equal(np.load(tmp_path / f"r{r}.npy"), want)
        assert float(np.load(tmp_path / f"t{r}.npy")[0]) == 0.5


def test_shard_range_partition():
    for n in (0, 1, 7, 256, 1001):
        for w in (1, 2, 3, 8):
            ranges = [pdist.shard_range(n, r, w) for r in range(w)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(w - 1))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        pdist.shard_range(4, 2, 2)

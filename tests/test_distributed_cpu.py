"""Ensemble sharding and the cross-rank statistics exchange, on CPU ranks.

Two gloo ranks (spawned processes, 127.0.0.1) stand in for two GPUs: each
takes its block of samples (SimpleLoadBalancer.cpp:63-97), forms its FP64
Welford moments, and gather_moments hands every rank all ranks' moments in
rank order; their Chan merge must equal the statistics of the whole
ensemble.  No GPU is touched.
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from alsvinn_b200 import distributed


def test_samples_for_rank_blocks_like_the_reference():
    blocks = [distributed.samples_for_rank(4096, 8, r) for r in range(8)]
    assert blocks[0] == (0, 512) and blocks[7] == (3584, 512)
    covered = np.concatenate([np.arange(f, f + c) for f, c in blocks])
    np.testing.assert_array_equal(covered, np.arange(4096))
    with pytest.raises(ValueError):
        distributed.samples_for_rank(100, 3, 0)     # world must divide the samples
    with pytest.raises(ValueError):
        distributed.samples_for_rank(100, 4, 4)


def _chan_merge(n_a, mean_a, m2_a, n_b, mean_b, m2_b):
    n = n_a + n_b
    if n_a == 0:
        return n_b, mean_b.copy(), m2_b.copy()
    delta = mean_b - mean_a
    return n, mean_a + delta * (n_b / n), m2_a + m2_b + delta * delta * (n_a * n_b / n)


def _all_samples(total, cells):
    rng = np.random.default_rng(1234)
    return 1.7 + 0.05 * rng.standard_normal((total, cells))


def _worker(rank, world, port, out_dir, total, cells):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        first, count = distributed.samples_for_rank(total, world, rank)
        mine = _all_samples(total, cells)[first:first + count]
        mean = mine.mean(axis=0)
        m2 = ((mine - mean) ** 2).sum(axis=0)
        ns, means, m2s = distributed.gather_moments(count, torch.from_numpy(mean),
                                                    torch.from_numpy(m2))
        n, mu, M2 = 0, np.zeros(cells), np.zeros(cells)
        for k in range(world):
            n, mu, M2 = _chan_merge(n, mu, M2, ns[k], means[k].numpy(), m2s[k].numpy())
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), n=n, mean=mu, var=M2 / n)
    finally:
        torch.distributed.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2])
def test_gathered_moments_merge_to_the_ensemble_statistics(world):
    total, cells = 96, 257
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(world, _free_port(), d, total, cells), nprocs=world, join=True)
        res = [np.load(os.path.join(d, "rank%d.npz" % r)) for r in range(world)]
    data = _all_samples(total, cells)
    for r in res:
        assert int(r["n"]) == total
        np.testing.assert_allclose(r["mean"], data.mean(axis=0), rtol=1e-14)
        np.testing.assert_allclose(r["var"], data.var(axis=0), rtol=1e-12)
    # every rank merged in the same order: identical bits
    np.testing.assert_array_equal(res[0]["mean"], res[1]["mean"])
    np.testing.assert_array_equal(res[0]["var"], res[1]["var"])

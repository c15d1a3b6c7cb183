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


def _failing_worker(rank, world, port, out_dir, mode):
    """Rank 1 fails before the statistics exchange: it reports the failure
    ("report") or exits without a word ("silent"); rank 0 must learn of it on
    the host through check_peers, within the time limit, and never enter the
    collective."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import time
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=20))
    result = "no error"
    t0 = time.time()
    try:
        if rank == 1:
            try:
                raise RuntimeError("injected failure of this rank's share")
            except RuntimeError:
                if mode == "report":
                    distributed.check_peers(False, "stats-step-1", timeout_seconds=3.0)
                result = "left"
                return
        distributed.check_peers(True, "stats-step-1", timeout_seconds=3.0)
        distributed.gather_moments(1, torch.zeros(4, dtype=torch.float64),
                                   torch.zeros(4, dtype=torch.float64))
    except distributed.PeerFailure as e:
        result = "PeerFailure failed=%s silent=%s" % (e.failed, e.silent)
    finally:
        with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
            f.write("%s|%.1f" % (result, time.time() - t0))
        if rank == 0:
            # keep the store (hosted by rank 0) alive until rank 1 is done
            time.sleep(1.0)
        torch.distributed.destroy_process_group()


@pytest.mark.parametrize("mode", ["report", "silent"])
def test_failed_rank_is_detected_on_the_host_before_the_exchange(mode):
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_failing_worker, args=(2, _free_port(), d, mode), nprocs=2, join=True)
        r0 = open(os.path.join(d, "rank0.txt")).read().split("|")
        r1 = open(os.path.join(d, "rank1.txt")).read().split("|")
    assert r1[0] in ("left", "PeerFailure failed=[1] silent=[]")
    if mode == "report":
        assert r0[0] == "PeerFailure failed=[1] silent=[]"
    else:
        assert r0[0] == "PeerFailure failed=[] silent=[1]"
        assert float(r0[1]) < 15.0      # the 3 s limit, not the 20 s group timeout

"""The multi-GPU ensemble path of the product on one GPU: two ranks.

Two processes (gloo over 127.0.0.1, spawned) each run
``distributed.kh_observable_ensemble`` on their block of Kelvin-Helmholtz
samples (SimpleLoadBalancer.cpp:63-97: contiguous blocks), both on cuda:0.
Their kernels are independent (nothing on the device waits for the other
process); the exchange is on the host: check_peers through the store, the
Welford moments and the observables through gloo all_gathers staged in
host memory, and the rank-ordered Chan merge on each rank's device.

Every rank must hold bit for bit what one process computes alone: the
observables of the whole ensemble solved as one batch, and the FP64 field
statistics formed block by block (each rank's block accumulated by itself,
then merged in rank order, which is the association the sharded run
defines).
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import alsvinn_b200 as als
from alsvinn_b200 import distributed, uq

pytestmark = pytest.mark.gpu

N = 32
TOTAL = 140          # 70 per rank: two 64-state chunks per block
END_TIME = 0.1


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    torch.cuda.set_device(0)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=120))
    try:
        params, y, info = distributed.kh_observable_ensemble(N, TOTAL, precision="fp64",
                                                             end_time=END_TIME)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), params=params, y=y,
                 mean=info["field_mean"], var=info["field_var"])
    finally:
        torch.distributed.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _single_process_reference(world):
    """One process: the whole ensemble as one batch; statistics block by block."""
    params, y, info = uq.kh_observable_ensemble(N, 0, TOTAL, precision="fp64", end_time=END_TIME)
    merged = als.MeanVariance(int(np.prod(info["shape"])))
    for r in range(world):
        first, count = distributed.samples_for_rank(TOTAL, world, r)
        with als.Simulator(2, (N, N), (0.0, 0.0), (1.0, 1.0), flux="hll3",
                           reconstruction="weno2", integrator="rungekutta3",
                           boundary="periodic", cfl=0.4, end_time=END_TIME,
                           members=count) as sim:
            sim.set_state(np.stack([als.kelvin_helmholtz(N, params[first + k], sim.ghosts)
                                    for k in range(count)]))
            sim.run()
            block = als.MeanVariance(merged.count)
            block.add_solver(sim, 0)
            n, mean_ptr, m2_ptr = block.moments()
            mean = distributed._device_view(mean_ptr, block.count, 0).clone()
            m2 = distributed._device_view(m2_ptr, block.count, 0).clone()
            merged.merge(n, mean, m2)
            torch.cuda.synchronize()
            block.close()
    mean = torch.zeros(merged.count, dtype=torch.float64, device="cuda")
    var = torch.zeros_like(mean)
    merged.result(mean, var)
    merged.close()
    shape = info["shape"]
    return params, y, mean.cpu().numpy().reshape(shape), var.cpu().numpy().reshape(shape)


def test_two_ranks_on_one_gpu_equal_the_single_process_ensemble():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank, args=(world, _free_port(), d), nprocs=world, join=True)
        res = [dict(np.load(os.path.join(d, "rank%d.npz" % r))) for r in range(world)]
    params, y, mean, var = _single_process_reference(world)
    for r in res:
        np.testing.assert_array_equal(r["params"], params)
        np.testing.assert_array_equal(r["y"], y)
        np.testing.assert_array_equal(r["mean"], mean)
        np.testing.assert_array_equal(r["var"], var)
    # and the statistics are the ensemble's own to rounding
    with als.Simulator(2, (N, N), (0.0, 0.0), (1.0, 1.0), flux="hll3", reconstruction="weno2",
                       integrator="rungekutta3", boundary="periodic", cfl=0.4,
                       end_time=END_TIME, members=TOTAL) as sim:
        sim.set_state(np.stack([als.kelvin_helmholtz(N, params[k], sim.ghosts)
                                for k in range(TOTAL)]))
        sim.run()
        states = sim.get_state()
    np.testing.assert_allclose(mean, states.mean(axis=0), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(var, states.var(axis=0), rtol=1e-10, atol=1e-15)

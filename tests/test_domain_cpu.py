"""Spatial decomposition on CPU: the Cartesian decomposition's bookkeeping
and the halo exchange of both transports on host tensors (the exchange is
torch slicing and torch.distributed, the same code that moves device
planes).  Two gloo ranks stand in for two GPUs."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from alsvinn_b200 import domain


def test_decomposition_bookkeeping():
    """rank = x + px (y + py z); neighbours; physical sides of Neumann grids."""
    dec = domain.CartesianDecomposition(2, (64, 48), (4, 2), 6, "periodic")
    assert dec.coords == (2, 1, 0) and dec.local_n == (16, 24) and dec.start == (32, 24)
    assert dec.neighbours[:4] == [5, 7, 2, 2]
    dec = domain.CartesianDecomposition(2, (64, 48), (4, 2), 4, "neumann")
    assert dec.coords == (0, 1, 0)
    assert dec.neighbours[:4] == [-1, 5, 0, -1]
    # one rank along a direction: its periodic sides are the boundary's, not exchanged
    dec = domain.CartesianDecomposition(2, (64, 48), (2, 1), 0, "periodic")
    assert dec.neighbours[:4] == [1, 1, -1, -1]
    with pytest.raises(ValueError):
        domain.CartesianDecomposition(2, (64, 48), (5, 1), 0)
    with pytest.raises(ValueError):
        domain.CartesianDecomposition(1, (64,), (2, 2), 0)


def _global_with_ghosts(dim, n, g, bc, seed=3):
    """A random global interior with its ghosts filled (x, then y, then z
    sides over the full extent, as the reference's boundary does)."""
    rng = np.random.default_rng(seed)
    shape = [dim + 2] + [1] * (3 - dim) + [n[d] + 2 * g for d in reversed(range(dim))]
    U = np.zeros(shape)
    inner = [slice(None)] + [slice(None)] * (3 - dim) + [slice(g, g + n[d]) for d in
                                                        reversed(range(dim))]
    U[tuple(inner)] = rng.standard_normal([dim + 2] + [1] * (3 - dim) +
                                          [n[d] for d in reversed(range(dim))])
    for d in range(dim):
        ax = 3 - d
        N = n[d] + 2 * g
        for k in range(g):
            lo = [slice(None)] * 4
            hi = [slice(None)] * 4
            src_lo = [slice(None)] * 4
            src_hi = [slice(None)] * 4
            lo[ax] = k
            hi[ax] = N - 1 - k
            if bc == "periodic":
                src_lo[ax] = k + n[d]
                src_hi[ax] = N - 1 - k - n[d]
            else:
                src_lo[ax] = 2 * g - 1 - k
                src_hi[ax] = N - 2 * g + k
            U[tuple(lo)] = U[tuple(src_lo)]
            U[tuple(hi)] = U[tuple(src_hi)]
    return U


def _scramble_exchanged_ghosts(planes, dec, g):
    """Overwrites every ghost layer that the exchange must supply."""
    for d in range(dec.dimension):
        for side in (0, 1):
            if dec.neighbours[2 * d + side] >= 0:
                lo, hi = domain._recv_rows(dec.local_n[d], g, side)
                domain._slab(planes, d, lo, hi).fill_(-999.0)


@pytest.mark.parametrize("dim,n,procs", [(1, (24,), (3,)), (2, (12, 10), (2, 2)),
                                         (3, (6, 8, 4), (1, 2, 2))])
@pytest.mark.parametrize("bc", ["periodic", "neumann"])
def test_local_exchange_restores_the_global_ghosts(dim, n, procs, bc):
    g = 2
    U = _global_with_ghosts(dim, n, g, bc)
    world = int(np.prod(procs))
    decs = [domain.CartesianDecomposition(dim, n, procs, r, bc) for r in range(world)]
    planes = [torch.from_numpy(np.ascontiguousarray(U[d.local_slice(g)])) for d in decs]
    for p, d in zip(planes, decs):
        _scramble_exchanged_ghosts(p, d, g)
    domain.LocalExchange(decs, g).exchange(planes)
    for p, d in zip(planes, decs):
        got = p.numpy()
        want = U[d.local_slice(g)]
        # every exchanged layer is the global one; corners of two exchanged
        # directions included (the later axis carries them)
        for dd in range(dim):
            for side in (0, 1):
                if d.neighbours[2 * dd + side] >= 0:
                    lo, hi = domain._recv_rows(d.local_n[dd], g, side)
                    sl = [slice(None)] * 4
                    sl[3 - dd] = slice(lo, hi)
                    np.testing.assert_array_equal(got[tuple(sl)], want[tuple(sl)])


def _subdomain_images(i, n, G, bc, c, p):
    """(padded position, member step) pairs of interior cell i along one
    direction of subdomain c of p: the integer logic of subdomain_images in
    alsvinn_b200/csrc/stage_kernel.cuh, restated for a CPU check."""
    out = [(i + G, 0)]
    low = p > 1 and (c > 0 or bc == "periodic")
    high = p > 1 and (c < p - 1 or bc == "periodic")
    if i < G:
        out.append((i + G + n, -1 if low else 0) if (low or bc == "periodic")
                   else (G - 1 - i, 0))
    if i >= n - G:
        out.append((i + G - n, 1 if high else 0) if (high or bc == "periodic")
                   else (2 * n + G - 1 - i, 0))
    return out


@pytest.mark.parametrize("dim,n,procs", [(1, (24,), (3,)), (1, (8,), (2,)), (2, (12, 10), (2, 2)),
                                         (2, (16, 8), (4, 1)), (2, (8, 12), (1, 3)),
                                         (3, (8, 8, 4), (2, 2, 1)), (3, (4, 8, 8), (1, 2, 2)),
                                         (3, (8, 8, 8), (2, 2, 2))])
@pytest.mark.parametrize("bc", ["periodic", "neumann"])
def test_stage_kernel_images_rebuild_every_split_block(dim, n, procs, bc):
    """The fused split solver's epilogue: every interior cell of every
    subdomain writes its images (own boundary images and the neighbours'
    ghost layers, corners as combined steps) into the members' blocks.
    Starting from blocks whose ghosts are garbage, this must give each
    block exactly its slice of the whole grid with the whole grid's ghosts,
    and every write must land inside the member buffers."""
    g = 2
    U = _global_with_ghosts(dim, n, g, bc)
    world = int(np.prod(procs))
    decs = [domain.CartesianDecomposition(dim, n, procs, r, bc) for r in range(world)]
    p3 = list(procs) + [1] * (3 - len(procs))
    blocks = np.stack([U[d.local_slice(g)] for d in decs])
    local = decs[0].local_n
    inner = [slice(None)] * 4
    for d in range(dim):
        inner[3 - d] = slice(g, g + local[d])
    work = np.full_like(blocks, -999.0)
    for r in range(world):
        work[r][tuple(inner)] = blocks[r][tuple(inner)]
    ln = list(local) + [1] * (3 - dim)
    for r, dec in enumerate(decs):
        c = dec.coords
        for gz in range(ln[2]):
            for gy in range(ln[1]):
                for gx in range(ln[0]):
                    per_axis = []
                    for d, i in enumerate((gx, gy, gz)):
                        if d < dim:
                            per_axis.append(_subdomain_images(i, ln[d], g, bc, c[d], p3[d]))
                        else:
                            per_axis.append([(0, 0)])
                    src = work[r][:, per_axis[2][0][0], per_axis[1][0][0], per_axis[0][0][0]]
                    for kz, (pz, sz) in enumerate(per_axis[2]):
                        for ky, (py, sy) in enumerate(per_axis[1]):
                            for kx, (px, sx) in enumerate(per_axis[0]):
                                if kx == ky == kz == 0:
                                    continue
                                t = [(c[0] + sx) % p3[0], (c[1] + sy) % p3[1], (c[2] + sz) % p3[2]]
                                m = t[0] + p3[0] * (t[1] + p3[1] * t[2])
                                assert 0 <= m < world
                                assert 0 <= pz < work.shape[2] and 0 <= py < work.shape[3] \
                                    and 0 <= px < work.shape[4]
                                work[m][:, pz, py, px] = src
    np.testing.assert_array_equal(work, blocks)


def _dist_worker(rank, world, port, out_dir, dim, n, procs, bc):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        g = 2
        U = _global_with_ghosts(dim, n, g, bc)
        dec = domain.CartesianDecomposition(dim, n, procs, rank, bc)
        planes = torch.from_numpy(np.ascontiguousarray(U[dec.local_slice(g)]))
        _scramble_exchanged_ghosts(planes, dec, g)
        ex = domain.DistExchange(dec, g)
        ex.exchange(planes)
        ws = ex.max_wave_speed([rank + 1.0, 10.0 * rank, 0.0])
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), got=planes.numpy(),
                 want=U[dec.local_slice(g)], ws=ws)
    finally:
        torch.distributed.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("dim,n,procs,bc", [(2, (12, 10), (1, 2), "periodic"),
                                            (2, (12, 10), (2, 1), "neumann"),
                                            (1, (16,), (2,), "periodic")])
def test_dist_exchange_on_gloo_ranks(dim, n, procs, bc):
    world = int(np.prod(procs))
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_dist_worker, args=(world, _free_port(), d, dim, n, procs, bc), nprocs=world,
                 join=True)
        res = [np.load(os.path.join(d, "r%d.npz" % r)) for r in range(world)]
    for r, z in enumerate(res):
        dec = domain.CartesianDecomposition(dim, n, procs, r, bc)
        for dd in range(dim):
            for side in (0, 1):
                if dec.neighbours[2 * dd + side] >= 0:
                    lo, hi = domain._recv_rows(dec.local_n[dd], 2, side)
                    sl = [slice(None)] * 4
                    sl[3 - dd] = slice(lo, hi)
                    np.testing.assert_array_equal(z["got"][tuple(sl)], z["want"][tuple(sl)])
        np.testing.assert_array_equal(z["ws"], [world, 10.0 * (world - 1), 0.0])

"""One grid split over several subdomains (spatial domain decomposition).

The reference's MPI path (alsfvm/src/mpi/): a Cartesian decomposition of the
grid over px x py x pz ranks (domain/CartesianDecomposition.cpp:40-135;
rank = x + px (y + py z), cartesian/rank_index.hpp), every side of a
subdomain either a neighbour (exchanged) or a physical boundary, the ghost
layers exchanged before every flux evaluation
(CartesianCellExchanger.cpp:51-100, ConservedSystem.cpp:45-63) and the
wave speed maximised over ranks before the time step
(CartesianCellExchanger.cpp:37-44).

Each subdomain runs the B200 plug-in calls (NumericalFlux, Integrator,
Boundary) on its own padded planes.  After a stage, a subdomain first fills
its ghosts locally (als_fill_ghosts with the global boundary type: right for
physical sides, overwritten on the others) and then the exchange overwrites,
axis by axis, every side that has a neighbour with that neighbour's
boundary slab -- full slabs, ghosts of the other axes included, so later
axes carry the corners.  Interior results equal the undivided grid's bit for
bit (the flux stencils are axis-aligned and read no corner ghosts).

`SplitSimulation` runs the same split in the fused solver instead
(als_solver_decompose): the subdomains are the members of one solver, one
launch per stage covers all of them, they share one time step, and each
stage kernel writes every updated cell's images straight into the
neighbouring subdomains' ghost layers, so no exchange step and no host
round trip remain between the stages.

Two transports for the plug-in path:

* ``LocalExchange``: every subdomain lives in this process (one GPU); halo
  slabs are device-to-device copies.
* ``DistExchange``: one subdomain per process (one GPU each);
  ``torch.distributed`` point-to-point sends of packed slabs (NCCL over
  NVLink for device tensors, gloo for host tensors) in two phases per axis
  (upward, then downward), so a pair of ranks never has two messages in
  flight in the same direction; the wave speed is an all-reduce (MAX).
"""
import numpy as np

from . import _lib
from .simulator import Boundary, Integrator, NumericalFlux, _ptr, _stream, INTEGRATOR


class CartesianDecomposition:
    """Subdomain `rank` of a grid of `n` cells split over `procs` ranks per
    direction (CartesianDecomposition.cpp:40-135)."""

    def __init__(self, dimension, n, procs, rank, boundary="periodic"):
        self.dimension = dimension
        self.n = tuple(int(v) for v in n)[:dimension]
        procs = tuple(int(v) for v in procs) + (1,) * (3 - len(procs))
        self.procs = procs[:3]
        world = self.procs[0] * self.procs[1] * self.procs[2]
        if not 0 <= rank < world:
            raise ValueError("rank %d outside %d subdomains" % (rank, world))
        for d in range(3):
            if d >= dimension and self.procs[d] != 1:
                raise ValueError("inactive direction %d cannot be split" % d)
            if d < dimension and self.n[d] % self.procs[d] != 0:
                raise ValueError("%d ranks do not divide %d cells in direction %d"
                                 % (self.procs[d], self.n[d], d))
        self.rank = rank
        self.world = world
        self.boundary = boundary
        self.coords = (rank % self.procs[0], (rank // self.procs[0]) % self.procs[1],
                       rank // (self.procs[0] * self.procs[1]))
        self.local_n = tuple(self.n[d] // self.procs[d] for d in range(dimension))
        self.start = tuple(self.local_n[d] * self.coords[d] for d in range(dimension))
        # neighbours[2d + s]: rank on side s (0 low, 1 high) of direction d, or -1
        self.neighbours = [-1] * 6
        for side in range(2 * dimension):
            d, s = side // 2, side % 2
            at_edge = (s == 0 and self.coords[d] == 0) or \
                      (s == 1 and self.coords[d] == self.procs[d] - 1)
            if at_edge and (boundary != "periodic" or self.procs[d] == 1):
                continue
            if self.procs[d] == 1:
                continue
            c = list(self.coords)
            c[d] = (c[d] + (1 if s else -1)) % self.procs[d]
            self.neighbours[side] = c[0] + self.procs[0] * (c[1] + self.procs[1] * c[2])

    def local_slice(self, ghosts):
        """Slices of the global padded array (nvar, Nz, Ny, Nx) holding this
        subdomain's padded block (its interior plus `ghosts` around it)."""
        sl = [slice(None)] * 4
        for d in range(self.dimension):
            axis = 3 - d
            sl[axis] = slice(self.start[d], self.start[d] + self.local_n[d] + 2 * ghosts)
        return tuple(sl)


def _slab(planes, d, lo, hi):
    """View of planes (nvar, Nz, Ny, Nx) restricted to [lo, hi) along direction d."""
    sl = [slice(None)] * planes.dim()
    sl[planes.dim() - 1 - d] = slice(lo, hi)
    return planes[tuple(sl)]


def _send_rows(local_n, g, side):
    """Rows a subdomain sends across `side`: its g boundary layers."""
    return (g, 2 * g) if side == 0 else (local_n, local_n + g)


def _recv_rows(local_n, g, side):
    """Its ghost rows on `side`."""
    return (0, g) if side == 0 else (local_n + g, local_n + 2 * g)


class LocalExchange:
    """All subdomains in this process: halo slabs copied between their planes."""

    def __init__(self, decompositions, ghosts):
        self.decs = decompositions
        self.g = ghosts

    def exchange(self, planes):
        """planes[r]: subdomain r's padded planes (device tensors)."""
        for d in range(self.decs[0].dimension):
            for side in (0, 1):
                for r, dec in enumerate(self.decs):
                    nb = dec.neighbours[2 * d + side]
                    if nb < 0:
                        continue
                    # my ghosts on `side` come from the neighbour's opposite boundary layers
                    lo, hi = _recv_rows(dec.local_n[d], self.g, side)
                    slo, shi = _send_rows(self.decs[nb].local_n[d], self.g, 1 - side)
                    _slab(planes[r], d, lo, hi).copy_(_slab(planes[nb], d, slo, shi))

    def max_wave_speed(self, speeds):
        return np.max(np.asarray(speeds, dtype=np.float64), axis=0)


class DistExchange:
    """One subdomain per process, torch.distributed point-to-point."""

    def __init__(self, decomposition, ghosts, group=None):
        self.dec = decomposition
        self.g = ghosts
        self.group = group

    def exchange(self, planes):
        import torch.distributed as dist
        dec, g = self.dec, self.g
        for d in range(dec.dimension):
            # phase 0: slabs travel up (to the high neighbour); phase 1: down
            for phase in (0, 1):
                send_side, recv_side = (1, 0) if phase == 0 else (0, 1)
                ops, recvs = [], []
                nb_send = dec.neighbours[2 * d + send_side]
                nb_recv = dec.neighbours[2 * d + recv_side]
                if nb_send >= 0:
                    lo, hi = _send_rows(dec.local_n[d], g, send_side)
                    ops.append(dist.P2POp(dist.isend, _slab(planes, d, lo, hi).contiguous(),
                                          nb_send, self.group))
                if nb_recv >= 0:
                    lo, hi = _recv_rows(dec.local_n[d], g, recv_side)
                    buf = _slab(planes, d, lo, hi).contiguous()
                    ops.append(dist.P2POp(dist.irecv, buf, nb_recv, self.group))
                    recvs.append((lo, hi, buf))
                if ops:
                    for req in dist.batch_isend_irecv(ops):
                        req.wait()
                for lo, hi, buf in recvs:
                    _slab(planes, d, lo, hi).copy_(buf)

    def max_wave_speed(self, speed):
        import torch
        import torch.distributed as dist
        t = torch.tensor(np.asarray(speed, dtype=np.float64))
        if dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return t.cpu().numpy()


class Subdomain:
    """The plug-in solver state of one subdomain."""

    def __init__(self, decomposition, flux, reconstruction, integrator, cfl, gamma):
        dec = decomposition
        self.dec = dec
        self.flux = NumericalFlux(dec.dimension, dec.local_n, flux, reconstruction, gamma)
        self.g = self.flux.getNumberOfGhostCells()
        self.boundary = Boundary(dec.dimension, dec.local_n, self.g, dec.boundary)
        self.integrator = Integrator(integrator, self.flux, cfl)
        self.volumes = None

    def set_state(self, global_padded):
        """Takes this subdomain's block of a global padded state (numpy)."""
        import torch
        block = np.ascontiguousarray(global_padded[self.dec.local_slice(self.g)])
        first = torch.from_numpy(block).cuda()
        self.volumes = [first] + [first.clone() for _ in
                                  range(self.integrator.getNumberOfSubsteps())]

    def interior(self, k=0):
        """Interior cells of volume k (numpy)."""
        v = self.volumes[k].cpu().numpy()
        sl = [slice(None)] * 4
        for d in range(self.dec.dimension):
            sl[3 - d] = slice(self.g, self.g + self.dec.local_n[d])
        return v[tuple(sl)]


class DecomposedSimulation:
    """The reference's time loop over decomposed subdomains
    (Simulator.cpp:191-214 with ConservedSystem's exchange and the
    wave-speed maximum).  `subdomains` are the ones of this process;
    `exchange` a LocalExchange (all of them) or a DistExchange (one)."""

    def __init__(self, subdomains, exchange, cell_lengths, cfl, end_time, stream=0):
        self.subs = subdomains
        self.exchange = exchange
        self.lengths = list(cell_lengths) + [0.0] * (3 - len(cell_lengths))
        self.cfl = cfl
        self.end_time = end_time
        self.t = 0.0
        self.steps = 0
        self.stream = stream
        self.dts = []

    def _exchange(self, k):
        planes = [s.volumes[k] for s in self.subs]
        for s, p in zip(self.subs, planes):
            s.boundary.applyBoundaryConditions(p, stream=self.stream)
        if isinstance(self.exchange, LocalExchange):
            self.exchange.exchange(planes)
        else:
            self.exchange.exchange(planes[0])

    def _max_speed(self, speeds):
        if isinstance(self.exchange, LocalExchange):
            return self.exchange.max_wave_speed(speeds)
        return self.exchange.max_wave_speed(speeds[0])

    def run(self, max_steps=10 ** 9):
        import torch
        lib = _lib.load()
        integ = self.subs[0].integrator
        substeps = integ.getNumberOfSubsteps()
        self._exchange(0)
        while self.t < self.end_time and self.steps < max_steps:
            dt = 0.0
            for s in range(substeps):
                speeds = [sub.flux.computeFlux(sub.volumes[s], sub.volumes[s + 1],
                                               stream=self.stream, compute_wave_speed=s == 0)
                          for sub in self.subs]
                if s == 0:
                    ws = self._max_speed(speeds)
                    dt = integ.computeTimestep(ws, self.lengths, self.t, self.end_time)
                c = dt / self.lengths[0]
                for sub in self.subs:
                    out = sub.volumes[s + 1]
                    if integ.integrator == INTEGRATOR["rungekutta4"] and s == 3:
                        _lib.check(lib.als_integrator_combine_rk4(
                            _ptr(out), _ptr(sub.volumes[0]), _ptr(sub.volumes[1]),
                            _ptr(sub.volumes[2]), _ptr(sub.volumes[3]), out.numel(), c,
                            _stream(self.stream)))
                    else:
                        _lib.check(lib.als_integrator_combine(
                            integ.integrator, s, _ptr(out), _ptr(sub.volumes[s]),
                            _ptr(sub.volumes[0]), out.numel(), c, _stream(self.stream)))
                self._exchange(s + 1)
            for sub in self.subs:
                sub.volumes[0], sub.volumes[substeps] = sub.volumes[substeps], sub.volumes[0]
            self.t += dt
            self.steps += 1
            self.dts.append(dt)
        torch.cuda.synchronize()
        return self.steps, self.t

    def gather(self, global_shape):
        """The global interior (numpy, nvar x interior shape) from the
        subdomains of this process (LocalExchange: all of them)."""
        nvar = global_shape[0]
        dim = self.subs[0].dec.dimension
        shape = [nvar] + [1] * (3 - dim) + [self.subs[0].dec.n[d] for d in reversed(range(dim))]
        out = np.zeros(shape)
        for sub in self.subs:
            sl = [slice(None)] * 4
            for d in range(dim):
                sl[3 - d] = slice(sub.dec.start[d], sub.dec.start[d] + sub.dec.local_n[d])
            out[tuple(sl)] = sub.interior()
        return out


class SplitSimulation:
    """A grid of ``n`` cells split over ``procs`` subdomains that advance in
    the fused solver (``Simulator.decompose``).  Subdomain r is member r
    (x fastest, CartesianDecomposition.cpp:40-135).  The solver's corners are
    subdomain 0's, as the reference computes them (origin, origin + dx *
    local cells, CartesianDecomposition.cpp:69-72), moved by as many ulps as
    it takes for (end - origin) / local cells to be the whole grid's cell
    length to the bit: the reference's ranks each recompute the length from
    their corners and can differ from the whole grid in the last bit; here
    every subdomain takes the whole grid's time step."""

    def __init__(self, dimension, n, procs, lower=None, upper=None, flux="hll3",
                 reconstruction="weno2", integrator="rungekutta3", boundary="periodic",
                 gamma=1.4, cfl=0.4, end_time=1.0, max_steps=0, precision="fp64", device=0):
        from .simulator import Simulator
        self.dimension = dimension
        self.n = tuple(int(v) for v in n)[:dimension]
        world = 1
        for p in procs:
            world *= int(p)
        self.decs = [CartesianDecomposition(dimension, self.n, procs, r, boundary)
                     for r in range(world)]
        self.boundary = boundary
        lower = list(lower or [0.0] * dimension)
        upper = list(upper or [1.0] * dimension)
        local_n = self.decs[0].local_n
        dx = [(upper[d] - lower[d]) / self.n[d] for d in range(dimension)]
        lo = [lower[d] for d in range(dimension)]
        hi = [lo[d] + dx[d] * local_n[d] for d in range(dimension)]
        for d in range(dimension):
            for _ in range(64):
                got = (hi[d] - lo[d]) / local_n[d]
                if got == dx[d]:
                    break
                hi[d] = np.nextafter(hi[d], np.inf if got < dx[d] else -np.inf)
            if (hi[d] - lo[d]) / local_n[d] != dx[d]:
                raise ValueError("no subdomain corner gives the whole grid's cell length")
        self.sim = Simulator(dimension, local_n, lo, hi, flux=flux, reconstruction=reconstruction,
                             integrator=integrator, boundary=boundary, gamma=gamma, cfl=cfl,
                             end_time=end_time, max_steps=max_steps, precision=precision,
                             members=world, device=device)
        self.sim.decompose(procs)
        self.ghosts = self.sim.ghosts

    def set_state(self, global_padded):
        """Takes the whole grid's padded state (numpy, nvar x padded extents):
        fills its ghosts with the boundary condition and hands every
        subdomain its block."""
        import torch
        x = torch.from_numpy(np.ascontiguousarray(global_padded, dtype=np.float64)).cuda()
        Boundary(self.dimension, self.n, self.ghosts, self.boundary).applyBoundaryConditions(x)
        whole = x.cpu().numpy()
        blocks = np.stack([whole[dec.local_slice(self.ghosts)] for dec in self.decs])
        self.sim.set_state(blocks)

    def gather(self):
        """The whole grid's padded state (numpy) from the subdomains' blocks;
        every cell, ghosts included, is taken from the subdomain whose block
        holds it first (their blocks overlap in the ghost layers)."""
        blocks = self.sim.get_state()
        g = self.ghosts
        shape = [blocks.shape[1]] + [1] * (3 - self.dimension) + \
            [self.n[d] + 2 * g for d in reversed(range(self.dimension))]
        out = np.zeros(shape)
        for r in reversed(range(len(self.decs))):
            out[self.decs[r].local_slice(g)] = blocks[r]
        return out

    def interior(self):
        """The whole grid's interior cells (numpy)."""
        full = self.gather()
        g = self.ghosts
        sl = [slice(None)] * 4
        for d in range(self.dimension):
            sl[3 - d] = slice(g, g + self.n[d])
        return full[tuple(sl)]

    def run(self):
        self.sim.run()
        return self.sim.info()

    def advance(self, steps):
        self.sim.advance(steps)

    def close(self):
        self.sim.close()

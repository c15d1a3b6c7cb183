"""Ensembles sharded over GPUs, one process per GPU (torch.distributed).

Samples are independent, so the only exchange is the statistics at the end:

* ``samples_for_rank``: contiguous blocks of total/world samples per rank, the
  reference's SimpleLoadBalancer (alsuq/src/mpi/SimpleLoadBalancer.cpp:35-97),
  including its requirement that the world size divides the sample count;
* ``gather_moments``: every rank's Welford (n, mean, M2) gathered on every
  rank with one all_gather per array (NCCL over NVLink straight from device
  memory; with a gloo group the arrays are staged through host memory);
* ``merge_statistics``: a fresh FP64 accumulator into which all ranks'
  moments are Chan-merged in rank order on the device, so every rank holds
  the same bits.  The reference instead MPI_Reduces raw sums S1, S2 to rank 0
  (alsuq/src/stats/StatisticsHelper.cpp:35-79).

No step of the solve itself communicates.

``check_peers`` is the failure check before that exchange: every rank posts
whether its share succeeded under a tag in the process group's key-value
store and waits, with a time limit, for everyone else's; a failed or silent
rank turns into a ``PeerFailure`` on every other rank, on the host, before
any collective is launched.
"""
import datetime


class PeerFailure(RuntimeError):
    """Raised by check_peers: ``failed`` ranks reported a failure, ``silent``
    ranks did not report within the time limit."""

    def __init__(self, tag, failed, silent):
        super().__init__("ranks %s failed and ranks %s did not report before %r"
                         % (failed, silent, tag))
        self.failed = failed
        self.silent = silent


def check_peers(ok, tag, timeout_seconds=30.0, store=None, group=None):
    """Posts this rank's status for ``tag`` and waits for every rank's.

    Returns when all ranks posted success; raises PeerFailure otherwise
    (after at most ``timeout_seconds`` per silent rank).  Each tag is used
    once per run (e.g. "stats-step-100")."""
    import torch.distributed as dist
    if store is None:
        store = dist.distributed_c10d._get_default_store()
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    store.set("%s/%d" % (tag, rank), b"1" if ok else b"0")
    failed, silent = [], []
    limit = datetime.timedelta(seconds=timeout_seconds)
    for r in range(world):
        key = "%s/%d" % (tag, r)
        try:
            store.wait([key], limit)
        except Exception:
            silent.append(r)
            continue
        if store.get(key) != b"1":
            failed.append(r)
    if failed or silent:
        raise PeerFailure(tag, failed, silent)


def samples_for_rank(total, world, rank):
    """Sample indices [first, first + count) of `rank` (contiguous blocks)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    if total % world != 0:
        raise ValueError("the number of processes (%d) must divide the number of samples (%d)"
                         % (world, total))
    per = total // world
    return rank * per, per


def _exchange_device(group=None):
    """Where the collectives of `group` take their tensors: the current CUDA
    device for NCCL, the host for gloo."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def all_gather_tensor(x, group=None):
    """All ranks' copies of tensor `x` (same shape on every rank), in rank
    order, on x's device; staged through the host for gloo."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    via = _exchange_device(group)
    xs = x.contiguous().to(via)
    parts = [torch.empty_like(xs) for _ in range(world)]
    dist.all_gather(parts, xs, group=group)
    return [p.to(x.device) for p in parts]


def gather_moments(n, mean, m2, group=None):
    """All ranks' (n, mean, M2), in rank order, on every rank.

    ``mean`` and ``m2`` are FP64 tensors of the same length on every rank;
    the gathered arrays are returned on their device (NCCL exchanges device
    memory directly, gloo through host copies)."""
    import torch
    ns = torch.tensor([int(n)], dtype=torch.int64, device=mean.device)
    n_all = all_gather_tensor(ns, group)
    mean_all = all_gather_tensor(mean, group)
    m2_all = all_gather_tensor(m2, group)
    return [int(v.item()) for v in n_all], mean_all, m2_all


def merge_statistics(local, group=None):
    """Chan merge of every rank's MeanVariance ``local`` into a new
    accumulator, identical on all ranks.  Returns the new MeanVariance."""
    import torch
    from .simulator import MeanVariance
    torch.cuda.synchronize()
    n, mean_ptr, m2_ptr = local.moments()
    device = torch.cuda.current_device()
    mean = _device_view(mean_ptr, local.count, device).clone()
    m2 = _device_view(m2_ptr, local.count, device).clone()
    ns, means, m2s = gather_moments(n, mean, m2, group)
    merged = MeanVariance(local.count, device=device)
    for k in range(len(ns)):
        if ns[k] > 0:
            merged.merge(ns[k], means[k], m2s[k])
    torch.cuda.synchronize()
    return merged


class _DeviceArray:
    """Zero-copy view of library-owned device memory (CUDA array interface)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3}


def _device_view(ptr, count, device):
    """FP64 tensor aliasing `count` doubles at a library device pointer."""
    import torch
    return torch.as_tensor(_DeviceArray(ptr, count), device="cuda:%d" % device)


_calls = 0


def kh_observable_ensemble(n, total_samples, precision="fp64", end_time=2.0, group=None, **kw):
    """The UQ ensemble of uq.kh_observable_ensemble sharded over the ranks of
    `group`: each rank solves its block of samples on its own GPU; the
    observables are all-gathered (sample order) and the FP64 field
    statistics merged.  Returns (params, y, info) on every rank, info with
    the merged "field_mean" / "field_var" and this rank's "solve_seconds".
    A rank whose solve fails makes every rank raise PeerFailure (check_peers)
    before any collective starts."""
    import torch
    import torch.distributed as dist
    from . import uq
    global _calls
    _calls += 1
    tag = "kh-ensemble-%d" % _calls
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    first, count = samples_for_rank(total_samples, world, rank)
    try:
        params, y, info = uq.kh_observable_ensemble(n, first, count, precision=precision,
                                                    end_time=end_time, keep_statistics=True,
                                                    **kw)
    except Exception:
        # the others learn of it before they launch the exchange
        check_peers(False, tag, group=group)
        raise
    check_peers(True, tag, group=group)
    local = info.pop("statistics")
    merged = merge_statistics(local, group)
    local.close()
    count_all = merged.count
    mean = torch.zeros(count_all, dtype=torch.float64, device="cuda")
    var = torch.zeros_like(mean)
    merged.result(mean, var)
    merged.close()
    ys = all_gather_tensor(torch.as_tensor(y, dtype=torch.float64, device="cuda"), group)
    ps = all_gather_tensor(torch.as_tensor(params, dtype=torch.float64, device="cuda"), group)
    shape = info["shape"]
    info["field_mean"] = mean.cpu().numpy().reshape(shape)
    info["field_var"] = var.cpu().numpy().reshape(shape)
    return torch.cat(ps).cpu().numpy(), torch.cat(ys).cpu().numpy(), info

"""Mock catalogs shared out over GPUs (one process per GPU, ``torch.distributed``).

A single spectrum does not shard (the estimator's mesh is never split: no exchange step), so
several GPUs work as replicas.  Sets of independent mocks do shard: each rank measures
its own subset (``batch.BatchedSpectra`` per mesh size) and one collective assembles the
per-mock float64 multipoles on every rank for the covariance.  Not in the reference,
which measures mocks one at a time.

- ``mock_cost``: the relative cost of one mock, N_p log2(N_r) (paint work per particle
  grows with the mesh's tile count only through the log factor; the FFTs add
  N_r log2(N_r), included).
- ``partition_mocks``: longest-processing-time-first greedy assignment, deterministic, so
  every rank computes the same partition without communicating.
- ``gather_multipoles``: every rank contributes the rows of its own mocks; one
  ``all_reduce`` (sum over disjoint rows) gives all ranks the full (nmocks, nells, nbins)
  array.  Works with the nccl backend (device tensors) and gloo (host tensors).
- ``ShardedMocks`` / ``measure_mocks``: the runner: this rank's share of the mocks, grouped by
  mesh size into batches of one ``BatchedSpectra`` each (one paint launch sequence, one
  batched FFT and one binning pass per batch, replayed from a CUDA graph), then the gather.
"""
import math

import numpy as np
import torch

__all__ = ['mock_cost', 'partition_mocks', 'local_mocks', 'gather_multipoles', 'covariance', 'ShardedMocks',
           'measure_mocks']


def mock_cost(nparticles, meshsize):
    """Relative cost of measuring one mock: N_p log2(N_r) + N_r log2(N_r)."""
    nr = float(np.prod(np.broadcast_to(np.asarray(meshsize, dtype='f8'), (3,))))
    lg = math.log2(max(nr, 2.))
    return float(nparticles) * lg + nr * lg


def partition_mocks(costs, world_size):
    """Split mock indices over ``world_size`` ranks, balancing the summed cost.

    Mocks are taken by decreasing cost (ties by index) and each goes to the rank with the
    smallest load so far (ties to the lowest rank); each rank's list is returned sorted.
    """
    costs = np.asarray(costs, dtype='f8')
    if world_size < 1:
        raise ValueError('world_size must be >= 1')
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.] * world_size
    parts = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def local_mocks(costs, rank=None, world_size=None):
    """Indices of the mocks this rank measures (``torch.distributed`` defaults)."""
    if world_size is None:
        world_size = torch.distributed.get_world_size() if torch.distributed.is_initialized() else 1
    if rank is None:
        rank = torch.distributed.get_rank() if torch.distributed.is_initialized() else 0
    return partition_mocks(costs, world_size)[rank]


def gather_multipoles(local, nmocks, shape, device=None):
    """Full (nmocks, *shape) float64 array from each rank's ``{mock index: array}``.

    Rows of mocks a rank does not own are zero on that rank; ranks own disjoint rows, so a
    sum over ranks assembles the array (the rows are exact copies, nothing is added to a
    non-zero value).
    """
    if device is None:
        device = torch.device('cuda', torch.cuda.current_device()) if (
            torch.distributed.is_initialized() and torch.distributed.get_backend() == 'nccl') else torch.device('cpu')
    full = torch.zeros((nmocks,) + tuple(shape), dtype=torch.float64, device=device)
    for i, value in local.items():
        full[i] = torch.as_tensor(value, dtype=torch.float64, device=device)
    if torch.distributed.is_initialized() and torch.distributed.get_world_size() > 1:
        torch.distributed.all_reduce(full, op=torch.distributed.ReduceOp.SUM)
    return full


def covariance(multipoles):
    """Sample covariance of flattened multipoles ((nmocks, ...) -> (nvalues, nvalues)), float64."""
    x = torch.as_tensor(multipoles, dtype=torch.float64)
    x = x.reshape(x.shape[0], -1)
    d = x - x.mean(dim=0, keepdim=True)
    return d.T @ d / max(x.shape[0] - 1, 1)


class ShardedMocks:
    """This rank's share of a set of mocks, ready to measure: ``ShardedMocks(specs, bins)(catalog)``.

    Parameters
    ----------
    specs : list of (meshsize, nparticles), one per mock, the same list on every rank (the
        particle counts only weigh the partition: expected counts will do)
    bins : dict meshsize -> ``BinMesh2SpectrumPoles`` (all with the same ells and number of bins)
    group : mocks per batch (one runner per mesh size and group of this rank's mocks)
    runner : ``runner(attrs, bin, counts, resampler=, interlacing=, compensate=, los=)`` returning a
        callable of the concatenated positions that gives (nmocks, nells, nbins) multipoles;
        default ``batch.BatchedSpectra`` (autotuned paint tiles, captured in a CUDA graph at its
        first call).  A batch's runner is built at the first call with the catalogs' counts, and
        rebuilt when they change.
    """

    def __init__(self, specs, bins, resampler='tsc', interlacing=2, compensate=True, los='z', group=32, runner=None):
        if runner is None:
            from .batch import BatchedSpectra as runner
        self.runner = runner
        self.kwargs = dict(resampler=resampler, interlacing=interlacing, compensate=compensate, los=los)
        self.specs = [(int(m), float(n)) for m, n in specs]
        self.mine = local_mocks([mock_cost(n, m) for m, n in self.specs])
        shapes = {(len(b.ells), b.nbins) for b in bins.values()}
        if len(shapes) != 1:
            raise ValueError('every mesh size must bin the same ells into the same number of bins')
        self.shape = shapes.pop()
        self.bins = bins
        self.batches = []  # [meshsize, mock indices, counts, runner]
        for meshsize in sorted({self.specs[i][0] for i in self.mine}):
            idx = [i for i in self.mine if self.specs[i][0] == meshsize]
            for start in range(0, len(idx), group):
                self.batches.append([meshsize, idx[start:start + group], None, None])

    def __call__(self, catalog):
        """(nmocks, nells, nbins) float64 multipoles of every mock, on every rank.  ``catalog(i)``
        gives mock i's positions ((nparticles, 3) float32) and is called for this rank's mocks."""
        local = {}
        for batch in self.batches:
            meshsize, sel = batch[0], batch[1]
            cats = [torch.as_tensor(catalog(i)) for i in sel]
            counts = [int(c.shape[0]) for c in cats]
            if batch[3] is None or batch[2] != counts:
                b = self.bins[meshsize]
                batch[2], batch[3] = counts, self.runner(b.mattrs, b, counts, **self.kwargs)
            out = batch[3](torch.cat(cats))
            for j, i in enumerate(sel):
                local[i] = out[j]
        return gather_multipoles(local, len(self.specs), self.shape)


def measure_mocks(specs, catalog, bins, resampler='tsc', interlacing=2, compensate=True, los='z', group=32,
                  runner=None):
    """Multipoles of every mock, measured by the ranks of the process group in parallel
    (``ShardedMocks`` built and run once).  Returns the (nmocks, nells, nbins) float64 tensor on
    every rank and the indices of the mocks this rank measured."""
    sharded = ShardedMocks(specs, bins, resampler=resampler, interlacing=interlacing, compensate=compensate,
                           los=los, group=group, runner=runner)
    return sharded(catalog), sharded.mine

"""Mock sharding over ranks: the partition and the gather of per-mock multipoles, run as
two gloo processes on CPU (the same host logic the nccl path uses on GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from jaxpower_b200.sharding import mock_cost, partition_mocks, gather_multipoles, covariance, local_mocks


def test_partition_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = [mock_cost(n, m) for n, m in zip(np.exp(rng.uniform(np.log(1e5), np.log(4e6), 256)),
                                             rng.choice([128, 192, 256], 256))]
    for world in (1, 2, 3, 8):
        parts = partition_mocks(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # greedy bound
        assert parts == partition_mocks(costs, world)  # deterministic
    with pytest.raises(ValueError):
        partition_mocks(costs, 0)


def _fake(i, shape):
    return np.sin(np.arange(np.prod(shape)).reshape(shape) + 0.37 * i)


def _worker(rank, world, port, costs, shape, out):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        mine = local_mocks(costs)
        full = gather_multipoles({i: _fake(i, shape) for i in mine}, len(costs), shape)
        out[rank] = (mine, full.numpy(), covariance(full).numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_gather_two_ranks_gloo():
    costs = [mock_cost(n, 128) for n in np.linspace(1e5, 2e6, 21)]
    shape = (3, 7)
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_worker, args=(2, _free_port(), costs, shape, out), nprocs=2, join=True,
                           start_method='spawn')
        out = dict(out)
    expected = np.stack([_fake(i, shape) for i in range(len(costs))])
    owned = sorted(out[0][0] + out[1][0])
    assert owned == list(range(len(costs))) and not set(out[0][0]) & set(out[1][0])
    for rank in (0, 1):
        assert np.array_equal(out[rank][1], expected)
        cov = np.cov(expected.reshape(len(costs), -1).T)
        assert np.allclose(out[rank][2], cov, rtol=1e-12, atol=1e-14)


class _StubSpectra:
    """Stands in for BatchedSpectra on CPU: multipoles made from each catalog's positions."""

    def __init__(self, attrs, bin, counts, **kwargs):
        self.counts, self.shape = counts, (len(bin.ells), bin.nbins)

    def __call__(self, positions):
        out, start = [], 0
        for n in self.counts:
            x = positions[start:start + n].double()
            start += n
            out.append(torch.full(self.shape, float(x.sum()) + n, dtype=torch.float64))
        return torch.stack(out)


class _StubBins:
    ells, nbins, mattrs = (0, 2, 4), 5, None


def _catalog(i):
    return torch.as_tensor(np.random.default_rng(i).uniform(0., 1., (100 + 37 * i, 3)).astype('f4'))


def _runner_worker(rank, world, port, specs, out):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from jaxpower_b200.sharding import measure_mocks
        full, mine = measure_mocks(specs, _catalog, {128: _StubBins(), 192: _StubBins()}, group=3,
                                   runner=_StubSpectra)
        out[rank] = (mine, full.numpy())
    finally:
        dist.destroy_process_group()


def test_measure_mocks_two_ranks_gloo():
    """The sharded mock runner's host path (partition, per-mesh-size batches of at most `group`
    mocks, gather) with the batched spectra stubbed: every rank ends with every mock's row."""
    specs = [(128 if i % 3 else 192, 100 + 37 * i) for i in range(11)]
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_runner_worker, args=(2, _free_port(), specs, out), nprocs=2, join=True,
                           start_method='spawn')
        out = dict(out)
    expected = np.stack([np.full((3, 5), float(_catalog(i).double().sum()) + specs[i][1]) for i in range(11)])
    assert sorted(out[0][0] + out[1][0]) == list(range(11))
    for rank in (0, 1):
        assert np.array_equal(out[rank][1], expected)

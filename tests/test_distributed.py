"""Shots across ranks: the cost-balanced partition and the stacked-gradient
all-reduce, run as two gloo ranks on the CPU (the GPU runner replaced by a
deterministic fake that fills each shot's gradient from its index)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rockseis_b200.distributed import fwi_gradient_sharded, partition_shots


def test_partition_covers_every_shot_once_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.uniform(1.0, 5.0, 37)
    for world in (1, 2, 3, 8):
        parts = partition_shots(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() if p else 0.0 for p in parts]
        # longest-processing-time bound: max load <= mean + largest single shot
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
        assert parts == partition_shots(costs, world)          # deterministic
    assert partition_shots([], 2) == [[], []]
    assert partition_shots([1.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        partition_shots([1.0], 0)


class _Img:
    def __init__(self, shape):
        self.a = np.zeros(shape)

    def getImagedata(self):
        return self.a


class _Model:
    def __init__(self, nx, nz):
        self.nx, self.nz = nx, nz

    def getNx_pml(self): return self.nx
    def getNz_pml(self): return self.nz
    def getNy_pml(self): return 1


class _Src:
    nt = 100


class _Job:
    def __init__(self, i, shape):
        self.i = i
        self.model = _Model(40 + 7 * (i % 5), 30)
        self.source = _Src()
        self.vpgrad, self.rhograd = _Img(shape), _Img(shape)
        self.misfit = 0.0


def _fill(jobs):
    for j in jobs:
        j.vpgrad.a[:] = np.arange(j.vpgrad.a.size).reshape(j.vpgrad.a.shape) * (j.i + 1)
        j.rhograd.a[:] = -0.5 * (j.i + 1)
        j.misfit = 10.0 * j.i


def _jobs():
    return [_Job(i, (6, 5)) for i in range(11)]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ran = []

        def runner(local):
            ran.extend(j.i for j in local)
            _fill(local)
        vp, rho, mis = fwi_gradient_sharded(_jobs(), rank, world, runner=runner)
        np.savez(os.path.join(out, f"r{rank}.npz"), vp=vp, rho=rho, mis=mis, ran=np.array(ran, int))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_stack_the_gradient(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    ref = _jobs()
    _fill(ref)
    vp_ref = sum(j.vpgrad.a for j in ref)
    rho_ref = sum(j.rhograd.a for j in ref)
    mis_ref = sum(j.misfit for j in ref)
    ran = []
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(d["vp"], vp_ref) and np.array_equal(d["rho"], rho_ref)
        assert float(d["mis"]) == mis_ref
        ran.extend(d["ran"].tolist())
    assert sorted(ran) == list(range(len(ref)))                 # each shot on exactly one rank


def test_single_rank_needs_no_process_group():
    jobs = _jobs()
    vp, rho, mis = fwi_gradient_sharded(jobs, 0, 1, runner=_fill)
    assert np.array_equal(vp, sum(j.vpgrad.a for j in jobs)) and mis == sum(j.misfit for j in jobs)

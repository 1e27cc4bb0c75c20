"""The runGrad scheduler's host logic (rockseis_b200/inversion.py) on the CPU: the
gather queue over a Sort map of a recorded-data file, batches, a failed batch's
gathers handed out again one at a time, a gather that keeps failing left out and
reported, and two gloo ranks sharing the gathers with one all-reduce.  The GPU work
is replaced by a fake runner that adds a per-gather pattern to the global images and
fails on request (failures are made on the host)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rockseis_b200 import abi
from rockseis_b200.inversion import InversionAcoustic2D
from rockseis_b200.rockseis import Data2D, ModelAcoustic2D

NSHOT, NREC, NT = 5, 4, 16


def make_survey(path):
    sx = np.array([310.0, 50.0, 490.0, 170.0, 250.0])
    rows = [(s, g) for s in sx for g in (100.0, 200.0, 300.0, 400.0)]
    d = Data2D(len(rows), NT, 1e-3, 0.0)
    d.scoords[:] = [[s, 10.0] for s, _ in rows]
    d.gcoords[:] = [[g, 0.0] for _, g in rows]
    d.data[:] = np.arange(d.data.size, dtype=np.float32).reshape(d.data.shape)
    d.setFile(str(path))
    d.write()
    return sorted(sx)


class FakeJob:
    def __init__(self, shot):
        self.sx = float(shot.scoords[0, 0])
        self.misfit = 0.0


def make_inv(path):
    g = ModelAcoustic2D(61, 21, 5, 10.0, 10.0, 0.0, 0.0, 0)
    g.createModel()
    w = Data2D(1, NT, 1e-3, 0.0)
    inv = InversionAcoustic2D(g, w, str(path))
    inv.build = FakeJob
    return inv


def fake_runner(fail=lambda sx, n: False):
    calls = {}

    def run(jobs, vpgrad, rhograd):
        for j in jobs:
            calls[j.sx] = calls.get(j.sx, 0) + 1
            if fail(j.sx, calls[j.sx]):
                raise abi.RsgpuError(abi.ERR_CUDA, f"injected failure of shot {j.sx}")
        for j in jobs:                      # a batch either stacks completely or not at all
            vpgrad[:, int(j.sx) // 10] += 1.0
            rhograd[0, int(j.sx) // 10] += j.sx
            j.misfit = j.sx / 10.0
    run.calls = calls
    return run


def expected(sxs):
    vp = np.zeros((21, 61), np.float32)
    rho = np.zeros_like(vp)
    for s in sxs:
        vp[:, int(s) // 10] += 1.0
        rho[0, int(s) // 10] += s
    return vp, rho


def test_every_gather_once_in_batches(tmp_path):
    sxs = make_survey(tmp_path / "p.rss")
    inv = make_inv(tmp_path / "p.rss")
    run = fake_runner()
    r = inv.runGrad(batch=2, runner=run)
    vp, rho = expected(sxs)
    assert np.array_equal(r["vpgrad"], vp) and np.array_equal(r["rhograd"], rho)
    assert r["batches"] == 3 and r["failed"] == []
    assert sorted(r["misfits"]) == list(range(NSHOT))
    assert r["misfit"] == pytest.approx(sum(sxs) / 10.0)
    assert all(n == 1 for n in run.calls.values())
    assert all(inv.sort.getStatus(k) == abi.GATHER_FINISHED for k in range(NSHOT))


def test_failed_batch_is_retried_gather_by_gather(tmp_path):
    sxs = make_survey(tmp_path / "p.rss")
    inv = make_inv(tmp_path / "p.rss")
    run = fake_runner(lambda sx, n: sx == 250.0 and n == 1)      # fails on its first attempt only
    r = inv.runGrad(batch=3, runner=run)
    vp, rho = expected(sxs)
    assert np.array_equal(r["vpgrad"], vp) and np.array_equal(r["rhograd"], rho)
    assert r["failed"] == [] and run.calls[250.0] == 2


def test_gather_that_keeps_failing_is_reported_and_left_out(tmp_path):
    sxs = make_survey(tmp_path / "p.rss")
    inv = make_inv(tmp_path / "p.rss")
    run = fake_runner(lambda sx, n: sx == 490.0)
    r = inv.runGrad(batch=2, retries=2, runner=run)
    bad = sorted(sxs).index(490.0)                                 # gathers run in source-x order
    vp, rho = expected([s for s in sxs if s != 490.0])
    assert np.array_equal(r["vpgrad"], vp) and np.array_equal(r["rhograd"], rho)
    assert r["failed"] == [bad] and run.calls[490.0] == 3
    assert inv.sort.getStatus(bad) == abi.GATHER_FAILED and bad not in r["misfits"]


def _worker(rank, world, port, path, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        inv = make_inv(path)
        run = fake_runner()
        r = inv.runGrad(batch=2, rank=rank, world=world, runner=run)
        np.savez(os.path.join(out, f"r{rank}.npz"), vp=r["vpgrad"], rho=r["rhograd"], mis=r["misfit"],
                 ran=np.array(sorted(run.calls), float))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_share_the_gathers(tmp_path):
    path = tmp_path / "p.rss"
    sxs = make_survey(path)
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(path), str(tmp_path)), nprocs=world, join=True)
    vp, rho = expected(sxs)
    ran = []
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(d["vp"], vp) and np.array_equal(d["rho"], rho)
        assert float(d["mis"]) == pytest.approx(sum(sxs) / 10.0)
        ran.extend(d["ran"].tolist())
    assert sorted(ran) == sorted(sxs)                              # every gather on exactly one rank

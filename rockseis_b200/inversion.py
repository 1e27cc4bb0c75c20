"""InversionAcoustic2D::runGrad as a GPU batch scheduler.

The reference computes one FWI gradient iteration (lib/inversion.cpp:231-602) with
an MPI master handing shot gathers to workers one at a time; each worker builds the
shot's local model window (Model::getLocal), positions the wavelet at the shot,
resamples the recorded gather onto the wavelet's time axis (Interp, SINC), runs
FwiAcoustic2D and writes the window gradient to a file, and the master stacks the
files into the global gradient (Image2D::stackImage).

Here the gathers come from a Sort map of the recorded data file and its queue
(NOT_STARTED / RUNNING / FINISHED / FAILED): a batch of up to `batch` gathers runs
through one resident rsgpu_adjoint batch, the window gradients are stacked into the
global images on the device (rsgpu_adjoint_stack, shots in gather order), the
modelled and residual gathers go to their output files through the Sort map, and the
batch's gathers are marked FINISHED.  A batch that fails is marked FAILED and its
gathers come back from the queue one at a time, up to `retries` more attempts each;
a gather that keeps failing is reported, as the reference's queue leaves it FAILED.
With several ranks (one process per GPU) every rank takes a cost-balanced share of
the gathers and one all-reduce stacks the global gradients and misfits.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .rockseis import (SMAP, GMAP, AdjointBatch, Data2D, FwiAcoustic2D, Image2D, Interp, ModelAcoustic2D, Sort,
                       check_stability)


class InversionAcoustic2D:
    """One gradient of InversionAcoustic2D<T>::runGrad on the GPU.

    gmodel: the global ModelAcoustic2D; wavelet: a one-trace Data2D; precord: path of
    the recorded pressure data (.rss, Data2D).  Optional output paths receive the
    modelled and residual gathers (same layout as precord, on the wavelet's time axis)."""

    def __init__(self, gmodel: ModelAcoustic2D, wavelet: Data2D, precord: str, order=8, apertx=0.0, snapinc=1,
                 ncheck=0, precision=None, misfit_type=abi.MISFIT_DIFFERENCE, ckpt=abi.CKPT_NATIVE,
                 accum=abi.ACCUM_REFERENCE):
        self.gmodel, self.wavelet, self.precord = gmodel, wavelet, str(precord)
        self.order, self.apertx, self.snapinc, self.ncheck = order, float(apertx), snapinc, ncheck
        self.precision = gmodel.precision if precision is None else precision
        self.misfit_type, self.ckpt, self.accum = misfit_type, ckpt, accum
        self.pmodelled = self.presidual = None
        self.interp = Interp(abi.INTERP_SINC)

    def setPmodelledfile(self, path): self.pmodelled = str(path)
    def setPresidualfile(self, path): self.presidual = str(path)

    # ---------------------------------------------------------------- one shot
    def job(self, shot: Data2D):
        """The FwiAcoustic2D job of one gather, as a worker of runGrad builds it
        (lib/inversion.cpp:345-450): local model, wavelet at the shot, the gather
        resampled onto the wavelet's time axis, modelled/residual containers."""
        lmodel = self.gmodel.getLocal(shot, self.apertx, SMAP)
        w = self.wavelet
        src = Data2D(1, w.nt, w.dt, w.ot, self.precision)
        src.data[:] = w.data[:1]
        src.scoords[0], src.gcoords[0] = shot.scoords[0], shot.gcoords[0]
        src.setField(abi.PRESSURE)
        src.makeMap(lmodel, SMAP)
        ntr = shot.ntrace
        shoti = Data2D(ntr, w.nt, w.dt, 0.0, self.precision)
        self.interp.interp(shot, shoti)
        shoti.makeMap(lmodel, GMAP)
        f = FwiAcoustic2D(lmodel, src, shoti, self.order, self.snapinc, precision=self.precision)
        f.setNcheck(self.ncheck)
        f.setMisfit_type(self.misfit_type)
        f.setCheckpointPrecision(self.ckpt)
        f.setAccumulation(self.accum)
        f.setVpgrad(Image2D("vpgrad", lmodel, 1, 1, self.precision))
        f.setRhograd(Image2D("rhograd", lmodel, 1, 1, self.precision))
        f.setWavgrad(Data2D(1, w.nt, w.dt, 0.0, self.precision))
        for name in ("datamod", "datares"):
            d = Data2D(ntr, w.nt, w.dt, 0.0, self.precision)
            d.scoords[:], d.gcoords[:] = shot.scoords, shot.gcoords
            d.makeMap(lmodel, GMAP)
            (f.setDatamodP if name == "datamod" else f.setDataresP)(d)
        return f

    def window_origin(self, lmodel) -> tuple[int, int]:
        """Image2D::stackImage's placement (lib/image.cpp:397-398):
        (int)(ox_local/dx - ox_global/dx) in the element type, and the same in z."""
        t = self.gmodel.dtype
        g = self.gmodel
        ix = int(t(t(lmodel.ox) / t(lmodel.dx)) - t(t(g.ox) / t(g.dx)))
        iz = int(t(t(lmodel.oz) / t(lmodel.dz)) - t(t(g.oz) / t(g.dz)))
        return ix, iz

    # ---------------------------------------------------------------- a batch on the GPU
    def run_batch(self, jobs, vpgrad, rhograd):
        """Runs the jobs in one resident batch, stacks their window gradients into the
        global vpgrad / rhograd on the device and reads the per-shot outputs."""
        check_stability(jobs[0].model, jobs[0].source.dt, "InversionAcoustic2D")
        b = AdjointBatch(jobs)
        try:
            b.run()
            b.read()
            # last, so that a batch that fails anywhere leaves the global images untouched
            org = [self.window_origin(j.model) for j in jobs]
            b.stack(self.gmodel.nx, self.gmodel.nz, [o[0] for o in org], [o[1] for o in org], vpgrad, rhograd)
        finally:
            b.close()

    # ---------------------------------------------------------------- the gradient
    def runGrad(self, batch=16, retries=2, rank=0, world=1, group=None, runner=None):
        """The stacked gradient of every gather of the recorded data.

        Returns dict(vpgrad, rhograd [nz][nx] of the element type, misfit (sum),
        misfits {gather: value}, failed [gathers that kept failing], batches).
        `runner(jobs, vpgrad, rhograd)` replaces run_batch (tests inject failures)."""
        runner = runner or self.run_batch
        build = getattr(self, "build", None) or self.job
        sort = Sort(self.precision)
        sort.createShotmap(self.precord)
        ng = sort.getNensemb()
        mine = self._share(sort, ng, rank, world)
        for k in range(ng):
            if k not in mine:
                sort.setStatus(k, abi.GATHER_FINISHED)     # another rank's gather
        if self.pmodelled and rank == 0:
            sort.createEmptydataset(self.pmodelled, self.wavelet.nt, self.wavelet.dt, 0.0)
        if self.presidual and rank == 0:
            sort.createEmptydataset(self.presidual, self.wavelet.nt, self.wavelet.dt, 0.0)
        t = self.gmodel.dtype
        vpgrad = np.zeros((self.gmodel.nz, self.gmodel.nx), t)
        rhograd = np.zeros_like(vpgrad)
        misfits: dict[int, float] = {}
        attempts = {k: 0 for k in mine}
        failed: list[int] = []
        nbatch = 0
        isolate: set[int] = set()          # gathers of a failed batch: retried one per batch
        while True:
            todo = []
            while len(todo) < batch:
                k = self._next(sort)
                if k is None or (k in isolate and todo):
                    break
                todo.append(k)
                sort.setStatus(k, abi.GATHER_RUNNING)
                if k in isolate:
                    break
            if not todo:
                break
            shots = [sort.get2DGather(k) for k in todo]
            jobs = [build(s) for s in shots]
            try:
                runner(jobs, vpgrad, rhograd)
            except abi.RsgpuError:
                for k in todo:
                    attempts[k] += 1
                    if attempts[k] <= retries:
                        sort.setStatus(k, abi.GATHER_FAILED)      # handed out again
                    else:
                        failed.append(k)                          # stays taken: not handed out again
                isolate.update(todo)
                continue
            isolate.difference_update(todo)
            nbatch += 1
            for k, s, j in zip(todo, shots, jobs):
                misfits[k] = float(j.misfit)
                for path, name in ((self.pmodelled, "datamodP"), (self.presidual, "dataresP")):
                    if path:
                        d = getattr(j, name)
                        d.setFile(path)
                        sort.put2DGather(d, k)
                sort.setStatus(k, abi.GATHER_FINISHED)
        for k in failed:
            sort.setStatus(k, abi.GATHER_FAILED)
        self.sort = sort
        misfit = float(sum(misfits[k] for k in sorted(misfits)))
        if world > 1:
            from .distributed import _allreduce_sum
            n = vpgrad.size
            vec = np.concatenate([vpgrad.reshape(-1).astype(np.float64), rhograd.reshape(-1).astype(np.float64),
                                  [misfit]])
            vec = _allreduce_sum(vec, group)
            vpgrad = vec[:n].reshape(vpgrad.shape).astype(t)
            rhograd = vec[n:2 * n].reshape(rhograd.shape).astype(t)
            misfit = float(vec[2 * n])
        return dict(vpgrad=vpgrad, rhograd=rhograd, misfit=misfit, misfits=misfits, failed=sorted(failed),
                    batches=nbatch)

    @staticmethod
    def _next(sort):
        k = abi.lib.rsgpu_sort_next(sort.h)
        return None if k < 0 else int(k)

    def _share(self, sort, ng, rank, world):
        """This rank's gathers: longest-processing-time partition by trace count
        (the window sizes follow the gathers' spreads)."""
        if world <= 1:
            return set(range(ng))
        from .distributed import partition_shots
        costs = [abi.lib.rsgpu_sort_gather_size(sort.h, k) for k in range(ng)]
        return set(partition_shots(costs, world)[rank])

"""torch.autograd binding of the acoustic 2D modelling and its adjoint.

`modelled_data(vp, rho, problem)` is differentiable: its forward pass is the GPU
forward modelling (ModellingAcoustic2D::run, lib/modelling.cpp:197-291) of the
pressure traces at the problem's receivers, and its backward pass is the GPU
adjoint plus gradient correlation of FwiAcoustic2D::run_optimal
(lib/fwi.cpp:1159-1332, crossCorr :511-571).  The backward pass turns the
incoming trace gradient g into the observed data d - g, so that the DIFFERENCE
residual (lib/fwi.cpp:798-806, mod - obs) the gradient driver back-propagates is
g itself; the driver's vp and rho gradients are then the vector-Jacobian
products J^T g.  Both passes go through the C ABI (rsgpu_modelling,
rsgpu_fwi_gradient) with host buffers, so the tensors live on the host.

The reference's gradient is built from the forward operator and two-point
correlation differences, not the exact transpose of the discrete forward
operator, so J^T g agrees with finite differences of the modelling to the
discretisation level (a few per cent), not to rounding.
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from . import abi
from .rockseis import Data2D, FwiAcoustic2D, Image2D, ModellingAcoustic2D, _Model


class AcousticProblem2D:
    """One acoustic 2D shot: a model container (whose Vp/R the autograd inputs
    replace), a source Data2D with its map, a receiver Data2D with its map, the
    stencil order, the arithmetic and the Revolve snapshot count of the adjoint."""

    def __init__(self, model: _Model, source: Data2D, receivers: Data2D, order: int = 8, precision=None,
                 ncheck: int = 0):
        self.model, self.source, self.receivers = model, source, receivers
        self.order = int(order)
        self.precision = model.precision if precision is None else int(precision)
        self.ncheck = int(ncheck)
        self.dtype = abi.real_dtype(self.precision)

    def _model_with(self, vp: torch.Tensor, rho: torch.Tensor) -> _Model:
        m = copy.copy(self.model)
        m._padded = {}                      # staggered copies are rebuilt from the new vp and rho
        shape = self.model.Vp.shape
        m.Vp = np.ascontiguousarray(vp.detach().cpu().numpy().astype(self.dtype).reshape(shape))
        m.R = np.ascontiguousarray(rho.detach().cpu().numpy().astype(self.dtype).reshape(shape))
        return m

    def _traces(self, data=None) -> Data2D:
        r = self.receivers
        d = Data2D(r.ntrace, r.nt, r.dt, r.ot, self.precision)
        d.gcoords[:] = r.gcoords
        d.setField(r.getField())
        d.gmap, d.gshift = r.gmap.copy(), r.gshift.astype(self.dtype)
        if data is not None:
            d.data[:] = data
        return d

    def model_traces(self, vp: torch.Tensor, rho: torch.Tensor) -> np.ndarray:
        m = self._model_with(vp, rho)
        rec = self._traces()
        mod = ModellingAcoustic2D(m, self.source, self.order, 1, self.precision)
        mod.setRecP(rec)
        mod.run()
        return rec.data.copy()

    def vjp(self, vp: torch.Tensor, rho: torch.Tensor, traces: np.ndarray, g: np.ndarray):
        """(J^T g) for vp and rho: the gradient driver run on observed data traces - g."""
        m = self._model_with(vp, rho)
        obs = self._traces(traces.astype(self.dtype) - g.astype(self.dtype))
        f = FwiAcoustic2D(m, self.source, obs, self.order, 1, precision=self.precision)
        f.setNcheck(self.ncheck)
        if self.precision == abi.F64:
            f.setAccumulation(abi.ACCUM_F64)
        f.setVpgrad(Image2D("vpgrad", m, 1, 1, self.precision))
        f.setRhograd(Image2D("rhograd", m, 1, 1, self.precision))
        f.run_optimal()
        return f.vpgrad.getImagedata()[0, 0].copy(), f.rhograd.getImagedata()[0, 0].copy()


class _ModelledData(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vp, rho, problem):
        traces = problem.model_traces(vp, rho)
        ctx.problem, ctx.traces = problem, traces
        ctx.save_for_backward(vp, rho)
        return torch.from_numpy(traces).to(device=vp.device, dtype=vp.dtype)

    @staticmethod
    def backward(ctx, g):
        vp, rho = ctx.saved_tensors
        gv, gr = ctx.problem.vjp(vp, rho, ctx.traces, g.detach().cpu().numpy())
        return (torch.from_numpy(gv).to(device=vp.device, dtype=vp.dtype).reshape(vp.shape),
                torch.from_numpy(gr).to(device=rho.device, dtype=rho.dtype).reshape(rho.shape), None)


def modelled_data(vp: torch.Tensor, rho: torch.Tensor, problem: AcousticProblem2D) -> torch.Tensor:
    """Pressure traces [ntrace, nt] modelled in (vp, rho) [nz, nx]; differentiable in vp and rho."""
    return _ModelledData.apply(vp, rho, problem)

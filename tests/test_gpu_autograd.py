"""The adjoint through torch.autograd: finite-difference checks of the GPU
gradient.  The reference's own check of its gradient is the forward-difference
program src/hello_fdgrad.cpp:230-252 (one perturbed parameter at a time).

The differentiable op is rockseis_b200.autograd.modelled_data (forward modelling
forward, FwiAcoustic2D adjoint + correlation backward), run in FP64 so that the
central differences carry no rounding noise.  The reference gradient is not the
exact transpose of the discrete forward operator (it correlates with two-point
time differences), so the bars are the discretisation level measured on these
cases, not rounding.
"""
import numpy as np
import pytest
import torch

from rockseis_b200 import abi
from rockseis_b200.autograd import AcousticProblem2D, modelled_data
from tests.cases import Case2D

pytestmark = pytest.mark.gpu

FD_TOL = 0.08      # relative disagreement of a directional derivative with central differences


def _case(dt=1e-3, nt=500):
    c = Case2D(abi.ACOUSTIC2D, nx=81, nz=61, nt=nt, dt=dt, precision=abi.F64, scoord=(400.3, 23.7), nrec=30)
    prob = AcousticProblem2D(c.model, c.src, c.rec, order=8, precision=abi.F64, ncheck=12)
    vp = torch.tensor(c.vp, dtype=torch.float64)
    rho = torch.tensor(c.rho, dtype=torch.float64)
    return c, prob, vp, rho


def _blob(shape, cz, cx, w):
    z, x = np.mgrid[0:shape[0], 0:shape[1]]
    return torch.tensor(np.exp(-((z - cz) ** 2 + (x - cx) ** 2) / (2.0 * w * w)), dtype=torch.float64)


def _central(f, x0, dm, eps):
    return (f(x0 + eps * dm) - f(x0 - eps * dm)) / (2.0 * eps)


def _misfit_errors(dt, nt):
    c, prob, vp0, rho0 = _case(dt, nt)
    vt = vp0.clone()
    vt[25:33, 30:42] *= 0.95
    with torch.no_grad():
        obs = modelled_data(vt, rho0, prob)

    def loss(vp, rho):
        return 0.5 * ((modelled_data(vp, rho, prob) - obs) ** 2).sum()

    vp = vp0.clone().requires_grad_(True)
    rho = rho0.clone().requires_grad_(True)
    loss(vp, rho).backward()
    errs = {}
    for name, grad, x0, make in (("vp", vp.grad, vp0, lambda x: loss(x, rho0)),
                                 ("rho", rho.grad, rho0, lambda x: loss(vp0, x))):
        dm = _blob(x0.shape, 29, 36, 4.0)
        with torch.no_grad():
            fd = float(_central(make, x0, dm, 5.0))
        ad = float((grad * dm).sum())
        assert fd != 0.0
        errs[name] = abs(ad - fd) / abs(fd)
        print(f"dt {dt}: {name} autograd {ad:.6e}  central difference {fd:.6e}  relative {errs[name]:.3e}")
    return errs


def test_misfit_gradient_against_central_differences(require_gpu):
    # The reference correlates the forward wavefield with a two-point time
    # difference of the adjoint one, which is first-order accurate in dt: the
    # disagreement is a few per cent at dt = 1 ms (15 Hz source) and shrinks in
    # proportion when dt is halved, the signature of that discretisation and not
    # of an indexing or sign error (which would not depend on dt).
    e1 = _misfit_errors(1e-3, 500)
    e2 = _misfit_errors(5e-4, 1000)
    for k in ("vp", "rho"):
        assert e1[k] <= FD_TOL, k
        assert e2[k] <= 0.65 * e1[k] + 2e-3, k


def test_vector_jacobian_product_dot_test(require_gpu):
    # <J dm, g> (central differences of the modelling) against <dm, J^T g> (backward)
    c, prob, vp0, rho0 = _case()
    rng = np.random.default_rng(5)
    with torch.no_grad():
        d0 = modelled_data(vp0, rho0, prob)
    g = torch.tensor(rng.standard_normal(d0.shape), dtype=torch.float64) * float(d0.abs().max())
    dm = _blob(vp0.shape, 30, 40, 5.0)
    vp = vp0.clone().requires_grad_(True)
    d = modelled_data(vp, rho0, prob)
    assert torch.equal(d.detach(), d0)
    d.backward(g)
    with torch.no_grad():
        jdm = _central(lambda x: modelled_data(x, rho0, prob), vp0, dm, 5.0)
    lhs = float((jdm * g).sum())
    rhs = float((dm * vp.grad).sum())
    err = abs(lhs - rhs) / abs(lhs)
    print(f"<J dm, g> {lhs:.6e}  <dm, J^T g> {rhs:.6e}  relative {err:.3e}")
    assert err <= FD_TOL

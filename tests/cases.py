"""Small seeded problems shared by the parity tests (sizes the CPU oracle runs in seconds)."""
from __future__ import annotations

import numpy as np

from oracle import api
from rockseis_b200 import abi, synth
from rockseis_b200.rockseis import Data2D, ModelAcoustic2D, ModelElastic2D


class Case2D:
    def __init__(self, physics, nx=81, nz=61, lpml=12, dx=10.0, dt=1e-3, nt=300, order=8, fs=0, seed=1,
                 sfield=abi.PRESSURE, rfield=abi.PRESSURE, scoord=(400.3, 23.7), nrec=30, rx0=13.1, rdx=20.0,
                 rz=5.2, f0=15.0, precision=abi.F32_EXACT, ox=0.0, oz=0.0):
        self.physics, self.nt, self.dt, self.order, self.precision = physics, nt, dt, order, precision
        dtype = abi.real_dtype(precision)
        vp = synth.layered_vp(nx, nz, dx, 1500, 3500, 4, 0.05, 100, seed)
        rho = synth.gardner(vp)
        vs = (vp / 1.8).astype(np.float32)
        self.vp, self.vs, self.rho = vp, vs, rho
        if physics == abi.ACOUSTIC2D:
            m = ModelAcoustic2D(nx, nz, lpml, dx, dx, ox, oz, fs, precision)
        else:
            m = ModelElastic2D(nx, nz, lpml, dx, dx, ox, oz, fs, precision)
        m.createModel()
        m.Vp[:] = vp
        m.R[:] = rho
        if physics == abi.ELASTIC2D:
            m.Vs[:] = vs
        self.model = m
        sc = np.atleast_2d(np.asarray(scoord, np.float64))
        self.scoords = sc
        self.gcoords = synth.surface_line(nrec, rx0, rdx, rz)
        src = Data2D(len(sc), nt, dt, 0.0, precision)
        src.scoords[:] = sc
        src.data[:] = synth.ricker(nt, dt, f0, dtype)[None, :]
        src.setField(sfield)
        src.makeMap(m, 0)
        rec = Data2D(len(self.gcoords), nt, dt, 0.0, precision)
        rec.gcoords[:] = self.gcoords
        rec.setField(rfield)
        rec.makeMap(m, 1)
        self.src, self.rec = src, rec
        self.pb = api.Problem2D(nx, nz, dx, dx, lpml, order, fs, dt, nt, vp, rho, vs, ox, oz)
        tab = np.zeros(12 * lpml, dtype)
        abi.check(abi.lib.rsgpu_pml_tables(lpml, dt, precision, tab.ctypes.data))
        self.tab = tab

    def oracle_traces(self, nsteps=None, want_state=False):
        s, r = self.src, self.rec
        if self.physics == abi.ACOUSTIC2D:
            return api.orc_modelling_a2d(self.pb, self.model.padded(), self.tab, s.smap, s.sshift, s.data, s.field,
                                         r.gmap, r.gshift, r.field, nsteps, want_state)
        return api.orc_modelling_e2d(self.pb, self.model.padded(), self.tab, s.smap, s.sshift, s.data, s.field,
                                     r.gmap, r.gshift, r.field, None, nsteps, want_state)


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fwi_case(nx=81, nz=61, nt=300, seed=1, precision=abi.F32_EXACT, scoord=(400.3, 23.7), dlens=0.92, **kw):
    """A Case2D in the starting model plus 'observed' data modelled (by the oracle)
    in a model with a slow lens, so residuals and gradients are nonzero."""
    from rockseis_b200.rockseis import ModelAcoustic2D
    c = Case2D(abi.ACOUSTIC2D, nx=nx, nz=nz, nt=nt, seed=seed, precision=precision, scoord=scoord, **kw)
    vt = c.vp.copy()
    vt[nz // 3: nz // 3 + 8, nx // 3: nx // 3 + 12] *= dlens
    # the observed data are always modelled in float, so cases of every precision share them
    mt = ModelAcoustic2D(nx, nz, c.model.lpml, c.model.dx, c.model.dz, c.model.ox, c.model.oz, c.model.fs)
    mt.createModel()
    mt.Vp[:], mt.R[:] = vt, c.rho
    pbt = api.Problem2D(nx, nz, c.model.dx, c.model.dz, c.model.lpml, c.order, c.model.fs, c.dt, nt, vt, c.rho)
    dtype = abi.real_dtype(precision)
    tab32 = np.zeros(12 * c.model.lpml, np.float32)
    abi.check(abi.lib.rsgpu_pml_tables(c.model.lpml, c.dt, abi.F32_EXACT, tab32.ctypes.data))
    obs = api.orc_modelling_a2d(pbt, mt.padded(), tab32, c.src.smap, c.src.sshift,
                                synth.ricker(nt, c.dt, 15.0)[None, :], abi.PRESSURE, c.rec.gmap, c.rec.gshift,
                                abi.PRESSURE)
    c.obs = obs.astype(dtype)
    return c


def oracle_fwi(c, misfit=0):
    return api.orc_fwi_a2d(c.pb, [a.astype(np.float32) for a in c.model.padded()], c.tab, c.src.smap, c.src.sshift,
                           c.src.data, c.rec.gmap, c.rec.gshift, c.obs, misfit)


def oracle_rtm(c, data, nhx=1, nhz=1):
    return api.orc_rtm_a2d(c.pb, [a.astype(np.float32) for a in c.model.padded()], c.tab, c.src.smap, c.src.sshift,
                           c.src.data, c.rec.gmap, c.rec.gshift, data, nhx, nhz)


class ElasticFwiCase:
    """Elastic 2D FWI problem: starting model, source, P/Ux/Uz receiver sets and
    observed data modelled by the oracle in a model with a slow lens."""

    def __init__(self, nx=61, nz=47, lpml=10, dx=10.0, dt=1e-3, nt=250, fs=0, seed=7, sfield=abi.PRESSURE,
                 scoord=(301.7, 28.3), nrec=20, rx0=13.0, rdx=30.0, rz=14.7, precision=abi.F32_EXACT):
        from rockseis_b200.rockseis import ModelElastic2D
        self.nt, self.dt, self.order, self.precision, self.sfield = nt, dt, 8, precision, sfield
        t = abi.real_dtype(precision)
        vp = synth.layered_vp(nx, nz, dx, 1800, 3200, 3, 0.05, 60, seed)
        vs = (vp / 1.8).astype(np.float32)
        rho = synth.gardner(vp)
        vt = vp.copy()
        vt[nz // 3: nz // 3 + 10, nx // 3: nx // 3 + 15] *= 0.93
        self.vp, self.vs, self.rho = vp, vs, rho
        m = ModelElastic2D(nx, nz, lpml, dx, dx, 0.0, 0.0, fs, precision)
        m.createModel()
        m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
        self.model = m
        src = Data2D(1, nt, dt, 0.0, precision)
        src.scoords[:] = [scoord]
        src.data[:] = synth.ricker(nt, dt, 20.0, t)[None, :]
        src.setField(sfield)
        src.makeMap(m, 0)
        self.src = src
        gc = synth.surface_line(nrec, rx0, rdx, rz)
        self.recs = []
        for f in (abi.PRESSURE, abi.VX, abi.VZ):
            r = Data2D(nrec, nt, dt, 0.0, precision)
            r.gcoords[:] = gc
            r.setField(f)
            r.makeMap(m, 1)
            self.recs.append(r)
        self.tab = np.zeros(12 * lpml, t)
        abi.check(abi.lib.rsgpu_pml_tables(lpml, dt, precision, self.tab.ctypes.data))
        self.pb = api.Problem2D(nx, nz, dx, dx, lpml, 8, fs, dt, nt, vp, rho, vs)
        # observed data: float oracle modelling in the true model
        mt = ModelElastic2D(nx, nz, lpml, dx, dx, 0.0, 0.0, fs)
        mt.createModel()
        mt.Vp[:], mt.Vs[:], mt.R[:] = vt, vs, rho
        pbt = api.Problem2D(nx, nz, dx, dx, lpml, 8, fs, dt, nt, vt, rho, vs)
        tab32 = np.zeros(12 * lpml, np.float32)
        abi.check(abi.lib.rsgpu_pml_tables(lpml, dt, abi.F32_EXACT, tab32.ctypes.data))
        wav32 = synth.ricker(nt, dt, 20.0)[None, :]
        self.obs = [api.orc_modelling_e2d(pbt, mt.padded(), tab32, src.smap, src.sshift.astype(np.float32), wav32,
                                          sfield, r.gmap, r.gshift.astype(np.float32), r.field).astype(t)
                    for r in self.recs]

    def oracle(self, misfit=0):
        return api.orc_fwi_e2d(self.pb, [a.astype(np.float32) for a in self.model.padded()],
                               self.tab.astype(np.float32), self.src.smap, self.src.sshift, self.src.data, self.sfield,
                               [r.gmap for r in self.recs], [r.gshift for r in self.recs],
                               [o.astype(np.float32) for o in self.obs], misfit)

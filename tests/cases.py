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

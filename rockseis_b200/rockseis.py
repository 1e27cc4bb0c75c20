"""Python mirror of the RockSeis driver classes on the hot path.

Same class and method names, argument meanings and return codes as the
reference's C++ API (include/model.h, data.h, modelling.h, fwi.h, rtm.h of the
RockSeis tree); every compute call goes through the C ABI of librsgpu
(include/rsgpu.h) to the sm_100a kernels.  Differences in error behaviour: the
reference's rs_error prints and calls exit(1); here the same conditions raise
rockseis_b200.abi.RsgpuError carrying the library's status code and message.

Precision: ``precision`` selects the propagator arithmetic (abi.F32_EXACT,
F32_FAST, F64); arrays are float32 for the F32 modes and float64 for F64.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi
from .abi import check, ptr

MOD_OK, MOD_ERR = 1, 0
FWI_OK, FWI_ERR = 1, 0
RTM_OK, RTM_ERR = 1, 0
SMAP, GMAP = 0, 1


def _f(dtype, x):
    """Round a Python float to the model's element type, as a T member would hold it."""
    return float(np.asarray(x, dtype=dtype))


class _Model:
    dim = 2
    physics = abi.ACOUSTIC2D
    names: tuple[str, ...] = ()

    def __init__(self, nx, ny, nz, lpml, dx, dy, dz, ox, oy, oz, fs, precision=abi.F32_EXACT):
        self.precision = precision
        self.dtype = abi.real_dtype(precision)
        self.nx, self.ny, self.nz, self.lpml = int(nx), int(ny), int(nz), int(lpml)
        t = self.dtype
        self.dx, self.dy, self.dz = _f(t, dx), _f(t, dy), _f(t, dz)
        self.ox, self.oy, self.oz = _f(t, ox), _f(t, oy), _f(t, oz)
        self.fs = bool(fs)
        self.realized = False
        self._padded: dict[str, np.ndarray] = {}

    # getters mirroring Model<T>
    def getNx(self): return self.nx
    def getNy(self): return self.ny
    def getNz(self): return self.nz
    def getLpml(self): return self.lpml
    def getDx(self): return self.dx
    def getDz(self): return self.dz
    def getFs(self): return self.fs
    def getNx_pml(self): return self.nx + 2 * self.lpml
    def getNz_pml(self): return self.nz + 2 * self.lpml
    def getNy_pml(self): return self.ny + 2 * self.lpml if self.dim == 3 else 1

    def _shape(self):
        return (self.nz, self.ny, self.nx) if self.dim == 3 else (self.nz, self.nx)

    def _pshape(self):
        if self.dim == 3:
            return (self.getNz_pml(), self.getNy_pml(), self.getNx_pml())
        return (self.getNz_pml(), self.getNx_pml())

    def geom(self):
        """(n, o, d) of the regular grid along the map axes, as Model::getGeom holds them."""
        if self.dim == 3:
            return (np.array([self.nx, self.ny, self.nz], np.int32), np.array([self.ox, self.oy, self.oz]),
                    np.array([self.dx, self.dy, self.dz]))
        return (np.array([self.nx, self.nz], np.int32), np.array([self.ox, self.oz]), np.array([self.dx, self.dz]))

    def staggerModels(self):
        """Pad, form moduli, stagger and invert density (Model*::staggerModels)."""
        if not self.realized:
            raise abi.RsgpuError(abi.ERR_STATE, f"{type(self).__name__}::staggerModels: Model is not allocated.")
        outs = [np.zeros(self._pshape(), self.dtype) for _ in self.names]
        arr = (C.c_void_p * 8)(*([o.ctypes.data for o in outs] + [None] * (8 - len(outs))))
        vs = getattr(self, "Vs", None)
        check(abi.lib.rsgpu_stagger_model(self.physics, self.nx, self.ny, self.nz, self.lpml, int(self.fs),
                                          self.precision, ptr(self.Vp), ptr(vs), ptr(self.R), arr))
        self._padded = dict(zip(self.names, outs))

    def padded(self):
        if not self._padded:
            self.staggerModels()
        return [self._padded[n] for n in self.names]

    def getVpmax(self):
        return float(self.Vp.max())

    # ---- aperture windows (Model::getLocalsize2d/3d, lib/model.cpp:272-470)
    def _local_axis(self, s, g, aperture, use_src, d, o):
        """Start and size of the local window along one axis.  The reference rounds
        with rintf, i.e. in float after double arithmetic; so does this."""
        f32 = np.float32
        s = np.asarray(s, np.float64)
        g = np.asarray(g, np.float64)
        dd, oo, ap = float(f32(d)), float(f32(o)), float(f32(aperture))
        if ap >= 0:
            v = s if use_src else g
            mn, mx = float(v.min()), float(v.max())
            off = float(np.abs(g - s).max())
            if ap > 0:
                size = int(f32(np.rint(f32((mx - mn + ap) / dd))) + f32(1))
                if size % 2 == 0:
                    size += 1
            else:
                size = int(f32(2) * f32(np.rint(f32(off / dd))) + f32(1))
            start = int(f32(np.rint(f32((mn - oo) / dd))) - f32((size - 1) // 2))
        else:
            mn, mx = float(min(s.min(), g.min())), float(max(s.max(), g.max()))
            size = int(f32(np.rint(f32((mx - mn + 2 * abs(ap)) / dd))) + f32(2))
            start = int(f32(np.rint(f32((mn - oo) / dd))) - f32(np.rint(f32(abs(ap / dd))))) - 1
        return start, size

    def getLocalsize2d(self, data, aperture, map_):
        """(start, size) of the x window (Model::getLocalsize2d, lib/model.cpp:272-343)."""
        return self._local_axis(data.scoords[:, 0], data.gcoords[:, 0], aperture, map_ == SMAP, self.dx, self.ox)

    def getLocalsize3d(self, data, aperture_x, aperture_y, map_):
        """((start_x, size_x), (start_y, size_y)) (Model::getLocalsize3d, lib/model.cpp:345-470)."""
        return (self._local_axis(data.scoords[:, 0], data.gcoords[:, 0], aperture_x, map_ == SMAP, self.dx, self.ox),
                self._local_axis(data.scoords[:, 1], data.gcoords[:, 1], aperture_y, map_ == SMAP, self.dy, self.oy))

    def _origin(self, o, start, d):
        """Origin of a local window, o + start*d evaluated in T as the reference does."""
        t = self.dtype
        return float(t(t(o) + t(t(start) * t(d))))

    def _window(self, arr, sx, nxw, sy=0, nyw=1):
        """Edge-clamped copy of a window (the copy loops of Model*::getLocal)."""
        ix = np.clip(np.arange(sx, sx + nxw), 0, self.nx - 1)
        if self.dim == 3:
            iy = np.clip(np.arange(sy, sy + nyw), 0, self.ny - 1)
            return np.ascontiguousarray(arr[:, iy][:, :, ix])
        return np.ascontiguousarray(arr[:, ix])


class ModelAcoustic2D(_Model):
    physics = abi.ACOUSTIC2D
    names = ("Rx", "Rz", "L")

    def __init__(self, nx, nz, lpml, dx, dz, ox, oz, fs, precision=abi.F32_EXACT):
        super().__init__(nx, 1, nz, lpml, dx, 1.0, dz, ox, 0.0, oz, fs, precision)

    def createModel(self):
        self.Vp = np.zeros(self._shape(), self.dtype)
        self.R = np.zeros(self._shape(), self.dtype)
        self.realized = True

    def getVp(self): return self.Vp
    def getR(self): return self.R
    def getRx(self): return self.padded()[0]
    def getRz(self): return self.padded()[1]
    def getL(self): return self.padded()[2]

    def getLocal(self, data, aperture, map_):
        """Local model around a shot's sources or receivers (ModelAcoustic2D::getLocal,
        lib/model.cpp:1443-1509): window from getLocalsize2d, edge-clamped copy."""
        sx, nxw = self.getLocalsize2d(data, aperture, map_)
        m = ModelAcoustic2D(nxw, self.nz, self.lpml, self.dx, self.dz, self._origin(self.ox, sx, self.dx), self.oz,
                            self.fs, self.precision)
        m.createModel()
        m.Vp[:], m.R[:] = self._window(self.Vp, sx, nxw), self._window(self.R, sx, nxw)
        return m


class ModelElastic2D(_Model):
    physics = abi.ELASTIC2D
    names = ("Rx", "Rz", "L", "L2M", "M")

    def __init__(self, nx, nz, lpml, dx, dz, ox, oz, fs, precision=abi.F32_EXACT):
        super().__init__(nx, 1, nz, lpml, dx, 1.0, dz, ox, 1.0, oz, fs, precision)

    def createModel(self):
        self.Vp = np.zeros(self._shape(), self.dtype)
        self.Vs = np.zeros(self._shape(), self.dtype)
        self.R = np.zeros(self._shape(), self.dtype)
        self.realized = True

    def getVp(self): return self.Vp
    def getVs(self): return self.Vs
    def getR(self): return self.R
    def getRx(self): return self.padded()[0]
    def getRz(self): return self.padded()[1]
    def getL(self): return self.padded()[2]
    def getL2M(self): return self.padded()[3]
    def getM(self): return self.padded()[4]

    def getLocal(self, data, aperture, map_):
        """ModelElastic2D::getLocal (lib/model.cpp:2840-2910)."""
        sx, nxw = self.getLocalsize2d(data, aperture, map_)
        m = ModelElastic2D(nxw, self.nz, self.lpml, self.dx, self.dz, self._origin(self.ox, sx, self.dx), self.oz,
                           self.fs, self.precision)
        m.createModel()
        m.Vp[:], m.Vs[:], m.R[:] = (self._window(a, sx, nxw) for a in (self.Vp, self.Vs, self.R))
        return m


class ModelAcoustic3D(_Model):
    """ModelAcoustic3D<T> (include/model.h): arrays [nz][ny][nx]."""
    dim = 3
    physics = abi.ACOUSTIC3D
    names = ("Rx", "Ry", "Rz", "L")

    def __init__(self, nx, ny, nz, lpml, dx, dy, dz, ox, oy, oz, fs, precision=abi.F32_EXACT):
        super().__init__(nx, ny, nz, lpml, dx, dy, dz, ox, oy, oz, fs, precision)

    def createModel(self):
        self.Vp = np.zeros(self._shape(), self.dtype)
        self.R = np.zeros(self._shape(), self.dtype)
        self.realized = True

    def getVp(self): return self.Vp
    def getR(self): return self.R
    def getDy(self): return self.dy
    def getRx(self): return self.padded()[0]
    def getRy(self): return self.padded()[1]
    def getRz(self): return self.padded()[2]
    def getL(self): return self.padded()[3]

    def getLocal(self, data, aperture_x, aperture_y, map_):
        """ModelAcoustic3D::getLocal (lib/model.cpp:2369-2450)."""
        (sx, nxw), (sy, nyw) = self.getLocalsize3d(data, aperture_x, aperture_y, map_)
        m = ModelAcoustic3D(nxw, nyw, self.nz, self.lpml, self.dx, self.dy, self.dz,
                            self._origin(self.ox, sx, self.dx), self._origin(self.oy, sy, self.dy), self.oz,
                            self.fs, self.precision)
        m.createModel()
        m.Vp[:], m.R[:] = self._window(self.Vp, sx, nxw, sy, nyw), self._window(self.R, sx, nxw, sy, nyw)
        return m


class ModelElastic3D(_Model):
    """ModelElastic3D<T> (include/model.h): arrays [nz][ny][nx]; staggered
    parameters Rx, Ry, Rz, L, L2M, M_yz, M_xz, M_xy (lib/model.cpp:3371-3475)."""
    dim = 3
    physics = abi.ELASTIC3D
    names = ("Rx", "Ry", "Rz", "L", "L2M", "M_yz", "M_xz", "M_xy")

    def __init__(self, nx, ny, nz, lpml, dx, dy, dz, ox, oy, oz, fs, precision=abi.F32_EXACT):
        super().__init__(nx, ny, nz, lpml, dx, dy, dz, ox, oy, oz, fs, precision)

    def createModel(self):
        self.Vp = np.zeros(self._shape(), self.dtype)
        self.Vs = np.zeros(self._shape(), self.dtype)
        self.R = np.zeros(self._shape(), self.dtype)
        self.realized = True

    def getVp(self): return self.Vp
    def getVs(self): return self.Vs
    def getR(self): return self.R
    def getDy(self): return self.dy
    def getRx(self): return self.padded()[0]
    def getRy(self): return self.padded()[1]
    def getRz(self): return self.padded()[2]
    def getL(self): return self.padded()[3]
    def getL2M(self): return self.padded()[4]
    def getM_yz(self): return self.padded()[5]
    def getM_xz(self): return self.padded()[6]
    def getM_xy(self): return self.padded()[7]


class Data2D:
    """Trace container (Data2D<T>): data[itr, it] == reference data[it + itr*nt]."""
    dim = 2

    def __init__(self, ntrace, nt, dt, ot, precision=abi.F32_EXACT):
        self.precision = precision
        self.dtype = abi.real_dtype(precision)
        self.ntrace, self.nt = int(ntrace), int(nt)
        self.dt, self.ot = _f(self.dtype, dt), _f(self.dtype, ot)
        self.data = np.zeros((self.ntrace, self.nt), self.dtype)
        self.scoords = np.zeros((self.ntrace, self.dim), self.dtype)   # (x, z)
        self.gcoords = np.zeros((self.ntrace, self.dim), self.dtype)
        self.smap = np.full((self.ntrace, self.dim), -1, np.int32)
        self.gmap = np.full((self.ntrace, self.dim), -1, np.int32)
        self.sshift = np.zeros((self.ntrace, self.dim), self.dtype)
        self.gshift = np.zeros((self.ntrace, self.dim), self.dtype)
        self.field = abi.PRESSURE
        self.reciprocity = False

    def getNtrace(self): return self.ntrace
    def getNt(self): return self.nt
    def getDt(self): return self.dt
    def getOt(self): return self.ot
    def getData(self): return self.data
    def getField(self): return self.field
    def setField(self, f): self.field = int(f)
    def setReciprocity(self, v): self.reciprocity = bool(v)
    def setFile(self, path): self.file = str(path)
    def getFile(self): return getattr(self, "file", "")

    def write(self):
        """Data2D::write / Data3D::write (lib/data.cpp:580-635, 1265-1320): the traces
        and their source/receiver coordinates to the .rss file set with setFile."""
        check(abi.lib.rsgpu_rss_write_traces(self.getFile().encode(), self.precision, self.dim, self.nt,
                                             float(self.dt), float(self.ot), self.ntrace,
                                             ptr(np.ascontiguousarray(self.scoords)),
                                             ptr(np.ascontiguousarray(self.gcoords)),
                                             ptr(np.ascontiguousarray(self.data))))
        return 1

    def read(self):
        """Data2D::read (lib/data.cpp:463-506): traces and coordinates from the file;
        the file's sample count must equal nt."""
        h = rss_header(self.getFile())
        if h.n[0] != self.nt:
            raise abi.RsgpuError(abi.ERR_ARG, f"Data2D::read: Nt in {self.getFile()} is different from nt")
        n = min(self.ntrace, int(h.n[1]))
        check(abi.lib.rsgpu_rss_read_traces(self.getFile().encode(), self.precision, 0, n, ptr(self.scoords),
                                            ptr(self.gcoords), ptr(self.data)))
        return 1

    @classmethod
    def fromFile(cls, path, precision=abi.F32_EXACT):
        """A container sized and filled from an .rss trace file."""
        h = rss_header(path)
        d = cls(int(h.n[1]), int(h.n[0]), h.d[0], h.o[0], precision)
        d.setFile(path)
        d.read()
        return d

    def makeMap(self, model: _Model, which=None):
        """Geometry2D::makeMap: coordinates -> (cell, fractional shift); -1 if off the grid."""
        whichs = (SMAP, GMAP) if which is None else (which,)
        n, o, d = model.geom()
        # staggered trace positions: -0.5 cell along the traced velocity component
        gs = np.zeros(self.dim)
        comp = {abi.VX: 0, abi.VY: 1, abi.VZ: self.dim - 1}.get(self.field)
        if comp is not None and not (self.dim == 2 and self.field == abi.VY):
            gs[comp] = -0.5
        for w in whichs:
            coords = np.ascontiguousarray((self.scoords if w == SMAP else self.gcoords).astype(np.float64))
            mp = np.full((self.ntrace, self.dim), -1, np.int32)
            sh = np.zeros((self.ntrace, self.dim), self.dtype)
            check(abi.lib.rsgpu_make_map(self.dim, self.precision, self.ntrace,
                                         coords.ctypes.data_as(C.POINTER(C.c_double)),
                                         n.ctypes.data_as(C.POINTER(C.c_int)),
                                         o.astype(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                         d.astype(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                         gs.ctypes.data_as(C.POINTER(C.c_double)),
                                         mp.ctypes.data_as(C.POINTER(C.c_int)), ptr(sh)))
            if w == SMAP:
                self.smap, self.sshift = mp, sh
            else:
                self.gmap, self.gshift = mp, sh


class Data3D(Data2D):
    """Trace container (Data3D<T>): coordinates and maps (x, y, z)."""
    dim = 3


def rss_header(path) -> abi.RssHeader:
    """File::readHeader (lib/file.cpp:221-250)."""
    h = abi.RssHeader()
    check(abi.lib.rsgpu_rss_read_header(str(path).encode(), C.byref(h)))
    return h


class Sort:
    """Sort<T> (include/sort.h, lib/sort.cpp): gathers of an .rss trace file by source,
    receiver or CMP position, and the gather queue (NOT_STARTED / RUNNING / FINISHED /
    FAILED) the MPI drivers hand out."""

    def __init__(self, precision=abi.F32_EXACT):
        self.precision = precision
        self.dtype = abi.real_dtype(precision)
        self.reciprocity = False
        self.h = C.c_void_p()
        self.dim = 2

    def __del__(self):
        if getattr(self, "h", None):
            abi.lib.rsgpu_sort_destroy(self.h)
            self.h = C.c_void_p()

    def setReciprocity(self, v): self.reciprocity = bool(v)
    def getReciprocity(self): return self.reciprocity

    def _create(self, path, key, dx=0.0, dy=0.0, order=0):
        if self.h:
            abi.lib.rsgpu_sort_destroy(self.h)
            self.h = C.c_void_p()
        check(abi.lib.rsgpu_sort_create(str(path).encode(), key, float(dx), float(dy), int(order), C.byref(self.h)))
        self.file = str(path)
        self.dim = 3 if rss_header(path).type == abi.RSS_DATA3D else 2
        return True

    def createShotmap(self, path, order=0): return self._create(path, abi.SORT_SOURCE, 0.0, 0.0, order)
    def createReceivermap(self, path, order=0): return self._create(path, abi.SORT_RECEIVER, 0.0, 0.0, order)
    def createCMPmap(self, path, dx, dy, order=0): return self._create(path, abi.SORT_CMP, dx, dy, order)

    def _info(self):
        ng, ntr, nt = C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(abi.lib.rsgpu_sort_info(self.h, C.byref(ng), C.byref(ntr), C.byref(nt)))
        return ng.value, ntr.value, nt.value

    def getNensemb(self): return self._info()[0]
    def getNtraces(self): return self._info()[1]
    def getStatus(self, number): return abi.lib.rsgpu_sort_status(self.h, int(number))
    def setStatus(self, number, status): check(abi.lib.rsgpu_sort_set_status(self.h, int(number), int(status)))

    def get2DGather(self, number=None):
        """Sort::get2DGather(number), or without a number the next gather not started or
        failed (None when every gather is running or finished); marks it RUNNING."""
        if number is None:
            number = abi.lib.rsgpu_sort_next(self.h)
            if number < 0:
                return None
        n = abi.lib.rsgpu_sort_gather_size(self.h, int(number))
        if n < 0:
            raise abi.RsgpuError(abi.ERR_ARG, f"Sort::get2DGather: no gather {number}")
        _, _, nt = self._info()
        h = rss_header(self.file)
        g = (Data3D if self.dim == 3 else Data2D)(n, nt, h.d[0], h.o[0], self.precision)
        check(abi.lib.rsgpu_sort_read_gather(self.h, int(number), int(self.reciprocity), ptr(g.scoords),
                                             ptr(g.gcoords), ptr(g.data)))
        g.setReciprocity(self.reciprocity)
        g.number = int(number)
        return g

    get3DGather = get2DGather

    def createEmptydataset(self, path, n1, d1, o1):
        """Sort::createEmptydataset (lib/sort.cpp:999-1055)."""
        check(abi.lib.rsgpu_sort_create_output(self.h, str(path).encode(), int(n1), float(d1), float(o1)))

    def put2DGather(self, data, number):
        """Sort::put2DGather (lib/sort.cpp:535-579): the gather into the file data.getFile()."""
        check(abi.lib.rsgpu_sort_write_gather(self.h, data.getFile().encode(), int(number), int(self.reciprocity),
                                              data.nt, ptr(np.ascontiguousarray(data.scoords)),
                                              ptr(np.ascontiguousarray(data.gcoords)),
                                              ptr(np.ascontiguousarray(data.data))))

    put3DGather = put2DGather


def check_stability(model: _Model, dt: float, cls: str) -> None:
    """Modelling*::checkStability (lib/modelling.cpp:181-194)."""
    t = model.dtype
    vpmax = t(model.getVpmax())
    dx, dz = t(model.dx), t(model.dz)
    if model.dim == 3:
        dy = t(model.dy)
        dt_stab = t(2.0 / (3.1415 * math.sqrt((1.0 / float(dx * dx)) + (1 / float(dy * dy)) + (1 / float(dz * dz)))
                           * float(vpmax)))
    else:
        dt_stab = t(2.0 / (3.1415 * math.sqrt((1.0 / float(dx * dx)) + (1 / float(dz * dz))) * float(vpmax)))
    if not t(dt) < dt_stab:
        raise abi.RsgpuError(abi.ERR_ARG, f"{cls}::run: Wavelet sampling interval (dt) does not match the "
                             f"stability criteria (limit {float(dt_stab)}).")


def _tile(tile, models, sources, receivers, order, precision) -> int:
    """The tile index to build with: `tile`, or the autotuner's pick for tile == -2 (2D only)."""
    if int(tile) != -2:
        return int(tile)
    if models[0].dim == 3:
        return -1
    from .autotune import tune_tile
    return tune_tile(models, sources, receivers, order, precision)


def make_config(model: _Model, order: int, nt: int, dt: float, precision: int, tile: int = -1) -> abi.Config:
    cfg = abi.Config()
    cfg.physics = model.physics
    cfg.precision = precision
    cfg.lpml = model.lpml
    cfg.order = int(order)
    cfg.fs = int(model.fs)
    cfg.nt = int(nt)
    cfg.dx, cfg.dy, cfg.dz = float(model.dx), float(model.dy), float(model.dz)
    cfg.dt = float(dt)
    cfg.pml = None
    cfg.tile = int(tile)
    return cfg


def make_shot(model: _Model, source: Data2D, rec: Data2D | None, keep: list) -> abi.Shot:
    """Fill one rsgpu_shot from mirror objects; `keep` holds arrays alive for the call."""
    s = abi.Shot()
    s.nx, s.ny, s.nz = model.nx, model.ny, model.nz
    pads = model.padded()
    keep.extend(pads)
    for k, a in enumerate(pads):
        s.model[k] = a.ctypes.data
    smap, sshift = np.ascontiguousarray(source.smap), np.ascontiguousarray(source.sshift)
    wav = np.ascontiguousarray(source.data)
    keep.extend([smap, sshift, wav])
    s.nsrc, s.smap, s.sshift, s.wavelet, s.src_field = source.ntrace, ptr(smap), ptr(sshift), ptr(wav), source.field
    if rec is not None:
        gmap, gshift = np.ascontiguousarray(rec.gmap), np.ascontiguousarray(rec.gshift)
        keep.extend([gmap, gshift])
        s.nrec, s.gmap, s.gshift, s.rec_field = rec.ntrace, ptr(gmap), ptr(gshift), rec.field
        s.rec_out = ptr(rec.data)
        if rec.reciprocity and model.physics == abi.ELASTIC2D:
            fac = reciprocity_factor(model, rec)
            keep.append(fac)
            s.rec_factor = ptr(fac)
        if model.physics == abi.ELASTIC3D and rec.field == abi.PRESSURE:
            fac = pressure_factor_3d(model, rec)
            keep.append(fac)
            s.rec_factor = ptr(fac)
    return s


def pressure_factor_3d(model: _Model, rec: Data2D) -> np.ndarray:
    """(3*R*Vp*Vp - 4*R*Vs*Vs)/3 at each receiver's map point, evaluated in double
    and stored in T: the divisor of WavesElastic3D::recordData's pressure
    (lib/waves.cpp:4285)."""
    fac = np.ones(rec.ntrace, model.dtype)
    for i, (mx, my, mz) in enumerate(rec.gmap):
        if mx >= 0 and my >= 0 and mz >= 0:
            r, vp, vs = (float(a[mz, my, mx]) for a in (model.R, model.Vp, model.Vs))
            fac[i] = (3.0 * r * vp * vp - 4.0 * r * vs * vs) / 3.0
    return fac


def reciprocity_factor(model: _Model, rec: Data2D) -> np.ndarray:
    """R*Vp*Vp - R*Vs*Vs at each receiver cell, in T (lib/waves.cpp:2218-2220)."""
    t = model.dtype
    fac = np.ones(rec.ntrace, t)
    for i, (mx, mz) in enumerate(rec.gmap):
        if mx >= 0 and mz >= 0:
            r, vp, vs = model.R[mz, mx], model.Vp[mz, mx], model.Vs[mz, mx]
            fac[i] = t(t(r * vp) * vp) - t(t(r * vs) * vs)
    return fac


class _Modelling:
    physics_name = "ModellingAcoustic2D"

    def __init__(self, model=None, source=None, order=4, snapinc=1, precision=None):
        self.model, self.source = model, source
        self.order = int(order) if 1 < int(order) < 9 else 4   # Modelling<T>::Modelling (lib/modelling.cpp:17-22)
        self.snapinc = snapinc if snapinc > 0 else 1
        self.precision = precision if precision is not None else (model.precision if model else abi.F32_EXACT)
        self.recP = self.recVx = self.recVy = self.recVz = None
        self.tile = -1
        self.zchunk = 0
        self.launch_mode = 0

    def setModel(self, m): self.model = m
    def setSource(self, s): self.source = s
    def setRecP(self, d): self.recP = d
    def setRecVx(self, d): self.recVx = d
    def setRecVy(self, d): self.recVy = d
    def setRecVz(self, d): self.recVz = d
    def getOrder(self): return self.order

    def checkStability(self):
        check_stability(self.model, self.source.dt, self.physics_name)
        return True

    def run(self):
        self.checkStability()
        recs = [r for r in (self.recP, self.recVx, self.recVy, self.recVz) if r is not None]
        tile = _tile(self.tile, [self.model] * len(recs or [None]), [self.source] * len(recs or [None]), recs or [None],
                     self.order, self.precision)
        cfg = make_config(self.model, self.order, self.source.nt, self.source.dt, self.precision, tile)
        cfg.zchunk = int(self.zchunk)
        cfg.launch_mode = int(self.launch_mode)
        keep: list = []
        # one shot per recorded field; the wavefield computation is shared by
        # the reference, here each receiver set is a separate batch entry
        rec_list = recs or [None]
        shots = (abi.Shot * len(rec_list))(*[make_shot(self.model, self.source, r, keep) for r in rec_list])
        check(abi.lib.rsgpu_modelling(C.byref(cfg), len(rec_list), shots))
        return MOD_OK


class ModellingAcoustic2D(_Modelling):
    physics_name = "ModellingAcoustic2D"


class ModellingElastic2D(_Modelling):
    physics_name = "ModellingElastic2D"


class ModellingAcoustic3D(_Modelling):
    physics_name = "ModellingAcoustic3D"


class ModellingElastic3D(_Modelling):
    """ModellingElastic3D<T>::run (lib/modelling.cpp:727-850)."""
    physics_name = "ModellingElastic3D"


def modelling_batch(models, sources, receivers, order, precision=abi.F32_EXACT, tile=-1, launch_mode=0, zchunk=0):
    """Many shots, each with its own model window, advanced together in one plan
    (the batched form of Modelling*::run).  Traces accumulate into receivers[i].data.
    launch_mode / zchunk: rsgpu_config's (0 = the library's choice)."""
    tile = _tile(tile, models, sources, receivers, order, precision)
    cfg = make_config(models[0], order, sources[0].nt, sources[0].dt, precision, tile)
    cfg.launch_mode, cfg.zchunk = int(launch_mode), int(zchunk)
    keep: list = []
    shots = (abi.Shot * len(models))(*[make_shot(m, s, r, keep) for m, s, r in zip(models, sources, receivers)])
    check(abi.lib.rsgpu_modelling(C.byref(cfg), len(models), shots))
    return MOD_OK


class Plan:
    """Device-resident batch (rsgpu_plan): upload once, run steps, read traces."""

    def __init__(self, models, sources, receivers, order, precision=abi.F32_EXACT, tile=-1, launch_mode=0, zchunk=0):
        tile = _tile(tile, models, sources, receivers, order, precision)
        self.cfg = make_config(models[0], order, sources[0].nt, sources[0].dt, precision, tile)
        self.cfg.launch_mode, self.cfg.zchunk = int(launch_mode), int(zchunk)
        self._keep: list = []
        self.n = len(models)
        self.receivers = receivers
        self.shots = (abi.Shot * self.n)(*[make_shot(m, s, r, self._keep) for m, s, r in zip(models, sources, receivers)])
        self.h = C.c_void_p()
        check(abi.lib.rsgpu_plan_create(C.byref(self.cfg), self.n, self.shots, C.byref(self.h)))

    def reset(self): check(abi.lib.rsgpu_plan_reset(self.h))
    def run(self, it0=0, nsteps=None):
        check(abi.lib.rsgpu_plan_run(self.h, it0, self.cfg.nt if nsteps is None else nsteps))
    def sync(self): check(abi.lib.rsgpu_plan_sync(self.h))
    def stream(self) -> int: return abi.lib.rsgpu_plan_stream(self.h) or 0
    def launch_count(self) -> int: return abi.lib.rsgpu_plan_launch_count(self.h)
    def enable_timing(self): check(abi.lib.rsgpu_plan_enable_timing(self.h))

    def kernel_times(self):
        """Mean (velocity, stress) half-step kernel durations in ms from the last graph replay."""
        v, s_ = C.c_float(), C.c_float()
        check(abi.lib.rsgpu_plan_kernel_times(self.h, C.byref(v), C.byref(s_)))
        return v.value, s_.value

    def info(self):
        """(launch mode in use, fused work items, rows per work item)."""
        m, n, b = C.c_int(), C.c_int(), C.c_int()
        check(abi.lib.rsgpu_plan_info(self.h, C.byref(m), C.byref(n), C.byref(b)))
        return m.value, n.value, b.value

    def read_traces(self, i, out=None):
        r = self.receivers[i]
        if out is None:
            out = np.zeros((r.ntrace, r.nt), abi.real_dtype(self.cfg.precision))
        check(abi.lib.rsgpu_plan_read_traces(self.h, i, ptr(out)))
        return out

    def read_field(self, i, field, shape):
        out = np.zeros(shape, abi.real_dtype(self.cfg.precision))
        check(abi.lib.rsgpu_plan_read_field(self.h, i, field, ptr(out)))
        return out

    def close(self):
        if self.h:
            abi.lib.rsgpu_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- FWI gradient / RTM image
class Image2D:
    """Image container (Image2D<T>, include/image.h): imagedata[ihz, ihx, iz, ix]."""

    def __init__(self, imagefile, model: _Model, nhx=1, nhz=1, precision=None):
        self.imagefile = imagefile
        self.nx, self.nz, self.nhx, self.nhz = model.nx, model.nz, int(nhx), int(nhz)
        self.dx, self.dz, self.ox, self.oz = model.dx, model.dz, model.ox, model.oz
        self.dtype = abi.real_dtype(model.precision if precision is None else precision)
        self.imagedata = None

    def allocateImage(self):
        if self.imagedata is None:
            self.imagedata = np.zeros((self.nhz, self.nhx, self.nz, self.nx), self.dtype)

    def getImagedata(self):
        self.allocateImage()
        return self.imagedata

    def getNhx(self): return self.nhx
    def getNhz(self): return self.nhz


class Image3D:
    """Image container (Image3D<T>, include/image.h): imagedata[ihz, ihy, ihx, iz, iy, ix]."""

    def __init__(self, imagefile, model: _Model, nhx=1, nhy=1, nhz=1, precision=None):
        self.imagefile = imagefile
        self.nx, self.ny, self.nz = model.nx, model.ny, model.nz
        self.nhx, self.nhy, self.nhz = int(nhx), int(nhy), int(nhz)
        self.dtype = abi.real_dtype(model.precision if precision is None else precision)
        self.imagedata = None

    def allocateImage(self):
        if self.imagedata is None:
            self.imagedata = np.zeros((self.nhz, self.nhy, self.nhx, self.nz, self.ny, self.nx), self.dtype)

    def getImagedata(self):
        self.allocateImage()
        return self.imagedata

    def getNhx(self): return self.nhx
    def getNhy(self): return self.nhy
    def getNhz(self): return self.nhz


class _Adjoint:
    """Settings shared by FwiAcoustic2D and RtmAcoustic2D (the reference's Fwi / Rtm bases)."""
    cls = "FwiAcoustic2D"

    def __init__(self, model, source, dataP, order=4, snapinc=1, precision=None):
        self.model, self.source, self.dataP = model, source, dataP
        self.order = int(order) if 1 < int(order) < 9 else 4
        self.snapinc = snapinc if snapinc > 0 else 1
        self.precision = precision if precision is not None else model.precision
        self.ncheck = 0
        self.ckpt_precision = abi.CKPT_NATIVE
        self.accum = abi.ACCUM_REFERENCE
        self.misfit_type = abi.MISFIT_DIFFERENCE
        self.tile = -1
        self.noreverse = False

    def setModel(self, m): self.model = m
    def setSource(self, s): self.source = s
    def setDataP(self, d): self.dataP = d
    def setSnapinc(self, n): self.snapinc = int(n) if int(n) > 0 else 1
    def getSnapinc(self): return self.snapinc
    def setNcheck(self, n): self.ncheck = int(n)
    def setMisfit_type(self, t): self.misfit_type = int(t)
    def setCheckpointPrecision(self, p): self.ckpt_precision = int(p)   # no reference counterpart
    def setAccumulation(self, a): self.accum = int(a)                  # no reference counterpart

    def checkStability(self):
        check_stability(self.model, self.source.dt, self.cls)
        return True

    def _opts(self, nhx=1, nhz=1, nhy=1, snapmethod=abi.SNAP_OPTIMAL) -> abi.AdjointOpts:
        o = abi.AdjointOpts()
        o.ncheck, o.ckpt_precision, o.accum, o.misfit, o.nhx, o.nhz = (self.ncheck, self.ckpt_precision, self.accum,
                                                                        self.misfit_type, nhx, nhz)
        o.nhy = nhy
        o.snapmethod = snapmethod
        o.snapinc, o.noreverse = self.snapinc, int(bool(self.noreverse))
        return o

    def _adjoint_shot(self, keep: list) -> abi.AdjointShot:
        a = abi.AdjointShot()
        a.shot = make_shot(self.model, self.source, self.dataP, keep)
        a.shot.rec_out = None
        data = np.ascontiguousarray(self.dataP.data)
        keep.append(data)
        a.data = ptr(data)
        return a


class FwiAcoustic2D(_Adjoint):
    """FwiAcoustic2D<T> (include/fwi.h:128-182): gradient of the DIFFERENCE misfit
    with respect to vp and rho (and the source wavelet), run on the GPU."""
    cls = "FwiAcoustic2D"

    def __init__(self, model=None, source=None, dataP=None, order=4, snapinc=1, precision=None):
        super().__init__(model, source, dataP, order, snapinc, precision)
        self.vpgrad = self.rhograd = self.wavgrad = self.datamodP = self.dataresP = self.srcilum = None
        self.misfit = 0.0

    def setSrcilum(self, img): self.srcilum = img
    def setNoreverse(self, v): self.noreverse = bool(v)
    def getNoreverse(self): return self.noreverse
    def setVpgrad(self, img): self.vpgrad = img
    def setRhograd(self, img): self.rhograd = img
    def setWavgrad(self, d): self.wavgrad = d
    def setDatamodP(self, d): self.datamodP = d
    def setDataresP(self, d): self.dataresP = d
    def getMisfit(self): return self.misfit

    def _adjoint_shot(self, keep):
        a = super()._adjoint_shot(keep)
        vp, rho = np.ascontiguousarray(self.model.Vp), np.ascontiguousarray(self.model.R)
        keep.extend([vp, rho])
        a.vp, a.rho = ptr(vp), ptr(rho)
        a.vpgrad = ptr(self.vpgrad.getImagedata()) if self.vpgrad is not None else None
        a.rhograd = ptr(self.rhograd.getImagedata()) if self.rhograd is not None else None
        a.wavgrad = ptr(self.wavgrad.data) if self.wavgrad is not None else None
        a.datares = ptr(self.dataresP.data) if self.dataresP is not None else None
        a.shot.rec_out = ptr(self.datamodP.data) if self.datamodP is not None else None
        a.srcilum = ptr(self.srcilum.getImagedata()) if self.srcilum is not None else None
        self._mis = C.c_double(0.0)
        a.misfit = C.pointer(self._mis)
        return a

    def run(self):
        """FwiAcoustic2D::run (lib/fwi.cpp:1030-1156): FULL snapshots every snapinc
        steps; with setNoreverse(True) the forward run, datamodP and the misfit only."""
        return fwi_gradient_batch([self], snapmethod=abi.SNAP_FULL)

    def run_optimal(self):
        return fwi_gradient_batch([self])


class FwiAcoustic3D(FwiAcoustic2D):
    """FwiAcoustic3D<T> (include/fwi.h:186-236): vp/rho gradients of the DIFFERENCE
    misfit on a 3D window (gradients in Image3D containers)."""
    cls = "FwiAcoustic3D"


class FwiElastic2D(_Adjoint):
    """FwiElastic2D<T> (include/fwi.h:240-300): vp/vs/rho (and wavelet) gradients of
    the DIFFERENCE misfit of P, Ux and Uz data, run on the GPU with the adjoint
    elastic propagator and Revolve checkpointing."""
    cls = "FwiElastic2D"

    def __init__(self, model=None, source=None, dataP=None, dataUx=None, dataUz=None, order=4, snapinc=1,
                 precision=None):
        super().__init__(model, source, dataP, order, snapinc, precision)
        self.dataUx, self.dataUz = dataUx, dataUz
        self.vpgrad = self.vsgrad = self.rhograd = self.wavgrad = None
        self.datamodP = self.datamodUx = self.datamodUz = None
        self.dataresP = self.dataresUx = self.dataresUz = None
        self.misfit = 0.0

    def setDataUx(self, d): self.dataUx = d
    def setDataUz(self, d): self.dataUz = d
    def setVpgrad(self, img): self.vpgrad = img
    def setVsgrad(self, img): self.vsgrad = img
    def setRhograd(self, img): self.rhograd = img
    def setWavgrad(self, d): self.wavgrad = d
    def setDatamodP(self, d): self.datamodP = d
    def setDatamodUx(self, d): self.datamodUx = d
    def setDatamodUz(self, d): self.datamodUz = d
    def setDataresP(self, d): self.dataresP = d
    def setDataresUx(self, d): self.dataresUx = d
    def setDataresUz(self, d): self.dataresUz = d
    def getMisfit(self): return self.misfit

    def _adjoint_shot(self, keep):
        a = super()._adjoint_shot(keep)
        m = self.model
        vp, vs, rho = (np.ascontiguousarray(x) for x in (m.Vp, m.Vs, m.R))
        keep.extend([vp, vs, rho])
        a.vp, a.vs, a.rho = ptr(vp), ptr(vs), ptr(rho)
        for d, mp, sh, dat in ((self.dataUx, "gmap_vx", "gshift_vx", "data_vx"),
                               (self.dataUz, "gmap_vz", "gshift_vz", "data_vz")):
            arrs = [np.ascontiguousarray(x) for x in (d.gmap, d.gshift, d.data)]
            keep.extend(arrs)
            setattr(a, mp, ptr(arrs[0]))
            setattr(a, sh, ptr(arrs[1]))
            setattr(a, dat, ptr(arrs[2]))
        out = lambda o: ptr(o.getImagedata()) if o is not None else None  # noqa: E731
        a.vpgrad, a.vsgrad, a.rhograd = out(self.vpgrad), out(self.vsgrad), out(self.rhograd)
        dat = lambda o: ptr(o.data) if o is not None else None  # noqa: E731
        a.wavgrad = dat(self.wavgrad)
        a.shot.rec_out, a.datamod_vx, a.datamod_vz = dat(self.datamodP), dat(self.datamodUx), dat(self.datamodUz)
        a.datares, a.datares_vx, a.datares_vz = dat(self.dataresP), dat(self.dataresUx), dat(self.dataresUz)
        self._mis = C.c_double(0.0)
        a.misfit = C.pointer(self._mis)
        return a

    def run_optimal(self):
        return fwi_gradient_batch([self])


class FwiElastic3D(_Adjoint):
    """FwiElastic3D<T> (include/fwi.h:318-390): vp/vs/rho (and wavelet) gradients of
    the DIFFERENCE misfit of the Ux, Uy and Uz data, run on the GPU with the
    adjoint elastic 3D propagator and Revolve checkpointing (run_optimal,
    lib/fwi.cpp:6770-6990).  Gradients are Image3D containers [1, 1, 1, nz, ny, nx]."""
    cls = "FwiElastic3D"

    def __init__(self, model=None, source=None, dataUx=None, dataUy=None, dataUz=None, order=4, snapinc=1,
                 precision=None):
        super().__init__(model, source, dataUx, order, snapinc, precision)
        self.dataUy, self.dataUz = dataUy, dataUz
        self.vpgrad = self.vsgrad = self.rhograd = self.wavgrad = None
        self.datamodUx = self.datamodUy = self.datamodUz = None
        self.dataresUx = self.dataresUy = self.dataresUz = None
        self.misfit = 0.0

    def setDataUx(self, d): self.dataP = d
    def setDataUy(self, d): self.dataUy = d
    def setDataUz(self, d): self.dataUz = d
    def setVpgrad(self, img): self.vpgrad = img
    def setVsgrad(self, img): self.vsgrad = img
    def setRhograd(self, img): self.rhograd = img
    def setWavgrad(self, d): self.wavgrad = d
    def setDatamodUx(self, d): self.datamodUx = d
    def setDatamodUy(self, d): self.datamodUy = d
    def setDatamodUz(self, d): self.datamodUz = d
    def setDataresUx(self, d): self.dataresUx = d
    def setDataresUy(self, d): self.dataresUy = d
    def setDataresUz(self, d): self.dataresUz = d
    def getMisfit(self): return self.misfit

    def _adjoint_shot(self, keep):
        a = super()._adjoint_shot(keep)
        m = self.model
        vp, vs, rho = (np.ascontiguousarray(x) for x in (m.Vp, m.Vs, m.R))
        keep.extend([vp, vs, rho])
        a.vp, a.vs, a.rho = ptr(vp), ptr(vs), ptr(rho)
        for d, mp, sh, dat in ((self.dataUy, "gmap_vy", "gshift_vy", "data_vy"),
                               (self.dataUz, "gmap_vz", "gshift_vz", "data_vz")):
            arrs = [np.ascontiguousarray(x) for x in (d.gmap, d.gshift, d.data)]
            keep.extend(arrs)
            setattr(a, mp, ptr(arrs[0]))
            setattr(a, sh, ptr(arrs[1]))
            setattr(a, dat, ptr(arrs[2]))
        out = lambda o: ptr(o.getImagedata()) if o is not None else None  # noqa: E731
        a.vpgrad, a.vsgrad, a.rhograd = out(self.vpgrad), out(self.vsgrad), out(self.rhograd)
        dat = lambda o: ptr(o.data) if o is not None else None  # noqa: E731
        a.wavgrad = dat(self.wavgrad)
        a.shot.rec_out, a.datamod_vy, a.datamod_vz = dat(self.datamodUx), dat(self.datamodUy), dat(self.datamodUz)
        a.datares, a.datares_vy, a.datares_vz = dat(self.dataresUx), dat(self.dataresUy), dat(self.dataresUz)
        self._mis = C.c_double(0.0)
        a.misfit = C.pointer(self._mis)
        return a

    def run_optimal(self):
        return fwi_gradient_batch([self])


class RtmAcoustic2D(_Adjoint):
    """RtmAcoustic2D<T> (include/rtm.h:97-127): (extended) cross-correlation image."""
    cls = "RtmAcoustic2D"

    def __init__(self, model=None, pimage=None, source=None, dataP=None, order=4, snapinc=1, precision=None):
        super().__init__(model, source, dataP, order, snapinc, precision)
        self.pimage = pimage

    def setImage(self, img): self.pimage = img

    def _adjoint_shot(self, keep):
        a = super()._adjoint_shot(keep)
        a.image = ptr(self.pimage.getImagedata())
        return a

    def run(self):
        """RtmAcoustic2D::run (lib/rtm.cpp:222-326): FULL snapshots every snapinc steps."""
        return rtm_image_batch([self], snapmethod=abi.SNAP_FULL)

    def run_edge(self):
        """RtmAcoustic2D::run_edge (lib/rtm.cpp:328-421): only the wavefield's four edge
        lines are kept every snapinc steps; the source wavefield is re-propagated from
        them during the adjoint pass."""
        return rtm_image_batch([self], snapmethod=abi.SNAP_EDGES)

    def run_optimal(self):
        return rtm_image_batch([self])


class RtmAcoustic3D(_Adjoint):
    """RtmAcoustic3D<T> (include/rtm.h:128-160): (extended) 3D cross-correlation image."""
    cls = "RtmAcoustic3D"

    def __init__(self, model=None, pimage=None, source=None, dataP=None, order=4, snapinc=1, precision=None):
        super().__init__(model, source, dataP, order, snapinc, precision)
        self.pimage = pimage

    def setImage(self, img): self.pimage = img

    def _adjoint_shot(self, keep):
        a = super()._adjoint_shot(keep)
        a.image = ptr(self.pimage.getImagedata())
        return a

    def run(self):
        """RtmAcoustic3D::run (lib/rtm.cpp:640-733): FULL snapshots every snapinc steps."""
        return rtm_image_batch([self], snapmethod=abi.SNAP_FULL)

    def run_optimal(self):
        return rtm_image_batch([self])


def _lags(j0):
    if isinstance(j0, (RtmAcoustic2D, RtmAcoustic3D)):
        img = j0.pimage
        return img.getNhx(), img.getNhz(), img.getNhy() if isinstance(img, Image3D) else 1
    return 1, 1, 1


def _adjoint_tile(jobs) -> int:
    # the adjoint reuses the forward kernels: tune on the forward modelling of the batch
    j0 = jobs[0]
    return _tile(j0.tile, [j.model for j in jobs], [j.source for j in jobs], [j.dataP for j in jobs], j0.order,
                 j0.precision)


def _adjoint_batch(jobs, fn, snapmethod):
    j0 = jobs[0]
    j0.checkStability()
    cfg = make_config(j0.model, j0.order, j0.source.nt, j0.source.dt, j0.precision, _adjoint_tile(jobs))
    opts = j0._opts(*_lags(j0), snapmethod=snapmethod)
    keep: list = []
    shots = (abi.AdjointShot * len(jobs))(*[j._adjoint_shot(keep) for j in jobs])
    check(fn(C.byref(cfg), C.byref(opts), len(jobs), shots))
    for j in jobs:
        if isinstance(j, (FwiAcoustic2D, FwiElastic2D, FwiElastic3D)):
            j.misfit += j._mis.value
    return FWI_OK


def fwi_gradient_batch(jobs, snapmethod=abi.SNAP_OPTIMAL):
    """Many FwiAcoustic2D shots (each with its own model window) in one batched
    gradient computation; per-shot outputs accumulate like run_optimal's (run's
    with SNAP_FULL: snapshots every snapinc steps of the first job)."""
    return _adjoint_batch(jobs, abi.lib.rsgpu_fwi_gradient, snapmethod)


def rtm_image_batch(jobs, snapmethod=abi.SNAP_OPTIMAL):
    """Many RtmAcoustic2D shots imaged in one batched run (SNAP_FULL: as
    RtmAcoustic2D::run, SNAP_EDGES: as RtmAcoustic2D::run_edge)."""
    return _adjoint_batch(jobs, abi.lib.rsgpu_rtm_image, snapmethod)


class AdjointBatch:
    """Device-resident gradient/image batch (rsgpu_adjoint_*): create once, run many times."""

    def __init__(self, jobs, kind=abi.KIND_FWI, snapmethod=abi.SNAP_OPTIMAL):
        j0 = jobs[0]
        self.jobs = jobs
        self.cfg = make_config(j0.model, j0.order, j0.source.nt, j0.source.dt, j0.precision, _adjoint_tile(jobs))
        self.opts = j0._opts(*_lags(j0), snapmethod=snapmethod)
        self._keep: list = []
        self.shots = (abi.AdjointShot * len(jobs))(*[j._adjoint_shot(self._keep) for j in jobs])
        self.h = C.c_void_p()
        check(abi.lib.rsgpu_adjoint_create(C.byref(self.cfg), C.byref(self.opts), kind, len(jobs), self.shots,
                                           C.byref(self.h)))

    def run(self): check(abi.lib.rsgpu_adjoint_run(self.h))

    def read(self):
        check(abi.lib.rsgpu_adjoint_read(self.h, len(self.jobs), self.shots))
        for j in self.jobs:
            if isinstance(j, (FwiAcoustic2D, FwiElastic2D, FwiElastic3D)):
                j.misfit += j._mis.value
                j._mis.value = 0.0

    def stack(self, nxg, nzg, ix_start, iz_start, out0, out1=None, out2=None):
        """Image2D::stackImage of every shot's result into global images, on the device
        (rsgpu_adjoint_stack); out* are the running global images (host arrays of the
        element type), updated in place."""
        x0 = np.ascontiguousarray(ix_start, np.int32)
        z0 = np.ascontiguousarray(iz_start, np.int32)
        check(abi.lib.rsgpu_adjoint_stack(self.h, int(nxg), int(nzg), x0.ctypes.data_as(C.POINTER(C.c_int)),
                                          z0.ctypes.data_as(C.POINTER(C.c_int)),
                                          *[ptr(o) if o is not None else None for o in (out0, out1, out2)]))

    def stats(self):
        v = [C.c_longlong() for _ in range(4)]
        check(abi.lib.rsgpu_adjoint_stats(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("fw_steps", "bw_steps", "ckpt_bytes", "launches"), [x.value for x in v]))

    def stream(self) -> int: return abi.lib.rsgpu_adjoint_stream(self.h) or 0

    def close(self):
        if self.h:
            abi.lib.rsgpu_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Interp:
    """Interp<T> (include/interp.h, lib/interp.cpp): resample a Data2D/Data3D onto
    another's time axis (its nt, dt, ot) on the GPU; coordinates are copied."""

    def __init__(self, mode=abi.INTERP_LINEAR):
        self.mode = int(mode)

    def interp(self, frm: Data2D, to: Data2D):
        if frm.ntrace != to.ntrace:
            raise abi.RsgpuError(abi.ERR_ARG, "Interp::interp: Number of traces in the two datasets mismatch.")
        to.scoords[:] = frm.scoords
        to.gcoords[:] = frm.gcoords
        src = np.ascontiguousarray(frm.data.astype(to.dtype))
        check(abi.lib.rsgpu_interp_traces(to.precision, self.mode, frm.ntrace, frm.nt, float(frm.ot), float(frm.dt),
                                          ptr(src), to.nt, float(to.ot), float(to.dt), ptr(to.data)))

"""Shot-gather files and gather sorting (rockseis_b200/csrc/rss.cpp) against the
reference's own File / Data2D / Data3D / ModelAcoustic2D writers and Sort
(lib/file.cpp, lib/data.cpp, lib/model.cpp, lib/sort.cpp), run in this process
through oracle/_ref.  Files written by either side must be byte-identical, each side
must read the other's files, and every gather of every sort key and order must hold
the same traces in the same order.  CPU only."""
import os

import numpy as np
import pytest

from oracle import api
from rockseis_b200 import abi
from rockseis_b200.rockseis import Data2D, Data3D, Sort, rss_header

needs_ref = pytest.mark.skipif(not api.ref_available(), reason="reference library oracle/_ref not built here")


def survey(dim, nshot=5, nrec=7, nt=23, seed=3, dtype=np.float32):
    """Traces of nshot shots with nrec receivers each, shuffled, with repeated
    receiver positions across shots (so receiver and CMP gathers hold several)."""
    rng = np.random.default_rng(seed)
    sx = rng.choice(np.arange(0.0, 800.0, 40.0), nshot, replace=False)
    gx = np.arange(nrec) * 50.0 + 10.0
    rows = []
    for s in sx:
        for g in gx:
            if dim == 2:
                rows.append(([s, 5.0], [g, 0.0]))
            else:
                rows.append(([s, 30.0 * (s // 200), 5.0], [g, 20.0 * (g // 100), 0.0]))
    perm = rng.permutation(len(rows))
    sc = np.array([rows[i][0] for i in perm], dtype)
    gc = np.array([rows[i][1] for i in perm], dtype)
    data = rng.standard_normal((len(rows), nt)).astype(dtype)
    return sc, gc, data


@needs_ref
@pytest.mark.parametrize("dim,dtype", [(2, np.float32), (2, np.float64), (3, np.float32), (3, np.float64)])
def test_trace_file_bytes_equal_reference(tmp_path, dim, dtype):
    sc, gc, data = survey(dim, dtype=dtype)
    ours, theirs = tmp_path / "ours.rss", tmp_path / "ref.rss"
    cls = Data3D if dim == 3 else Data2D
    d = cls(len(data), data.shape[1], 2e-3, -0.25, abi.F64 if dtype == np.float64 else abi.F32_EXACT)
    d.scoords[:], d.gcoords[:], d.data[:] = sc, gc, data
    d.setFile(str(ours))
    d.write()
    api.ref_data_write(theirs, dim, data.shape[1], 2e-3, -0.25, sc, gc, data, dtype=dtype)
    assert ours.read_bytes() == theirs.read_bytes()
    h = rss_header(theirs)
    assert (h.type, h.nheader, h.n[0], h.n[1]) == ((abi.RSS_DATA3D if dim == 3 else abi.RSS_DATA2D), 2 * dim,
                                                  data.shape[1], len(data))


@needs_ref
def test_each_side_reads_the_others_traces(tmp_path):
    sc, gc, data = survey(2)
    theirs, ours = tmp_path / "ref.rss", tmp_path / "ours.rss"
    api.ref_data_write(theirs, 2, data.shape[1], 1e-3, 0.0, sc, gc, data)
    d = Data2D.fromFile(str(theirs))
    assert np.array_equal(d.data, data) and np.array_equal(d.scoords, sc) and np.array_equal(d.gcoords, gc)
    d.setFile(str(ours))
    d.write()
    rs, rg, rd = api.ref_data_read2d(ours, data.shape[1], len(data))
    assert np.array_equal(rd, data) and np.array_equal(rs, sc) and np.array_equal(rg, gc)
    # a trace range
    part = np.zeros((3, data.shape[1]), np.float32)
    abi.check(abi.lib.rsgpu_rss_read_traces(str(ours).encode(), abi.F32_EXACT, 4, 3, None, None, part.ctypes.data))
    assert np.array_equal(part, data[4:7])


@needs_ref
def test_model_file_bytes_equal_reference(tmp_path):
    vp = np.random.default_rng(1).uniform(1500, 4000, (13, 17)).astype(np.float32)
    ours, theirs = tmp_path / "ours.rss", tmp_path / "ref.rss"
    abi.check(abi.lib.rsgpu_rss_write_model(str(ours).encode(), abi.F32_EXACT, 17, 0, 13, 10.0, 0.0, 12.5, -50.0, 0.0,
                                            3.0, vp.ctypes.data))
    api.ref_model_write(theirs, vp, 10.0, 12.5, -50.0, 3.0)
    assert ours.read_bytes() == theirs.read_bytes()
    back = np.zeros_like(vp)
    abi.check(abi.lib.rsgpu_rss_read_model(str(theirs).encode(), abi.F32_EXACT, vp.size, back.ctypes.data))
    assert np.array_equal(back, vp)


@needs_ref
@pytest.mark.parametrize("dim,dtype", [(2, np.float32), (2, np.float64), (3, np.float32)])
@pytest.mark.parametrize("key,order", [(abi.SORT_SOURCE, 0), (abi.SORT_RECEIVER, 0), (abi.SORT_CMP, 0),
                                       (abi.SORT_SOURCE, 1), (abi.SORT_RECEIVER, 2), (abi.SORT_CMP, 2)])
def test_sort_gathers_equal_reference(tmp_path, dim, dtype, key, order):
    sc, gc, data = survey(dim, dtype=dtype)
    path = tmp_path / "survey.rss"
    api.ref_data_write(path, dim, data.shape[1], 1e-3, 0.0, sc, gc, data, dtype=dtype)
    prec = abi.F64 if dtype == np.float64 else abi.F32_EXACT
    s = Sort(prec)
    dx, dy = (25.0, 30.0) if key == abi.SORT_CMP else (0.0, 0.0)
    s._create(str(path), key, dx, dy, order)
    ng, _, _, _ = api.ref_sort_gather(path, dim, key, -1, data.shape[1], dx, dy, order, dtype=dtype)
    assert s.getNensemb() == ng and ng > 1
    for k in range(ng):
        for rec in (0, 1):
            s.setReciprocity(rec)
            g = s.get2DGather(k)
            _, rs, rg, rd = api.ref_sort_gather(path, dim, key, k, data.shape[1], dx, dy, order, rec, dtype=dtype)
            assert np.array_equal(g.data, rd), (k, rec)
            assert np.array_equal(g.scoords, rs) and np.array_equal(g.gcoords, rg), (k, rec)


def test_sort_queue_hands_out_failed_gathers_again(tmp_path):
    sc, gc, data = survey(2, nshot=3)
    path = tmp_path / "survey.rss"
    d = Data2D(len(data), data.shape[1], 1e-3, 0.0)
    d.scoords[:], d.gcoords[:], d.data[:] = sc, gc, data
    d.setFile(str(path))
    d.write()
    s = Sort()
    s.createShotmap(str(path))
    assert s.getNensemb() == 3
    g0 = s.get2DGather()                  # the first gather not started
    assert g0.number == 0 and s.getStatus(0) == abi.GATHER_RUNNING
    g1 = s.get2DGather()
    assert g1.number == 1
    s.setStatus(0, abi.GATHER_FAILED)     # a failed gather goes back to the queue
    assert s.get2DGather().number == 0
    for k in range(3):
        s.setStatus(k, abi.GATHER_FINISHED)
    assert s.get2DGather() is None
    # every trace of the survey lands in exactly one gather, shots sorted by source x
    xs = [s.get2DGather(k).scoords[0, 0] for k in range(3)]
    assert xs == sorted(xs)


@needs_ref
def test_put_gather_file_equals_reference(tmp_path):
    sc, gc, data = survey(2, nshot=4)
    path = tmp_path / "survey.rss"
    api.ref_data_write(path, 2, data.shape[1], 1e-3, 0.0, sc, gc, data)
    n1 = 11
    s = Sort()
    s.createShotmap(str(path))
    ours, theirs = tmp_path / "ours.rss", tmp_path / "ref.rss"
    s.createEmptydataset(str(ours), n1, 4e-3, 0.5)
    number = 2
    g = s.get2DGather(number)
    out = Data2D(g.ntrace, n1, 4e-3, 0.5)
    out.scoords[:], out.gcoords[:] = g.scoords, g.gcoords
    out.data[:] = np.random.default_rng(5).standard_normal(out.data.shape).astype(np.float32)
    out.setFile(str(ours))
    s.put2DGather(out, number)
    assert api.ref_sort_put2d(path, theirs, number, n1, 4e-3, 0.5, out.data) == g.ntrace
    assert ours.read_bytes() == theirs.read_bytes()
    assert os.path.getsize(ours) > 0

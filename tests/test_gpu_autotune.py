"""Tile autotuner on the GPU: it measures every built shape, caches its pick, and
the picked shape models the same traces bit for bit as the library default."""
import json

import numpy as np
import pytest

from rockseis_b200 import abi, autotune
from rockseis_b200.rockseis import Data2D, modelling_batch
from tests.cases import Case2D

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("physics", [abi.ACOUSTIC2D, abi.ELASTIC2D])
def test_autotuned_tile_models_identical_traces(require_gpu, tmp_path, monkeypatch, physics):
    monkeypatch.setenv("RSGPU_TILE_CACHE", str(tmp_path / "tiles.json"))
    cases = [Case2D(physics, nx=81 + 16 * i, nz=61, nt=120, seed=i + 1) for i in range(3)]
    out = {}
    for tile in (-1, autotune.AUTO):
        recs = []
        for c in cases:
            r = Data2D(c.rec.ntrace, c.nt, c.dt, 0.0)
            r.gcoords[:] = c.rec.gcoords
            r.setField(c.rec.field)
            r.gmap, r.gshift = c.rec.gmap, c.rec.gshift
            recs.append(r)
        modelling_batch([c.model for c in cases], [c.src for c in cases], recs, 8, abi.F32_EXACT, tile=tile)
        out[tile] = [r.data.copy() for r in recs]
    for a, b in zip(out[-1], out[autotune.AUTO]):
        assert np.abs(a).max() > 0
        assert np.array_equal(a, b)
    table = json.load(open(tmp_path / "tiles.json"))
    (entry,) = table.values()
    shapes = autotune.tile_shapes(abi.F32_EXACT)
    assert entry["tile"] in shapes and len(entry["ms_per_step"]) == len(shapes)
    assert all(v > 0 for v in entry["ms_per_step"].values())
    assert entry["ms_per_step"][str(entry["tile"])] == min(entry["ms_per_step"].values())

"""Tile autotuner host logic: the shape table the library reports, the JSON cache,
and the choice of the fastest shape (measurements faked on the CPU)."""
import json

from rockseis_b200 import abi, autotune
from rockseis_b200.rockseis import ModelAcoustic2D


def test_tile_table_matches_library():
    f32 = autotune.tile_shapes(abi.F32_FAST)
    assert len(f32) == abi.lib.rsgpu_tile_count(abi.F32_FAST) >= 2
    for tx, tz, rz, mb in f32.values():
        assert tx % 4 == 0 and tz % rz == 0 and mb >= 1
    f64 = autotune.tile_shapes(abi.F64)
    assert sorted(f64) == [0, 3]
    import ctypes as C
    v = [C.c_int() for _ in range(4)]
    assert abi.lib.rsgpu_tile_shape(abi.F64, 1, *[C.byref(x) for x in v]) == abi.ERR_ARG
    assert abi.lib.rsgpu_tile_shape(abi.F32_FAST, 99, *[C.byref(x) for x in v]) == abi.ERR_ARG


def _models(n=3):
    ms = []
    for i in range(n):
        m = ModelAcoustic2D(60 + 10 * i, 40, 10, 10.0, 10.0, 0.0, 0.0, 0)
        ms.append(m)
    return ms


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
    calls = []
    fake = {0: 3.0, 3: 1.5, 5: 2.0}
    monkeypatch.setattr(autotune, "tile_shapes", lambda p: {k: (32, 32, 2, 1) for k in fake})

    def measure(models, sources, receivers, order, precision, tile, warm, steps):
        calls.append(tile)
        return fake[tile]
    monkeypatch.setattr(autotune, "measure_tile", measure)
    path = str(tmp_path / "tiles.json")
    ms = _models()
    assert autotune.tune_tile(ms, [None] * 3, [None] * 3, 8, abi.F32_FAST, cache=path) == 3
    assert sorted(calls) == [0, 3, 5]
    table = json.load(open(path))
    (key, entry), = table.items()
    assert entry["tile"] == 3 and key == autotune.problem_key(ms, 8, abi.F32_FAST)
    # cached: no new measurement
    calls.clear()
    assert autotune.tune_tile(ms, [None] * 3, [None] * 3, 8, abi.F32_FAST, cache=path) == 3
    assert calls == []
    # another problem class (one shot fewer) is measured and stored beside it
    assert autotune.tune_tile(ms[:2], [None] * 2, [None] * 2, 8, abi.F32_FAST, cache=path) == 3
    assert len(json.load(open(path))) == 2
    # refresh re-measures
    fake[0] = 0.5
    assert autotune.tune_tile(ms, [None] * 3, [None] * 3, 8, abi.F32_FAST, cache=path, refresh=True) == 0


def test_problem_key_separates_precision_and_order():
    ms = _models(2)
    keys = {autotune.problem_key(ms, o, p) for o in (4, 8) for p in (abi.F32_EXACT, abi.F32_FAST)}
    assert len(keys) == 4

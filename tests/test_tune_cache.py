"""The autotuner's result cache (pcx_tune_cache_*): entries keyed by GPU name,
size, element type and batch (power-of-two bucket), saved to JSON and merged
back.  Host code only, so this runs on CPU."""
import ctypes
import json

from packed_b200 import _lib


def _put(L, gpu, n, dtype, batch, **kw):
    r = _lib.TuneResult(**kw)
    assert L.pcx_tune_cache_put(gpu, n, dtype, batch, ctypes.byref(r)) == _lib.PCX_OK


def _get(L, gpu, n, dtype, batch):
    r = _lib.TuneResult()
    rc = L.pcx_tune_cache_get(gpu, n, dtype, batch, ctypes.byref(r))
    return rc, r


def test_round_trip_through_json(tmp_path):
    L = _lib.lib()
    L.pcx_tune_cache_clear()
    _put(L, b"NVIDIA B200", 1 << 20, _lib.PCX_F32, 128, form=2, rounds=3, log_n1=10, log_n2=10, blocks_per_sm=1,
         stages=2, ms=0.2375)
    _put(L, b"NVIDIA B200", 1 << 16, _lib.PCX_F64, 16, form=3, rounds=3, chunk_bytes=48 << 20, ms=1.5)
    _put(L, b'odd "name" \\ gpu', 1 << 14, _lib.PCX_F32, 3, form=2, rounds=6, log_n1=7, log_n2=7, blocks_per_sm=2,
         stages=3, ms=0.01)
    # the same key again replaces the entry (batch 200 falls in the 128..255 bucket)
    _put(L, b"NVIDIA B200", 1 << 20, _lib.PCX_F32, 200, form=2, rounds=2, log_n1=10, log_n2=10, blocks_per_sm=1,
         stages=3, ms=0.2)
    assert L.pcx_tune_cache_size() == 3
    path = tmp_path / "tune.json"
    assert L.pcx_tune_cache_save(str(path).encode()) == _lib.PCX_OK
    doc = json.loads(path.read_text())
    assert doc["version"] == 1 and len(doc["entries"]) == 3
    assert {e["gpu"] for e in doc["entries"]} == {"NVIDIA B200", 'odd "name" \\ gpu'}

    L.pcx_tune_cache_clear()
    assert L.pcx_tune_cache_size() == 0
    assert L.pcx_tune_cache_load(str(path).encode()) == _lib.PCX_OK
    assert L.pcx_tune_cache_size() == 3
    rc, r = _get(L, b"NVIDIA B200", 1 << 20, _lib.PCX_F32, 255)
    assert rc == _lib.PCX_OK
    assert (r.form, r.rounds, r.log_n1, r.log_n2, r.blocks_per_sm, r.stages) == (2, 2, 10, 10, 1, 3)
    assert abs(r.ms - 0.2) < 1e-9
    rc, r = _get(L, b"NVIDIA B200", 1 << 16, _lib.PCX_F64, 31)
    assert rc == _lib.PCX_OK and r.form == 3 and r.chunk_bytes == 48 << 20
    rc, r = _get(L, b'odd "name" \\ gpu', 1 << 14, _lib.PCX_F32, 2)
    assert rc == _lib.PCX_OK and (r.log_n1, r.blocks_per_sm, r.stages, r.rounds) == (7, 2, 3, 6)
    # misses: other batch bucket, other type, other GPU
    assert _get(L, b"NVIDIA B200", 1 << 20, _lib.PCX_F32, 64)[0] == _lib.PCX_ERR_INVALID
    assert _get(L, b"NVIDIA B200", 1 << 20, _lib.PCX_F64, 128)[0] == _lib.PCX_ERR_INVALID
    assert _get(L, b"NVIDIA H100", 1 << 20, _lib.PCX_F32, 128)[0] == _lib.PCX_ERR_INVALID
    # loading merges: the file again leaves three entries
    assert L.pcx_tune_cache_load(str(path).encode()) == _lib.PCX_OK
    assert L.pcx_tune_cache_size() == 3
    L.pcx_tune_cache_clear()


def test_malformed_or_missing_file(tmp_path):
    L = _lib.lib()
    L.pcx_tune_cache_clear()
    bad = tmp_path / "bad.json"
    bad.write_text('{"version": 1, "entries": [{"gpu": "x", "n": 1024,')
    assert L.pcx_tune_cache_load(str(bad).encode()) == _lib.PCX_ERR_INVALID
    assert b"malformed" in L.pcx_last_error()
    assert L.pcx_tune_cache_load(str(tmp_path / "none.json").encode()) == _lib.PCX_ERR_INVALID
    assert L.pcx_tune_cache_size() == 0
    # unknown keys are skipped
    ok = tmp_path / "ok.json"
    ok.write_text('{"version": 1, "note": {"a": [1, 2]}, "entries": [{"gpu": "G", "n": 65536, "dtype": "f32", '
                  '"batch_log2": 4, "form": 2, "rounds": 3, "chunk_bytes": 0, "split": [8, 8], '
                  '"blocks_per_sm": 2, "stages": 3, "ms": 0.5, "extra": "ignored"}]}')
    assert L.pcx_tune_cache_load(str(ok).encode()) == _lib.PCX_OK
    rc, r = _get(L, b"G", 65536, _lib.PCX_F32, 16)
    assert rc == _lib.PCX_OK and (r.log_n1, r.log_n2, r.blocks_per_sm, r.stages) == (8, 8, 2, 3)
    L.pcx_tune_cache_clear()

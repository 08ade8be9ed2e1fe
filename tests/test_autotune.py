"""Autotuner host logic (no GPU): shape classes, candidate generation, the
JSON cache. The GPU test measures real candidates."""
import json

import pytest

from hb_hammerbench_b200 import autotune, tiles


@pytest.fixture
def cache(tmp_path, monkeypatch):
    p = tmp_path / "tune.json"
    monkeypatch.setenv("HBSG_AUTOTUNE_CACHE", str(p))
    autotune.clear_memory_cache()
    yield p
    autotune.clear_memory_cache()


def test_shape_classes():
    assert autotune.shape_key(8192, 8192, 8192, "bf16x6") == "bf16x6:m13:n13:k13"
    assert autotune.shape_key(5000, 8000, 8192, "ffma") == autotune.shape_key(4097, 8192, 8192, "ffma")
    assert autotune.shape_key(4096, 8192, 8192, "ffma") != autotune.shape_key(4097, 8192, 8192, "ffma")


@pytest.mark.parametrize("variant,parts", [("ffma", 0), ("bf16x6", 3), ("bf16x3_scaled", 2)])
def test_candidates_use_matching_family(variant, parts):
    tl = {t["tile"]: t for t in tiles()}
    c = autotune.candidates(8192, 8192, 8192, variant, list(tl.values()))
    assert c
    for cfg in c:
        t = tl[cfg["tile"]]
        assert t["parts"] == parts
        if variant == "ffma":
            assert cfg["split_k"] in (0, 1)  # full output: keep one FMA chain per element


def test_small_output_candidates_slice_k():
    c = autotune.candidates(256, 256, 1 << 20, "bf16x6", tiles())
    assert any(cfg["split_k"] > 1 for cfg in c)


def test_cache_roundtrip(cache):
    assert autotune.lookup(1024, 1024, 1024, "bf16x6") is None
    autotune._store(autotune.shape_key(1024, 1024, 1024, "bf16x6"),
                    {"config": {"tile": 10, "split_k": 0, "chunk_k": 32, "raster_group": 8},
                     "ms": 1.0, "candidates": []})
    assert autotune.lookup(1000, 1000, 1000, "bf16x6")["tile"] == 10
    assert json.load(open(cache))["bf16x6:m10:n10:k10"]["ms"] == 1.0
    autotune.clear_memory_cache()
    assert autotune.lookup(1024, 1024, 1024, "bf16x6")["chunk_k"] == 32  # reloaded from disk

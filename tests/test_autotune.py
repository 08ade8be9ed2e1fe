"""Autotuner host logic (no GPU): shape classes, candidate generation, the
JSON cache. The GPU test measures real candidates."""
import json

import pytest

from hb_hammerbench_b200 import autotune, tiles


@pytest.fixture
def cache(tmp_path, monkeypatch):
    # an empty user cache and no shipped table
    p = tmp_path / "tune.json"
    monkeypatch.setenv("HBSG_AUTOTUNE_CACHE", str(p))
    monkeypatch.setattr(autotune, "SHIPPED_PATH", str(tmp_path / "none.json"))
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


def test_shipped_table_is_the_default(tmp_path, monkeypatch):
    # the host interface answers from the user cache first, then from the
    # package's shipped table; HBSG_AUTOTUNE=0 turns the lookup off
    from hb_hammerbench_b200 import resolve_config
    shipped = tmp_path / "shipped.json"
    shipped.write_text(json.dumps({autotune.shape_key(8192, 8192, 8192, "bf16x6"): {
        "config": {"tile": 20, "split_k": 0, "chunk_k": 64, "raster_group": 8}, "ms": 4.0}}))
    monkeypatch.setattr(autotune, "SHIPPED_PATH", str(shipped))
    monkeypatch.setenv("HBSG_AUTOTUNE_CACHE", str(tmp_path / "user.json"))
    monkeypatch.setenv("HBSG_AUTOTUNE", "1")
    autotune.clear_memory_cache()
    try:
        assert resolve_config(8192, 8192, 8192, "bf16x6", False, None)["tile"] == 20
        assert resolve_config(8000, 8100, 8192, 2, False, None)["tile"] == 20  # enum form
        assert resolve_config(8192, 8192, 8192, "bf16x6", True, None) is None  # transposed
        assert resolve_config(8192, 8192, 8192, "bf16x6", False, {"tile": 10}) == {"tile": 10}
        assert resolve_config(100, 100, 100, "bf16x6", False, None) is None  # no class
        autotune._store(autotune.shape_key(8192, 8192, 8192, "bf16x6"),
                        {"config": {"tile": 10}, "ms": 3.0})
        assert resolve_config(8192, 8192, 8192, "bf16x6", False, None)["tile"] == 10
        monkeypatch.setenv("HBSG_AUTOTUNE", "0")
        assert resolve_config(8192, 8192, 8192, "bf16x6", False, None) is None
    finally:
        autotune.clear_memory_cache()


def test_shipped_table_parses():
    # every shipped entry names a tile of the library's table for its variant
    data = json.load(open(autotune.SHIPPED_PATH))
    tl = {t["tile"]: t for t in tiles()}
    for key, e in data.items():
        cfg = e["config"]
        if "tile" in cfg and cfg["tile"]:
            t = tl[cfg["tile"]]
            variant = key.split(":")[1] if key.startswith("grouped:") else key.split(":")[0]
            want = "ffma" if variant == "ffma" else "bf16"
            assert t["family"] == want, key

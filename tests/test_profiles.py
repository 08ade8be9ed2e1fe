"""The committed profile summaries and the traffic table the bench line reads
(CPU only): each summary names the command that made it with the clocks left
unlocked, the traffic table points at summaries that exist, and bench.py's
lookup resolves the keys of its own lines."""
import glob
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = os.path.join(ROOT, "profiles")


def _summaries():
    return sorted(p for p in glob.glob(os.path.join(PROFILES, "*.md"))
                  if os.path.basename(p) != "README.md")


@pytest.mark.parametrize("path", _summaries(), ids=os.path.basename)
def test_summary_gives_its_command(path):
    text = open(path).read()
    assert "ncu " in text, "a summary names the ncu command it comes from"
    assert "--clock-control none" in text


def test_index_lists_every_summary():
    index = open(os.path.join(PROFILES, "README.md")).read()
    for path in _summaries():
        assert os.path.basename(path) in index


def test_profiles_hold_text_only():
    for name in os.listdir(PROFILES):
        assert os.path.splitext(name)[1] in (".md", ".txt", ".json"), name


def test_traffic_table_points_at_summaries():
    table = json.load(open(os.path.join(PROFILES, "traffic.json")))
    entries = {k: v for k, v in table.items() if not k.startswith("_")}
    assert entries
    for key, entry in entries.items():
        assert isinstance(entry["dram_bytes_per_launch"], int), key
        assert entry["dram_bytes_per_launch"] > 0, key
        assert os.path.exists(os.path.join(PROFILES, entry["capture"])), key


def test_bench_resolves_its_traffic_keys():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    table = json.load(open(os.path.join(PROFILES, "traffic.json")))
    # the headline (tensor-core kernel, 6 products, 8192^3) and the FFMA leg
    assert bench._profile_traffic("tc_gemm_bf16x6_n8192") == \
        table["tc_gemm_bf16x6_n8192"]["dram_bytes_per_launch"]
    assert bench._profile_traffic("ffma_sgemm_n8192") == \
        table["ffma_sgemm_n8192"]["dram_bytes_per_launch"]
    assert bench._profile_traffic("no_such_kernel_n1") is None

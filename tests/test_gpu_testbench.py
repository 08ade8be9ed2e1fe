"""The C++ testbench (tests/testbench/sgemm_main.cpp) run as the reference
runs its launch directories: N_<n>__NITER_<k> with a PASS/FAIL banner."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TB = os.path.join(HERE, "testbench")


@pytest.fixture(scope="module")
def binary():
    subprocess.run(["make", "-s", "-C", TB], check=True)
    return os.path.join(TB, "sgemm_testbench")


@pytest.mark.parametrize("args", [["512", "2"], ["256", "3", "uniform"], ["100", "1", "uniform"]])
def test_testbench_passes(binary, args):
    r = subprocess.run([binary] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "HBSG REGRESSION TEST PASSED" in r.stdout
    if args[-1] != "uniform":
        assert "differing elements: 0," in r.stdout  # integer fixture: exact

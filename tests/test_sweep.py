"""Host logic of the benchmark driver (no GPU): case-name parsing in the
reference's N_<n>__NITER_<k> launch-directory convention and the seeded
uneven-batch generator."""
import numpy as np
import pytest

from hb_hammerbench_b200 import sweep


def test_reference_case_name():
    assert sweep.parse_case("N_512__NITER_2") == {"N": 512, "NITER": 2}


def test_general_and_grouped_names():
    c = sweep.parse_case("M_256__N_256__K_1048576__V_bf16x6__SPLITK_74")
    assert c == {"M": 256, "N": 256, "K": 1048576, "V": "bf16x6", "SPLITK": 74}
    g = sweep.parse_case("GROUPED_512__SEED_0__V_ffma")
    assert g["GROUPED"] == 512 and g["SEED"] == 0
    s = sweep.parse_case("M_8192__N_8192__K_8192__V_bf16x6__TILE_10__SPLITK_0__CHUNK_64__RASTER_16")
    assert sweep._config(s) == {"split_k": 0, "tile": 10, "chunk_k": 64, "raster_group": 16}
    assert sweep._config(sweep.parse_case("N_512__NITER_2")) is None


def test_blackscholes_names():
    # apps/blackscholes/tests.mk:1 registers num-option_32768
    assert sweep.parse_case("num-option_32768") == {"NUM-OPTION": 32768}
    c = sweep.parse_case("num-option_10000000__LAYOUT_arrays")
    assert c == {"NUM-OPTION": 10000000, "LAYOUT": "arrays"}


def test_jacobi_names():
    # apps/jacobi/tests.mk:1-2 registers nx_64__ny_8__nz_512 and nx_32__ny_8__nz_512
    assert sweep.parse_case("nx_64__ny_8__nz_512") == {"NX": 64, "NY": 8, "NZ": 512}


@pytest.mark.parametrize("bad", ["N_512__V_fp64", "NITER_2", "N__512", "SEED_1__V_ffma"])
def test_bad_names(bad):
    with pytest.raises(ValueError):
        sweep.parse_case(bad)


def test_grouped_dims_distribution():
    d = sweep.grouped_dims(512, 0)
    assert d.shape == (512, 3)
    assert d.min() >= 64 and d.max() <= 2048 and not (d % 32).any()
    assert np.array_equal(d, sweep.grouped_dims(512, 0))
    assert not np.array_equal(d, sweep.grouped_dims(512, 1))

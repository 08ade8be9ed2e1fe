"""Generate the golden fixtures under tests/golden/ from the reference's own
host reference product, host_mm (apps/sgemm/main.cpp:15-26), compiled from the
reference source tree by `make -C oracle ref`.

Run in a container that has the reference tree:  python tests/golden/make_golden.py
The fixtures are committed; the tests never need the reference tree.

Fixtures
  sgemm_mod_N512_NITER2.json    the benchmark's own launch N_512__NITER_2 with its
                                inputs mat1[i] = i % 7, mat2[i] = i % 3
                                (main.cpp:49-52, tests.mk:1): SHA-256 of the
                                expected float32 result bytes and sampled values.
  sgemm_ramp_identity_N512.json legacy sgemm_512 fixture, A[i] = i, B = I, C = A
                                (apps/legacy/gemm/sgemm_512/main.cpp:69-80).
  sgemm_uniform_N64_NITER2.npz  seeded U[-1,1) inputs (numpy PCG64, seed 42) and
  sgemm_uniform_N128_NITER1.npz the reference host_mm outputs, per matrix.
  jacobi_mod_64x8x512.json      the Jacobi benchmark's launch nx_64__ny_8__nz_512
                                (apps/jacobi/tests.mk:1) on its input A0[i] = i % 13,
                                c0 = 2, c1 = 4 (main.cpp:62-73): SHA-256 of the
                                reference host_jacobi's output (main.cpp:19-48).
  blackscholes_32768.json       the Black-Scholes benchmark's launch num-option_32768
                                (apps/blackscholes/tests.mk:1) on seeded synthetic
                                option records (hb_hammerbench_b200.blackscholes.
                                option_records(32768, seed 3)): SHA-256 of the inputs,
                                of the reference host BlkSchlsEqEuroNoDiv's call/put
                                (bs.hpp:60-125) and of the oracle's restatement of the
                                device kernel's arithmetic (bs_kernel.hpp:163-198),
                                with the testbench's error between the two
                                (main.cpp:119-141).

    python tests/golden/make_golden.py [--jacobi | --blackscholes]   (only that fixture)
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle  # noqa: E402


def sha(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest()


REFERENCE_ROOT = os.environ.get("HB_REFERENCE_ROOT", "/root/reference")


def jacobi_fixture():
    assert oracle.ref_jacobi_available(), "reference host_jacobi not built"
    nx, ny, nz, c0, c1 = 64, 8, 512, 2, 4
    a = oracle.fill_jacobi(nx * ny * nz)
    out = oracle.ref_host_jacobi(a, nx, ny, nz, c0, c1)
    rng = np.random.Generator(np.random.PCG64(11))
    idx = np.sort(rng.choice(out.size, 32, replace=False))
    with open(os.path.join(HERE, "jacobi_mod_64x8x512.json"), "w") as f:
        json.dump({
            "source": "reference host_jacobi (apps/jacobi/main.cpp:19-48) compiled from the reference tree",
            "inputs": "A0[i] = i % 13 (apps/jacobi/main.cpp:70-73), c0 = 2, c1 = 4 (main.cpp:62-63)",
            "nx": nx, "ny": ny, "nz": nz, "c0": c0, "c1": c1,
            "sha256_anext_f32": sha(out),
            "samples": [[int(i), float(out[i])] for i in idx],
        }, f, indent=1)


def blackscholes_fixture():
    from hb_hammerbench_b200.blackscholes import option_records
    assert oracle.ref_bs_available(), "reference Black-Scholes host library not built"
    n, seed = 32768, 3
    rec = option_records(n, seed)
    host = oracle.ref_bs_host(rec)
    assert np.array_equal(host, oracle.bs_host(rec))
    dev = oracle.bs_device(rec)
    rng = np.random.Generator(np.random.PCG64(13))
    idx = np.sort(rng.choice(n, 32, replace=False))
    with open(os.path.join(HERE, "blackscholes_32768.json"), "w") as f:
        json.dump({
            "source": "reference BlkSchlsEqEuroNoDiv (apps/blackscholes/bs.hpp:60-125) compiled "
                      "from the reference tree; device arithmetic: oracle_bs_device "
                      "(bs_kernel.hpp:163-198 restated)",
            "inputs": "option_records(32768, seed=3): (n, 8) float32 records s, strike, r, v, t, "
                      "call, put, unused",
            "num_option": n, "seed": seed,
            "sha256_inputs_f32": sha(rec),
            "sha256_host_call_put_f32": sha(host[:, 5:7]),
            "sha256_device_call_put_f32": sha(dev[:, 5:7]),
            "validation_error_device_vs_host": oracle.bs_validation_error(dev, host),
            "samples": [[int(i), float(host[i, 5]), float(host[i, 6]), float(dev[i, 5]),
                         float(dev[i, 6])] for i in idx],
        }, f, indent=1)


def main():
    oracle.build(REFERENCE_ROOT)
    if "--jacobi" in sys.argv:
        jacobi_fixture()
        return
    if "--blackscholes" in sys.argv:
        blackscholes_fixture()
        return
    assert oracle.ref_available(), "reference host_mm not built"

    # 1. the benchmark's own fixture, N=512 NITER=2
    n, niter = 512, 2
    m1, m2 = oracle.fill_mod(niter * n * n)
    outs = {}
    for opt in ("O3", "O0"):
        outs[opt] = np.concatenate([
            oracle.ref_host_mm(m1[i * n * n:(i + 1) * n * n], m2[i * n * n:(i + 1) * n * n], n, opt).ravel()
            for i in range(niter)])
    assert np.array_equal(outs["O3"], outs["O0"])
    c = outs["O3"]
    rng = np.random.Generator(np.random.PCG64(7))
    idx = np.sort(rng.choice(c.size, 64, replace=False))
    fix = {
        "source": "reference host_mm (apps/sgemm/main.cpp:15-26) compiled from the reference tree, -O3 and -O0 agree",
        "inputs": "mat1[i] = i % 7, mat2[i] = i % 3 for i < NITER*N*N (apps/sgemm/main.cpp:49-52)",
        "N": n, "NITER": niter,
        "sha256_result_f32": sha(c),
        "first": float(c[0]), "last": float(c[-1]),
        "sum_per_matrix": [float(np.sum(c[i * n * n:(i + 1) * n * n].astype(np.float64))) for i in range(niter)],
        "samples": [[int(i), float(c[i])] for i in idx],
    }
    with open(os.path.join(HERE, "sgemm_mod_N512_NITER2.json"), "w") as f:
        json.dump(fix, f, indent=1)

    # 2. legacy sgemm_512 fixture: C = A
    a, b = oracle.fill_ramp_identity(n)
    cr = oracle.ref_host_mm(a, b, n, "O3")
    assert np.array_equal(cr, a)
    with open(os.path.join(HERE, "sgemm_ramp_identity_N512.json"), "w") as f:
        json.dump({
            "source": "reference host_mm compiled from the reference tree",
            "inputs": "A[i] = i, B = identity (apps/legacy/gemm/sgemm_512/main.cpp:69-80)",
            "N": n, "sha256_result_f32": sha(cr), "result_equals_A": True,
        }, f, indent=1)

    # 3. seeded uniform inputs with the reference's outputs
    for n, niter in ((64, 2), (128, 1)):
        A, B = oracle.uniform_inputs((niter, n, n), (niter, n, n), seed=42)
        C = np.stack([oracle.ref_host_mm(A[i], B[i], n, "O3") for i in range(niter)])
        C0 = np.stack([oracle.ref_host_mm(A[i], B[i], n, "O0") for i in range(niter)])
        assert np.array_equal(C, C0)
        np.savez_compressed(os.path.join(HERE, f"sgemm_uniform_N{n}_NITER{niter}.npz"),
                            A=A, B=B, C_ref=C, seed=np.int64(42))
    jacobi_fixture()
    blackscholes_fixture()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

"""Records golden vectors from the reference itself.

Runs the reference built from its own sources for sm_100a
(oracle/_ref/libMHCUDA.so, see oracle/Makefile) on a B200 through its C ABI
and stores, per case, the parameters it used, the CSR input, the device logf
of every weight and the reference's output.  tests/test_oracle.py checks the
CPU oracle against these files without a GPU.

    python tests/golden/make_golden.py [--out DIR]
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
from wmh_testlib import CGen, device_logf, gamma_params, random_csr, reference_lib  # noqa: E402


def record(out_dir, name, m, samples, seed=None, params=None):
    lib = reference_lib()
    assert lib is not None, "build the reference first: make -C oracle ref"
    dim = m.shape[1]
    gen = CGen(lib, dim, samples, seed=seed or 1, deferred=params is not None, devices=1)
    try:
        if params is not None:
            gen.assign(*params)
        rs, ln_cs, betas = gen.retrieve()
        ref_out = gen.calc_csr(m)
    finally:
        gen.close()
    path = os.path.join(out_dir, name + ".npz")
    np.savez_compressed(path, rs=rs, ln_cs=ln_cs, betas=betas,
                        weights=m.data.astype(np.float32), cols=m.indices.astype(np.uint32),
                        rows=m.indptr.astype(np.uint32), lnw=device_logf(m.data),
                        ref_out=ref_out, seed=np.int64(seed or -1))
    print(name, m.shape, m.nnz, samples, os.path.getsize(path), "bytes")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import scipy.sparse as sp
    # test.py:126-152 / 154-182: the tiny vectors with seeded parameters.
    tiny = sp.csr_matrix(np.array([O.TINY_V1, O.TINY_V2], np.float32))
    record(args.out, "tiny_seed_default", tiny, 128, seed=1)
    # test.py:184-210: the real-valued vector, seed 7.
    record(args.out, "float_seed7", sp.csr_matrix(np.array([O.FLOAT_V], np.float32)), 128, seed=7)
    # test.py:92-101: first 300 rows of the seed-1 6400x130 matrix, seed 1.
    _, m = O.reference_small_matrix(1)
    record(args.out, "small_seed1_rows300", m[:300], 128, seed=1)
    # Near-tie cells that separate the fused and unfused float forms.
    from test_gpu_reference import crafted_form_case
    rs, lc, b, cm = crafted_form_case(np.random.default_rng(11), rows=16, samples=64)
    record(args.out, "fma_form_crafted", cm, 64, params=(rs, lc, b))
    # Lognormal weights, a long row, empty rows, 256 samples.
    rng = np.random.default_rng(2024)
    rm = random_csr(rng, 40, 200, 25, empty_frac=0.05, long_rows=[(3, 190)])
    record(args.out, "lognormal_s256", rm, 256, params=gamma_params(rng, 200, 256))


if __name__ == "__main__":
    main()

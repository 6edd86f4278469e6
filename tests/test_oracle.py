"""CPU checks of the oracle itself (no GPU).

The oracle (oracle/wmh_oracle.c and its numpy twin in oracle/oracle.py)
restates kernel.cu:95-110 of the reference.  These tests pin it:
  * the C and numpy restatements agree bit for bit, in both FMA forms, on
    random inputs and on the edge cases the reference's semantics define;
  * on the reference's own fixtures (test.py:13-14, 35-39, 185-189) it agrees
    with a float64 restatement of the datasketch algorithm the reference's
    tests compare against (test.py:22-26, 51-56, 142-146, 201-204);
  * on golden vectors recorded from the reference build on a B200
    (tests/golden/, made by tests/golden/make_golden.py) it reproduces the
    reference's output exactly.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from wmh_testlib import gamma_params, random_csr, selected

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("form", [O.FORM_UNFUSED, O.FORM_FUSED])
@pytest.mark.parametrize("samples", [1, 3, 64, 128])
def test_c_matches_numpy_random(form, samples):
    rng = np.random.default_rng(100 + samples)
    dim = 300
    rs, lc, b = gamma_params(rng, dim, samples)
    m = random_csr(rng, 200, dim, 20, empty_frac=0.05, zero_frac=0.05)
    co = O.COracle(rs, lc, b)
    a = co.hash_csr(m, form=form)
    n = O.hash_numpy(rs, lc, b, m.data, m.indices, m.indptr, form=form)
    assert a.shape == (200, samples, 2)
    np.testing.assert_array_equal(a, n)


def test_forms_differ_on_crafted_cells():
    """The crafted near-tie cells the GPU test uses really separate the forms."""
    from test_gpu_reference import crafted_form_case
    rs, lc, b, m = crafted_form_case(np.random.default_rng(5), rows=8, samples=32)
    co = O.COracle(rs, lc, b)
    f = co.hash_csr(m, form=O.FORM_FUSED)
    u = co.hash_csr(m, form=O.FORM_UNFUSED)
    assert (f != u).any(axis=2).mean() > 0.9
    nf = O.hash_numpy(rs, lc, b, m.data, m.indices, m.indptr, form=O.FORM_FUSED)
    nu = O.hash_numpy(rs, lc, b, m.data, m.indices, m.indptr, form=O.FORM_UNFUSED)
    np.testing.assert_array_equal(f, nf)
    np.testing.assert_array_equal(u, nu)


def test_edge_semantics():
    """kernel.cu:79,106: strict '<' against FLT_MAX; first position wins ties;
    zero / negative / NaN weights are never selected; empty rows give the
    sentinel; the column is reported as stored."""
    dim, samples = 8, 4
    rs = np.ones((samples, dim), np.float32)
    lc = np.zeros((samples, dim), np.float32)
    b = np.full((samples, dim), 0.5, np.float32)
    # Row 0: two identical entries in columns 3 and 5 -> column 3 (first) wins.
    # Row 1: empty.  Row 2: zero, negative, NaN weights only.  Row 3: the same
    # column twice with equal weights -> first occurrence (same k either way).
    data = np.array([2.0, 2.0, 0.0, -1.0, np.nan, 4.0, 4.0], np.float32)
    cols = np.array([3, 5, 1, 2, 3, 6, 6], np.uint32)
    rows = np.array([0, 2, 2, 5, 7], np.uint32)
    co = O.COracle(rs, lc, b)
    for form in (0, 1):
        out = co.hash(data, cols, rows, form=form)
        nout = O.hash_numpy(rs, lc, b, data, cols, rows, form=form)
        np.testing.assert_array_equal(out, nout)
        assert (out[0, :, 0] == 3).all()
        assert (out[1] == 0xFFFFFFFF).all()
        assert (out[2] == 0xFFFFFFFF).all()
        assert (out[3, :, 0] == 6).all()
        t = np.floor(np.log(np.float32(2.0)) / 1 + 0.5)
        assert (out[0, :, 1] == np.uint32(int(t))).all()


def test_rows_offset_is_absolute():
    """rows[0] != 0 addresses weights/cols absolutely (minhashcuda.cc:447-452)."""
    rng = np.random.default_rng(7)
    rs, lc, b = gamma_params(rng, 50, 16)
    m = random_csr(rng, 30, 50, 6)
    co = O.COracle(rs, lc, b)
    full = co.hash_csr(m)
    part = co.hash(m.data, m.indices, m.indptr[10:21])
    np.testing.assert_array_equal(part, full[10:20])


def test_negative_t_and_saturation():
    """(uint32)(int32)t keeps negative t as two's complement (test.py:198),
    and the conversion saturates like the GPU's."""
    t = np.array([-1.0, -2.5, 3e9, -3e9, np.nan, 7.9], np.float32)
    np.testing.assert_array_equal(O.gpu_f2i(t), [-1, -2, 2**31 - 1, -2**31, 0, 7])
    rs = np.full((2, 2), 0.5, np.float32)
    lc = np.zeros((2, 2), np.float32)
    b = np.zeros((2, 2), np.float32)
    co = O.COracle(rs, lc, b)
    out = co.hash(np.array([0.1], np.float32), np.array([1], np.uint32),
                  np.array([0, 1], np.uint32))
    t = int(np.floor(np.log(np.float32(0.1)) / np.float32(0.5)))
    assert t < 0
    assert out[0, 0, 1] == np.uint32(t & 0xFFFFFFFF)


def _ds_params(dim, samples=128, seed=1):
    rs, lc, b = O.datasketch_params(dim, samples, seed)
    return rs, lc, b


def test_tiny_fixture_against_datasketch_restatement():
    """test.py:12-32: datasketch parameters injected (as float32), exact
    equality with datasketch's float64 hashes of the two tiny vectors."""
    rs, lc, b = _ds_params(len(O.TINY_V1))
    import scipy.sparse as sp
    m = sp.csr_matrix(np.array([O.TINY_V1, O.TINY_V2], np.float32))
    out = O.COracle(rs.astype(np.float32), lc.astype(np.float32), b.astype(np.float32)).hash_csr(m)
    want = np.stack([O.datasketch_f64(rs, lc, b, O.TINY_V1),
                     O.datasketch_f64(rs, lc, b, O.TINY_V2)]).astype(np.uint32)
    np.testing.assert_array_equal(out, want)


def test_float_fixture_against_datasketch_restatement():
    """test.py:184-210 with float32 parameters on both sides, compared as int32."""
    rng = np.random.default_rng(7)
    rs, lc, b = gamma_params(rng, len(O.FLOAT_V), 128)
    import scipy.sparse as sp
    m = sp.csr_matrix(np.array([O.FLOAT_V], np.float32))
    out = O.COracle(rs, lc, b).hash_csr(m).astype(np.int32)
    v32 = np.array(O.FLOAT_V, np.float32).astype(np.float64)
    want = O.datasketch_f64(rs, lc, b, v32)[None].astype(np.int32)
    np.testing.assert_array_equal(out, want)


def test_small_matrix_against_datasketch_restatement():
    """test.py:34-64 (seed 0, 6400x130, datasketch parameters): the reference
    claims bit equality with datasketch; the oracle must agree on this
    fixture.  Checked on every 8th row to keep the CPU suite short."""
    data, m = O.reference_small_matrix(0)
    rs, lc, b = _ds_params(130)
    out = O.COracle(rs.astype(np.float32), lc.astype(np.float32), b.astype(np.float32)).hash_csr(m)
    for r in range(0, 6400, 8):
        want = O.datasketch_f64(rs, lc, b, data[r]).astype(np.uint32)
        np.testing.assert_array_equal(out[r], want, err_msg=f"row {r}")


def test_golden_vectors():
    """Golden outputs recorded from the reference build on a B200."""
    files = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
    if not files:
        pytest.skip("no golden vectors recorded yet")
    for f in files:
        g = np.load(f)
        co = O.COracle(g["rs"], g["ln_cs"], g["betas"])
        out = co.hash(g["weights"], g["cols"], g["rows"], form=O.REFERENCE_FORM, lnw=g["lnw"])
        ref = g["ref_out"]
        mask = selected(out)
        np.testing.assert_array_equal(out[mask], ref[mask], err_msg=os.path.basename(f))
        # Cells with no selectable entry are undefined in the reference.
        assert mask.mean() > 0.5


def test_every_recorded_golden_case_is_committed():
    """Each case tests/golden/make_golden.py records from the reference build
    has its file here, so test_golden_vectors pins all of them."""
    import re
    src = open(os.path.join(GOLDEN, "make_golden.py")).read()
    names = set(re.findall(r'record\(args\.out, "([a-z0-9_]+)"', src))
    have = {os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    assert names and names <= have, sorted(names - have)

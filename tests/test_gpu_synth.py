"""The synthetic workloads are pure functions of (seed, row): any row range
regenerates bit for bit, which the benchmark relies on to check and time a
CPU sample of rows it hashed on the GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["large", "streamed", "batched"])
def test_row_ranges_regenerate_identically(name):
    from minhashcuda_b200 import synth
    w = synth.WORKLOADS[name]
    ip, cols, wts = synth.host_csr(w, 0, 3000)
    ip2, cols2, wts2 = synth.host_csr(w, 1000, 1000)
    a, b = ip[1000], ip[2000]
    np.testing.assert_array_equal(ip2, ip[1000:2001] - a)
    np.testing.assert_array_equal(cols2, cols[a:b])
    np.testing.assert_array_equal(wts2, wts[a:b])
    ip3, cols3, wts3 = synth.host_csr(w, 0, 3000)
    np.testing.assert_array_equal(cols3, cols)
    # rows hold distinct, sorted, in-range columns
    for r in range(0, 3000, 97):
        c = cols[ip[r]:ip[r + 1]].astype(np.int64)
        assert (np.diff(c) > 0).all() and (c < w.dim).all()
    lens = np.diff(ip.astype(np.int64))
    assert lens.min() >= w.nnz_lo

"""Device-side LSH band keys and Jaccard estimates over device-resident
hashes, against their numpy restatements; and the estimate against the true
weighted Jaccard similarity as the reference's integration test checks it
(test.py:92-110)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _hash_on_device(lib, gen, m, samples):
    import torch
    ip = torch.from_numpy(m.indptr.astype(np.int64).astype(np.uint32).view(np.int32)).cuda()
    cols = torch.from_numpy(m.indices.astype(np.uint32).view(np.int32)).cuda()
    w = torch.from_numpy(m.data.astype(np.float32)).cuda()
    out = torch.empty((m.shape[0], samples, 2), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert lib.mhcuda_calc_device(gen, w.data_ptr(), cols.data_ptr(), ip.data_ptr(), m.shape[0],
                                  m.nnz, out.data_ptr(), None) == 0
    assert lib.mhcuda_device_status(gen) == 0
    return out


def test_bands_and_jaccard_match_restatement_and_truth():
    import torch
    import minhashcuda_b200 as mb
    lib = mb.capi()
    data, m = O.reference_small_matrix(1)
    gen = lib.mhcuda_init(130, 128, 1, 0, 1, 0, None)
    assert gen
    try:
        d_out = _hash_on_device(lib, gen, m, 128)
        hashes = d_out.cpu().numpy().view(np.uint32)
        for width in (1, 4, 16, 128):
            keys = torch.empty((m.shape[0], 128 // width), dtype=torch.int64, device="cuda")
            assert lib.mhcuda_lsh_bands(gen, d_out.data_ptr(), m.shape[0], width,
                                        keys.data_ptr(), None) == 0
            np.testing.assert_array_equal(keys.cpu().numpy().view(np.uint64),
                                          O.lsh_band_keys(hashes, width))
        rng = np.random.default_rng(3)
        pairs = rng.integers(0, m.shape[0], (5000, 2)).astype(np.uint32)
        pairs[0] = (0, 1)
        pairs[1] = (7, 7)
        pairs[2] = (0, 6400)  # out of range -> -1
        d_pairs = torch.from_numpy(pairs.view(np.int32)).cuda()
        est = torch.empty(len(pairs), dtype=torch.float32, device="cuda")
        assert lib.mhcuda_jaccard(gen, d_out.data_ptr(), m.shape[0], d_pairs.data_ptr(),
                                  len(pairs), est.data_ptr(), None) == 0
        got = est.cpu().numpy()
        assert got[2] == -1.0 and got[1] == 1.0
        keep = np.ones(len(pairs), bool)
        keep[2] = False
        np.testing.assert_array_equal(got[keep], O.jaccard_estimate(hashes, pairs[keep]))
        # test.py:104-110: estimate of rows 0 and 1 within 0.005 of the truth
        truth = np.minimum(data[0], data[1]).sum() / np.maximum(data[0], data[1]).sum()
        assert abs(got[0] - truth) < 0.005
    finally:
        lib.mhcuda_fini(gen)

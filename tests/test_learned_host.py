"""Host-side logic of the 128-wide learned index (no GPU): the query rows
the selection kernel reads, the merge of its two columns per query back to
one candidate list, and the principal-direction projection."""
import numpy as np
import torch

from sseqs_b200 import learned


def _index(n, dim=128):
    idx = object.__new__(learned.LearnedIndex)
    idx.n, idx.dim = n, dim
    return idx


def test_wide_query_rows_hold_each_code_in_one_half():
    q = torch.arange(3 * 128, dtype=torch.int64).reshape(3, 128).to(torch.uint8)
    w = _index(10)._wide(q)
    assert w.shape == (6, 256)
    for i in range(3):
        assert torch.equal(w[2 * i, :128], q[i]) and not w[2 * i, 128:].any()
        assert torch.equal(w[2 * i + 1, 128:], q[i]) and not w[2 * i + 1, :128].any()
    full = torch.ones((2, 256), dtype=torch.uint8)
    assert torch.equal(_index(10, 256)._wide(full), full)


def test_merge_columns_maps_pairs_back_to_codes():
    """Row r of column 2i is code 2r and of column 2i + 1 code 2r + 1; the
    spare zero row (code n when n is odd) and entries past a column's count
    are dropped; each query's entries come first in its row, column 2i's
    before column 2i + 1's."""
    n, cap = 9, 4                          # codes 0..8, spare row 9
    cand = torch.tensor([[0, 3, 4, 7],     # query 0, even codes: 0 6 8 (14: past count)
                         [4, 1, 0, 0],     # query 0, odd codes: 9 (spare) 3
                         [2, 2, 2, 2],     # query 1, even: count 0
                         [0, 1, 2, 3]])    # query 1, odd: 1 3 5 7 (count 6 > cap)
    cs = cand.to(torch.float32) + 0.5
    cnt = np.array([3, 2, 0, 6])
    out, out_s, counts, cap2 = _index(n)._merge_columns(cand, cs, cnt, cap)
    assert cap2 == 2 * cap
    assert counts.tolist() == [4, 4]
    assert out[0, :4].tolist() == [0, 6, 8, 3]
    assert out[1, :4].tolist() == [1, 3, 5, 7]
    assert out_s[0, :4].tolist() == [0.5, 3.5, 4.5, 1.5]
    assert out_s[1, :4].tolist() == [0.5, 1.5, 2.5, 3.5]


def test_merge_keeps_odd_code_after_even_of_same_query():
    cand = torch.tensor([[1, 0], [1, 0]])
    cs = torch.tensor([[1.0, 0.0], [2.0, 0.0]])
    out, out_s, counts, _ = _index(4)._merge_columns(cand, cs, np.array([1, 1]), 2)
    assert counts.tolist() == [2]
    assert out[0, :2].tolist() == [2, 3]
    assert out_s[0, :2].tolist() == [1.0, 2.0]


def test_principal_directions_keep_the_dominant_subspace():
    """Embeddings that live in an 8-dimensional subspace keep their dot
    products exactly after projection onto 8 principal directions."""
    g = torch.Generator().manual_seed(0)
    basis, _ = torch.linalg.qr(torch.randn(256, 8, generator=g, dtype=torch.float64))
    x = torch.randn(2000, 8, generator=g, dtype=torch.float64) @ basis.T
    x = (x / x.norm(dim=1, keepdim=True)).to(torch.float32)
    p = learned.principal_directions(x, 8)
    assert p.shape == (256, 8)
    assert torch.allclose(p.T @ p, torch.eye(8), atol=1e-5)
    y = learned.project(x, p)
    assert torch.allclose(y.norm(dim=1), torch.ones(2000), atol=1e-5)
    assert torch.allclose(y @ y.T, x @ x.T, atol=1e-4)

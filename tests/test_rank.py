"""Global ranking of batch hits (sseqs/msa.py:411-427): the vectorised
``rank_hits`` equals a plain row-by-row restatement of the reference's sort,
ties between batches included; CPU tensors, no GPU."""
import importlib

import numpy as np
import pytest
import torch

M = importlib.import_module("sseqs_b200.msa")


def _plain(query, per_batch, num_msas):
    rows = []
    for bh in per_batch:
        if bh is None:
            continue
        g, aff, lin = bh.g.numpy(), bh.affine.numpy(), bh.linear.numpy()
        hb, hl = bh.hits.numpy(), bh.hit_len.numpy()
        norm = M._norm(aff, len(query), bh.maxlen)
        for r in range(g.size):
            rows.append((float(norm[r]), bh.batch, int(g[r]), int(aff[r]), int(lin[r]),
                         hb[r, :hl[r]].tobytes().decode("latin-1")))
    rows.sort(key=lambda x: (-x[0], x[1], x[2]))
    return rows[:num_msas]


def _batches(rng, n_batches, per, maxlens):
    out = []
    for bi in range(n_batches):
        n = int(per[bi])
        g = np.sort(rng.choice(100_000, n, replace=False)).astype(np.int32)
        aff = rng.integers(0, 40, n).astype(np.int32)          # many equal scores
        lin = rng.integers(0, 400, n).astype(np.int32)
        hl = rng.integers(0, 33, n).astype(np.int32)
        hits = rng.integers(64, 96, (n, 32)).astype(np.uint8)
        hits[:, :3] = [0xe9, 0x40, 0x7a]                       # latin-1, '@', lower case
        out.append(M.BatchHits(bi, torch.from_numpy(g), torch.from_numpy(aff),
                               torch.from_numpy(lin), torch.from_numpy(hits),
                               torch.from_numpy(hl), int(maxlens[bi]), 0, 0))
    return out


@pytest.mark.parametrize("seed", range(5))
@pytest.mark.parametrize("num_msas", [1, 50, 4096])
def test_rank_hits_equals_plain_sort(seed, num_msas):
    rng = np.random.default_rng(seed)
    nb = 4
    per = rng.integers(0, 300, nb)
    maxlens = [500, 500, 800, 500]                             # equal norms across batches
    batches = _batches(rng, nb, per, maxlens)
    batches.insert(2, None)                                   # a batch without hits
    q = "M" * int(rng.integers(20, 900))
    assert M.rank_hits(q, batches, num_msas) == _plain(q, batches, num_msas)


def test_rank_hits_empty():
    assert M.rank_hits("MKT", [None], 10) == []
    empty = M.BatchHits(0, torch.zeros(0, dtype=torch.int32), torch.zeros(0, dtype=torch.int32),
                        torch.zeros(0, dtype=torch.int32), torch.zeros((0, 8), dtype=torch.uint8),
                        torch.zeros(0, dtype=torch.int32), 10, 0, 0)
    assert M.rank_hits("MKT", [empty], 10) == []


def test_timings_have_the_reference_keys():
    """msa(..., return_timings=True) returns the reference's dict: the keys
    of sseqs/msa.py:442-446, seconds as floats, stages this build does not
    have at 0."""
    ref_keys = {"t_dec", "t_prep1", "t_prep2", "t_fft", "t_prep_fft", "t_sw", "t_out",
                "t_out_cpu", "t_log", "t_topk1", "t_topk2", "t_save", "t_prep_sw", "t_a3m",
                "t_to_vram"}
    st = M.SearchStats()
    st.add("t_sw", 0.25)
    st.add("t_sw", 0.5)
    st.add("t_search", 1.0)             # internal, not part of the reference's dict
    t = st.timings()
    assert set(t) == ref_keys
    assert t["t_sw"] == 0.75 and t["t_fft"] == 0.0
    assert all(isinstance(v, float) for v in t.values())

"""GPU tests of the batched path: many queries of one stripe width in one
launch give exactly the scores of their single-query launches, and the
bucketed, graph-replayed search gives exactly the per-query top-k."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _db(n_seqs=3000, chunk_bytes=120_000, seed=3):
    from sseqs_b200 import dbtools
    from sseqs_b200.database import Database
    q = dbtools.random_query(300, seed)
    syn = dbtools.synthetic_db([q], n_seqs, 0.02, (0.3, 0.9), seed=seed, device="cpu",
                               chunk_bytes=chunk_bytes)
    return q, Database(syn.chunks, bs=chunk_bytes)


def _pack(queries):
    sw = importlib.import_module("sseqs_b200.sw")
    enc = [sw.encode_query(q) for q in queries]
    buf = torch.zeros((len(enc), 2048), dtype=torch.uint8, device="cuda")
    for i, e in enumerate(enc):
        buf[i, :e.numel()] = e
    lens = torch.tensor([e.numel() for e in enc], dtype=torch.int32, device="cuda")
    return enc, buf, lens


@pytest.fixture(params=[False, True], ids=["one_per_row", "pairs"])
def pairing(request):
    """Run a test with the query-pair kernel off, then on, at every width."""
    from sseqs_b200 import tune
    before = [tune.get_query_pairing(t) for t in range(1, 65)]
    tune.set_query_pairing(0, request.param)
    yield request.param
    for t, on in enumerate(before, 1):
        tune.set_query_pairing(t, on)


@pytest.mark.parametrize("lengths", [[300, 289, 320, 300, 305], [40, 33, 64], [2048, 2017],
                                     [7, 1, 32, 20]])
@pytest.mark.parametrize("affine", [False, True])
def test_scan_queries_equals_single_query_scans(lengths, affine, pairing):
    from sseqs_b200 import batched, dbtools
    sw = importlib.import_module("sseqs_b200.sw")
    _, db = _db()
    b = db.batches[0]
    queries = [dbtools.random_query(L, 50 + i) for i, L in enumerate(lengths)]
    enc, buf, lens = _pack(queries)
    tpt = (lengths[0] + 31) // 32
    kw = dict(affine=affine, skip=1 if affine else 0, gap_a=11 if affine else -1, gap_b=1)
    n = b.n_segments - 2
    got = batched.sw_scan_queries(buf, lens, tpt, b.ascii, b.delim, g0=1, n_targets=n, **kw)
    # gathered targets too: every third segment, out of order
    idx = torch.arange(n, 0, -3, dtype=torch.int32, device="cuda")
    got_i = batched.sw_scan_queries(buf, lens, tpt, b.ascii, b.delim, good_idx=idx, **kw)
    # and one list per query
    gen = torch.Generator(device="cpu")
    gen.manual_seed(len(lengths))
    idx2 = torch.randint(1, n + 1, (len(enc), 257), generator=gen, dtype=torch.int32).cuda()
    got_2 = batched.sw_scan_queries(buf, lens, tpt, b.ascii, b.delim, good_idx=idx2, **kw)
    for i, e in enumerate(enc):
        exp = sw.sw_scan(e, b.ascii, b.delim, g0=1, n_targets=n, **kw)
        assert torch.equal(got[i, :n], exp), i
        exp_i = sw.sw_scan(e, b.ascii, b.delim, good_idx=idx, **kw)
        assert torch.equal(got_i[i, :idx.numel()], exp_i), i
        exp_2 = sw.sw_scan(e, b.ascii, b.delim, good_idx=idx2[i], **kw)
        assert torch.equal(got_2[i, :257], exp_2), i


def test_length_outside_the_launch_width_is_not_scored(pairing):
    from sseqs_b200 import batched, dbtools
    _, db = _db()
    b = db.batches[0]
    enc, buf, lens = _pack([dbtools.random_query(100, 1), dbtools.random_query(100, 2)])
    lens[1] = 130                      # ceil(130/32) = 5, the launch is tpt 4
    out = batched.sw_scan_queries(buf, lens, 4, b.ascii, b.delim, affine=True, g0=1,
                                  n_targets=500, skip=1, gap_a=11, gap_b=1)
    assert bool((out[1, :500] == torch.iinfo(torch.int32).min).all())
    assert bool((out[0, :500] >= 0).all())


def _per_query_topk(db, enc, k):
    from sseqs_b200 import select
    sw = importlib.import_module("sseqs_b200.sw")
    rows = []
    for bi, b in enumerate(db.batches):
        n = b.n_segments - 2
        if n <= 0:
            continue
        s = sw.sw_scan(enc, b.ascii, b.delim, affine=True, g0=1, n_targets=n, skip=1,
                       gap_a=11, gap_b=1)
        kk = min(k, n)
        p = select.topk_indices(s, kk).long()
        for t, v in zip(p.cpu().numpy(), s[p].cpu().numpy()):
            rows.append((-int(v), bi, int(t) + 1))
    rows.sort()
    return rows[:k]


@pytest.mark.parametrize("use_graphs", [True, False])
def test_search_queries_matches_per_query_topk(use_graphs, pairing):
    from sseqs_b200 import batched, dbtools
    _, db = _db()
    rng = np.random.default_rng(11)
    lengths = [int(x) for x in np.clip(np.round(np.exp(rng.normal(np.log(300), 0.7, 9))), 16,
                                       2048)]
    lengths += [lengths[0], lengths[0] + 1, lengths[0]]   # same width: groups of 2 replay
    queries = [dbtools.random_query(L, 200 + i) for i, L in enumerate(lengths)]
    got = batched.search_queries(queries, db, top_k=50, use_graphs=use_graphs, group=2)
    sw = importlib.import_module("sseqs_b200.sw")
    for i, q in enumerate(queries):
        exp = _per_query_topk(db, sw.encode_query(q), 50)
        h = got[i]
        mine = list(zip((-h.scores.astype(np.int64)).tolist(), h.batch.tolist(),
                        h.segment.tolist()))
        assert mine == exp, i


PAIR_LENGTHS = [1, 17, 33, 64, 65, 100, 129, 200, 257, 300, 416, 500, 545, 640, 700, 858, 929,
                1000, 1024, 1100, 1500, 1800, 2048]


@pytest.mark.parametrize("gaps", [(11, 1), (5, 2)], ids=["msa_gaps", "other_gaps"])
@pytest.mark.parametrize("L", PAIR_LENGTHS)
def test_query_pairs_equal_unpaired_launches(L, gaps):
    """Affine queries that share their targets are scored two per launch row
    (query 2y in the low, 2y + 1 in the high half of every word); the scores
    equal the one-query-per-row launch in both lane layouts, with an odd
    query count and with one half of a pair outside the launch width -- at
    msa()'s gaps (kernels with them built in) and at others."""
    from sseqs_b200 import batched, dbtools, tune
    _, db = _db()
    b = db.batches[0]
    tpt = (L + 31) // 32
    lengths = [L, max(32 * (tpt - 1) + 1, L - 7), L, 32 * tpt, max(32 * (tpt - 1) + 1, L - 3)]
    queries = [dbtools.random_query(x, 900 + i) for i, x in enumerate(lengths)]
    enc, buf, lens = _pack(queries)
    lens[3] = 32 * tpt + 1             # another width: not scored in either form
    n = b.n_segments - 2
    kw = dict(affine=True, g0=1, n_targets=n, skip=1, gap_a=gaps[0], gap_b=gaps[1])
    before = tune.get_variant(3, tpt), tune.get_query_pairing(tpt)
    try:
        tune.set_query_pairing(tpt, False)
        ref = batched.sw_scan_queries(buf, lens, tpt, b.ascii, b.delim, **kw)
        tune.set_query_pairing(tpt, True)
        for wide in (0, 1):
            tune.set_variant(3, tpt, wide)
            got = batched.sw_scan_queries(buf, lens, tpt, b.ascii, b.delim, **kw)
            assert torch.equal(got[:, :n], ref[:, :n]), wide
    finally:
        tune.set_variant(3, tpt, before[0])
        tune.set_query_pairing(tpt, before[1])
    assert bool((ref[3, :n] == torch.iinfo(torch.int32).min).all())

"""GPU test of the search server: requests that arrive while others are in
flight share engine steps, and each result equals the one-query-at-a-time
search of the same query (identical integer scores and hit lists)."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_single_query_search():
    from sseqs_b200 import dbtools, select, serve
    from sseqs_b200.database import Database
    sw = importlib.import_module("sseqs_b200.sw")
    q0 = dbtools.random_query(250, 7)
    syn = dbtools.synthetic_db([q0], 3000, 0.02, (0.3, 0.9), seed=7, device="cpu",
                               chunk_bytes=100_000)
    db = Database(syn.chunks, bs=100_000)
    rng = np.random.default_rng(5)
    queries = [q0] + [dbtools.random_query(int(L), 300 + i)
                      for i, L in enumerate(rng.integers(20, 700, 9))]
    ex = serve.GpuExecutor(db, top_k=64)
    srv = serve.SearchServer(ex, top_k=64, max_slots=4)
    reqs = [srv.submit(q) for q in queries[:3]]
    srv.step()
    reqs += [srv.submit(q) for q in queries[3:6]]
    srv.step()
    reqs += [srv.submit(q) for q in queries[6:]]
    while srv.step():
        pass
    assert len(db.batches) > 1
    for q, r in zip(queries, reqs):
        enc = sw.encode_query(q)
        rows = []
        for bi, b in enumerate(db.batches):
            n = b.n_segments - 2
            if n <= 0:
                continue
            s = sw.sw_scan(enc, b.ascii, b.delim, affine=True, g0=1, n_targets=n, skip=1,
                           gap_a=11, gap_b=1)
            p = select.topk_indices(s, min(64, n)).long()
            for t, v in zip(p.cpu().numpy(), s[p].cpu().numpy()):
                rows.append((-int(v), bi, int(t) + 1))
        rows.sort()
        exp = rows[:64]
        h = r.result
        got = list(zip((-h.scores.astype(np.int64)).tolist(), h.batch.tolist(),
                       h.segment.tolist()))
        assert got == exp


def test_learned_executor_results_do_not_depend_on_the_mix():
    from sseqs_b200 import dbtools, learned, serve
    from sseqs_b200.database import Database
    q0 = dbtools.random_query(200, 17)
    syn = dbtools.synthetic_db([q0], 3000, 0.02, (0.5, 0.95), seed=17, device="cpu",
                               chunk_bytes=100_000)
    db = Database(syn.chunks, bs=100_000)
    model = learned.Embedder(seed=4)
    learned.train(model, learned.training_pairs(16, 32, seed=4), queries_per_step=8,
                  targets_per_query=16)
    index = learned.LearnedIndex(model, db, chunk=1000)
    rng = np.random.default_rng(3)
    queries = [q0] + [dbtools.random_query(int(L), 500 + i)
                      for i, L in enumerate(rng.integers(30, 600, 5))]
    alone = []
    for q in queries:
        srv = serve.SearchServer(serve.LearnedExecutor(index, top_k=40, n_cand=200), top_k=40)
        r = srv.submit(q)
        while srv.step():
            pass
        alone.append(r.result)
    srv = serve.SearchServer(serve.LearnedExecutor(index, top_k=40, n_cand=200), top_k=40)
    reqs = [srv.submit(q) for q in queries[:2]]
    srv.step()
    reqs += [srv.submit(q) for q in queries[2:]]
    while srv.step():
        pass
    for a, r in zip(alone, reqs):
        assert np.array_equal(a.scores, r.result.scores)
        assert np.array_equal(a.batch, r.result.batch)
        assert np.array_equal(a.segment, r.result.segment)

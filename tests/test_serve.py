"""Host-side tests of the search server's scheduling (no GPU): admission by
slots and memory, one database batch per engine step for every request in
flight, completion after one full cycle, and results that do not depend on
which requests ran together."""
import threading
import zlib

import numpy as np
import pytest

from sseqs_b200 import serve


class HostExecutor:
    """Deterministic stand-in for the GPU step: a segment's score is a hash
    of (query, batch, segment); top-k per batch with index tie-break."""

    def __init__(self, n_batches=5, n_segments=300, top_k=20):
        self._nb, self.nseg, self.top_k = n_batches, n_segments, top_k
        self.calls = []

    @property
    def n_batches(self):
        return self._nb

    @staticmethod
    def request_bytes(top_k, n_batches):
        return 1000

    def prepare(self, req):
        if not req.query or not req.query.isalpha():
            raise ValueError("bad query")
        req.enc = req.query

    def scores(self, query, bi):
        seed = zlib.crc32(f"{query}/{bi}".encode())
        return np.random.default_rng(seed).integers(0, 50, self.nseg).astype(np.int32)

    def step(self, bi, reqs):
        self.calls.append((bi, [r.rid for r in reqs]))
        out = []
        for r in reqs:
            s = self.scores(r.enc, bi)
            order = np.lexsort((np.arange(s.size), -s.astype(np.int64)))[:self.top_k]
            out.append(((order + 1).astype(np.int32), s[order]))
        return out


def _alone(query, **kw):
    ex = HostExecutor(**kw)
    srv = serve.SearchServer(ex, top_k=ex.top_k)
    r = srv.submit(query)
    while srv.step():
        pass
    return r.result


def test_result_is_the_same_alone_and_in_the_mix():
    ex = HostExecutor()
    srv = serve.SearchServer(ex, top_k=ex.top_k, max_slots=3)
    queries = ["ACDE", "MKV", "WWWY", "PLKQ", "GGA", "TT", "HHHH"]
    reqs = [srv.submit(queries[0]), srv.submit(queries[1])]
    srv.step()
    reqs.append(srv.submit(queries[2]))          # arrives while two are in flight
    srv.step()
    srv.step()
    reqs += [srv.submit(q) for q in queries[3:]]  # more than the free slots
    while srv.step():
        pass
    assert not srv.inflight and not srv.pending
    for q, r in zip(queries, reqs):
        exp = _alone(q)
        assert np.array_equal(r.result.scores, exp.scores)
        assert np.array_equal(r.result.batch, exp.batch)
        assert np.array_equal(r.result.segment, exp.segment)
        assert r.done.is_set()


def test_every_request_sees_each_batch_once_from_where_it_joined():
    ex = HostExecutor(n_batches=4)
    srv = serve.SearchServer(ex, top_k=ex.top_k, max_slots=8)
    a = srv.submit("AAA")
    srv.step()
    b = srv.submit("CCC")
    while srv.step():
        pass
    seen = {a.rid: [], b.rid: []}
    for bi, rids in ex.calls:
        for rid in rids:
            seen[rid].append(bi)
    assert seen[a.rid] == [0, 1, 2, 3]
    assert seen[b.rid] == [1, 2, 3, 0]
    assert a.start_batch == 0 and b.start_batch == 1


def test_admission_respects_slots_and_memory():
    ex = HostExecutor(n_batches=3)
    free = {"bytes": 10_500}
    srv = serve.SearchServer(ex, top_k=ex.top_k, max_slots=2, memory_reserve=8_000,
                             free_memory=lambda: free["bytes"])
    reqs = [srv.submit(q) for q in ["AA", "CC", "DD"]]
    srv.step()
    assert len(srv.inflight) == 2 and len(srv.pending) == 1       # slot limit
    free["bytes"] = 8_500                                          # < reserve + 1000
    while srv.inflight:
        srv.step()
    assert len(srv.pending) == 1                                   # memory limit holds it
    free["bytes"] = 20_000
    while srv.step():
        pass
    assert all(r.done.is_set() for r in reqs)


def test_bad_request_fails_alone():
    ex = HostExecutor(n_batches=2)
    srv = serve.SearchServer(ex, top_k=ex.top_k)
    good, bad = srv.submit("ACD"), srv.submit("12")
    while srv.step():
        pass
    assert isinstance(bad.result, ValueError)
    assert isinstance(good.result, serve.Hits) and good.result.scores.size == ex.top_k


def test_threaded_server_with_poisson_arrivals():
    ex = HostExecutor(n_batches=3)
    srv = serve.SearchServer(ex, top_k=ex.top_k, max_slots=4).start()
    try:
        queries = [("ACDEFGHIKL"[i % 10] * (1 + i % 5)) for i in range(40)]
        offs = serve.poisson_arrivals(len(queries), rate=2000.0, seed=1)
        reqs = serve.replay(srv, queries, offs)
    finally:
        srv.stop()
    st = serve.stats(reqs, max(1e-6, max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)))
    assert st.completed == 40 and st.p99_ms >= st.p50_ms > 0
    for q, r in zip(queries, reqs):
        exp = _alone(q, n_batches=3)
        assert np.array_equal(r.result.segment, exp.segment)


def test_learned_request_bytes_follow_the_index_width():
    """Admission by memory counts a 128-wide index's two selection columns
    and merged list per query (4x the candidate bytes of a 256-wide one)."""
    class Index:
        def __init__(self, dim):
            self.dim = dim
    wide = serve.LearnedExecutor(Index(256), top_k=4096, n_cand=32768)
    half = serve.LearnedExecutor(Index(128), top_k=4096, n_cand=32768)
    assert wide.request_bytes(4096, 5) == 8 * 12 * 32768 + 16 * 4096
    assert half.request_bytes(4096, 5) == 4 * 8 * 12 * 32768 + 16 * 4096

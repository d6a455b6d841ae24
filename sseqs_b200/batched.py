"""Many queries of uneven length against the resident database.

The reference searches one query at a time (sseqs/msa.py:235: a Python loop
over queries, each sweeping every batch).  Here the queries are grouped by
stripe width (tpt = ceil(len/32), which fixes the score kernel's shape and
the reference's stripe rule), and each group of up to 128 queries sweeps a
database batch in ONE launch (``sseqs_sw_scan_queries``: blockIdx.y picks
the query, each query has its own target counter), followed by the per-query
top-k.  The launches of a group over all batches are captured once into a
CUDA graph keyed by (tpt, group size); a later group of the same shape copies
its queries into the graph's query buffer and replays it.  The lane layout
of each width is chosen by the autotuner (``tune.autotune``) before capture.

Scores are those of the per-query path: every query's score of every target
equals its own ``sw.sw_scan`` call (both run the same kernel template; the
batched launch only changes which query a block reads).
"""
from __future__ import annotations

import importlib
from dataclasses import dataclass

import numpy as np
import torch

from . import select, tune
from ._lib import check, lib, ptr, stream_ptr, to_device, to_host

_sw = importlib.import_module("sseqs_b200.sw")

MAX_QUERY = 2048
GROUP = 128                 # queries per launch (kMaxLaunchQueries)


def sw_scan_queries(queries: torch.Tensor, lens: torch.Tensor, tpt: int, ascii: torch.Tensor,
                    delim: torch.Tensor, *, affine: bool, good_idx: torch.Tensor | None = None,
                    g0: int = 0, n_targets: int | None = None, skip: int = 0, gap_a: int = -1,
                    gap_b: int = 0, out: torch.Tensor | None = None,
                    tickets: torch.Tensor | None = None) -> torch.Tensor:
    """Scores ``[len(lens), n]`` of several queries of stripe width ``tpt``.

    ``queries`` is a uint8 device tensor ``[>= len(lens), stride]`` of residue
    classes, row i holding ``lens[i]`` of them (``lens``: device int32, every
    ``ceil(len/32) == tpt``; a row that breaks this is filled with INT32_MIN);
    target selection and gap parameters are those of ``sw.sw_scan``, except
    that a 2-D ``good_idx`` gives every query its own row of targets.
    """
    nq = lens.numel()
    idx_stride = 0
    if good_idx is not None:
        good_idx = good_idx.to(torch.int32).contiguous()
        if good_idx.dim() == 2:
            idx_stride = good_idx.stride(0)
            n = good_idx.shape[1]
        else:
            n = good_idx.numel()
    else:
        n = int(n_targets)
    if out is None:
        out = torch.empty((nq, max(n, 1)), dtype=torch.int32, device=ascii.device)
    if tickets is None:
        tickets = torch.empty(max(nq, 1), dtype=torch.int32, device=ascii.device)
    check(lib().sseqs_sw_scan_queries(1 if affine else 0, nq, int(tpt), ptr(queries),
                                      queries.stride(0), ptr(lens), ptr(good_idx), idx_stride,
                                      int(g0), n,
                                      ptr(ascii), ptr(delim), int(skip), ptr(out), out.stride(0),
                                      int(gap_a), int(gap_b), ptr(tickets), stream_ptr()),
          "sw_scan_queries")
    return out


def buckets(lengths) -> dict:
    """Query indices grouped by stripe width, each group in length order."""
    out: dict = {}
    for i, L in sorted(enumerate(lengths), key=lambda x: (x[1], x[0])):
        out.setdefault(tune.tpt_of(L), []).append(i)
    return out


@dataclass
class QueryHits:
    """Top-k of one query over the database: score desc, then (batch, segment)
    (or normalised score desc when searched with ``rank="norm"``)."""
    scores: np.ndarray      # int32
    batch: np.ndarray       # int32
    segment: np.ndarray     # int32 (delimiter-based segment index g)
    norm: np.ndarray | None = None   # float32 score / sqrt(Lq * maxlen of the batch)


class _Scratch:
    """Buffers every group shares: one group runs at a time on the stream,
    so the score rows of one batch, the top-k workspace and the target
    counters are reused by all groups (and by their graphs)."""

    def __init__(self, db, rows: int):
        dev = db.device
        self.n = [max(b.n_segments - 2, 0) for b in db.batches]
        nmax = max(self.n + [1])
        self.scores = torch.empty((rows, nmax), dtype=torch.int32, device=dev)
        self.tickets = torch.empty(rows, dtype=torch.int32, device=dev)
        self.ws = torch.empty(lib().sseqs_topk_workspace_bytes(nmax), dtype=torch.uint8,
                              device=dev)


class _GroupPlan:
    """Static buffers and (optionally) the CUDA graph of one group shape."""

    def __init__(self, db, scratch: _Scratch, tpt: int, nq: int, top_k: int, gaps,
                 use_graph: bool):
        dev = db.device
        self.db, self.tpt, self.nq, self.top_k, self.gaps = db, tpt, nq, top_k, gaps
        self.q = torch.zeros((nq, MAX_QUERY), dtype=torch.uint8, device=dev)
        self.lens = torch.full((nq,), tpt * 32, dtype=torch.int32, device=dev)
        self.n = scratch.n
        self.scores = scratch.scores[:nq]
        self.tickets = scratch.tickets[:nq]
        self.ws = scratch.ws
        self.kb = [min(top_k, n) for n in self.n]
        self.idx = [torch.empty((nq, max(k, 1)), dtype=torch.int32, device=dev) for k in self.kb]
        self.val = [torch.empty((nq, max(k, 1)), dtype=torch.int32, device=dev) for k in self.kb]
        self.graph = None
        self.use_graph = use_graph

    def _launches(self):
        open_, ext = self.gaps
        for bi, batch in enumerate(self.db.batches):
            n, k = self.n[bi], self.kb[bi]
            if n <= 0 or k <= 0:
                continue
            sw_scan_queries(self.q, self.lens, self.tpt, batch.ascii, batch.delim, affine=True,
                            g0=1, n_targets=n, skip=1, gap_a=open_, gap_b=ext,
                            out=self.scores, tickets=self.tickets)
            for i in range(self.nq):
                row = self.scores[i, :n]
                select.topk_indices(row, k, out=self.idx[bi][i], ws=self.ws)
                torch.gather(row, 0, self.idx[bi][i, :k].long(), out=self.val[bi][i, :k])

    def run(self, enc: list[torch.Tensor]):
        """Scores the queries ``enc`` (device class tensors of this width):
        their residues and lengths go into the static buffers, then the
        captured graph replays (captured on first use, after one eager run
        that also serves as its warm-up)."""
        assert len(enc) == self.nq
        for i, e in enumerate(enc):
            assert tune.tpt_of(e.numel()) == self.tpt
            self.q[i, :e.numel()].copy_(e)
        self.lens.copy_(to_device(torch.tensor([int(e.numel()) for e in enc], dtype=torch.int32),
                                  self.lens.device))
        if not self.use_graph:
            self._launches()
            return
        if self.graph is None:
            self._launches()
            torch.cuda.synchronize()
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._launches()
            return
        self.graph.replay()


class BatchedSearcher:
    """Keeps the group plans (static buffers and captured graphs) of a
    database across calls, so later query sets replay the graphs."""

    def __init__(self, db, *, top_k: int = 4096, gap_open: int = 11, gap_extend: int = 1,
                 use_graphs: bool = True, autotune: bool = True, group: int = GROUP):
        self.db, self.top_k = db, int(top_k)
        self.gaps = (int(gap_open), int(gap_extend))
        self.use_graphs, self.autotune = use_graphs, autotune
        self.group = max(1, min(int(group), GROUP))
        self.plans: dict = {}
        self.scratch = _Scratch(db, self.group)

    def search(self, queries, rank: str = "score") -> list[QueryHits]:
        """Top-k per query over every batch: by affine score (``rank="score"``)
        or by normalised score (``"norm"``: float32 score over float32
        sqrt(Lq * maxlen of the hit's batch), the ranking of the exhaustive
        search, sseqs/msa.py:339-345), ties by batch, then segment.  A
        batch's own top-k is the same under both (one maxlen per batch)."""
        if rank not in ("score", "norm"):
            raise ValueError("rank is 'score' or 'norm'")
        if isinstance(queries, str):
            queries = [queries]
        db = self.db
        enc = [_sw.encode_query(q, device=db.device) for q in queries]
        lengths = [int(e.numel()) for e in enc]
        for L in lengths:
            if not 1 <= L <= MAX_QUERY:
                raise ValueError(f"query length {L} outside 1..{MAX_QUERY}")
        if self.autotune and db.batches:
            tune.autotune(lengths, db.batches[0])
            tune.autotune_pairing(lengths, db.batches[0])
        per_query: list = [None] * len(enc)
        for tpt, members in buckets(lengths).items():
            for s in range(0, len(members), self.group):
                grp = members[s:s + self.group]
                key = (tpt, len(grp))
                plan = self.plans.get(key)
                if plan is None:
                    plan = self.plans[key] = _GroupPlan(db, self.scratch, tpt, len(grp),
                                                        self.top_k, self.gaps, self.use_graphs)
                plan.run([enc[i] for i in grp])
                for j, qi in enumerate(grp):
                    per_query[qi] = _collect(plan, j, self.top_k,
                                             lengths[qi] if rank == "norm" else None)
        return per_query


def search_queries(queries, db, *, top_k: int = 4096, gap_open: int = 11, gap_extend: int = 1,
                   use_graphs: bool = True, autotune: bool = True,
                   group: int = GROUP) -> list[QueryHits]:
    """Affine scores of every query against every segment of ``db`` (the
    exact sweep of the affine stage, sseqs/msa.py:327-337, for all queries at
    once); returns each query's ``top_k`` hits over all batches.  ``group``
    (<= 128) bounds the queries of one launch."""
    return BatchedSearcher(db, top_k=top_k, gap_open=gap_open, gap_extend=gap_extend,
                           use_graphs=use_graphs, autotune=autotune, group=group).search(queries)


def _collect(plan: _GroupPlan, j: int, top_k: int, qlen: int | None = None) -> QueryHits:
    sc, bt, sg = [], [], []
    for bi, k in enumerate(plan.kb):
        if k <= 0 or plan.n[bi] <= 0:
            continue
        idx = to_host(plan.idx[bi][j, :k])
        sc.append(to_host(plan.val[bi][j, :k]))
        bt.append(np.full(k, bi, dtype=np.int32))
        sg.append((idx + 1).astype(np.int32))       # target t is segment g = t + 1
    if not sc:
        z = np.zeros(0, dtype=np.int32)
        return QueryHits(z, z, z)
    sc, bt, sg = np.concatenate(sc), np.concatenate(bt), np.concatenate(sg)
    if qlen is None:
        order = np.lexsort((sg, bt, -sc.astype(np.int64)))[:top_k]
        return QueryHits(sc[order], bt[order], sg[order])
    ml = np.array([b.maxlen for b in plan.db.batches], dtype=np.int64)[bt]
    norm = (sc.astype(np.float32) / np.sqrt((qlen * ml).astype(np.float32))).astype(np.float32)
    order = np.lexsort((sg, bt, -norm.astype(np.float64)))[:top_k]
    return QueryHits(sc[order], bt[order], sg[order], norm[order])

"""Search server: continuous batching of queries against the resident database.

The reference serves one request at a time (sseqs/server.py:30-110: a
ticket, a tar of a3m files, one ``msa()`` call per request).  Here requests
share the GPU while they run:

* the database stays resident in HBM (``database.Database``);
* an engine thread sweeps the database batches in a cycle; one engine step
  scores ONE batch for every request in flight (queries grouped by stripe
  width, up to 128 per launch, ``batched.sw_scan_queries``) and keeps each
  request's top-k of that batch;
* a request that arrives while others run is admitted at the next step, as
  soon as a slot and the device memory for its buffers are free; it then
  visits every batch once, starting wherever the cycle is, and completes
  after ``len(db.batches)`` steps -- so its work overlaps with that of the
  requests already in flight (continuous batching at batch granularity);
* a request's result does not depend on which requests it ran with: the
  per-batch top-k lists are merged in a fixed order (score desc, batch,
  segment), and every query's scores come from the same kernel either way.

``ServerStats`` reports completions, queries/s and latency percentiles.  The
per-step scoring is a replaceable ``executor`` so the scheduling can be run
without a GPU (tests use a host executor).
"""
from __future__ import annotations

import itertools
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    query: str
    t_submit: float
    t_admit: float | None = None
    t_done: float | None = None
    start_batch: int | None = None
    seen: int = 0                                  # batches scored so far
    parts: list = field(default_factory=list)      # (batch, segments, scores) per batch
    result: object = None
    done: threading.Event = field(default_factory=threading.Event)
    enc: object = None                             # executor-side state

    @property
    def latency(self) -> float | None:
        return None if self.t_done is None else self.t_done - self.t_submit


@dataclass
class Hits:
    """Merged top-k of one request: score desc, then batch, then segment."""
    scores: np.ndarray
    batch: np.ndarray
    segment: np.ndarray


def merge_parts(parts, top_k: int) -> Hits:
    if not parts:
        z = np.zeros(0, dtype=np.int32)
        return Hits(z, z, z)
    sc = np.concatenate([p[2] for p in parts]).astype(np.int32)
    bt = np.concatenate([np.full(len(p[1]), p[0], np.int32) for p in parts])
    sg = np.concatenate([p[1] for p in parts]).astype(np.int32)
    order = np.lexsort((sg, bt, -sc.astype(np.int64)))[:top_k]
    return Hits(sc[order], bt[order], sg[order])


class GpuExecutor:
    """Scores one database batch for a set of requests on the GPU."""

    def __init__(self, db, *, top_k: int = 4096, gap_open: int = 11, gap_extend: int = 1,
                 max_slots: int = 128):
        import torch

        from . import batched, tune
        self.torch, self.batched, self.tune = torch, batched, tune
        self.db, self.top_k, self.gaps = db, int(top_k), (int(gap_open), int(gap_extend))
        self.n = [max(b.n_segments - 2, 0) for b in db.batches]
        self.rows = min(int(max_slots), batched.GROUP)
        nmax = max(self.n + [1])
        dev = db.device
        self.q = torch.zeros((self.rows, batched.MAX_QUERY), dtype=torch.uint8, device=dev)
        self.lens = torch.zeros(self.rows, dtype=torch.int32, device=dev)
        self.scores = torch.empty((self.rows, nmax), dtype=torch.int32, device=dev)
        self.tickets = torch.empty(self.rows, dtype=torch.int32, device=dev)
        from ._lib import lib
        self.ws = torch.empty(lib().sseqs_topk_workspace_bytes(nmax), dtype=torch.uint8,
                              device=dev)
        self.idx = torch.empty(max(self.top_k, 1), dtype=torch.int32, device=dev)

    @property
    def n_batches(self) -> int:
        return len(self.db.batches)

    @staticmethod
    def request_bytes(top_k: int, n_batches: int) -> int:
        """Device memory a request holds while in flight (query + its hits)."""
        return 2048 + 2 * 4 * top_k * max(n_batches, 1)

    def prepare(self, req: Request) -> None:
        import importlib
        sw = importlib.import_module("sseqs_b200.sw")
        req.enc = sw.encode_query(req.query, device=self.db.device)
        if not 1 <= req.enc.numel() <= self.batched.MAX_QUERY:
            raise ValueError(f"query length {req.enc.numel()} outside 1..2048")

    def step(self, bi: int, reqs: list) -> list:
        """Top-k (segments, scores) of batch ``bi`` for each request."""
        torch, batched = self.torch, self.batched
        from . import select
        from ._lib import to_host
        batch, n = self.db.batches[bi], self.n[bi]
        k = min(self.top_k, n)
        out: list = [None] * len(reqs)
        if n <= 0 or k <= 0:
            return [(np.zeros(0, np.int32), np.zeros(0, np.int32)) for _ in reqs]
        groups: dict = {}
        for i, r in enumerate(reqs):
            groups.setdefault(self.tune.tpt_of(r.enc.numel()), []).append(i)
        for tpt, members in groups.items():
            for s in range(0, len(members), self.rows):
                grp = members[s:s + self.rows]
                for j, i in enumerate(grp):
                    e = reqs[i].enc
                    self.q[j, :e.numel()].copy_(e)
                lens = torch.tensor([reqs[i].enc.numel() for i in grp], dtype=torch.int32)
                self.lens[:len(grp)].copy_(lens)
                sc = self.scores[:len(grp)]
                batched.sw_scan_queries(self.q, self.lens[:len(grp)], tpt, batch.ascii,
                                        batch.delim, affine=True, g0=1, n_targets=n, skip=1,
                                        gap_a=self.gaps[0], gap_b=self.gaps[1], out=sc,
                                        tickets=self.tickets)
                for j, i in enumerate(grp):
                    row = sc[j, :n]
                    p = select.topk_indices(row, k, out=self.idx, ws=self.ws)
                    vals = row[p.long()]
                    out[i] = ((to_host(p) + 1).astype(np.int32), to_host(vals))
        return out


class LearnedExecutor:
    """The learned-prefilter pipeline as one engine step: every request in
    flight gets its candidates from the FP8 index (all requests of the step
    in one selection GEMM), exact affine SW of the candidates and its top-k;
    requests complete in the step that admits them.  The database and its
    codes stay resident (``learned.LearnedIndex``)."""

    n_batches = 1

    def __init__(self, index, *, top_k: int = 4096, n_cand: int = 32768):
        self.index, self.top_k, self.n_cand = index, int(top_k), int(n_cand)

    def request_bytes(self, top_k: int, n_batches: int) -> int:
        # candidate lists (row + score, 12 bytes) at the selection cap (8x the
        # candidates), and the hits; a 128-wide index selects two columns
        # per query and merges them into a list twice as long (4x the bytes)
        lists = 4 if getattr(self.index, "dim", 256) < 256 else 1
        return lists * 8 * 12 * self.n_cand + 16 * top_k

    def prepare(self, req: Request) -> None:
        if not 1 <= len(req.query) <= 2048:
            raise ValueError(f"query length {len(req.query)} outside 1..2048")
        req.enc = req.query

    def step(self, bi: int, reqs: list) -> list:
        res = self.index.search_arrays([r.enc for r in reqs], n_cand=self.n_cand, top=self.top_k)
        # (segment, score, batch) per request; the server's merge sorts by
        # score, then batch, then segment
        return [(seg.astype(np.int32), aff.astype(np.int32), bt.astype(np.int32))
                for _, bt, seg, aff in res]


class SearchServer:
    """Continuous-batching request loop over a resident database."""

    def __init__(self, executor, *, max_slots: int = 64, top_k: int = 4096,
                 memory_reserve: int = 1 << 30, free_memory=None, clock=time.monotonic):
        self.ex = executor
        self.max_slots = int(max_slots)
        self.top_k = int(top_k)
        self.reserve = int(memory_reserve)
        self._free_memory = free_memory           # callable -> free bytes, or None
        self.clock = clock
        self.pending: deque = deque()
        self.inflight: list = []
        self.completed: list = []
        self._ids = itertools.count()
        self._cv = threading.Condition()
        self._stop = False
        self._thread = None
        self.cursor = 0                           # batch the next step scores
        self.steps = 0
        self.error: BaseException | None = None

    # ------------------------------------------------------------ client side
    def submit(self, query: str) -> Request:
        req = Request(next(self._ids), query, self.clock())
        with self._cv:
            self.pending.append(req)
            self._cv.notify_all()
        return req

    def start(self):
        self._thread = threading.Thread(target=self._run, name="sseqs-serve", daemon=True)
        self._thread.start()
        return self

    def stop(self, wait: bool = True):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        if wait and self._thread is not None:
            self._thread.join()

    def drain(self, timeout: float | None = None) -> bool:
        """Waits until nothing is pending or in flight."""
        end = None if timeout is None else time.monotonic() + timeout
        with self._cv:
            while self.pending or self.inflight:
                if self.error is not None:
                    raise self.error
                left = None if end is None else end - time.monotonic()
                if left is not None and left <= 0:
                    return False
                self._cv.wait(0.05 if left is None else min(left, 0.05))
        return True

    # ------------------------------------------------------------ engine side
    def _memory_ok(self, n_new: int) -> bool:
        if self._free_memory is None:
            return True
        need = n_new * self.ex.request_bytes(self.top_k, self.ex.n_batches)
        return self._free_memory() - self.reserve >= need

    def _admit(self):
        """Moves pending requests into flight while slots and memory allow."""
        while self.pending and len(self.inflight) < self.max_slots and self._memory_ok(1):
            req = self.pending.popleft()
            try:
                self.ex.prepare(req)
            except Exception as e:                     # a bad request fails alone
                req.result = e
                req.t_done = self.clock()
                req.done.set()
                self.completed.append(req)
                continue
            req.t_admit = self.clock()
            req.start_batch = self.cursor
            self.inflight.append(req)

    def step(self) -> bool:
        """One engine step (admission + one batch for everyone in flight);
        returns False when there was nothing to do."""
        with self._cv:
            self._admit()
            reqs = list(self.inflight)
        if not reqs:
            return False
        nb = self.ex.n_batches
        bi = self.cursor
        res = self.ex.step(bi, reqs) if nb else []
        now = self.clock()
        finished = []
        for r, part in zip(reqs, res):
            if len(part) == 3:            # executor that covers every batch at once
                for b in np.unique(part[2]):
                    m = part[2] == b
                    r.parts.append((int(b), part[0][m], part[1][m]))
            else:
                r.parts.append((bi, part[0], part[1]))
            r.seen += 1
        for r in reqs:
            if r.seen >= nb:
                r.result = merge_parts(r.parts, self.top_k)
                r.parts = []
                r.enc = None
                r.t_done = now
                finished.append(r)
        with self._cv:
            for r in finished:
                self.inflight.remove(r)
                self.completed.append(r)
                r.done.set()
            self.cursor = (bi + 1) % max(nb, 1)
            self.steps += 1
            self._cv.notify_all()
        return True

    def _run(self):
        try:
            while True:
                with self._cv:
                    if self._stop:
                        return
                    if not self.pending and not self.inflight:
                        self._cv.wait(0.01)
                        continue
                self.step()
        except BaseException as e:                   # surfaced by drain()
            self.error = e
            with self._cv:
                for r in self.inflight + list(self.pending):
                    r.result = e
                    r.done.set()
                self._cv.notify_all()


@dataclass
class ServerStats:
    completed: int
    seconds: float
    queries_per_s: float
    p50_ms: float
    p99_ms: float
    mean_ms: float


def stats(requests, seconds: float) -> ServerStats:
    lat = np.array([r.latency for r in requests if r.latency is not None]) * 1e3
    if lat.size == 0:
        return ServerStats(0, seconds, 0.0, float("nan"), float("nan"), float("nan"))
    return ServerStats(int(lat.size), seconds, lat.size / seconds, float(np.percentile(lat, 50)),
                       float(np.percentile(lat, 99)), float(lat.mean()))


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    """Submission offsets (seconds) of n requests at Poisson rate ``rate``."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def replay(server: SearchServer, queries, offsets) -> list:
    """Submits ``queries[i]`` at ``offsets[i]`` seconds from now (the server
    must be running); returns the requests once all have completed."""
    t0 = time.monotonic()
    reqs = []
    for q, off in zip(queries, offsets):
        dt = t0 + off - time.monotonic()
        if dt > 0:
            time.sleep(dt)
        reqs.append(server.submit(q))
    for r in reqs:
        r.done.wait()
    if server.error is not None:
        raise server.error
    return reqs

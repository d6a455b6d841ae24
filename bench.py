#!/usr/bin/env python
"""Benchmark of the sseqs_b200 database search on B200.

Workload (one "step" = one query): exact search of a query of the
64-query set (lengths uniform 50..1000, seed 0) against the resident
synthetic database of 20M sequences (log-normal lengths, 0.5% planted
homologs per query at 20-95% identity): linear (gap -1) and affine (11/1)
BLOSUM62 Smith-Waterman over every segment (prefilter off: top_fft=1,
top_sw=1), top-4096 per batch, global top-4096, CUDA traceback and a3m of
the 4096 best.  Metric: SW GCUPS = query length x segment residues, counted
once per SW variant, per second of step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

``--impl reference`` times the CPU oracle (the reference has no CPU
implementation of this path; the oracle restates its kernels) on all host
threads over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUERIES = 64
DB_SEQS = 20_000_000
HOMOLOG_FRAC = 0.005
IDENT = (0.20, 0.95)
TOP_K = 4096
BS = 1_000_000_000


def query_set():
    from sseqs_b200 import dbtools
    rng = np.random.default_rng(0)
    lens = rng.integers(50, 1001, N_QUERIES)
    return [dbtools.random_query(int(n), 1000 + i) for i, n in enumerate(lens)]


def step_queries(queries, steps, warmup):
    """Timed step i uses query i; warm-up steps use queries from the end."""
    warm = [queries[(N_QUERIES - 1 - i) % N_QUERIES] for i in range(warmup)]
    timed = [queries[i % N_QUERIES] for i in range(steps)]
    return warm, timed


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 8:
                    continue
                try:
                    sm.append(float(p[0]))
                    mx = float(p[1])
                except ValueError:
                    continue
                for name, v in zip(names, p[4:8]):
                    if v.lower() == "active":
                        reasons.add(name)
        finally:
            os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- GPU side
# DRAM traffic of the affine score kernel per target residue, from its ncu
# capture at 1M sequences, stripe width 27 (381.9 MB read + 10.0 MB written,
# 372.7M residues)
TRAFFIC_BYTES_PER_RESIDUE = (381.879296e6 + 10.014464e6) / 372662216


def build_database(queries, db_seqs, seed=0):
    import torch
    from sseqs_b200 import dbtools
    from sseqs_b200.database import Database
    syn = dbtools.synthetic_db(queries, db_seqs, HOMOLOG_FRAC, IDENT, seed=seed, device="cuda")
    db = Database(syn.chunks, bs=BS, keep_packed=True)
    info = {"db_sequences": syn.n_seqs, "db_residues": syn.n_residues, "db_chunks": len(syn.chunks),
            "db_packed_bytes": len(syn.chunks) * BS}
    del syn
    torch.cuda.empty_cache()
    return db, info


def segment_cells(db):
    """Residues of the segments every step scores (1 .. nseg-2 of each batch)."""
    tot = 0
    for b in db.batches:
        ln = b.lengths
        if b.n_segments > 2:
            tot += int(ln[1:b.n_segments - 1].sum(dtype=__import__("torch").int64).item())
    return tot


def run_step(M, query, db, timer=None, world=1, rank=0):
    """Device part of one step: search, rank, traceback (no file I/O).  With
    several GPUs every rank searches its own shard, the ranked hits are merged
    across ranks, and rank 0 aligns the merged list."""
    from sseqs_b200.to_a3m import traceback_all
    rows = M.search([query], db, num_msas=TOP_K, top_fft=1, top_sw=1, top_sw_affine=TOP_K,
                    timer=timer)[0]
    if world > 1:
        from sseqs_b200 import shard
        rows = [r[:1] + r[2:] for r in shard.gather_hits(rows, TOP_K)]
    al = traceback_all(query, [r[5] for r in rows]) if rank == 0 else None
    return rows, al


def prefiltered_leg(M, db, queries, exact_rows, per_query=32768):
    """The prefiltered search: the reference's prefilter keeping ~per_query candidates
    per query (top_fft = segments per batch // (per_query / batches)), exact
    linear + affine SW of the candidates, top-4096, traceback.  Reports
    queries/s and recall of the exact search's top-1000 hits."""
    import torch
    from sseqs_b200.to_a3m import traceback_all
    nb = len(db.batches)
    seg_per_batch = max(b.n_segments for b in db.batches)
    top_fft = max(1, seg_per_batch // max(1, per_query // nb))
    M.search([queries[0]], db, num_msas=TOP_K, top_fft=top_fft, top_sw=1,
             top_sw_affine=TOP_K)                       # warm-up (query spectra, LUTs)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    results = []
    for q in queries:
        rows = M.search([q], db, num_msas=TOP_K, top_fft=top_fft, top_sw=1,
                        top_sw_affine=TOP_K)[0]
        traceback_all(q, [r[5] for r in rows])
        results.append(rows)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    rec = []
    for q, rows in zip(queries, results):
        ex = exact_rows.get(q)
        if not ex:
            continue
        want = {(r[1], r[2]) for r in ex[:1000]}
        got = {(r[1], r[2]) for r in rows}
        rec.append(len(want & got) / max(1, len(want)))
    return {"queries_per_s": round(len(queries) / (ms * 1e-3), 3),
            "ms_per_query": round(ms / len(queries), 1),
            "top_fft": top_fft, "candidates_per_query": (seg_per_batch // top_fft) * nb,
            "recall_of_exact_top1000": round(float(np.mean(rec)), 4) if rec else None,
            "queries": len(queries)}


def batched_leg(db, n_queries, seed=3):
    """Batched uneven queries: lengths log-normal (median 300, sigma 0.6)
    clipped to 16..2048, affine 11/1 over every segment of the resident
    database, top-4096 per query.  Times the bucketed, graph-replayed path
    (``batched.BatchedSearcher``; its first call captures the graphs) against
    the same work one query at a time (``sw.sw_scan`` + top-k per batch), and
    checks that both give identical hit lists."""
    import torch
    from sseqs_b200 import batched, dbtools, select
    sw = importlib.import_module("sseqs_b200.sw")
    rng = np.random.default_rng(seed)
    lengths = np.clip(np.round(np.exp(rng.normal(np.log(300), 0.6, n_queries))), 16, 2048)
    queries = [dbtools.random_query(int(L), 5000 + i) for i, L in enumerate(lengths)]
    rows_aff = 0
    for b in db.batches:
        if b.n_segments > 2:
            ln = b.lengths[1:b.n_segments - 1].to(torch.int64)
            rows_aff += int((ln - 1).clamp_(min=0).sum().item())
    cells = int(sum(int(L) for L in lengths)) * rows_aff
    from sseqs_b200 import tune
    searcher = batched.BatchedSearcher(db, top_k=TOP_K)
    searcher.search(queries)                         # autotune + graph capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    got = searcher.search(queries)
    e1.record()
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    # the same batched launches with one query per launch row at every width
    pairing = {t: tune.get_query_pairing(t) for t in range(1, 65)}
    tune.set_query_pairing(0, False)
    unpaired = batched.BatchedSearcher(db, top_k=TOP_K, autotune=False)
    unpaired.search(queries)
    torch.cuda.synchronize()
    e0.record()
    got_u = unpaired.search(queries)
    e1.record()
    torch.cuda.synchronize()
    ms_u = e0.elapsed_time(e1)
    for t, on in pairing.items():
        tune.set_query_pairing(t, on)
    del unpaired

    def one(q):
        enc = sw.encode_query(q)
        rows = []
        for bi, b in enumerate(db.batches):
            n = b.n_segments - 2
            if n <= 0:
                continue
            s = sw.sw_scan(enc, b.ascii, b.delim, affine=True, g0=1, n_targets=n, skip=1,
                           gap_a=11, gap_b=1)
            p = select.topk_indices(s, min(TOP_K, n)).long()
            rows.append((s[p], bi, p + 1))
        return rows

    one(queries[0])
    torch.cuda.synchronize()
    e0.record()
    ref = [one(q) for q in queries]
    e1.record()
    torch.cuda.synchronize()
    ms_q = e0.elapsed_time(e1)
    same = all(np.array_equal(a.scores, b.scores) and np.array_equal(a.batch, b.batch)
               and np.array_equal(a.segment, b.segment) for a, b in zip(got, got_u))
    for h, rows in zip(got, ref):
        sc = np.concatenate([r[0].cpu().numpy() for r in rows])
        bt = np.concatenate([np.full(r[0].numel(), r[1], np.int32) for r in rows])
        sg = np.concatenate([r[2].cpu().numpy() for r in rows])
        o = np.lexsort((sg, bt, -sc.astype(np.int64)))[:TOP_K]
        same &= (np.array_equal(h.scores, sc[o]) and np.array_equal(h.batch, bt[o])
                 and np.array_equal(h.segment, sg[o]))
    return {"queries": n_queries,
            "lengths": "log-normal median 300 sigma 0.6, clipped 16..2048, seed %d" % seed,
            "length_range": [int(lengths.min()), int(lengths.max())],
            "buckets": len(batched.buckets([int(L) for L in lengths])),
            "graphs": len(searcher.plans),
            "gcups_batched": round(cells / (ms_b * 1e-3) / 1e9, 1),
            "gcups_batched_one_query_per_row": round(cells / (ms_u * 1e-3) / 1e9, 1),
            "gcups_one_query_at_a_time": round(cells / (ms_q * 1e-3) / 1e9, 1),
            "ms_batched": round(ms_b, 1), "ms_one_query_at_a_time": round(ms_q, 1),
            "paired_widths": sorted(t for t, on in pairing.items() if on),
            "cells": cells, "identical_hits": bool(same)}


def serving_leg(db, n_requests, rate, seed=4, index=None):
    """Request loop over the resident database (``serve.SearchServer`` with
    the GPU executor): Poisson arrivals at ``rate`` queries/s, query lengths
    U(50, 1000), exact affine scoring of every segment and top-4096 per
    request, continuous batching at database-batch granularity.  Reports
    completed queries/s and latency percentiles (submission to result)."""
    from sseqs_b200 import dbtools, serve
    rng = np.random.default_rng(seed)
    queries = [dbtools.random_query(int(L), 9000 + i)
               for i, L in enumerate(rng.integers(50, 1001, n_requests))]
    if index is None:
        ex = serve.GpuExecutor(db, top_k=TOP_K)
        pipeline = "exact affine SW of every segment, top-4096"
    else:
        ex = serve.LearnedExecutor(index, top_k=TOP_K)
        pipeline = "learned prefilter (FP8 index, 32768 candidates) + exact affine SW, top-4096"
    import torch
    free = (lambda: torch.cuda.mem_get_info()[0])
    srv = serve.SearchServer(ex, top_k=TOP_K, max_slots=64, memory_reserve=2 << 30,
                             free_memory=free)
    # warm-up outside the measurement (autotune of the widths, first launches)
    from sseqs_b200 import tune
    tune.autotune([len(q) for q in queries], db.batches[0])
    srv.submit(queries[0])
    while srv.step():
        pass
    srv.completed.clear()
    srv.start()
    try:
        offs = serve.poisson_arrivals(n_requests, rate, seed=seed)
        reqs = serve.replay(srv, queries, offs)
    finally:
        srv.stop()
    span = max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)
    st = serve.stats(reqs, span)
    return {"requests": n_requests, "arrival_rate_qps": rate,
            "queries_per_s": round(st.queries_per_s, 3), "p50_ms": round(st.p50_ms, 1),
            "p99_ms": round(st.p99_ms, 1), "mean_ms": round(st.mean_ms, 1),
            "engine_steps": srv.steps, "pipeline": pipeline,
            "lengths": "U(50, 1000), seed %d" % seed}


def learned_leg(db, exact_rows, n_pairs, n_queries, epochs=1, seed=5, target_power=0.5):
    """Learned prefilter: train the conv embedder on ``n_pairs`` seeded
    (query, target) pairs labelled by this package's exact SW, embed every
    database segment into FP8 codes, then per query take 32768 candidates by
    the FP8 GEMM, re-score them by exact affine SW, keep the top 4096 and
    align them (the same tail as the exact step).  Queries/s over
    ``n_queries`` queries U(50, 1000) (the exact leg's timed queries first);
    recall of the exact search's top-1000 over the exact leg's queries."""
    import torch
    from sseqs_b200 import dbtools, learned
    from sseqs_b200.to_a3m import traceback_all
    per_query = 256
    t0 = time.time()
    pairs = learned.training_pairs(max(1, n_pairs // per_query), per_query, seed=seed)
    torch.cuda.synchronize()
    t1 = time.time()
    model = learned.Embedder(seed=seed)
    hist = learned.train(model, pairs, epochs=epochs, seed=seed, target_power=target_power)
    torch.cuda.synchronize()
    t2 = time.time()
    index = learned.LearnedIndex(model, db)
    torch.cuda.synchronize()
    t3 = time.time()
    rng = np.random.default_rng(seed)
    qs = list(exact_rows)
    qs += [dbtools.random_query(int(L), 7000 + i)
           for i, L in enumerate(rng.integers(50, 1001, max(0, n_queries - len(qs))))]

    def step(batch_q):
        res = index.search(batch_q, n_cand=32768, top=TOP_K)
        for q, rows in zip(batch_q, res):
            traceback_all(q, learned.hit_strings(db, rows))
        return res

    step(qs[:2])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res = step(qs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    rec = []
    for q, rows in zip(qs, res):
        ex = exact_rows.get(q)
        if not ex:
            continue
        want = {(r[1], r[2]) for r in ex[:1000]}
        got = {(r[1], r[2]) for r in rows[:1000]}
        rec.append(len(want & got) / max(1, len(want)))
    learned_leg.index = index
    return {"queries": len(qs), "queries_per_s": round(len(qs) / (ms * 1e-3), 3),
            "ms_per_query": round(ms / len(qs), 2),
            "recall_of_exact_top1000": round(float(np.mean(rec)), 4) if rec else None,
            "recall_min": round(float(np.min(rec)), 4) if rec else None,
            "recall_queries": len(rec), "candidates_per_query": 32768,
            "train_pairs": int(pairs.y.numel()), "train_epochs": epochs,
            "train_steps": hist["steps"], "train_labelled_pairs": hist["labelled_pairs"],
            "train_loss_first_last": [hist["losses"][0][1], hist["losses"][-1][1]],
            "params": model.n_params, "seconds_pairs": round(t1 - t0, 1),
            "seconds_train": round(t2 - t1, 1), "seconds_index": round(t3 - t2, 1),
            "index_rows": index.n, "index_bytes": int(index.codes.numel())}


def kernels_one_batch_leg(db, queries):
    """GCUPS of this build's drop-in score operators (``sw_cuda_blosum62``,
    gap -1, windows of sseqs/msa.py:313-319; ``sw_cuda_affine``, 11/1,
    windows of :327-332) over segments 1 .. n-2 of the first database batch,
    per query of at most 1024 residues: the call form and inputs the
    reference arm times its own kernels on."""
    import torch
    sw = importlib.import_module("sseqs_b200.sw")
    b = db.batches[0]
    nseg = b.n_segments
    good = torch.arange(1, nseg - 1, dtype=torch.int32, device="cuda")
    residues = int(b.lengths[1:nseg - 1].sum(dtype=torch.int64).item())
    dp1 = (b.delim + 1).contiguous()
    lin_ms = aff_ms = 0.0
    cells = 0
    qs = [q for q in queries if len(q) <= 1024]
    for q in qs:
        qe = sw.encode_query(q)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        sw.sw_cuda_blosum62(qe, good, b.ascii, b.delim, gap_penalty_param=-1)
        ev[1].record()
        sw.sw_cuda_affine(qe, good, b.ascii, dp1, 11, 1)
        ev[2].record()
        torch.cuda.synchronize()
        lin_ms += ev[0].elapsed_time(ev[1])
        aff_ms += ev[1].elapsed_time(ev[2])
        cells += len(q) * residues
    return {"gcups_linear": round(cells / (lin_ms * 1e-3) / 1e9, 1),
            "gcups_affine": round(cells / (aff_ms * 1e-3) / 1e9, 1),
            "segments": nseg - 2, "residues": residues, "queries": len(qs)}


def linear_gap4_leg(db, queries, res_cells):
    """BLOSUM62 with linear gap 4 (the benchmark's "linear (gap 4)"
    variant) over every segment 1 .. n-2 of every batch: GCUPS."""
    import torch
    sw = importlib.import_module("sseqs_b200.sw")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for q in queries:
        qe = sw.encode_query(q)
        for b in db.batches:
            if b.n_segments > 2:
                sw.sw_scan(qe, b.ascii, b.delim, affine=False, g0=1, n_targets=b.n_segments - 2,
                           skip=0, gap_a=-4)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cells = sum(len(q) for q in queries) * res_cells
    return {"gcups": round(cells / (ms * 1e-3) / 1e9, 1), "queries": len(queries),
            "gap": -4}


def search_defaults_leg(M, db, queries):
    """The reference's defaults (bs = 5e7, top_fft = 200, top_sw = 10,
    top_sw_affine = 2, sseqs/msa.py:71-85) over the whole database: packed
    database bytes searched per second, the reference's own figure
    (README.md:11-12: GB/s over its chunk loop; the a3m after the loop is
    not in it).  The database is decoded once more with bs = 5e7 and stays
    resident."""
    import torch
    from sseqs_b200.database import Database
    db50 = Database(db.packed, bs=50_000_000)
    packed = sum(c.numel() for c in db.packed)
    M.search([queries[-1]], db50, num_msas=TOP_K)            # warm-up (LUTs, first launches)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    hits = 0
    for q in queries:
        hits += len(M.search([q], db50, num_msas=TOP_K, top_fft=200, top_sw=10,
                             top_sw_affine=2)[0])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    del db50
    torch.cuda.empty_cache()
    return {"GB_per_s": round(packed * len(queries) / (ms * 1e-3) / 1e9, 2),
            "ms_per_query": round(ms / len(queries), 1), "queries": len(queries),
            "packed_bytes": packed, "hits": hits,
            "settings": "bs=5e7, top_fft=200, top_sw=10, top_sw_affine=2, database resident"}


SWEEP_RATES = (10, 50, 100, 250, 500)


def serving_sweep(index, rates, seconds, seed=6, n_alone=4):
    """The learned-prefilter request loop (``serve.SearchServer`` +
    ``serve.LearnedExecutor``, continuous batching, up to 64 requests in
    flight, admission by free device memory) under Poisson arrivals at each
    rate for about ``seconds`` seconds (at least 20 requests), query lengths
    U(50, 1000): served queries/s and latency percentiles per rate.  Then
    ``n_alone`` requests of the last rate are scored again alone, and their
    hits must equal the ones they got in the mix."""
    import torch
    from sseqs_b200 import dbtools, serve
    ex = serve.LearnedExecutor(index, top_k=TOP_K)
    free = (lambda: torch.cuda.mem_get_info()[0])
    srv = serve.SearchServer(ex, top_k=TOP_K, max_slots=64, memory_reserve=2 << 30,
                             free_memory=free)
    rng = np.random.default_rng(seed)
    srv.submit(dbtools.random_query(300, 1))                  # warm-up
    while srv.step():
        pass
    srv.completed.clear()
    out, last = [], None
    srv.start()
    try:
        for rate in rates:
            n = max(20, int(rate * seconds))
            qs = [dbtools.random_query(int(L), 20000 + 997 * rate + i)
                  for i, L in enumerate(rng.integers(50, 1001, n))]
            offs = serve.poisson_arrivals(n, rate, seed=seed + rate)
            steps0 = srv.steps
            reqs = serve.replay(srv, qs, offs)
            span = max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)
            st = serve.stats(reqs, span)
            out.append({"arrival_rate_qps": rate, "requests": n,
                        "queries_per_s": round(st.queries_per_s, 2),
                        "p50_ms": round(st.p50_ms, 1), "p99_ms": round(st.p99_ms, 1),
                        "mean_ms": round(st.mean_ms, 1), "engine_steps": srv.steps - steps0,
                        "saturated": st.queries_per_s < 0.9 * rate})
            last = reqs
    finally:
        srv.stop()
    same = True
    alone = serve.SearchServer(ex, top_k=TOP_K, max_slots=64)
    for r in last[:n_alone]:
        a = alone.submit(r.query)
        while alone.step():
            pass
        ra, rb = a.result, r.result
        same &= (np.array_equal(ra.scores, rb.scores) and np.array_equal(ra.batch, rb.batch)
                 and np.array_equal(ra.segment, rb.segment))
    return {"rates": out, "identical_alone_vs_mix": bool(same), "checked_alone": n_alone,
            "pipeline": "learned prefilter (FP8 index, 32768 candidates) + exact affine SW, "
                        "top-4096; up to 64 requests in flight",
            "index_rows": index.n, "lengths": "U(50, 1000)"}


RECALL_BANDS = ((0.20, 0.30), (0.30, 0.45), (0.45, 0.60), (0.60, 0.95))


def bench_learned_scale(args):
    """``--learned-scale``: the learned prefilter at its stated size.  The
    embedder is trained on ``--learned-pairs`` seeded pairs; the database is
    20M synthetic sequences in which each of ``--recall-queries`` queries has
    ``--recall-homologs`` planted homologs (identity U(20%, 95%), the
    benchmark's length and composition model); ``--learned-queries`` queries
    are timed (the recall queries first, then U(50, 1000) queries without
    homologs).  The exact reference is the exhaustive affine sweep of every
    segment (``batched.BatchedSearcher``, ranked by normalised score like the
    learned path), timed on the recall queries.  Recall of the exact top-1000
    over the recall queries, overall and per identity band of the planted
    homologs among those 1000.  Neither path aligns its hits here.  One JSON
    line."""
    import torch
    from sseqs_b200 import batched, dbtools, learned
    from sseqs_b200.database import Database
    torch.cuda.set_device(0)
    t0 = time.time()
    rng = np.random.default_rng(41)
    nr = int(args.recall_queries)
    recall_qs = [dbtools.random_query(int(L), 40000 + i)
                 for i, L in enumerate(rng.integers(50, 1001, nr))]
    n_seqs = int(args.db_seqs)
    syn = dbtools.synthetic_db(recall_qs, n_seqs, args.recall_homologs / n_seqs, IDENT,
                               seed=77, device="cuda")
    db = Database(syn.chunks, bs=BS)
    batch_of_chunk = {b.chunk: bi for bi, b in enumerate(db.batches) if b.index == 0}
    seq_chunk, seq_rank = syn.seq_chunk.cpu().numpy(), syn.seq_rank.cpu().numpy()
    planted = {}                         # query -> {(batch, segment): identity}
    for qi in range(nr):
        sid = syn.planted[qi].cpu().numpy()
        u = syn.planted_identity[qi].cpu().numpy()
        planted[qi] = {(batch_of_chunk[int(seq_chunk[s])], int(seq_rank[s])): float(x)
                       for s, x in zip(sid, u)}
    n_res = syn.n_residues
    del syn
    torch.cuda.empty_cache()
    t1 = time.time()
    pairs = learned.training_pairs(max(1, args.learned_pairs // 256), 256, seed=5)
    t2 = time.time()
    model = learned.Embedder(seed=5)
    hist = learned.train(model, pairs, epochs=args.learned_epochs, seed=5,
                         target_power=args.learned_target_power)
    n_pairs = int(pairs.y.numel())
    del pairs
    torch.cuda.empty_cache()
    torch.cuda.synchronize()
    t3 = time.time()
    index = learned.LearnedIndex(model, db)
    torch.cuda.synchronize()
    t4 = time.time()
    qs = recall_qs + [dbtools.random_query(int(L), 60000 + i) for i, L in
                      enumerate(rng.integers(50, 1001, max(0, args.learned_queries - nr)))]
    chunk = 256
    index.search_arrays(qs[:4], n_cand=32768, top=TOP_K)            # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    got = []
    for s0 in range(0, len(qs), chunk):
        got += index.search_arrays(qs[s0:s0 + chunk], n_cand=32768, top=TOP_K)
    e1.record()
    torch.cuda.synchronize()
    ms_learned = e0.elapsed_time(e1)
    e0.record()
    got_r = []
    for s0 in range(0, nr, chunk):
        got_r += index.search_arrays(recall_qs[s0:s0 + chunk], n_cand=32768, top=TOP_K)
    e1.record()
    torch.cuda.synchronize()
    ms_learned_r = e0.elapsed_time(e1)
    # exhaustive sweep (eager launches; the autotuner runs on two queries first)
    exact = batched.BatchedSearcher(db, top_k=TOP_K, use_graphs=False)
    exact.search(recall_qs[:2], rank="norm")
    torch.cuda.synchronize()
    e0.record()
    ref = exact.search(recall_qs, rank="norm")
    e1.record()
    torch.cuda.synchronize()
    ms_exact = e0.elapsed_time(e1)
    def recall(hits, depth_label):
        rec, same = [], True
        band_want = np.zeros(len(RECALL_BANDS), np.int64)
        band_got = np.zeros(len(RECALL_BANDS), np.int64)
        band_planted = np.zeros(len(RECALL_BANDS), np.int64)
        hom_want = hom_got = 0
        for qi in range(nr):
            h = ref[qi]
            want = set(zip(h.batch[:1000].tolist(), h.segment[:1000].tolist()))
            mine = hits[qi]
            gset = set(zip(mine[1][:1000].tolist(), mine[2][:1000].tolist()))
            rec.append(len(want & gset) / max(1, len(want)))
            # every learned hit's score is the exact score of the same segment
            ex = dict(zip(zip(h.batch.tolist(), h.segment.tolist()), h.scores.tolist()))
            for bt, sg, a in zip(mine[1].tolist(), mine[2].tolist(), mine[3].tolist()):
                if (bt, sg) in ex and ex[(bt, sg)] != a:
                    same = False
            for key, u in planted[qi].items():
                for k, (lo, hi) in enumerate(RECALL_BANDS):
                    if lo <= u < hi or (k == len(RECALL_BANDS) - 1 and u == hi):
                        band_planted[k] += 1
                        if key in want:
                            band_want[k] += 1
                            band_got[k] += key in gset
                            hom_want += 1
                            hom_got += key in gset
        bands = [{"identity": [lo, hi], "planted": int(p), "in_exact_top1000": int(w),
                  "recall": round(float(g) / w, 4) if w else None}
                 for (lo, hi), p, w, g in zip(RECALL_BANDS, band_planted, band_want, band_got)]
        return {"candidates_per_query": depth_label,
                "recall_of_exact_top1000": round(float(np.mean(rec)), 4),
                "recall_min": round(float(np.min(rec)), 4),
                "recall_of_planted_homologs_in_exact_top1000":
                    round(hom_got / max(1, hom_want), 4),
                "recall_by_identity_band": bands, "scores_equal_exact": same}

    r32 = recall(got_r, 32768)
    depths = [dict(r32, queries_per_s=round(nr / (ms_learned_r * 1e-3), 2))]
    for depth in (131072, 524288):
        e0.record()
        hits = []
        for s0 in range(0, nr, 64):
            hits += index.search_arrays(recall_qs[s0:s0 + 64], n_cand=depth, top=TOP_K)
        e1.record()
        torch.cuda.synchronize()
        depths.append(dict(recall(hits, depth),
                           queries_per_s=round(nr / (e0.elapsed_time(e1) * 1e-3), 2)))
    # the same embedder with a 128-wide index (the embeddings projected onto
    # their 128 leading principal directions), at the default depth
    del index
    torch.cuda.empty_cache()
    index128 = learned.LearnedIndex(model, db, dim=128)
    index128.search_arrays(recall_qs[:4], n_cand=32768, top=TOP_K)    # warm-up
    torch.cuda.synchronize()
    e0.record()
    hits = []
    for s0 in range(0, nr, chunk):
        hits += index128.search_arrays(recall_qs[s0:s0 + chunk], n_cand=32768, top=TOP_K)
    e1.record()
    torch.cuda.synchronize()
    r128 = dict(recall(hits, 32768), queries_per_s=round(nr / (e0.elapsed_time(e1) * 1e-3), 2),
                index_bytes=int(index128.codes.numel()))
    qps_l = len(qs) / (ms_learned * 1e-3)
    qps_lr = nr / (ms_learned_r * 1e-3)
    qps_e = nr / (ms_exact * 1e-3)
    out = {
        "metric": "queries/s of the learned prefilter at >= 0.99 recall of the exact top-1000",
        "value": round(qps_l, 2), "unit": "queries/s", "n_gpus": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp8 e4m3 + int16x2",
        "data": "synthetic",
        "config": {"workload": "learned prefilter at its stated size",
                   "db_sequences": n_seqs, "db_residues": int(n_res),
                   "queries": len(qs), "recall_queries": nr,
                   "planted_homologs_per_recall_query": int(args.recall_homologs),
                   "identity": list(IDENT), "candidates_per_query": 32768, "top_k": TOP_K,
                   "train_pairs": n_pairs, "train_epochs": args.learned_epochs,
                   "train_target_power": args.learned_target_power},
        "queries_per_s_recall_queries": round(qps_lr, 2),
        "exact_queries_per_s": round(qps_e, 3),
        "speedup_vs_exact": round(qps_lr / qps_e, 2),
        "recall_of_exact_top1000": r32["recall_of_exact_top1000"],
        "recall_min": r32["recall_min"],
        "recall_by_identity_band": r32["recall_by_identity_band"],
        "scores_equal_exact": all(d["scores_equal_exact"] for d in depths + [r128]),
        "candidate_depths": depths,
        "index_128": r128,
        "train_loss_first_last": [hist["losses"][0][1], hist["losses"][-1][1]],
        "train_steps": hist["steps"],
        "seconds_build_db": round(t1 - t0, 1), "seconds_pairs": round(t2 - t1, 1),
        "seconds_train": round(t3 - t2, 1), "seconds_index": round(t4 - t3, 1),
        "ms_learned": round(ms_learned, 1), "ms_exact": round(ms_exact, 1),
    }
    print(json.dumps(out), flush=True)


def exact_saturation(db, n_q=16, n_batches=3, seed=7):
    """Saturation rate of the exact pipeline (``serve.GpuExecutor``: affine
    SW of every segment, top-k per batch) at this database size: ``n_q``
    requests of lengths U(50, 1000) scored together over the first
    ``n_batches`` batches, timed with CUDA events, and the rate scaled to the
    whole database by residues (the exact pipeline's cost is linear in
    them)."""
    import torch
    from sseqs_b200 import dbtools, serve
    ex = serve.GpuExecutor(db, top_k=TOP_K, max_slots=64)
    rng = np.random.default_rng(seed)
    reqs = [serve.Request(i, dbtools.random_query(int(L), 31000 + i), 0.0)
            for i, L in enumerate(rng.integers(50, 1001, n_q))]
    for r in reqs:
        ex.prepare(r)
    nb = min(n_batches, len(db.batches))
    ex.step(0, reqs[:2])                                   # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for bi in range(nb):
        ex.step(bi, reqs)
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    res_sub = sum(b.n_residues for b in db.batches[:nb])
    cells = sum(len(r.query) for r in reqs) * res_sub
    whole = sec * db.n_residues / max(res_sub, 1)
    return {"queries_per_s": round(n_q / whole, 4), "seconds_per_query": round(whole / n_q, 2),
            "gcups": round(cells / sec / 1e9, 1), "queries": n_q,
            "timed_batches": nb, "timed_residues": int(res_sub),
            "note": "timed on the first batches, scaled to all residues"}


def bench_serving_scale(args):
    """``--serving-scale N``: a database of N synthetic sequences built in
    shards of 20M (each with its own seed, decoded into the resident
    database as it is made), the embedder trained as in the learned leg, the
    FP8 index of every segment, and the serving sweep over it.  One JSON
    line."""
    import torch
    from sseqs_b200 import dbtools, learned
    from sseqs_b200.database import Database
    torch.cuda.set_device(0)
    t0 = time.time()
    queries = query_set()
    db = Database([], bs=BS)
    n_left, shard = int(args.serving_scale), 0
    n_res = 0
    while n_left > 0:
        n = min(20_000_000, n_left)
        syn = dbtools.synthetic_db(queries[:8], n, 0.0005, IDENT, seed=1000 + shard, device="cuda")
        n_res += syn.n_residues
        db.add_chunks(syn.chunks)
        del syn
        torch.cuda.empty_cache()
        n_left -= n
        shard += 1
    t1 = time.time()
    pairs = learned.training_pairs(max(1, args.learned_pairs // 256), 256, seed=5)
    model = learned.Embedder(seed=5)
    learned.train(model, pairs, epochs=args.learned_epochs, seed=5,
                  target_power=args.learned_target_power)
    del pairs
    torch.cuda.empty_cache()
    t2 = time.time()
    index = learned.LearnedIndex(model, db, dim=args.index_dim)
    torch.cuda.synchronize()
    t3 = time.time()
    sweep = serving_sweep(index, SWEEP_RATES, args.sweep_seconds)
    sweep["exact_pipeline_saturation"] = exact_saturation(db)
    # recall of the exhaustive search's top-1000 for queries with planted
    # homologs (each query has 0.05% of every shard)
    M = importlib.import_module("sseqs_b200.msa")
    rec = []
    for q in queries[:args.scale_recall_queries]:
        ex = M.search([q], db, num_msas=TOP_K, top_fft=1, top_sw=1, top_sw_affine=TOP_K)[0]
        got = index.search([q], n_cand=32768, top=TOP_K)[0]
        want = {(r[1], r[2]) for r in ex[:1000]}
        rec.append(len(want & {(r[1], r[2]) for r in got[:1000]}) / max(1, len(want)))
    best = max(r["queries_per_s"] for r in sweep["rates"])
    free, total = torch.cuda.mem_get_info()
    out = {
        "metric": "queries/s of the learned serving loop under Poisson arrivals (max over rates)",
        "value": best, "unit": "queries/s", "n_gpus": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp8 e4m3 + int16x2",
        "data": "synthetic",
        "config": {"workload": "serving at the benchmark's serving scale",
                   "db_sequences": int(args.serving_scale), "db_residues": int(n_res),
                   "db_shards": shard, "index_bytes": int(index.codes.numel()),
                   "index_dim": index.dim, "device_bytes_in_use": int(total - free)},
        "serving_sweep": sweep,
        "recall_of_exact_top1000": [round(r, 4) for r in rec],
        "recall_candidates_per_query": 32768,
        "seconds_build_db": round(t1 - t0, 1), "seconds_train": round(t2 - t1, 1),
        "seconds_index": round(t3 - t2, 1),
    }
    print(json.dumps(out), flush=True)


def measured_peak(name):
    """sseqs_dpx_peak (ALU-pipe DPX issue rate) or sseqs_int16x2_peak (both
    int pipes), in int16x2 lane-instructions per second."""
    import torch
    from sseqs_b200 import _lib
    sink = torch.zeros(1, dtype=torch.int32, device="cuda")
    v = ctypes.c_double()
    _lib.check(getattr(_lib.lib(), name)(sink.data_ptr(), ctypes.byref(v), _lib.stream_ptr()),
               name)
    return v.value


def cpu_sample_gcups(queries, budget_s, seed=0):
    """The CPU oracle (all host threads) over a bounded sample: the first
    query against a freshly generated database of the same distribution."""
    from oracle import oracle as O
    from sseqs_b200 import dbtools
    q = queries[0]
    qi = O.encode_query(q)
    nt = os.cpu_count() or 1

    def sample(n):
        syn = dbtools.synthetic_db([q], n, HOMOLOG_FRAC, IDENT, seed=seed, device="cpu",
                                   chunk_bytes=max(1 << 20, n * 700))
        a = O.xbit_decompress(syn.chunks[0].numpy(), syn.chunks[0].numel() * 8 // 5, 0)
        seg = O.segment(a)
        return a, np.flatnonzero(a == 64).astype(np.int32), seg

    a, d, seg = sample(2000)
    good = np.arange(1, len(seg["lengths"]) - 1, dtype=np.int32)
    t0 = time.time()
    O.sw_affine(qi, good, a, d + 1, 11, 1, nt)
    rate = len(q) * float(seg["lengths"][1:-1].sum()) / max(time.time() - t0, 1e-3)
    n = int(min(400_000, max(2000, rate * budget_s / 2 / (len(q) * 280))))
    a, d, seg = sample(n)
    good = np.arange(1, len(seg["lengths"]) - 1, dtype=np.int32)
    cells = len(q) * float(seg["lengths"][1:-1].sum())
    t0 = time.time()
    O.sw_linear(qi, good, a, d, -1, nt)
    O.sw_affine(qi, good, a, d + 1, 11, 1, nt)
    dt = time.time() - t0
    return 2 * cells / dt / 1e9, nt, f"query 0 (length {len(q)}) vs {len(good)} sequences " \
        f"({int(cells)} residue-columns x 2 variants) of a same-distribution database", dt


def small_exact_leg(M, reps=20):
    """The CPU-runnable exact search: one query of 200 residues
    (seed 0) against 100k synthetic sequences (same length model, 1% planted
    homologs at 30-90% identity), exact linear (-1) + affine (11/1) search,
    top 100 with alignments.  The GPU path (``msa.search`` + traceback, CUDA
    events over ``reps`` searches) beside the CPU oracle on all host threads
    over the same decoded database, both counted in SW cell updates of the
    two variants."""
    import torch
    from oracle import oracle as O
    from sseqs_b200 import dbtools
    from sseqs_b200.database import Database
    from sseqs_b200.to_a3m import traceback_all
    q = dbtools.random_query(200, 0)
    cb = 25_000_000                      # one chunk holds the ~30M residues
    syn = dbtools.synthetic_db([q], 100_000, 0.01, (0.30, 0.90), seed=0, device="cuda",
                               chunk_bytes=cb)
    chunk = syn.chunks[0]
    db = Database(syn.chunks, bs=cb)
    del syn
    cells = 2 * len(q) * segment_cells(db)

    def once():
        rows = M.search([q], db, num_msas=100, top_fft=1, top_sw=1, top_sw_affine=100)[0]
        traceback_all(q, [r[5] for r in rows])

    once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        once()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    a = O.xbit_decompress(chunk.cpu().numpy(), chunk.numel() * 8 // 5, 0)
    seg = O.segment(a)
    d = np.flatnonzero(a == 64).astype(np.int32)
    good = np.arange(1, len(seg["lengths"]) - 1, dtype=np.int32)
    cpu_cells = 2 * len(q) * float(seg["lengths"][1:-1].sum())
    qi = O.encode_query(q)
    nt = os.cpu_count() or 1
    t0 = time.time()
    O.sw_linear(qi, good, a, d, -1, nt)
    O.sw_affine(qi, good, a, d + 1, 11, 1, nt)
    dt = time.time() - t0
    return {"workload": "1 query of 200 residues vs 100k sequences, exact linear + affine, "
                        "top 100 with alignments",
            "gpu_ms_per_query": round(ms, 2), "gpu_gcups": round(cells / (ms * 1e-3) / 1e9, 1),
            "cpu_seconds": round(dt, 2), "cpu_gcups": round(cpu_cells / dt / 1e9, 3),
            "cpu_cores": nt, "cpu_kind": "port",
            "gpu_over_cpu": round((cells / (ms * 1e-3)) / (cpu_cells / dt), 1)}


def bench_b200(args):
    import torch
    import torch.distributed as dist
    from sseqs_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    M = importlib.import_module("sseqs_b200.msa")
    L = _lib.lib()
    queries = query_set()
    # weak scaling: every rank holds its own database shard of DB_SEQS sequences
    db, info = build_database(queries, args.db_seqs, seed=rank)
    res_cells = segment_cells(db)
    from sseqs_b200 import tune
    tuned = tune.autotune([len(q) for q in queries], db.batches[0])
    warm, timed = step_queries(queries, args.steps, args.warmup)
    for q in warm:
        run_step(M, q, db, world=world, rank=rank)
    torch.cuda.synchronize()

    events = {"affine": [], "both": []}

    def timer(kind, start):
        if kind not in events:
            return None
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        if start:
            events[kind].append([e, None])
        else:
            events[kind][-1][1] = e

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    n0 = L.sseqs_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    cells = 0
    exact_rows = {}
    for q in timed:
        rows, _ = run_step(M, q, db, timer=timer, world=world, rank=rank)
        exact_rows.setdefault(q, rows)
        cells += 2 * len(q) * res_cells
    e1.record()
    torch.cuda.synchronize()
    n_launch = L.sseqs_launch_count() - n0
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_cells = cells * world
    gcups = total_cells / (ms * 1e-3) / 1e9
    aff_ms = [a.elapsed_time(b) for a, b in events["affine"]]
    both_ms = [a.elapsed_time(b) for a, b in events["both"]]
    # queries of up to 736 residues score both variants in one fused launch;
    # longer ones launch the affine kernel on its own
    aff_cells = sum(len(q) * res_cells for q in timed if not tune.fused(len(q)))
    both_cells = sum(len(q) * res_cells for q in timed if tune.fused(len(q)))

    # end to end through the public call (host query in, a3m file out)
    import sseqs_b200
    e2e_ms = 0.0
    tmp = tempfile.mkdtemp()
    h0, d0 = _lib.transfer_bytes["h2d"], _lib.transfer_bytes["d2h"]
    for q in timed:
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        sseqs_b200.msa(q, os.path.join(tmp, "out.a3m"), num_msas=TOP_K, top_fft=1, top_sw=1,
                       top_sw_affine=TOP_K, bs=BS, db=db, verbose=False)
        s1.record()
        torch.cuda.synchronize()
        e2e_ms += s0.elapsed_time(s1)
    h2d = _lib.transfer_bytes["h2d"] - h0
    d2h = _lib.transfer_bytes["d2h"] - d0
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_gcups = total_cells / (e2e_ms * 1e-3) / 1e9

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    alu_peak = measured_peak("sseqs_dpx_peak")
    dual_peak = measured_peak("sseqs_int16x2_peak")
    aff_rate = aff_cells / max(sum(aff_ms) * 1e-3, 1e-9)  # cells/s of the affine launches
    both_rate = both_cells / max(sum(both_ms) * 1e-3, 1e-9)  # cell positions/s, fused launches
    # The affine kernel issues 3.5 ALU-pipe (max-type DPX) + 2 FMA-pipe
    # (int16x2 add) instructions per int16x2 word, i.e. per 2 cells; the ALU
    # pipe is its limit.
    achieved = aff_rate * 3.5 / 2
    out = {
        "metric": "SW GCUPS on 1 B200",
        "value": round(gcups, 1),
        "unit": "GCUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int16x2",
        "data": "synthetic",
        "config": {
            "workload": "exact search, one query per step: linear (gap -1) + affine (11/1) "
                        "BLOSUM62 SW of every segment of the resident database (top_fft=1, "
                        "top_sw=1), top-4096 per batch, global top-4096, CUDA traceback + a3m",
            **info,
            "queries": "64 seeded, lengths U(50,1000); timed step i uses query i",
            "homologs": "0.5% per query at 20-95% identity, indels 0.02 geometric(0.5)",
            "l2": "inputs larger than L2: the whole resident database is swept every step",
            "parallelism": "one database shard per GPU (weak)" if world > 1 else "1 GPU",
        },
        "queries_per_s": round(len(timed) * world / (ms * 1e-3), 3),
        "gcups_affine_kernel": round(aff_rate / 1e9, 1),
        "gcups_fused_kernel": round(2 * both_rate / 1e9, 1),
        "roofline": {
            "bound": "int-pipe (ALU, DPX)",
            "kernel": "sw_stream_kernel<affine> (dominant launch of the step; queries of more "
                      "than 736 residues)",
            "achieved": round(achieved / 1e9, 1),
            "peak": round(alu_peak / 1e9, 1),
            "unit": "Gop/s",
            "frac": round(achieved / alu_peak, 4),
            # DRAM bytes of one affine launch (one database batch): the ncu
            # capture of this kernel on a 1M-sequence batch read 381.9 MB and
            # wrote 10.0 MB for 372.7M residues, i.e. ~1.05 B per residue,
            # scaled here to the residues of an average batch of this database
            "traffic": int(TRAFFIC_BYTES_PER_RESIDUE * res_cells / max(1, len(db.batches))),
            "traffic_source": "ncu dram__bytes_read+write of the affine launch at 1M sequences "
                              "(391.9 MB / 372.7M residues), scaled to an average batch",
            "algorithmic_bytes": int(res_cells / max(1, len(db.batches))),
            "ops_model": "3.5 ALU-pipe DPX int16x2 instructions per 2 cells (affine kernel)",
            "peak_source": "sseqs_dpx_peak measured in this run: ALU-pipe int16x2 DPX issue rate",
            "dual_pipe": {"achieved": round(aff_rate * 5.5 / 2 / 1e9, 1),
                          "peak": round(dual_peak / 1e9, 1),
                          "frac": round(aff_rate * 5.5 / 2 / dual_peak, 4),
                          "ops_model": "5.5 int16x2 instructions per 2 cells (3.5 ALU + 2 FMA)"},
            "fused": {"kernel": "sw_stream_kernel<both> (queries of up to 736 residues)",
                      "achieved": round(both_rate * 2.5 / 1e9, 1),
                      "peak": round(alu_peak / 1e9, 1),
                      "frac": round(both_rate * 2.5 / alu_peak, 4),
                      "ops_model": "1.5 (linear) + 3.5 (affine) ALU-pipe DPX int16x2 "
                                   "instructions per 2 cells"},
            "survey_model": {"peak_cells_per_s": round(alu_peak * 2 / 7 / 1e9, 1),
                             "frac": round(aff_rate / (alu_peak * 2 / 7), 4),
                             "ops_model": "7 DPX ops per 2 cells"},
        },
        "autotune": {f"{m}_tpt{t}": ("wide" if w else "narrow")
                     for (m, t), w in sorted(tuned.items())},
        "e2e": {"value": round(e2e_gcups, 1), "unit": "GCUPS",
                "h2d_bytes_per_step": int(h2d / len(timed)),
                "d2h_bytes_per_step": int(d2h / len(timed)),
                "path": "sseqs_b200.msa(query, file) with the database resident in HBM"},
        "gpu_launches": int(n_launch),
        "clocks": clk,
    }
    if world == 1 and args.reference_legs:
        out["kernels_one_batch"] = kernels_one_batch_leg(db, timed[:4])
        out["linear_gap4"] = linear_gap4_leg(db, timed[:2], res_cells)
        out["search_defaults"] = search_defaults_leg(M, db, timed[:4])
    if world == 1 and args.prefilter_steps > 0:
        out["prefiltered"] = prefiltered_leg(M, db, timed[:args.prefilter_steps], exact_rows)
    if world == 1 and args.batched_queries > 0:
        out["batched"] = batched_leg(db, args.batched_queries)
    if world == 1 and args.serve_requests > 0:
        out["serving"] = serving_leg(db, args.serve_requests, args.serve_rate)
    if world == 1 and args.learned_pairs > 0:
        out["learned"] = learned_leg(db, exact_rows, args.learned_pairs, args.learned_queries,
                                     epochs=args.learned_epochs,
                                     target_power=args.learned_target_power)
        out["learned"]["speedup_vs_exact_step"] = round(
            out["learned"]["queries_per_s"] / out["queries_per_s"], 2)
        if args.serve_requests > 0:
            out["serving_learned"] = serving_leg(db, 4 * args.serve_requests,
                                                 args.serve_rate_learned,
                                                 index=learned_leg.index)
        if args.sweep_seconds > 0:
            out["serving_sweep"] = serving_sweep(learned_leg.index, SWEEP_RATES,
                                                 args.sweep_seconds)
        learned_leg.index = None
    if world == 1 and not args.no_cpu_baseline:
        v, cores, sample, dt = cpu_sample_gcups(queries, args.cpu_seconds)
        out["cpu_baseline"] = {"value": round(v, 3), "unit": "GCUPS", "cores": cores,
                               "kind": "port", "sample": sample, "seconds": round(dt, 1)}
        out["exact_q200_100k"] = small_exact_leg(M)
    print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def bench_reference(args):
    """CPU oracle (restatement of the reference kernels) on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    queries = query_set()
    budget = max(5.0, 10.0 * 1.0)
    vals = []
    t_all = time.time()
    warm, timed = step_queries(queries, args.steps, args.warmup)
    last = None
    for i in range(args.warmup + args.steps):
        v, cores, sample, dt = cpu_sample_gcups(queries, budget, seed=i)
        if i >= args.warmup:
            vals.append((v, dt))
        last = (cores, sample)
    gcups = sum(v * dt for v, dt in vals) / sum(dt for v, dt in vals)
    out = {
        "metric": "SW GCUPS on 1 B200",
        "value": round(gcups, 3),
        "unit": "GCUPS",
        "impl": "reference",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1000 * sum(dt for _, dt in vals) / len(vals), 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int16",
        "data": "synthetic",
        "config": {"workload": "exact search (linear -1 + affine 11/1 SW of every segment) of "
                               "query 0 per step on a bounded same-distribution sample",
                   "wall_s": round(time.time() - t_all, 1)},
        "cpu_baseline": {"value": round(gcups, 3), "unit": "GCUPS", "cores": last[0],
                         "kind": "port", "sample": last[1]},
        "e2e": {"value": round(gcups, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if args.reference_legs:
        out["reference_gpu"] = reference_gpu_legs(queries, args)
    print(json.dumps(out), flush=True)


def reference_gpu_legs(queries, args):
    """The reference's own CUDA kernels (oracle/_ref, compiled from its
    sources) on this GPU, beside the CPU value above: its score kernels over
    the first batch of the benchmark database (the inputs the b200 arm's
    ``kernels_one_batch`` leg times), and its search loop at its defaults
    (oracle/ref_search.py: sseqs/msa.py:196-405 restated around its kernels,
    the database streamed from pinned host memory as the reference does)."""
    try:
        import torch
        from oracle import ref_search, refkernels
        if not (torch.cuda.is_available() and refkernels.available()):
            return {"unavailable": "no GPU or oracle/_ref not built"}
        from sseqs_b200 import dbtools
        syn = dbtools.synthetic_db(queries, args.db_seqs, HOMOLOG_FRAC, IDENT, seed=0,
                                   device="cuda")
        _, timed = step_queries(queries, args.steps, args.warmup)
        res = {"kernels_one_batch": ref_search.kernels_one_batch(timed[:4], syn.chunks[0])}
        pinned = ref_search.pinned_copies(syn.chunks)
        del syn
        torch.cuda.empty_cache()
        ref_search.search_chunks(queries[-1], pinned[:1])             # warm-up
        qs = timed[:4]
        t0 = time.time()
        for q in qs:
            ref_search.search_chunks(q, pinned)
        dt = time.time() - t0
        packed = sum(p.numel() for p in pinned)
        res["search_defaults"] = {
            "GB_per_s": round(packed * len(qs) / dt / 1e9, 2),
            "ms_per_query": round(dt * 1e3 / len(qs), 1),
            "queries": len(qs), "packed_bytes": packed,
            "settings": "bs=5e7, top_fft=200, top_sw=10, top_sw_affine=2, chunks streamed "
                        "from pinned host memory (the reference's loop)"}
        return res
    except Exception as e:      # a measurement aid: report, do not fail the arm
        return {"unavailable": f"{type(e).__name__}: {e}"[:300]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--db-seqs", type=int, default=DB_SEQS)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-legs", dest="reference_legs", action="store_false",
                    help="skip the legs that time the reference's kernels (reference arm) and "
                         "this build on the same inputs (b200 arm)")
    ap.add_argument("--prefilter-steps", type=int, default=4,
                    help="queries of the prefiltered (FFT) leg; 0 skips it")
    ap.add_argument("--batched-queries", type=int, default=16,
                    help="queries of the batched uneven-length leg; 0 skips it")
    ap.add_argument("--serve-requests", type=int, default=24,
                    help="requests of the serving leg; 0 skips it")
    ap.add_argument("--serve-rate", type=float, default=0.8,
                    help="Poisson arrival rate (queries/s) of the serving leg (the exact "
                         "pipeline serves about 1.2 q/s at 20M sequences)")
    ap.add_argument("--serve-rate-learned", type=float, default=10.0,
                    help="Poisson arrival rate (queries/s) of the learned serving leg")
    ap.add_argument("--learned-pairs", type=int, default=1_000_000,
                    help="training pairs of the learned-prefilter leg; 0 skips it")
    ap.add_argument("--learned-queries", type=int, default=64,
                    help="queries timed in the learned-prefilter leg")
    ap.add_argument("--learned-epochs", type=int, default=2,
                    help="training epochs over the learned leg's pairs")
    ap.add_argument("--learned-target-power", type=float, default=0.5,
                    help="the embedder's training target is the normalised SW score to this "
                         "power (below 1 spreads remote homologs from unrelated pairs)")
    ap.add_argument("--sweep-seconds", type=float, default=4.0,
                    help="seconds of Poisson arrivals per rate of the learned serving sweep "
                         "(rates %s q/s); 0 skips it" % (SWEEP_RATES,))
    ap.add_argument("--serving-scale", type=int, default=0,
                    help="instead of the benchmark: build a database of this many sequences, "
                         "its learned index, and run the serving sweep over it")
    ap.add_argument("--learned-scale", action="store_true",
                    help="instead of the benchmark: the learned prefilter at its stated size "
                         "(training on --learned-pairs pairs, --learned-queries timed queries, "
                         "recall over --recall-queries queries with planted homologs)")
    ap.add_argument("--index-dim", type=int, default=256, choices=(128, 256),
                    help="--serving-scale: width of the FP8 index codes (128: the embeddings "
                         "projected onto their 128 leading principal directions)")
    ap.add_argument("--scale-recall-queries", type=int, default=2,
                    help="--serving-scale: planted-homolog queries whose recall of the exact "
                         "top-1000 is measured (each needs one exhaustive search)")
    ap.add_argument("--recall-queries", type=int, default=128,
                    help="queries with planted homologs whose recall --learned-scale reports")
    ap.add_argument("--recall-homologs", type=int, default=500,
                    help="planted homologs per recall query in --learned-scale")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        bench_reference(args)
    elif args.serving_scale > 0:
        bench_serving_scale(args)
    elif args.learned_scale:
        bench_learned_scale(args)
    else:
        bench_b200(args)


if __name__ == "__main__":
    main()

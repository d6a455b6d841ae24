"""``msa(queries, filenames, ...)`` -- database search and a3m output.

Same signature, defaults and output files as sseqs/msa.py:71-446.  Per query
and per database batch the stages of sseqs/msa.py:227-370 run on the GPU
against the HBM-resident database:

  prefilter (skipped when ``top_fft == 1``: every segment passes)
  -> top-k (#segments // top_fft) -> drop the lowest and highest index
  -> linear SW, gap -1 -> top-k (// top_sw) -> affine SW, 11/1
  -> top-k (top_sw_affine) -> score / sqrt(len(query) * longest segment)
  -> hit strings (first 500 residues)

then the hits of all batches are ranked and the best ``num_msas`` go through
the CUDA traceback into the a3m file (sseqs/msa.py:411-437).

Where the reference leaves an order unspecified (ties inside torch.topk and
numpy's argsort), hits are ordered by score, then by database position.
"""
from __future__ import annotations

import hashlib
import importlib
import math
import os
import pickle
import threading
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import select, tune
from ._lib import check, lib, ptr, stream_ptr, to_host
from .database import Database, default_database
from .to_a3m import to_a3m

_sw = importlib.import_module("sseqs_b200.sw")

HIT_WIDTH = 500           # sseqs/msa.py:183
_last_call: dict = {}     # gpu -> thread of the last non-blocking msa() call

# The keys of msa(..., return_timings=True) (sseqs/msa.py:442-446).  Here
# t_fft is the prefilter, t_topk1 its top-k, t_sw the linear and affine
# scoring with their top-k, t_out the hit gather, t_a3m the traceback and
# file; decompression and host-to-device copies happen once, when the
# database is loaded, so those keys and the reference's other
# per-batch preparation keys stay 0.
TIMING_KEYS = ("t_dec", "t_prep1", "t_prep2", "t_fft", "t_prep_fft", "t_sw", "t_out",
               "t_out_cpu", "t_log", "t_topk1", "t_topk2", "t_save", "t_prep_sw", "t_a3m",
               "t_to_vram")


@dataclass
class BatchHits:
    batch: int
    g: torch.Tensor          # filtered segment index of each hit (device, increasing)
    affine: torch.Tensor
    linear: torch.Tensor
    hits: torch.Tensor       # [n, HIT_WIDTH] bytes
    hit_len: torch.Tensor
    maxlen: int
    cells_linear: int
    cells_affine: int
    pos: torch.Tensor | None = None     # position of each hit in the candidate list
    fft: torch.Tensor | None = None     # prefilter scores of the batch (None: not computed)


class SearchStats:
    """Host seconds per stage; with ``sync`` every stage waits for the GPU
    before its clock is read (the reference's ``sync_time``)."""

    def __init__(self, sync: bool = False):
        self.cells = 0
        self.stage = {}
        self.sync = sync

    def add(self, key, dt):
        self.stage[key] = self.stage.get(key, 0.0) + dt

    def clock(self) -> float:
        if self.sync:
            torch.cuda.synchronize()
        return time.time()

    def timings(self) -> dict:
        """The reference's timings dict: every key of TIMING_KEYS."""
        return {k: float(self.stage.get(k, 0.0)) for k in TIMING_KEYS}


def _gather_hits(batch, g, n):
    out = torch.empty((max(n, 1), HIT_WIDTH), dtype=torch.uint8, device=batch.ascii.device)
    ln = torch.empty(max(n, 1), dtype=torch.int32, device=batch.ascii.device)
    check(lib().sseqs_gather_windows(ptr(batch.ascii), ptr(batch.offsets), ptr(batch.lengths),
                                     ptr(g), n, HIT_WIDTH, ptr(out), ptr(ln), stream_ptr()),
          "gather_windows")
    return out[:n], ln[:n]


def search_batch(q_enc: torch.Tensor, query: str, batch, bi: int, *, top_fft=200, top_sw=10,
                 top_sw_affine=2, fft_rank=4, luts=None, stats: SearchStats | None = None,
                 timer=None):
    """One query against one resident batch (sseqs/msa.py:235-370)."""
    nseg = batch.n_segments
    dev = batch.ascii.device
    k1 = nseg // top_fft
    n_c = k1 - 2                                            # [1:-1] (msa.py:307)
    if n_c <= 0:
        return None
    if top_fft == 1:
        cand = None                                         # segments 1 .. nseg-2
    else:
        from . import conv
        t0 = stats.clock() if stats is not None else 0.0
        scores = conv.prefilter_batch(query, batch, luts, fft_rank)
        t1 = stats.clock() if stats is not None else 0.0
        cand = select.topk_indices(scores, k1)[1:-1]
        if stats is not None:
            stats.add("t_fft", t1 - t0)
            stats.add("t_topk1", stats.clock() - t1)
    t_sw0 = stats.clock() if stats is not None else 0.0
    Lq = q_enc.numel()
    k2 = n_c // top_sw
    if top_sw == 1 and tune.fused(Lq):
        # every candidate gets both scores: one fused pass (same scores as
        # the two calls below)
        if timer is not None:
            timer("both", True)
        tgt = dict(g0=1, n_targets=n_c) if cand is None else dict(good_idx=cand)
        lin, aff = _sw.sw_scan_both(q_enc, batch.ascii, batch.delim, affine_skip=1, gap=-1,
                                    gap_open=11, gap_extend=1, **tgt)
        if timer is not None:
            timer("both", False)
        p2, cand2 = None, cand
    else:
        if cand is None:
            lin = _sw.sw_scan(q_enc, batch.ascii, batch.delim, affine=False, g0=1,
                              n_targets=n_c, skip=0, gap_a=-1)
        else:
            lin = _sw.sw_scan(q_enc, batch.ascii, batch.delim, affine=False, good_idx=cand,
                              skip=0, gap_a=-1)
        if k2 <= 0:
            if stats is not None:
                stats.add("t_sw", stats.clock() - t_sw0)
            return None
        if top_sw == 1:
            p2, cand2 = None, cand
        else:
            p2 = select.topk_indices(lin, k2)
            cand2 = (p2 + 1) if cand is None else cand[p2.long()]
        if timer is not None:
            timer("affine", True)
        if cand2 is None:
            aff = _sw.sw_scan(q_enc, batch.ascii, batch.delim, affine=True, g0=1, n_targets=k2,
                              skip=1, gap_a=11, gap_b=1)
        else:
            aff = _sw.sw_scan(q_enc, batch.ascii, batch.delim, affine=True, good_idx=cand2,
                              skip=1, gap_a=11, gap_b=1)
        if timer is not None:
            timer("affine", False)
    # torch.topk raises when top_sw_affine exceeds the list (msa.py:335);
    # here the list is kept whole instead.
    k3 = min(top_sw_affine, k2)
    # The reference scores the affine candidates in the order its linear
    # top-k returned them (msa.py:324-332), so with top-k ties falling to the
    # lower position an affine tie goes to the higher linear score, then to
    # the lower segment: select on the key (affine, linear).  Both scores lie
    # in [-1, 11 * 2048], so (affine + 1) * 2^15 + linear + 1 fits in int32.
    lin_c = lin if p2 is None else lin[p2.long()]
    key = ((aff + 1) << 15) | (lin_c + 1)
    p3 = select.topk_indices(key, k3).long()
    if cand2 is None:
        g = (p3 + 1).to(torch.int32)
    else:
        g = cand2[p3].to(torch.int32)
    pos = p3 if p2 is None else p2.long()[p3]
    if stats is not None:
        t_out0 = stats.clock()
        stats.add("t_sw", t_out0 - t_sw0)
    hits, hlen = _gather_hits(batch, g, k3)
    if stats is not None:
        stats.add("t_out", stats.clock() - t_out0)
    return BatchHits(bi, g, aff[p3], lin[pos], hits, hlen, batch.maxlen, 0, 0, pos,
                     None if top_fft == 1 else scores)


def _norm(aff: np.ndarray, Lq: int, maxlen: int) -> np.ndarray:
    """int32 score / sqrt(len(query) * maxlen) in float32 (msa.py:345)."""
    return (aff.astype(np.float32) / np.sqrt(np.float32(Lq * maxlen))).astype(np.float32)


def rank_hits(query: str, per_batch: list, num_msas: int):
    """Concatenate batch hits, order by normalised score (desc), then batch
    and segment position (asc); keep ``num_msas`` (msa.py:411-427).

    The order is one stable ``np.lexsort`` on those keys (segments are
    unique within a batch, so it is the order of the reference's sort), and
    only the kept rows' hit bytes are gathered and decoded.
    """
    parts = [bh for bh in per_batch if bh is not None and bh.g.numel() > 0]
    if not parts:
        return []
    cols = {k: [] for k in ("norm", "batch", "g", "aff", "lin", "part", "row")}
    for j, bh in enumerate(parts):
        g, aff, lin = to_host(bh.g), to_host(bh.affine), to_host(bh.linear)
        cols["norm"].append(_norm(aff, len(query), bh.maxlen))
        cols["batch"].append(np.full(g.size, bh.batch, dtype=np.int64))
        cols["g"].append(g.astype(np.int64))
        cols["aff"].append(aff)
        cols["lin"].append(lin)
        cols["part"].append(np.full(g.size, j, dtype=np.int64))
        cols["row"].append(np.arange(g.size, dtype=np.int64))
    c = {k: np.concatenate(v) for k, v in cols.items()}
    keep = np.lexsort((c["g"], c["batch"], -c["norm"].astype(np.float64)))[:num_msas]
    kpart, krow = c["part"][keep], c["row"][keep]
    hits = [None] * keep.size
    for j, bh in enumerate(parts):
        pos = np.flatnonzero(kpart == j)
        if pos.size == 0:
            continue
        idx = torch.from_numpy(krow[pos]).to(bh.hits.device)
        hb, hl = to_host(bh.hits.index_select(0, idx)), to_host(bh.hit_len.index_select(0, idx))
        blob, w = hb.tobytes(), hb.shape[1]
        for r, (p, n) in enumerate(zip(pos.tolist(), hl.tolist())):
            hits[p] = blob[r * w:r * w + min(max(n, 0), w)].decode("latin-1")
    return list(zip(c["norm"][keep].tolist(), c["batch"][keep].tolist(), c["g"][keep].tolist(),
                    c["aff"][keep].tolist(), c["lin"][keep].tolist(), hits))


def raw_hits(query: str, per_batch: list):
    """Every batch's hits in the layout of the reference's ``save_raw`` pickle
    (sseqs/msa.py:413-422): [query, hit strings, linear scores, prefilter
    scores, normalised affine scores], batches in order.

    Inside a batch the hits are in the order the reference's top-k calls
    produce when their ties fall to the lower position: affine score, then
    linear score (descending), then segment.  The prefilter column repeats
    the reference's indexing (``scores[good_idx]`` with ``good_idx`` the hit's
    position in the candidate list, sseqs/msa.py:362-363); with
    ``top_fft == 1`` no prefilter runs here and the column holds NaN.
    """
    matches, lin_all, fft_all, norm_all = [], [], [], []
    for bh in per_batch:
        if bh is None or bh.g.numel() == 0:
            continue
        g, aff, lin = to_host(bh.g), to_host(bh.affine), to_host(bh.linear)
        order = np.lexsort((g, -lin.astype(np.int64), -aff.astype(np.int64)))
        idx = torch.from_numpy(order).to(bh.hits.device)
        hb, hl = to_host(bh.hits.index_select(0, idx)), to_host(bh.hit_len.index_select(0, idx))
        w = hb.shape[1]
        blob = hb.tobytes()
        for r, n in enumerate(hl.tolist()):
            matches.append(blob[r * w:r * w + min(max(n, 0), w)].decode("latin-1"))
        norm = _norm(aff[order], len(query), bh.maxlen)
        if bh.fft is None:
            fft = np.full(order.size, np.nan, np.float16)
        else:
            fft = to_host(bh.fft.index_select(0, bh.pos.index_select(0, idx)))
        lin_all.extend(lin[order])
        fft_all.extend(fft)
        norm_all.extend(norm)
    return [query, matches, lin_all, fft_all, norm_all]


def search(queries, db: Database | None = None, *, num_msas=4096, top_fft=200, top_sw=10,
           top_sw_affine=2, fft_rank=4, dlength=1e6, stats: SearchStats | None = None,
           timer=None, bs: int | None = None, per_batch_out: list | None = None):
    """Ranked hits of every query: list (per query) of tuples
    (normalised score, batch, segment, affine, linear, hit string).

    ``per_batch_out``, if given, receives each query's list of per-batch
    ``BatchHits`` (None for a batch that gave none)."""
    if isinstance(queries, str):
        queries = [queries]
    db = default_database(bs) if db is None else db
    from . import conv
    out = []
    for query in queries:
        q_enc = _sw.encode_query(query, device=db.device)
        luts = conv.prefilter_luts(query, fft_rank) if top_fft != 1 else None
        per = []
        for bi, batch in enumerate(db.batches):
            if abs(len(query) - batch.maxlen) > dlength:   # msa.py:252
                continue
            per.append(search_batch(q_enc, query, batch, bi, top_fft=top_fft, top_sw=top_sw,
                                    top_sw_affine=top_sw_affine, fft_rank=fft_rank, luts=luts,
                                    stats=stats, timer=timer))
        out.append(rank_hits(query, per, num_msas))
        if per_batch_out is not None:
            per_batch_out.append(per)
    return out


def msa(queries, filenames=None, num_msas=4096, save_raw="", verbose=True, bs=50_000_000,
        fft_rank=4, top_fft=200, top_sw=10, top_sw_affine=2, return_timings=False,
        sync_time=False, dlength=1e6, gpu: int = 0, blocking: bool = True, db=None):
    """Search every query and write one a3m file per query (sseqs/msa.py:71-446).

    ``bs`` is the batch size the database was decoded with (a resident
    ``Database`` fixes it at load time); ``db`` selects a database other than
    the DBPATH/CHUNKS default.  ``blocking=False`` runs in a thread and
    returns it, as the reference does.
    """
    if not blocking:
        # one call in flight per GPU: a new call first waits for the last one
        # started on the same GPU (sseqs/msa.py:87-101)
        prev = _last_call.get(gpu)
        if prev is not None and prev.is_alive():
            prev.join()
        t = threading.Thread(target=msa, args=(queries, filenames, num_msas, save_raw, verbose,
                                               bs, fft_rank, top_fft, top_sw, top_sw_affine,
                                               return_timings, sync_time, dlength, gpu, True, db))
        _last_call[gpu] = t
        t.start()
        return t
    with torch.cuda.device(gpu):
        if isinstance(queries, str):
            queries = [queries]
        if isinstance(filenames, str):
            filenames = [filenames]
        if filenames is None:
            filenames = [hashlib.sha256(q.encode()).hexdigest()[:8] + ".a3m" for q in queries]
        for f in filenames:
            if f is not None and os.path.exists(f):
                os.remove(f)
        stats = SearchStats(sync=sync_time)
        t0 = time.time()
        per_batch = [] if save_raw != "" else None
        ranked = search(queries, db, num_msas=num_msas, top_fft=top_fft, top_sw=top_sw,
                        top_sw_affine=top_sw_affine, fft_rank=fft_rank, dlength=dlength,
                        stats=stats, bs=bs, per_batch_out=per_batch)
        if sync_time:
            torch.cuda.synchronize()
        stats.add("t_search", time.time() - t0)
        for qi, (query, fname, rows) in enumerate(zip(queries, filenames, ranked)):
            if save_raw != "":
                # one file, rewritten per query, as sseqs/msa.py:420-422 does
                ts = time.time()
                with open(save_raw, "wb") as fh:
                    pickle.dump(raw_hits(query, per_batch[qi]), fh)
                stats.add("t_save", time.time() - ts)
            t1 = time.time()
            if fname is not None:
                if verbose:
                    print(f"Saving result to {fname}")
                to_a3m(query, [r[5] for r in rows], fname)
            stats.add("t_a3m", time.time() - t1)
        if verbose:
            print(f"searched {len(queries)} queries, {sum(len(r) for r in ranked)} hits")
        if return_timings:
            return stats.timings()

"""GPU tests of the search pipeline: prefilter (tolerance), and the whole
per-batch search and a3m output against the CPU oracle (exact)."""
import importlib
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refkernels

pytestmark = pytest.mark.gpu

# Least share of segments whose reference fp16 prefilter score is finite, per
# case (a B200 measured 1.0 for each case but the last, 0.491 there: the
# overflow is a property of the reference kernel, not of this build).
FINITE_SHARE_MIN = {(64, 40): 1.0, (128, 100): 1.0, (256, 180): 1.0, (512, 300): 1.0,
                    (1024, 180): 1.0, (1024, 600): 0.45}


def _db(n_seqs=4000, chunk_bytes=150_000, Lq=180, seed=0, frac=0.02):
    from sseqs_b200 import dbtools
    q = dbtools.random_query(Lq, seed)
    syn = dbtools.synthetic_db([q], n_seqs, frac, (0.3, 0.9), seed=seed, device="cpu",
                               chunk_bytes=chunk_bytes)
    return q, syn


def _host_batches(syn, bs):
    """Decoded batches exactly as sseqs/msa.py:217-220 slices the chunks."""
    out = []
    for c in syn.chunks:
        c = c.numpy()
        for j in range(c.size // bs):
            out.append(O.xbit_decompress(c, int(bs * 8 / 5), j * bs))
    return out


# (transform length N, query length, longest segment): one case per N the
# reference instantiates (sseqs/filter.cu:182-312), plus N = 2048 (none there)
# with the query or a segment longer than 1024
PREFILTER_CASES = [(64, 40, 50), (128, 100, 128), (256, 180, 256), (512, 300, 512),
                   (1024, 180, 1000), (1024, 600, 1000), (2048, 1500, 1000),
                   (2048, 300, 1800), (2048, 2000, 2048)]


@pytest.mark.parametrize("N,Lq,maxlen", PREFILTER_CASES)
def test_prefilter_matches_float64_oracle_and_reference(N, Lq, maxlen):
    """fp32 direct sums vs the float64 restatement (tight), and vs the
    reference's own fp16 FFT kernel wherever that kernel's score is finite:
    its spectrum products overflow fp16 for long inputs, so the finite share
    is printed and asserted, and on the finite scores the values correlate
    and a 1/10 selection keeps the same segments."""
    from sseqs_b200 import conv, dbtools
    rng = np.random.default_rng(N + Lq)
    query = dbtools.random_query(Lq, Lq)
    lens = rng.integers(5, maxlen + 1, 700)
    lens[0] = maxlen
    segs = [dbtools.random_query(int(n), 100 + i) for i, n in enumerate(lens)]
    for i in range(5, 700, 37):           # planted pieces of the query
        a = int(rng.integers(0, max(1, Lq - 30)))
        piece = query[a:a + int(min(len(segs[i]), Lq - a))]
        segs[i] = piece + segs[i][len(piece):]
    segs[3] = (segs[3][:10] + "XXXBZ" + segs[3][15:])[:len(segs[3])]
    ascii = np.frombuffer(("@".join(segs) + "@").encode(), np.uint8).copy()
    seg = O.segment(ascii)
    n = conv.transform_length(Lq, int(seg["lengths"].max()))
    assert n == N
    A, B = O.prefilter_luts(query, 4)
    exp = O.prefilter_scores(query, A, B, ascii, seg["offsets"], seg["lengths"], n, 4)
    luts = conv.prefilter_luts(query, 4)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    got = conv.prefilter_scores(luts, d(ascii), d(seg["offsets"]), d(seg["lengths"].astype(np.int32)),
                                len(seg["lengths"]), n, 4).float().cpu().numpy()
    tol = 2e-3 * np.maximum(1.0, np.abs(exp))
    assert np.all(np.abs(got - exp) <= tol), np.max(np.abs(got - exp) / np.maximum(1, np.abs(exp)))
    if N > 1024:
        return                            # the reference computes nothing at N = 2048
    if not refkernels.available():
        pytest.skip("oracle/_ref/libsseqs_ref.so not built")
    ref = refkernels.warp_corr(query, A, B, d(ascii), d(seg["offsets"]),
                               d(seg["lengths"]), n, 4).float().cpu().numpy()
    fin = np.isfinite(ref)
    k = len(exp) // 10
    top_ref = set(np.argsort(-np.where(fin, ref, -np.inf), kind="stable")[:k])
    top_got = set(np.argsort(-got, kind="stable")[:k])
    overlap = len(top_ref & top_got) / k
    corr = np.corrcoef(ref[fin], got[fin])[0, 1] if fin.sum() > 2 else float("nan")
    print(f"N={N} Lq={Lq}: reference finite on {fin.mean():.3f} of segments, "
          f"corr {corr:.4f} on those, top-1/10 overlap {overlap:.3f}")
    assert fin.mean() >= FINITE_SHARE_MIN[(N, Lq)]
    assert corr > 0.99
    if fin.all():
        assert overlap >= 0.9


@pytest.mark.parametrize("k", [1, 3, 6])
def test_prefilter_other_ranks_match_float64_oracle(k):
    """Ranks 1-4 take the tensor-core form, higher ranks the direct form; both
    give the float64 restatement's scores (rank 1 clamps BLOSUM62 at 0,
    sseqs/msa.py:125)."""
    from sseqs_b200 import conv, dbtools
    rng = np.random.default_rng(k)
    query = dbtools.random_query(300, k)
    segs = [dbtools.random_query(int(n), 300 + i) for i, n in enumerate(rng.integers(1, 500, 400))]
    ascii = np.frombuffer(("@".join(segs) + "@").encode(), np.uint8).copy()
    seg = O.segment(ascii)
    n = conv.transform_length(len(query), int(seg["lengths"].max()))
    A, B = O.prefilter_luts(query, k)
    exp = O.prefilter_scores(query, A, B, ascii, seg["offsets"], seg["lengths"], n, k)
    luts = conv.prefilter_luts(query, k)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    got = conv.prefilter_scores(luts, d(ascii), d(seg["offsets"]), d(seg["lengths"].astype(np.int32)),
                                len(seg["lengths"]), n, k).float().cpu().numpy()
    tol = 2e-3 * np.maximum(1.0, np.abs(exp))
    assert np.all(np.abs(got - exp) <= tol)


def _oracle_search(query, batches, prefilter_fn=None, **kw):
    """Oracle restatement over the non-empty batches (numbered in order)."""
    rows = []
    bi = 0
    for a in batches:
        seg = O.segment(a)
        if seg["lengths"].size == 0:
            continue
        scores = prefilter_fn(bi) if prefilter_fn else None
        for g, aff, lin, norm, s in O.search_batch(query, a, prefilter=scores, **kw):
            rows.append((norm, bi, g, aff, lin, s))
        bi += 1
    rows.sort(key=lambda x: (-x[0], x[1], x[2]))
    return rows


@pytest.mark.parametrize("top_sw,top_sw_affine", [(1, 60), (3, 25)])
def test_exact_search_matches_oracle(top_sw, top_sw_affine):
    from sseqs_b200.database import Database
    M = importlib.import_module("sseqs_b200.msa")
    q, syn = _db()
    bs = 50_000
    db = Database(syn.chunks, bs=bs)
    got = M.search([q], db, num_msas=10_000, top_fft=1, top_sw=top_sw,
                   top_sw_affine=top_sw_affine)[0]
    exp = _oracle_search(q, _host_batches(syn, bs), top_fft=1, top_sw=top_sw,
                         top_sw_affine=top_sw_affine)
    assert len(got) == len(exp)
    for a, b in zip(got, exp):
        assert a[1:] == b[1:]
        assert a[0] == pytest.approx(b[0], rel=0, abs=0)


def test_prefiltered_search_matches_oracle_given_scores():
    from sseqs_b200 import conv
    from sseqs_b200.database import Database
    M = importlib.import_module("sseqs_b200.msa")
    q, syn = _db(seed=3)
    bs = 75_000
    db = Database(syn.chunks, bs=bs)
    got = M.search([q], db, num_msas=10_000, top_fft=7, top_sw=2, top_sw_affine=10)[0]
    luts = conv.prefilter_luts(q, 4)
    batches = _host_batches(syn, bs)
    scores = [conv.prefilter_batch(q, b, luts, 4).float().cpu().numpy() for b in db.batches]
    assert sum(1 for b in batches if O.segment(b)["lengths"].size) == len(scores)
    exp = _oracle_search(q, batches, top_fft=7, top_sw=2, top_sw_affine=10,
                         prefilter_fn=lambda bi: scores[bi])
    assert [r[1:] for r in got] == [r[1:] for r in exp]


def test_msa_writes_oracle_a3m(tmp_path):
    from sseqs_b200.database import Database
    import sseqs_b200
    q, syn = _db(n_seqs=3000, seed=5)
    db = Database(syn.chunks, bs=150_000)
    f = tmp_path / "out.a3m"
    t = sseqs_b200.msa(q, str(f), num_msas=200, top_fft=1, top_sw=1, top_sw_affine=200,
                       bs=150_000, db=db, verbose=False, return_timings=True, sync_time=True)
    # the reference's timings dict (sseqs/msa.py:442-446)
    assert set(t) == set(importlib.import_module("sseqs_b200.msa").TIMING_KEYS)
    assert t["t_sw"] > 0 and t["t_a3m"] > 0 and t["t_out"] > 0 and t["t_fft"] == 0
    rows = _oracle_search(q, _host_batches(syn, 150_000), top_fft=1, top_sw=1,
                          top_sw_affine=200)[:200]
    _, al = O.sw_affine_backtrack(q, [r[5] for r in rows])
    assert f.read_text() == O.to_a3m_text(q, al)
    # planted homologs dominate the top of the list
    assert sum(1 for r in rows[:20] if r[3] > 100) >= 15


def test_msa_non_blocking_runs_one_call_per_gpu(tmp_path):
    """blocking=False returns the thread; a second call on the same GPU first
    waits for the one before it (sseqs/msa.py:87-101), and both write the
    same a3m as a blocking call."""
    from sseqs_b200.database import Database
    import sseqs_b200
    q, syn = _db(n_seqs=2000, seed=6)
    db = Database(syn.chunks, bs=150_000)
    kw = dict(num_msas=100, top_fft=1, top_sw=1, top_sw_affine=100, bs=150_000, db=db,
              verbose=False)
    f0, f1, f2 = (tmp_path / f"{i}.a3m" for i in range(3))
    sseqs_b200.msa(q, str(f0), **kw)
    t1 = sseqs_b200.msa(q, str(f1), blocking=False, **kw)
    t2 = sseqs_b200.msa(q, str(f2), blocking=False, **kw)
    assert not t1.is_alive()
    t2.join()
    assert f1.read_text() == f0.read_text() == f2.read_text()


def test_fasta_database_names_its_hits(tmp_path):
    """A FASTA file packed with its sidecar index, loaded with batches smaller
    than a chunk: every ranked hit's string lies inside the sequence its
    name (from the index) points at, and planted homologs are named."""
    from sseqs_b200 import dbtools
    from sseqs_b200.database import Database
    M = importlib.import_module("sseqs_b200.msa")
    rng = np.random.default_rng(9)
    q = dbtools.random_query(150, 9)
    seqs = {}
    lines = []
    for i in range(1500):
        if i % 97 == 0:        # planted homolog: a mutated copy of the query
            s = "".join(c if rng.random() < 0.8 else "ACDEFGHIKLMNPQRSTVWY"[rng.integers(20)]
                        for c in q)
            name = f"hom{i} planted"
        else:
            s = dbtools.random_query(int(rng.integers(20, 400)), 5000 + i)
            name = f"bg{i}"
        seqs[name] = s
        lines.append(f">{name}\n{s[:60]}\n{s[60:]}\n")
    fa = tmp_path / "db.fasta"
    fa.write_text("".join(lines))
    xb = str(tmp_path / "db.xbit")
    idx = dbtools.fasta_to_xbit(str(fa), xb, chunk_bytes=100_000)
    assert idx.n_chunks >= 3
    db = Database.from_file(xb, bs=50_000, chunk_bytes=100_000)
    assert db.index is not None
    rows = M.search([q], db, num_msas=300, top_fft=1, top_sw=1, top_sw_affine=300)[0]
    names = db.hit_names(rows)
    assert len(names) == len(rows)
    for row, name in zip(rows, names):
        assert name is not None and row[5] in seqs[name], (row[1], row[2], name)
    # 16 planted; the first and last segment of every batch are not searched
    # (sseqs/msa.py:307), which can take out a few
    planted = [n for n in names[:16] if n.startswith("hom")]
    assert len(planted) >= 12

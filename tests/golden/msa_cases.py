"""Seeded end-to-end search cases shared by ``make_msa_golden.py`` (which runs
the reference's ``msa()`` on them, here on the CPU) and
``tests/test_gpu_msa_golden.py`` (which runs ``sseqs_b200.msa`` on them on
the GPU and compares with the stored outputs).

Each case is one 1e9-byte .xbit chunk, the unit the reference reads into
pinned memory (sseqs/msa.py:50-55), searched with the reference's default
batch size bs = 5e7 packed bytes, i.e. 20 batches (sseqs/msa.py:217).  The
sequences are split into 20 consecutive groups and group j is packed at
packed offset j * bs, so every batch starts with a whole sequence and ends in
zero ('@') padding.  No batch is padding only: the reference fails on such a
batch (``lengths.max()`` of an empty tensor, sseqs/msa.py:261).

The database is the benchmark's synthetic model (``dbtools.synthetic_db``:
background composition, log-normal lengths clipped to 30..1000, planted
homologs of the query), optionally with empty sequences ('@@', which move the
reference's filtered segment indices against its delimiter positions,
sseqs/msa.py:253 vs :313-319) and non-standard letters (X, B, Z, U).
"""
from __future__ import annotations

import hashlib

import numpy as np

CHUNK = 1_000_000_000
BS = 50_000_000
N_BATCHES = CHUNK // BS

CASES = {
    # the CPU-runnable benchmark configuration, searched exactly: every
    # segment is scored by both SW variants, 50 best per batch, top 1000
    "exact": dict(Lq=200, n_seqs=100_000, homolog_frac=0.01, ident=(0.3, 0.9), seed=0,
                  empty_frac=0.0, odd_frac=0.0,
                  params=dict(top_fft=1, top_sw=1, top_sw_affine=50, num_msas=1000)),
    # empty segments and non-standard letters, exact search
    "empty_segments": dict(Lq=150, n_seqs=20_000, homolog_frac=0.01, ident=(0.3, 0.9), seed=1,
                           empty_frac=0.03, odd_frac=0.005,
                           params=dict(top_fft=1, top_sw=1, top_sw_affine=20, num_msas=400)),
    # the reference's defaults: prefilter keeps 1/200, linear SW 1/10, 2 per batch
    "prefilter_defaults": dict(Lq=200, n_seqs=100_000, homolog_frac=0.01, ident=(0.3, 0.9),
                               seed=2, empty_frac=0.0, odd_frac=0.0,
                               params=dict(top_fft=200, top_sw=10, top_sw_affine=2,
                                           num_msas=4096)),
}


def _unpack(packed: np.ndarray, n: int) -> np.ndarray:
    """5-bit symbols of ``packed`` as ASCII bytes (layout of sseqs/xbit.cu:8-34)."""
    g = (n + 7) // 8
    p = np.zeros(g * 5, np.uint8)
    m = min(packed.size, p.size)
    p[:m] = packed[:m]
    w = np.zeros(g, np.uint64)
    for b in range(5):
        w = (w << np.uint64(8)) | p[b::5].astype(np.uint64)
    out = np.empty((g, 8), np.uint8)
    for k in range(8):
        out[:, k] = ((w >> np.uint64(35 - 5 * k)) & np.uint64(31)).astype(np.uint8) + 64
    return out.reshape(-1)[:n]


def case_sequences(name: str):
    """(query, list of sequence byte strings) of a case, in file order."""
    from sseqs_b200 import dbtools
    c = CASES[name]
    q = dbtools.random_query(c["Lq"], c["seed"])
    syn = dbtools.synthetic_db([q], c["n_seqs"], c["homolog_frac"], c["ident"], seed=c["seed"],
                               device="cpu", chunk_bytes=BS)
    assert len(syn.chunks) == 1
    n_sym = syn.n_residues + syn.n_seqs
    stream = _unpack(syn.chunks[0].numpy(), n_sym).tobytes()
    seqs = stream.split(b"@")[:-1]
    assert len(seqs) == syn.n_seqs
    rng = np.random.default_rng(1000 + c["seed"])
    if c["odd_frac"] > 0:
        odd = np.frombuffer(b"XBZU", np.uint8)
        out = []
        for s in seqs:
            a = np.frombuffer(s, np.uint8).copy()
            m = rng.random(a.size) < c["odd_frac"]
            a[m] = rng.choice(odd, int(m.sum()))
            out.append(a.tobytes())
        seqs = out
    if c["empty_frac"] > 0:
        out = []
        for s in seqs:
            if rng.random() < c["empty_frac"]:
                out.append(b"")
            out.append(s)
        seqs = out
    return q, seqs


def case_chunk(name: str):
    """(query, 1e9-byte packed chunk as uint8 numpy array, its sha256)."""
    from sseqs_b200 import dbtools
    q, seqs = case_sequences(name)
    chunk = np.zeros(CHUNK, np.uint8)
    bounds = np.linspace(0, len(seqs), N_BATCHES + 1).round().astype(np.int64)
    for j in range(N_BATCHES):
        group = seqs[bounds[j]:bounds[j + 1]]
        sym = np.frombuffer(b"".join(s + b"@" for s in group), np.uint8)
        packed = dbtools.pack_symbols_host(sym)
        assert packed.size <= BS
        chunk[j * BS:j * BS + packed.size] = packed
    return q, chunk, hashlib.sha256(chunk.tobytes()).hexdigest()

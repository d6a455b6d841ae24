"""HBM-resident sequence database.

The reference streams 1e9-byte .xbit chunks from pinned host RAM to the GPU
on every search and re-derives the segment structure of every batch
(sseqs/msa.py:13-64, :196-267).  Here a database is decoded once: for every
batch (``bs`` packed bytes of a chunk, decoded to ``bs*8/5`` symbols exactly as
sseqs/msa.py:217-220 slices it) the decoded bytes, the '@' positions and the
non-empty segment table stay resident in HBM, so a search touches no host
memory except its own results.

Trailing '@' padding of a batch (the zero fill of a chunk) is trimmed after
the first delimiter: padding only forms empty segments, which the reference
drops (sseqs/msa.py:253), after every real segment, so no index or result
changes.  A batch that is padding only is skipped (the reference fails on it
at sseqs/msa.py:261).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import select, xbit

CHUNK_BYTES = 1_000_000_000


@dataclass
class Batch:
    chunk: int
    index: int                 # batch number inside its chunk
    ascii: torch.Tensor        # decoded bytes, trimmed (device)
    n_symbols: int             # untrimmed batch size (bs*8/5)
    delim: torch.Tensor        # '@' positions, int32 (device)
    seg_index: torch.Tensor    # non-empty segment k of each filtered index
    lengths: torch.Tensor      # int32 lengths of the non-empty segments
    offsets: torch.Tensor      # int64 start of each (running sum of length+1)
    maxlen: int
    n_segments: int
    n_residues: int


def _effective_length(ascii: torch.Tensor) -> int:
    """Index after the delimiter that closes the last non-'@' byte."""
    n = ascii.numel()
    if n == 0:
        return 0
    blk = 1 << 16
    nb = (n + blk - 1) // blk
    pad = nb * blk - n
    a = torch.nn.functional.pad(ascii, (0, pad), value=64) if pad else ascii
    any_res = (a.view(nb, blk) != 64).any(1)
    nzb = torch.nonzero(any_res).flatten()
    if nzb.numel() == 0:
        return 0
    b = int(nzb[-1].item())
    row = a[b * blk:(b + 1) * blk]
    last = b * blk + int(torch.nonzero(row != 64).flatten()[-1].item())
    return min(n, last + 2)


class Database:
    """A list of packed chunks, decoded into resident batches."""

    def __init__(self, chunks, bs: int = CHUNK_BYTES, device="cuda", keep_packed: bool = False):
        self.device = torch.device(device)
        self.bs = int(bs)
        self.batches: list[Batch] = []
        self.packed = [] if keep_packed else None
        self.n_residues = 0
        self.index = None          # sidecar segment index (from_file), if any
        self.n_chunks = 0
        self.add_chunks(chunks)

    def add_chunks(self, chunks) -> None:
        """Decode more packed chunks into resident batches (after the ones
        already loaded), so a large database can be built a part at a time
        without holding all of it packed."""
        for ch in chunks:
            ci = self.n_chunks
            ch = ch if isinstance(ch, torch.Tensor) else torch.from_numpy(np.asarray(ch, np.uint8))
            ch = ch.to(self.device, torch.uint8)
            if ch.numel() % self.bs:
                raise ValueError("chunk size must be a multiple of bs (sseqs/msa.py:216)")
            if self.packed is not None:
                self.packed.append(ch)
            for j in range(ch.numel() // self.bs):
                self._add_batch(ci, j, ch)
            self.n_chunks += 1
            del ch

    def _add_batch(self, ci, j, ch):
        n_sym = int(self.bs * 8 / 5)
        full = xbit.decompress(ch, n_sym, j * self.bs)
        eff = _effective_length(full)
        if eff == 0:
            return
        ascii = full[:eff].clone() if eff < full.numel() else full
        del full
        delim = select.find_delims(ascii)
        tab = select.segment_table(ascii, delim)
        if tab["n_segments"] == 0:
            return
        res = int(tab["lengths"].sum(dtype=torch.int64).item())
        self.n_residues += res
        self.batches.append(Batch(ci, j, ascii, n_sym, delim, tab["seg_index"], tab["lengths"],
                                  tab["offsets"], tab["maxlen"], tab["n_segments"], res))

    @classmethod
    def from_file(cls, path: str, chunks: int | None = None, bs: int = CHUNK_BYTES,
                  device="cuda", chunk_bytes: int = CHUNK_BYTES):
        """Read ``chunks`` chunks of ``chunk_bytes`` from an .xbit file
        (sseqs/msa.py:50-55); bytes past the end of the file read as 0.  A
        sidecar segment index next to the file (``dbtools.fasta_to_xbit``)
        is loaded as ``index`` when its chunk size matches."""
        from .dbtools import SeqIndex, index_path
        size = os.path.getsize(path)
        n = math.ceil(size / chunk_bytes) if chunks is None else int(chunks)
        out = []
        with open(path, "rb") as fh:
            for i in range(n):
                buf = np.zeros(chunk_bytes, np.uint8)
                fh.seek(i * chunk_bytes)
                fh.readinto(memoryview(buf))
                out.append(torch.from_numpy(buf))
        db = cls(out, bs=bs, device=device)
        if os.path.exists(index_path(path)):
            idx = SeqIndex.load(index_path(path))
            if idx.chunk_bytes == chunk_bytes:
                db.index = idx
        return db

    def hit_names(self, hits) -> list:
        """FASTA names of ranked hits ((…, batch, segment, …) rows as
        ``msa.search`` returns them): the sequence holding the first byte of
        the hit's window (``offsets[g]`` of its batch, the bytes the hit
        string shows), from the sidecar index; None where a position is not
        inside a sequence."""
        if self.index is None:
            raise ValueError("no sidecar segment index loaded for this database")
        if (self.bs * 8) % 5:
            raise ValueError("batch boundaries fall inside a 5-byte group (bs % 5 != 0)")
        by_batch: dict = {}
        for r, row in enumerate(hits):
            by_batch.setdefault(int(row[1]), []).append((r, int(row[2])))
        names = [None] * len(hits)
        for bi, items in by_batch.items():
            b = self.batches[bi]
            g = torch.tensor([x[1] for x in items], dtype=torch.int64, device=b.offsets.device)
            off = b.offsets.index_select(0, g).cpu().numpy()
            base = b.index * self.bs * 8 // 5
            for (r, _), o in zip(items, off.tolist()):
                k = self.index.locate(b.chunk, base + o)
                names[r] = self.index.names[k] if k >= 0 else None
        return names

    @property
    def n_segments(self) -> int:
        return sum(b.n_segments for b in self.batches)


_default: dict = {}


def default_database(bs: int | None = None) -> Database:
    """The database named by DBPATH / CHUNKS, decoded with batch size ``bs``
    and loaded on first use (sseqs/msa.py:13-25 loads it at import time and
    exits if it is missing)."""
    bs = 50_000_000 if bs is None else int(bs)
    if bs not in _default:
        path = os.environ.get("DBPATH", "uniref_bfd_mgy_cf.xbit")
        chunks = int(os.environ.get("CHUNKS", 4))
        if not os.path.exists(path):
            raise FileNotFoundError(f"Didn't find MSA database at `{path}` (set DBPATH)")
        _default.clear()
        _default[bs] = Database.from_file(path, chunks=chunks, bs=bs)
    return _default[bs]

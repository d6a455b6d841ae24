"""Smith-Waterman scoring and traceback on the B200.

Mirrors two reference modules:

* the ``sw`` torch extension (sseqs/sw_bind.cpp:111-131):
  ``sw_cuda_blosum62(query_indices_tensor, good_idx, ascii_tensor,
  lengths_tensor, gap_penalty_param=-10)`` and ``sw_cuda_affine(...,
  gap_open=11, gap_extend=1)`` return int32 CUDA tensors;
* ``sseqs/sw.py``: ``sw(query, targets, gap_open=11, gap_extend=1)`` and
  ``sw_affine_backtrack(query, targets, gap_open=11, gap_extend=1,
  device="cuda", scores=False)``.

All kernels run on the current torch CUDA stream; there is no CPU path.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import check, lib, ptr, require_cuda, stream_ptr, to_device, to_host, workspace

AA = "ARNDCQEGHILKMFPSTWYV"
AA_MAP = {aa: i for i, aa in enumerate(AA)}


def _i32(t: torch.Tensor) -> torch.Tensor:
    t = t.to(dtype=torch.int32)
    return t if t.is_contiguous() else t.contiguous()


def _u8(t: torch.Tensor) -> torch.Tensor:
    t = t.to(dtype=torch.uint8)
    return t if t.is_contiguous() else t.contiguous()


def sw_cuda_blosum62(query_indices_tensor: torch.Tensor, good_idx: torch.Tensor,
                     ascii_tensor: torch.Tensor, lengths_tensor: torch.Tensor,
                     gap_penalty_param: int = -10) -> torch.Tensor:
    """Linear-gap score of every window (sseqs/sw_bind.cpp:32-73).

    ``lengths_tensor`` holds window boundaries: target t scores
    ``ascii[lengths[g-1]+1 : lengths[g]]`` for ``g = good_idx[t]``.
    """
    q, g = _u8(query_indices_tensor), _i32(good_idx)
    a, s = _u8(ascii_tensor), _i32(lengths_tensor)
    require_cuda(q, g, a, s)
    out = torch.empty(g.numel(), dtype=torch.int32, device=q.device)
    check(lib().sseqs_sw_linear(ptr(q), q.numel(), ptr(g), ptr(a), ptr(s), g.numel(), ptr(out),
                                int(gap_penalty_param), stream_ptr()), "sw_cuda_blosum62")
    return out


def sw_cuda_affine(query_indices_tensor: torch.Tensor, good_idx: torch.Tensor,
                   ascii_tensor: torch.Tensor, lengths_tensor: torch.Tensor,
                   gap_open: int = 11, gap_extend: int = 1) -> torch.Tensor:
    """Affine-gap score of every window (sseqs/sw_bind.cpp:78-108)."""
    q, g = _u8(query_indices_tensor), _i32(good_idx)
    a, s = _u8(ascii_tensor), _i32(lengths_tensor)
    require_cuda(q, g, a, s)
    out = torch.empty(g.numel(), dtype=torch.int32, device=q.device)
    check(lib().sseqs_sw_affine(ptr(q), q.numel(), ptr(g), ptr(a), ptr(s), g.numel(), ptr(out),
                                int(gap_open), int(gap_extend), stream_ptr()), "sw_cuda_affine")
    return out


def sw_scan(query_idx: torch.Tensor, ascii: torch.Tensor, delim: torch.Tensor, *,
            affine: bool, good_idx: torch.Tensor | None = None, g0: int = 0,
            n_targets: int | None = None, skip: int = 0, gap_a: int = -1, gap_b: int = 0,
            out: torch.Tensor | None = None) -> torch.Tensor:
    """Scores of database segments of one batch held in HBM.

    Segment g is the bytes between the '@' at ``delim[g-1]`` and ``delim[g]``;
    targets are ``good_idx`` (or ``g0 .. g0+n_targets-1``); the first ``skip``
    bytes of every segment are not scored.  ``skip=0`` with the linear gap is
    the call at sseqs/msa.py:313-319, ``skip=1`` with open/extend the one at
    sseqs/msa.py:327-332.
    """
    if good_idx is not None:
        good_idx = _i32(good_idx)
        n = good_idx.numel()
    else:
        n = int(n_targets)
    if out is None:
        out = torch.empty(n, dtype=torch.int32, device=ascii.device)
    check(lib().sseqs_sw_scan(1 if affine else 0, ptr(query_idx), query_idx.numel(),
                              ptr(good_idx), int(g0), n, ptr(ascii), ptr(delim), int(skip),
                              ptr(out), int(gap_a), int(gap_b), stream_ptr()), "sw_scan")
    return out


def sw_scan_both(query_idx: torch.Tensor, ascii: torch.Tensor, delim: torch.Tensor, *,
                 good_idx: torch.Tensor | None = None, g0: int = 0,
                 n_targets: int | None = None, affine_skip: int = 1, gap: int = -1,
                 gap_open: int = 11, gap_extend: int = 1):
    """Linear (windows of ``sw_scan`` with skip 0) and affine (windows
    ``affine_skip`` bytes later) scores of the same targets in one pass:
    returns ``(linear, affine)``, each equal to its own ``sw_scan`` call."""
    if good_idx is not None:
        good_idx = _i32(good_idx)
        n = good_idx.numel()
    else:
        n = int(n_targets)
    lin = torch.empty(n, dtype=torch.int32, device=ascii.device)
    aff = torch.empty(n, dtype=torch.int32, device=ascii.device)
    check(lib().sseqs_sw_scan_both(ptr(query_idx), query_idx.numel(), ptr(good_idx), int(g0), n,
                                   ptr(ascii), ptr(delim), int(affine_skip), ptr(lin), ptr(aff),
                                   int(gap), int(gap_open), int(gap_extend), stream_ptr()),
          "sw_scan_both")
    return lin, aff


def encode_query(query: str, device="cuda") -> torch.Tensor:
    """Class indices of the standard residues of ``query`` (sseqs/sw.py:11)."""
    return to_device(torch.tensor([AA_MAP[c] for c in query if c in AA_MAP], dtype=torch.uint8),
                     device)


def encode_seq(s: str, device="cuda") -> torch.Tensor:
    """The sequence as int16 character codes behind one leading 0, the
    layout sseqs/sw.py:262-265 feeds its traceback (kept for callers of that
    helper; the traceback here takes the strings themselves)."""
    codes = torch.tensor([0] + [ord(c) for c in s], dtype=torch.int16)
    return codes if str(device) == "cpu" else codes.to(device)


def pack_targets(targets: list[str], device="cuda"):
    """Targets as an int16 [B, W] matrix of character codes, each row a 0
    then its sequence then zeros, with int32 lengths (sequence + 1) and the
    width W = longest + 1 (sseqs/sw.py:267-276)."""
    W = max(len(t) for t in targets) + 1
    T = torch.zeros((len(targets), W), dtype=torch.int16)
    for i, t in enumerate(targets):
        T[i, 1:len(t) + 1] = torch.tensor([ord(c) for c in t], dtype=torch.int16)
    lens = torch.tensor([len(t) + 1 for t in targets], dtype=torch.int32)
    if str(device) != "cpu":
        T, lens = T.to(device), lens.to(device)
    return T, lens, W


def sw(query: str, targets: list[str], gap_open: int = 11, gap_extend: int = 1) -> torch.Tensor:
    """Affine score of ``query`` against each target (sseqs/sw.py:10-23).

    Target 0 scores its own window; the reference reads ``starts[-1]``
    there (out of bounds) and has no defined result.
    """
    q = encode_query(query)
    ascii = torch.from_numpy(np.frombuffer("".join(t + "@" for t in targets).encode("latin-1"),
                                           dtype=np.uint8).copy()).cuda()
    starts = torch.nonzero(ascii == 64, as_tuple=False).flatten()
    good_idx = torch.arange(len(targets), dtype=torch.int32, device="cuda")
    return sw_cuda_affine(q, good_idx, ascii, starts.to(torch.int32), gap_open=gap_open,
                          gap_extend=gap_extend)


# ------------------------------------------------------------------ traceback
class Alignments:
    """Device results of one traceback launch (kept for lazy host decoding)."""

    def __init__(self, best, info, q_al, t_al, cap, m_full):
        self.best, self.info, self.q_al, self.t_al = best, info, q_al, t_al
        self.cap, self.m_full = cap, m_full

    def to_dicts(self) -> list[dict]:
        best, info = to_host(self.best), to_host(self.info)
        q_al, t_al = to_host(self.q_al), to_host(self.t_al)
        out = []
        for b in range(best.shape[0]):
            n = int(info[b, 0])
            if n:
                qs = q_al[b, self.cap - n:].tobytes().decode("latin-1")
                ts = t_al[b, self.cap - n:].tobytes().decode("latin-1")
            else:
                qs = ts = ""
            out.append({
                "q_aligned": qs,
                "t_aligned": ts,
                "q_start_orig_0based": int(info[b, 1]),
                "q_end_orig_0based": int(info[b, 2]),
                "t_start_orig_0based": int(info[b, 3]),
                "t_end_orig_0based": int(info[b, 4]),
                "score": float(best[b]),
            })
        return out


def _bytes(s: str) -> bytes:
    return s.encode("latin-1", errors="replace")


def backtrack(query: str, targets: list[str], gap_open: int = 11, gap_extend: int = 1,
              device="cuda", with_matrix: bool = False) -> Alignments:
    """Launch the CUDA DP + traceback for a batch of targets."""
    B = len(targets)
    qb = _bytes(query)
    tbs = [_bytes(t) for t in targets]
    tlen_h = np.array([len(t) for t in tbs], dtype=np.int32)
    tmax = int(tlen_h.max()) if B else 0
    toff_h = np.zeros(B, dtype=np.int64)
    if B > 1:
        toff_h[1:] = np.cumsum(tlen_h[:-1])
    blob = b"".join(tbs)
    dev = torch.device(device)
    tbytes = to_device(torch.from_numpy(np.frombuffer(blob + b"\0" * 16, dtype=np.uint8).copy()), dev)
    toff = to_device(torch.from_numpy(toff_h), dev)
    tlen = to_device(torch.from_numpy(tlen_h), dev)
    q = to_device(torch.from_numpy(np.frombuffer(qb + b"\0", dtype=np.uint8).copy()), dev)
    cap = len(qb) + tmax + 1
    best = torch.zeros(B, dtype=torch.int32, device=dev)
    info = torch.empty((B, 5), dtype=torch.int32, device=dev)
    q_al = torch.zeros((B, cap), dtype=torch.uint8, device=dev)
    t_al = torch.zeros((B, cap), dtype=torch.uint8, device=dev)
    m_full = None
    tcols = tmax + 1
    if with_matrix:
        m_full = torch.zeros((B, len(qb) + 1, tcols), dtype=torch.int32, device=dev)
    L = lib()
    nbytes = L.sseqs_backtrack_workspace_bytes(len(qb), tmax, B)
    ws = workspace(nbytes, dev)
    check(L.sseqs_backtrack_affine(ptr(q), len(qb), ptr(tbytes), ptr(toff), ptr(tlen), tmax, B,
                                   int(gap_open), int(gap_extend), ptr(best), ptr(info), ptr(q_al),
                                   ptr(t_al), cap, ptr(m_full), tcols, ptr(ws), ws.numel(),
                                   stream_ptr()), "sw_affine_backtrack")
    return Alignments(best, info, q_al, t_al, cap, m_full)


def sw_affine_backtrack(query: str, targets: list[str], gap_open: int = 11, gap_extend: int = 1,
                        device="cuda", scores: bool = False):
    """Affine local alignments with traceback (sseqs/sw.py:27-219).

    Returns ``(M_full int32[B, Q+1, T+1], best int32[B], list[dict])`` like the
    reference, or only ``best`` when ``scores=True``.
    """
    res = backtrack(query, targets, gap_open, gap_extend, device=device, with_matrix=not scores)
    if scores:
        return res.best
    return res.m_full, res.best, res.to_dicts()

"""Learned prefilter: a 1D-conv sequence embedder and an FP8 candidate search.

The reference narrows the database with a gapless FFT correlation before
exact SW (sseqs/msa.py:281-307).  This module offers a learned alternative
for the same stage (it has no reference counterpart):

* ``Embedder`` -- residue embedding (21 classes -> 32), four width-5
  convolutions to 256 channels with GELU, mean over the sequence, L2
  normalisation: 1.03M parameters.  Forward and backward run on the tensor
  cores through ``sseqs_gemm_bf16`` (BF16 operands, fp32 accumulation) with
  fused bias/GELU/mask epilogues; the optimiser is Adam on fp32 master
  weights (``sseqs_adam_conv`` / ``sseqs_adam_flat``).
* ``training_pairs`` / ``train`` -- the embedder learns the exact affine SW
  score of (query, target) pairs divided by the query's self-score, on
  seeded planted-homolog data whose scores come from this package's own SW
  kernels (``batched.sw_scan_queries``); the loss is the squared error of
  the embeddings' cosine.
* ``LearnedIndex`` -- the embeddings of every database segment as FP8 e4m3
  codes resident in HBM (256 bytes per segment, or 128 after a projection
  onto the embeddings' leading principal directions); a query's candidates
  are the rows whose code dot product reaches a per-query threshold
  (estimated from a sample so that
  about ``factor`` times the wanted count pass), selected inside the FP8
  GEMM's epilogue (``sseqs_score_select``), cut to the wanted count, and
  re-scored by exact affine SW.  Every reported score is an exact integer SW
  score; recall against the exhaustive search is measured by the caller.
"""
from __future__ import annotations

import ctypes
import importlib
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import select, tune
from ._lib import check, lib, ptr, stream_ptr, to_host

D = 256            # channels and embedding width
E = 32             # residue embedding width
NCLS = 21
MAX_LEN = 2048     # residues of a sequence the embedder reads
CODE_SCALE = 16.0  # FP8 codes hold 16 x the unit-norm embedding

(_EPI_F32, _EPI_BF16, _EPI_BIAS_GELU, _EPI_GELU_GRAD, _EPI_F32_ADD, _EPI_BIAS_GELU_RES,
 _EPI_GELU_GRAD_RES) = range(7)


def _gemm(a_t, b_t, epi, M, N, K, A, lda, B, ldb, C, ldc, C2=None, bias=None, aux=None,
          mask=None, res=None):
    check(lib().sseqs_gemm_bf16(a_t, b_t, epi, M, N, K, A, lda, B, ldb, C, ldc, C2,
                                ptr(bias), aux, ptr(mask), res, stream_ptr()), "gemm_bf16")


@dataclass
class Layout:
    """Padded row layout of a set of sequences (see sseqs_embed_layout)."""
    P: int
    cls: torch.Tensor        # uint8 [P]
    mask: torch.Tensor       # uint8 [P], 1 on residue rows
    start: torch.Tensor      # int64 [S], first row of each sequence
    length: torch.Tensor     # int32 [S]

    @property
    def n(self) -> int:
        return self.start.numel()


def layout_rows(lengths: torch.Tensor, max_len: int = MAX_LEN) -> torch.Tensor:
    """Rows a layout of these sequences needs before rounding (device int64
    scalar): 2 leading zero rows and each sequence's rows plus 2."""
    return 2 + (lengths.to(torch.int64).clamp(0, max_len) + 2).sum()


def make_layout(ascii: torch.Tensor, offsets: torch.Tensor, lengths: torch.Tensor,
                max_len: int = MAX_LEN, rows: int | None = None) -> Layout:
    """Layout of the sequences ascii[offsets[s] : + lengths[s]] (device).
    ``rows`` is ``layout_rows(lengths)`` when the caller knows it already
    (which saves a device-to-host copy)."""
    dev = ascii.device
    L = lengths.to(torch.int64).clamp(0, max_len)
    sizes = L + 2
    row0 = torch.cumsum(sizes, 0) - sizes + 2
    P = int(layout_rows(lengths, max_len).item()) if rows is None else int(rows)
    P = (P + 31) // 32 * 32
    cls = torch.full((P,), 255, dtype=torch.uint8, device=dev)
    n = L.numel()
    L32 = L.to(torch.int32)
    off = offsets.to(torch.int64).contiguous()
    check(lib().sseqs_embed_layout(ptr(ascii), ptr(off), ptr(L32), ptr(row0), n, ptr(cls),
                                   stream_ptr()), "embed_layout")
    mask = (cls != 255).to(torch.uint8)
    return Layout(P, cls, mask, row0, L32)


class _Buffers:
    """Activation buffers with 2 zero rows of slack on both sides."""

    def __init__(self, rows: int, train: bool, dev):
        self.rows = rows
        z = lambda c: torch.zeros((rows + 4, c), dtype=torch.bfloat16, device=dev)
        # inference keeps two layer outputs (alternating), no embedded rows
        # and no pre-activations
        self.X0 = z(E) if train else None
        self.Y = [z(D) for _ in range(4 if train else 2)]
        self.Z = [z(D) for _ in range(4)] if train else None
        self.dZ = [z(D) for _ in range(4)] if train else None
        self.G = [z(D) for _ in range(4)] if train else None
        self.dX0 = z(E) if train else None


def _base(buf: torch.Tensor) -> int:
    """Address of layout row 0 (buffer row 2)."""
    return buf.data_ptr() + 2 * buf.shape[1] * buf.element_size()


class Embedder:
    """The 1D-conv embedder with its Adam state (all parameters on device).

    With ``residual`` (the default) layers 2-4 add their input to their
    output (Y_l = GELU(Z_l) + Y_{l-1}), so the pooled embedding keeps the
    first layer's short-window features, which substitutions disturb far
    less than the deeper layers' ~17-residue ones."""

    def __init__(self, seed: int = 0, device="cuda", residual: bool = True):
        dev = torch.device(device)
        self.device = dev
        self.residual = residual
        g = torch.Generator(device="cpu")
        g.manual_seed(seed)
        self.cin = [E, D, D, D]
        self.emb = (torch.randn(NCLS, E, generator=g) * 0.5).to(dev)
        self.W = [(torch.randn(D, 5, c, generator=g) * math.sqrt(2.0 / (5 * c))).to(dev)
                  for c in self.cin]
        self.b = [torch.zeros(D, device=dev) for _ in self.cin]
        self._opt = None
        self.step = 0
        self._bufs = None
        self._sync_bf16()

    @property
    def n_params(self) -> int:
        return self.emb.numel() + sum(w.numel() + b.numel() for w, b in zip(self.W, self.b))

    def _sync_bf16(self):
        self.emb_b = self.emb.to(torch.bfloat16).contiguous()
        self.Wb = [w.reshape(D, -1).to(torch.bfloat16).contiguous() for w in self.W]
        # the first convolution as a table: T[t][k] = E[k] . W1[:, t, :]^T from
        # the same bf16 values the GEMM form would multiply
        self.T1 = torch.einsum("kc,otc->tko", self.emb_b.float(),
                               self.Wb[0].float().reshape(D, 5, E)).contiguous()
        self.Wf = [w.flip(1).permute(2, 1, 0).reshape(c, -1).to(torch.bfloat16).contiguous()
                   for w, c in zip(self.W, self.cin)]

    def state_dict(self) -> dict:
        return {"emb": self.emb.cpu(), "W": [w.cpu() for w in self.W],
                "b": [b.cpu() for b in self.b]}

    def load_state_dict(self, st: dict):
        self.emb = st["emb"].to(self.device)
        self.W = [w.to(self.device) for w in st["W"]]
        self.b = [b.to(self.device) for b in st["b"]]
        self._sync_bf16()

    def _buffers(self, rows: int, train: bool) -> _Buffers:
        b = self._bufs
        if b is None or b.rows < rows or (train and b.dZ is None):
            self._bufs = None
            torch.cuda.empty_cache()
            b = self._bufs = _Buffers(max(rows, 1024), train, self.device)
        return b

    # ---------------------------------------------------------------- forward
    def forward(self, lay: Layout, train: bool = False):
        """Unit-norm embeddings [S, 256] (fp32) of the layout's sequences."""
        bufs = self._buffers(lay.P, train)
        P = lay.P
        L = lib()
        if train:    # the backward pass reads the embedded rows
            check(L.sseqs_embed_lookup(ptr(lay.cls), P, ptr(self.emb_b), E, _base(bufs.X0),
                                       stream_ptr()), "embed_lookup")
        # layer 1 from its table (a K = 160 GEMM otherwise); the pre-activations
        # Z are kept for the backward pass only
        check(L.sseqs_embed_conv1_table(ptr(lay.cls), P, ptr(self.T1), ptr(self.b[0]),
                                        ptr(lay.mask), D, _base(bufs.Y[0]),
                                        _base(bufs.Z[0]) if train else None, stream_ptr()),
              "conv1_table")
        prev = bufs.Y[0]
        for l in range(1, 4):
            Y = bufs.Y[l % len(bufs.Y)]
            # im2col(prev) row p starts at layout row p-2 = buffer row p
            res = self.residual
            _gemm(0, 0, _EPI_BIAS_GELU_RES if res else _EPI_BIAS_GELU, P, D, 5 * D,
                  prev.data_ptr(), D, self.Wb[l].data_ptr(), 5 * D, _base(Y), D,
                  _base(bufs.Z[l]) if train else None, self.b[l], None, lay.mask,
                  _base(prev) if res else None)
            prev = Y
        S = lay.n
        pooled = torch.empty((S, D), dtype=torch.float32, device=self.device)
        emb = torch.empty((S, D), dtype=torch.float32, device=self.device)
        inv = torch.empty(S, dtype=torch.float32, device=self.device)
        check(L.sseqs_pool_normalize(_base(prev), D, ptr(lay.start), ptr(lay.length), S,
                                     ptr(pooled), ptr(emb), ptr(inv), stream_ptr()),
              "pool_normalize")
        if train:
            self._cache = (lay, emb, inv)
        return emb

    # --------------------------------------------------------------- backward
    def backward(self, dE: torch.Tensor):
        """Gradients of every parameter from dLoss/d(embeddings) (after a
        ``forward(..., train=True)``); returns them as a dict."""
        lay, emb, inv = self._cache
        bufs, P, L = self._bufs, lay.P, lib()
        bufs.dZ[3][2:2 + P].zero_()
        bufs.G[3][2:2 + P].zero_()
        check(L.sseqs_pool_backward(ptr(emb), ptr(dE), ptr(inv), ptr(lay.start),
                                    ptr(lay.length), lay.n, D, _base(bufs.Z[3]),
                                    _base(bufs.dZ[3]), _base(bufs.G[3]), stream_ptr()),
              "pool_backward")
        grads = {"W": [None] * 4, "b": [None] * 4}
        for l in range(3, -1, -1):
            cin = self.cin[l]
            prev = bufs.Y[l - 1] if l > 0 else bufs.X0
            dZ = bufs.dZ[l]
            dWT = torch.zeros((5 * cin, D), dtype=torch.float32, device=self.device)
            # dW^T = im2col(prev)^T . dZ over the P rows (split over positions)
            _gemm(1, 1, _EPI_F32_ADD, 5 * cin, D, P, prev.data_ptr(), cin, _base(dZ), D,
                  dWT.data_ptr(), D)
            db = torch.zeros(D, dtype=torch.float32, device=self.device)
            check(L.sseqs_bias_grad(_base(dZ), P, D, ptr(db), stream_ptr()), "bias_grad")
            grads["W"][l], grads["b"][l] = dWT, db
            # data gradient through the transposed (flipped) kernel
            if l > 0 and self.residual:
                # G_{l-1} = conv_back(dZ_l) + G_l, dZ_{l-1} = G_{l-1} * GELU'(Z_{l-1})
                _gemm(0, 0, _EPI_GELU_GRAD_RES, P, cin, 5 * D, dZ.data_ptr(), D,
                      self.Wf[l].data_ptr(), 5 * D, _base(bufs.dZ[l - 1]), cin,
                      _base(bufs.G[l - 1]), None, _base(bufs.Z[l - 1]), lay.mask,
                      _base(bufs.G[l]))
            elif l > 0:
                _gemm(0, 0, _EPI_GELU_GRAD, P, cin, 5 * D, dZ.data_ptr(), D,
                      self.Wf[l].data_ptr(), 5 * D, _base(bufs.dZ[l - 1]), cin, None, None,
                      _base(bufs.Z[l - 1]), lay.mask)
            else:
                _gemm(0, 0, _EPI_BF16, P, cin, 5 * D, dZ.data_ptr(), D, self.Wf[0].data_ptr(),
                      5 * D, _base(bufs.dX0), cin, None, None, None, lay.mask)
        dEmb = torch.zeros((NCLS, E), dtype=torch.float32, device=self.device)
        check(L.sseqs_embed_grad(ptr(lay.cls), P, _base(bufs.dX0), E, ptr(dEmb), stream_ptr()),
              "embed_grad")
        grads["emb"] = dEmb
        return grads

    def apply(self, grads: dict, lr: float, b1=0.9, b2=0.999, eps=1e-8):
        """One Adam step with the gradients of ``backward``."""
        if self._opt is None:
            z = lambda t: torch.zeros_like(t)
            self._opt = {"emb": (z(self.emb), z(self.emb)),
                         "W": [(z(w), z(w)) for w in self.W],
                         "b": [(z(b), z(b)) for b in self.b]}
        self.step += 1
        L, st = lib(), stream_ptr()
        for l in range(4):
            m, v = self._opt["W"][l]
            check(L.sseqs_adam_conv(ptr(self.W[l]), ptr(m), ptr(v), ptr(grads["W"][l]), D,
                                    self.cin[l], lr, b1, b2, eps, self.step, ptr(self.Wb[l]),
                                    ptr(self.Wf[l]), st), "adam_conv")
            m, v = self._opt["b"][l]
            check(L.sseqs_adam_flat(ptr(self.b[l]), ptr(m), ptr(v), ptr(grads["b"][l]), D, lr,
                                    b1, b2, eps, self.step, None, st), "adam_flat")
        m, v = self._opt["emb"]
        check(L.sseqs_adam_flat(ptr(self.emb), ptr(m), ptr(v), ptr(grads["emb"]),
                                self.emb.numel(), lr, b1, b2, eps, self.step, ptr(self.emb_b),
                                st), "adam_flat")

    def embed(self, ascii, offsets, lengths, chunk: int = 32768) -> torch.Tensor:
        """Embeddings [n, 256] of many sequences, ``chunk`` at a time (the
        row counts of all chunks come to the host in one copy, so the chunks
        are queued without waiting for one another)."""
        n = lengths.numel()
        out = torch.empty((n, D), dtype=torch.float32, device=self.device)
        starts = list(range(0, n, chunk))
        if not starts:
            return out
        L = lengths.to(torch.int64).clamp(0, MAX_LEN) + 2
        bounds = torch.tensor(starts[1:] + [n], dtype=torch.int64, device=L.device)
        cum = torch.cumsum(L, 0)
        ends = cum[bounds - 1]
        rows = to_host(2 + ends - torch.cat([torch.zeros(1, dtype=torch.int64, device=L.device),
                                             ends[:-1]]))
        for s, r in zip(starts, rows.tolist()):
            lay = make_layout(ascii, offsets[s:s + chunk], lengths[s:s + chunk], rows=r)
            out[s:s + lay.n] = self.forward(lay)
        return out


# ------------------------------------------------------------- training data
@dataclass
class PairSet:
    """Sequences (queries and targets) in one byte buffer, and the pairs."""
    ascii: torch.Tensor      # device bytes, sequences separated by '@'
    offsets: torch.Tensor    # int64 [n_seqs]
    lengths: torch.Tensor    # int32 [n_seqs]
    qa: torch.Tensor         # int32 [B] query sequence of each pair
    tb: torch.Tensor         # int32 [B] target sequence of each pair
    y: torch.Tensor          # float32 [B]: SW(q, t) / SW(q, q)
    n_queries: int
    per_query: int
    delim: torch.Tensor      # int32 '@' positions (segment g = sequence g)
    query_enc: list          # residue classes of every query (device)
    self_score: torch.Tensor  # float32 [n_queries]
    qbuf: torch.Tensor = None    # uint8 [n_queries, 2048]: query classes, one row each
    qlen: torch.Tensor = None    # int32 [n_queries]


def training_pairs(n_queries: int, per_query: int, seed: int = 0, ident=(0.15, 1.0),
                   homolog_frac: float = 0.5, device="cuda", gap_open=11,
                   gap_extend=1) -> PairSet:
    """Seeded pairs: queries with lengths U(50, 1000); per query a fraction
    ``homolog_frac`` of mutated copies (identity U(ident), indels) and
    unrelated sequences (log-normal lengths, median 250) for the rest.  The
    target of a pair is the exact affine SW score of (query, target) divided
    by the query's self-score, computed with the score kernels."""
    from . import batched, dbtools
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rng = np.random.default_rng(seed)
    qlens = rng.integers(50, 1001, n_queries)
    nh = int(round(per_query * homolog_frac))
    parts, lens = [], []
    for qi in range(n_queries):
        q = dbtools.random_residues(int(qlens[qi]), gen, dev)
        parts.append(q)
        lens.append(torch.tensor([q.numel()], device=dev))
        qs = q.cpu().numpy().tobytes().decode()
        res, ln = dbtools.plant_homologs(qs, nh, ident[0], ident[1], gen, dev)
        parts.append(res)
        lens.append(ln)
        bl = dbtools.lognormal_lengths(per_query - nh, gen, dev)
        parts.append(dbtools.random_residues(int(bl.sum().item()), gen, dev))
        lens.append(bl)
    lengths = torch.cat(lens).to(torch.int64)
    residues = torch.cat(parts)
    n = lengths.numel()
    # interleave '@' after every sequence
    offsets = torch.cumsum(lengths + 1, 0) - (lengths + 1)
    ascii = torch.full((int((lengths + 1).sum().item()),), 64, dtype=torch.uint8, device=dev)
    seq_of = torch.repeat_interleave(torch.arange(n, device=dev), lengths)
    pos = torch.arange(residues.numel(), device=dev) - \
        (torch.cumsum(lengths, 0) - lengths)[seq_of]
    ascii[offsets[seq_of] + pos] = residues
    delim = (offsets + lengths).to(torch.int32)
    stride = 1 + per_query
    qa = torch.arange(n_queries, device=dev).repeat_interleave(per_query) * stride
    tb = qa + torch.arange(per_query, device=dev).repeat(n_queries) + 1
    # exact scores: target g of segment index g (window between delim[g-1]
    # and delim[g]); each query against [itself, its targets]
    sw = importlib.import_module("sseqs_b200.sw")
    scores = torch.empty((n_queries, stride), dtype=torch.int32, device=dev)
    encs = [sw.encode_query(bytes(ascii[int(offsets[i * stride]):int(offsets[i * stride]) +
                                        int(lengths[i * stride])].cpu().numpy()).decode(), dev)
            for i in range(n_queries)]
    for tpt, members in batched.buckets([e.numel() for e in encs]).items():
        for s in range(0, len(members), batched.GROUP):
            grp = members[s:s + batched.GROUP]
            qbuf = torch.zeros((len(grp), batched.MAX_QUERY), dtype=torch.uint8, device=dev)
            for j, qi in enumerate(grp):
                qbuf[j, :encs[qi].numel()] = encs[qi]
            ql = torch.tensor([encs[qi].numel() for qi in grp], dtype=torch.int32, device=dev)
            idx = torch.stack([torch.arange(qi * stride, (qi + 1) * stride, device=dev)
                               for qi in grp]).to(torch.int32)
            out = batched.sw_scan_queries(qbuf, ql, tpt, ascii, delim, affine=True,
                                          good_idx=idx, skip=0, gap_a=gap_open,
                                          gap_b=gap_extend)
            scores[torch.tensor(grp, device=dev)] = out[:, :stride]
    self_s = scores[:, 0:1].clamp(min=1).to(torch.float32)
    y = (scores[:, 1:].to(torch.float32) / self_s).clamp_(0, 1).flatten()
    qbuf = torch.zeros((n_queries, batched.MAX_QUERY), dtype=torch.uint8, device=dev)
    for i, e in enumerate(encs):
        qbuf[i, :e.numel()] = e
    qlen = torch.tensor([e.numel() for e in encs], dtype=torch.int32, device=dev)
    return PairSet(ascii, offsets, lengths.to(torch.int32), qa.to(torch.int32),
                   tb.to(torch.int32), y, n_queries, per_query, delim, encs,
                   self_s.flatten(), qbuf, qlen)


def _cross_scores(pairs: PairSet, qids, tseq, gap_open=11, gap_extend=1) -> torch.Tensor:
    """Exact affine SW of every query in ``qids`` (all of one stripe width)
    against every sequence in ``tseq`` (segment indices of the pair
    buffer), divided by the query's self-score: float32 [len(qids),
    len(tseq)].  One batched launch."""
    from . import batched
    dev = pairs.ascii.device
    tg = torch.as_tensor(tseq, dtype=torch.int32, device=dev)
    q = torch.as_tensor(qids, dtype=torch.int64, device=dev)
    tpt = tune.tpt_of(int(pairs.query_enc[qids[0]].numel()))
    sc = batched.sw_scan_queries(pairs.qbuf[q], pairs.qlen[q], tpt, pairs.ascii, pairs.delim,
                                 affine=True, good_idx=tg, skip=0, gap_a=gap_open,
                                 gap_b=gap_extend)
    return (sc[:, :tg.numel()].to(torch.float32) / pairs.self_score[q][:, None]).clamp_(0, 1)


def train(model: Embedder, pairs: PairSet, *, queries_per_step: int = 32,
          targets_per_query: int = 32, epochs: int = 1, lr: float = 2e-3,
          lr_end: float = 1e-4, floor: float = 0.5, target_power: float = 0.5, seed: int = 0,
          log=None) -> dict:
    """Adam on the squared error between embedding cosines and normalised
    SW scores.  A step takes ``queries_per_step`` queries with
    ``targets_per_query`` of each one's targets, and labels EVERY (query,
    target) pair of the step -- the targets of the other queries serve as
    negatives -- with the exact affine SW score of the pair divided by the
    query's self-score, computed for the step by the score kernels.

    The cosine is fitted to ``floor + (1 - floor) * y``: only the order of
    cosines matters for the search, and asking unrelated pairs for a cosine
    near 0 drives the pooled features towards cancelling out, after which
    the normalised embedding of a sequence is mostly noise and some close
    homologs come out nearly orthogonal.  The normalised score y enters as
    y**p (``target_power``, 0.5 by default), which spreads the low scores of
    remote homologs away from those of unrelated pairs (y of 0.05-0.15 at
    20-30% identity against ~0.01 for unrelated pairs) and compresses the
    high end, whose order matters less: close homologs are found anyway.
    Measured on 20M sequences with 500 planted homologs per query (10M
    training pairs, 32768 candidates): recall of the planted homologs in the
    exact top-1000 0.72 with p = 1, 0.79 with p = 0.5 (20-30% identity: 0.09
    -> 0.21)."""
    dev = model.device
    rng = np.random.default_rng(seed)
    nq, pq = pairs.n_queries, pairs.per_query
    tq = min(targets_per_query, pq)
    # a step's queries share one stripe width, so that one launch scores
    # all its (query, target) pairs
    qtpt = [tune.tpt_of(int(e.numel())) for e in pairs.query_enc]
    by_tpt: dict = {}
    for q in range(nq):
        for t0 in range(0, pq - tq + 1, tq):
            by_tpt.setdefault(qtpt[q], []).append((q, t0))

    def plan():
        steps = []
        for sl in by_tpt.values():
            perm = rng.permutation(len(sl))
            for s0 in range(0, len(sl), queries_per_step):
                steps.append([sl[i] for i in perm[s0:s0 + queries_per_step]])
        return [steps[i] for i in rng.permutation(len(steps))]

    total = epochs * len(plan())
    losses, step, labelled = [], 0, 0
    loss_acc = torch.zeros(1, dtype=torch.float32, device=dev)
    stride = 1 + pq
    for ep in range(epochs):
        for pick in plan():
            qids = [q for q, _ in pick]
            tseq = [q * stride + 1 + t0 + k for q, t0 in pick for k in range(tq)]
            seq = [q * stride for q in qids] + tseq
            sidx = torch.tensor(seq, dtype=torch.int64, device=dev)
            lay = make_layout(pairs.ascii, pairs.offsets[sidx], pairs.lengths[sidx])
            emb = model.forward(lay, train=True)
            y = _cross_scores(pairs, qids, tseq)
            if target_power != 1.0:
                y = y.pow_(target_power)
            y = (floor + (1.0 - floor) * y).flatten().contiguous()
            nqs, nt = len(qids), len(tseq)
            ia_t = torch.arange(nqs, dtype=torch.int32, device=dev).repeat_interleave(nt)
            ib_t = (nqs + torch.arange(nt, dtype=torch.int32, device=dev)).repeat(nqs)
            # half the weight on each query's own targets (homologs and
            # unrelated), half on the other queries' targets (negatives)
            owner = torch.arange(nt, device=dev) // tq
            own = (owner[None, :] == torch.arange(nqs, device=dev)[:, None]).flatten()
            w = torch.where(own, 0.5 / (nqs * tq), 0.5 / (nqs * max(nt - tq, 1))).to(
                torch.float32).contiguous()
            dE = torch.zeros_like(emb)
            loss_acc.zero_()
            check(lib().sseqs_pair_loss(ptr(emb), D, ptr(ia_t), ptr(ib_t), ptr(y), ptr(w),
                                        ia_t.numel(), ptr(dE), ptr(loss_acc), None, stream_ptr()),
                  "pair_loss")
            grads = model.backward(dE)
            frac = step / max(total - 1, 1)
            cur = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * frac))
            model.apply(grads, cur)
            labelled += ia_t.numel()
            if step % 50 == 0 or step == total - 1:
                losses.append((step, float(loss_acc.item())))
                if log:
                    log(f"step {step}/{total} loss {losses[-1][1]:.5f} lr {cur:.2e}")
            step += 1
    return {"steps": step, "losses": losses, "labelled_pairs": labelled}


# ----------------------------------------------------------------- search
def principal_directions(emb: torch.Tensor, k: int, max_rows: int = 1 << 20) -> torch.Tensor:
    """The k leading eigenvectors [256, k] (fp32, on emb's device) of the
    second-moment matrix of unit embeddings (rows of ``emb``, evenly
    subsampled to at most ``max_rows``): the k-dimensional subspace that
    keeps the most of their dot products."""
    step = max(1, emb.shape[0] // max_rows)
    x = emb[::step].to(torch.float64)
    c = (x.T @ x).cpu().numpy() / max(1, x.shape[0])
    w, v = np.linalg.eigh(c)                       # ascending eigenvalues
    top = v[:, np.argsort(w)[::-1][:k]]
    return torch.from_numpy(np.ascontiguousarray(top)).to(torch.float32).to(emb.device)


def project(emb: torch.Tensor, proj: torch.Tensor) -> torch.Tensor:
    """Rows of ``emb`` projected by ``proj`` and scaled back to unit norm."""
    y = emb @ proj
    return (y / y.norm(dim=1, keepdim=True).clamp_min(1e-12)).contiguous()


class LearnedIndex:
    """FP8 codes of every database segment, resident in HBM.

    ``dim`` is the code width: 256 (the embedding itself) or 128 (its
    projection onto the 128 leading principal directions of the database's
    embeddings, renormalised), which halves the index (200M segments: 25.6
    instead of 51.2 GB).  The selection kernel reads 256-byte rows; a
    128-wide index is read as rows of two consecutive codes, against two
    query columns per query, [q, 0] and [0, q], whose scores are those of the
    even and the odd code of every pair."""

    def __init__(self, model: Embedder, db, chunk: int = 32768, dim: int = D):
        if dim not in (D, D // 2):
            raise ValueError(f"code width {dim}: 256 or 128")
        self.model, self.db, self.dim = model, db, dim
        counts = [b.n_segments for b in db.batches]
        self.cum = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        n = int(self.cum[-1])
        # a 128-wide index holds an even number of rows (the spare one all
        # zero), so that it can be read as 256-byte rows
        rows = max(n, 1) if dim == D else max(n + (n & 1), 2)
        self.codes = torch.zeros((rows, dim), dtype=torch.uint8, device=db.device)
        self.proj = None
        L = lib()
        for bi, b in enumerate(db.batches):
            if b.n_segments == 0:
                continue
            # a whole batch per call: its chunks are queued back to back
            emb = model.embed(b.ascii, b.offsets[:b.n_segments], b.lengths[:b.n_segments],
                              chunk=chunk)
            if dim < D:
                if self.proj is None:
                    self.proj = principal_directions(emb, dim)
                emb = project(emb, self.proj)
            row = int(self.cum[bi])
            check(L.sseqs_quantize_e4m3(ptr(emb), emb.numel(), CODE_SCALE,
                                        self.codes[row:row + b.n_segments].data_ptr(),
                                        stream_ptr()), "quantize")
            del emb
        if dim < D and self.proj is None:     # no segments: any projection will do
            self.proj = torch.eye(D, dim, dtype=torch.float32, device=db.device)
        self.n = n

    def query_codes(self, enc_queries) -> torch.Tensor:
        """FP8 codes [nq, dim] of queries given as ASCII strings."""
        dev = self.db.device
        buf = "".join(q + "@" for q in enc_queries).encode()
        ascii = torch.from_numpy(np.frombuffer(buf, np.uint8).copy()).to(dev)
        lens = torch.tensor([len(q) for q in enc_queries], dtype=torch.int64, device=dev)
        offs = torch.cumsum(lens + 1, 0) - (lens + 1)
        emb = self.model.embed(ascii, offs, lens)
        if self.dim < D:
            emb = project(emb, self.proj)
        codes = torch.empty((len(enc_queries), self.dim), dtype=torch.uint8, device=dev)
        check(lib().sseqs_quantize_e4m3(ptr(emb), emb.numel(), CODE_SCALE, ptr(codes),
                                        stream_ptr()), "quantize")
        return codes

    def _wide(self, qcodes: torch.Tensor) -> torch.Tensor:
        """256-byte query rows: the codes themselves, or for a 128-wide index
        [q, 0] and [0, q] per query (rows 2i and 2i + 1)."""
        if self.dim == D:
            return qcodes.contiguous()
        nq = qcodes.shape[0]
        w = torch.zeros((2 * nq, D), dtype=torch.uint8, device=qcodes.device)
        w[0::2, :self.dim] = qcodes
        w[1::2, self.dim:] = qcodes
        return w

    def _select(self, qcodes: torch.Tensor, n_cand: int, sample: int, factor: float,
                cap_factor: int):
        """Threshold per query from a sample of the codes, then every row at
        or above it by the FP8 selection GEMM: (cand [nq, cap], scores,
        host counts, cap)."""
        dev = self.db.device
        nq = qcodes.shape[0]
        L = lib()
        # threshold: the k-th largest score over an evenly spaced sample
        S = min(sample, self.n)
        # evenly spaced rows in integer arithmetic (float32 cannot hold
        # every row index of a 20M-row index)
        rows = torch.arange(S, dtype=torch.int64, device=dev) * (self.n - 1) // max(S - 1, 1)
        samp = self.codes[rows]
        qwide = self._wide(qcodes)
        if self.dim < D:
            # zero-padded to 256 bytes: [q, 0] . [s, 0] = q . s
            samp = torch.cat([samp, torch.zeros_like(samp)], dim=1)
            qs = qwide[0::2].contiguous()
        else:
            qs = qwide
        samp = samp.contiguous()
        dense = torch.empty((nq, S), dtype=torch.float32, device=dev)
        check(L.sseqs_score_dense(ptr(qs), nq, ptr(samp), S, ptr(dense), stream_ptr()),
              "score_dense")
        k_s = max(1, min(S, int(math.ceil(factor * n_cand * S / max(self.n, 1)))))
        tau = torch.empty(nq, dtype=torch.float32, device=dev)
        check(L.sseqs_kth_largest_rows(ptr(dense), nq, S, k_s, ptr(tau), stream_ptr()),
              "kth_largest")
        # the selection over 256-byte rows: query columns and index rows as
        # the kernel reads them
        half = self.dim < D
        ncol = qwide.shape[0]
        tau_c = tau.repeat_interleave(2) if half else tau
        n_rows = self.codes.shape[0] // 2 if half else self.n
        cap = int(min(self.n, max(n_cand * cap_factor, 1024)))
        while True:
            count = torch.zeros(ncol, dtype=torch.int32, device=dev)
            cand = torch.empty((ncol, cap), dtype=torch.int64, device=dev)
            cs = torch.empty((ncol, cap), dtype=torch.float32, device=dev)
            check(L.sseqs_score_select(ptr(qwide), ncol, ptr(self.codes), n_rows, ptr(tau_c),
                                       ptr(count), ptr(cand), ptr(cs), cap, stream_ptr()),
                  "score_select")
            cnt = to_host(count)
            flag = ctypes.c_int(0)
            check(L.sseqs_gemm_error(ctypes.byref(flag)), "gemm_error")
            if flag.value:
                raise RuntimeError("score_select: a bounded wait of the selection kernel ran out")
            if int(cnt.max(initial=0)) <= cap or cap >= self.n:
                break
            cap = int(min(self.n, 2 * int(cnt.max())))
        if not half:
            return cand, cs, cnt, cap
        return self._merge_columns(cand, cs, cnt, cap)

    def _merge_columns(self, cand, cs, cnt, cap):
        """The two query columns of a 128-wide index back to one list per
        query: row r of column 2i is code 2r, of column 2i + 1 code 2r + 1;
        the spare zero row is dropped.  Returns (cand [nq, 2 cap], scores,
        host counts, 2 cap), each query's entries first in its row."""
        dev = cand.device
        ncol = cand.shape[0]
        nq = ncol // 2
        took = torch.from_numpy(np.minimum(cnt, cap).astype(np.int64)).to(dev)
        live = torch.arange(cap, device=dev)[None, :] < took[:, None]
        col = torch.arange(ncol, device=dev)
        code = 2 * cand + (col & 1)[:, None]
        keep = live & (code < self.n)
        qid = (col // 2)[:, None].expand(ncol, cap)[keep]         # query-major
        code, score = code[keep], cs[keep]
        cntq = torch.bincount(qid, minlength=nq)
        pos = torch.arange(qid.numel(), device=dev) - (torch.cumsum(cntq, 0) - cntq)[qid]
        out = torch.zeros((nq, 2 * cap), dtype=torch.int64, device=dev)
        out_s = torch.zeros((nq, 2 * cap), dtype=torch.float32, device=dev)
        out[qid, pos] = code
        out_s[qid, pos] = score
        return out, out_s, to_host(cntq).astype(np.int64), 2 * cap

    def candidates_flat(self, qcodes: torch.Tensor, n_cand: int, sample: int = 8192,
                        factor: float = 2.5, cap_factor: int = 8):
        """Per query the database rows of its ``n_cand`` highest code scores
        (fewer when fewer pass the threshold; ties at the cut go to the lower
        rows), as device arrays sorted by (query, row): ``(qid, rows)``
        (int64), and the host count per query."""
        dev = self.db.device
        nq = qcodes.shape[0]
        cand, cs, cnt, cap = self._select(qcodes, n_cand, sample, factor, cap_factor)
        took = np.minimum(cnt, cap).astype(np.int64)
        tk = torch.from_numpy(took).to(dev)
        live = torch.arange(cap, device=dev)[None, :] < tk[:, None]
        rows = cand[live]                                   # query-major
        keys = cs[live].to(torch.float16)
        qid = torch.repeat_interleave(torch.arange(nq, device=dev), tk)
        # the lists are appended in no fixed order: order by (query, row),
        # then stably by key (desc) and query, so that inside a query the
        # keys fall and equal keys keep the lower rows first
        o = torch.argsort(qid * max(self.n, 1) + rows)
        o = o[torch.sort(keys[o], descending=True, stable=True).indices]
        o = o[torch.sort(qid[o], stable=True).indices]
        start = torch.cumsum(tk, 0) - tk
        rank = torch.arange(o.numel(), device=dev) - start[qid[o]]
        o = o[rank < n_cand]
        kq, kr = qid[o], rows[o]
        o = torch.argsort(kq * max(self.n, 1) + kr)
        return kq[o], kr[o], np.minimum(took, n_cand)

    def candidates(self, qcodes: torch.Tensor, n_cand: int, sample: int = 8192,
                   factor: float = 2.5, cap_factor: int = 8):
        """``candidates_flat`` as a list of row tensors (increasing), one per
        query, and the host counts of rows at or above each threshold."""
        kq, kr, counts = self.candidates_flat(qcodes, n_cand, sample, factor, cap_factor)
        return list(torch.split(kr, [int(c) for c in counts])), counts

    def _batch_tables(self):
        if getattr(self, "_tabs", None) is None:
            dev = self.db.device
            bs = self.db.batches
            seg = [b.seg_index[:b.n_segments].to(torch.int32) for b in bs]
            nd = [b.delim.numel() for b in bs]
            self._tabs = {
                "cum": torch.from_numpy(self.cum).to(dev),
                "nseg": torch.tensor([b.n_segments for b in bs] or [0], dtype=torch.int64,
                                     device=dev),
                "maxlen": torch.tensor([b.maxlen for b in bs] or [0], dtype=torch.int64,
                                       device=dev),
                # segment number of every index row (the delimiter-based index
                # the exhaustive search reports)
                "seg": torch.cat(seg) if seg else torch.zeros(1, dtype=torch.int32, device=dev),
                # every batch's '@' positions, one after another, and where
                # each batch's begin; the batches' device addresses
                "delim": torch.cat([b.delim for b in bs]) if bs else
                         torch.zeros(1, dtype=torch.int32, device=dev),
                "doff": torch.tensor(np.concatenate([[0], np.cumsum(nd)[:-1]]) if nd else [0],
                                     dtype=torch.int64, device=dev),
                "bases": torch.tensor([b.ascii.data_ptr() for b in bs] or [0],
                                      dtype=torch.int64, device=dev),
            }
        return self._tabs

    # packed candidate bytes per rescoring call, at most (segment windows are
    # addressed with int32 delimiter positions)
    PACK_LIMIT = 1_500_000_000

    def rescore_flat(self, queries, qid: torch.Tensor, rows: torch.Tensor, top: int = 4096,
                     gap_open=11, gap_extend=1) -> list:
        """Exact affine SW of every query against its candidate rows (the
        affine stage of sseqs/msa.py:327-337: skip 1 residue, first and last
        segment of a batch excluded).  ``qid``/``rows``: device int64, sorted
        by (query, row).  Returns per query the ``top`` hits as host arrays
        ``(norm float32, batch, segment, affine int64)`` sorted by normalised
        score desc, then batch, then segment.

        The distinct candidate segments of all queries, from whatever
        batches they lie in, are first packed into one '@'-separated buffer
        (``sseqs_pack_segments``), so every stripe-width group of queries is
        scored by one SW launch over all its candidates whatever the number
        of database batches; a segment scores the same there as in its batch
        (the same bytes, the same skip).  The target rows, their positions
        and the ranking are built with a fixed number of whole-array
        operations, and the hits come back in one copy per field."""
        from . import batched
        sw = importlib.import_module("sseqs_b200.sw")
        dev = self.db.device
        nq, nb = len(queries), len(self.db.batches)
        empty = (np.zeros(0, np.float32), np.zeros(0, np.int64), np.zeros(0, np.int64),
                 np.zeros(0, np.int64))
        if nq == 0 or rows.numel() == 0 or nb == 0:
            return [empty for _ in range(nq)]
        T = self._batch_tables()
        batch = torch.searchsorted(T["cum"][1:], rows, right=True)
        local = rows - T["cum"][batch]
        ok = (local >= 1) & (local <= T["nseg"][batch] - 2)
        qid, rows, batch = qid[ok], rows[ok], batch[ok]
        n = qid.numel()
        if n == 0:
            return [empty for _ in range(nq)]
        seg = T["seg"][rows]
        # the distinct candidate segments and their windows (segment g of a
        # batch: bytes delim[g-1] + 1 .. delim[g]; every candidate has g >= 1)
        urows, inv = torch.unique(rows, return_inverse=True)
        ub = torch.searchsorted(T["cum"][1:], urows, right=True)
        dpos = T["doff"][ub] + T["seg"][urows].to(torch.int64)
        end = T["delim"][dpos].to(torch.int64)
        start = T["delim"][dpos - 1].to(torch.int64) + 1
        ulen = end - start
        dst = torch.cumsum(ulen + 1, 0) - (ulen + 1)
        per_q = to_host(torch.bincount(qid, minlength=nq)).astype(np.int64)
        total = int((dst[-1] + ulen[-1] + 1).item())
        if total > self.PACK_LIMIT and nq > 1:
            # too many bytes for one packed buffer: score the queries in two halves
            h = nq // 2
            cut = int(per_q[:h].sum())
            lo = self.rescore_flat(queries[:h], qid[:cut], rows[:cut], top, gap_open, gap_extend)
            hi = self.rescore_flat(queries[h:], qid[cut:] - h, rows[cut:], top, gap_open,
                                   gap_extend)
            return lo + hi
        if total > self.PACK_LIMIT:
            raise ValueError("candidate segments of one query exceed the packing limit")
        packed = torch.empty(total, dtype=torch.uint8, device=dev)
        # the int32 copies are held by names until the launch has been queued
        # (a temporary freed earlier could hand its memory to the next one)
        ub32, ulen32 = ub.to(torch.int32), ulen.to(torch.int32)
        check(lib().sseqs_pack_segments(ptr(T["bases"]), ptr(ub32), ptr(start), ptr(ulen32),
                                        ptr(dst), urows.numel(), ptr(packed), stream_ptr()),
              "pack_segments")
        pdelim = (dst + ulen).to(torch.int32)
        enc = [sw.encode_query(q, device=dev) for q in queries]
        lens = [e.numel() for e in enc]
        qstart_h = np.cumsum(per_q) - per_q
        # one launch per stripe-width group of up to GROUP queries; every
        # query row holds its own targets (indices into the packed buffer),
        # padded with its last one
        plan, pos_parts, qid_parts = [], [], []
        pos_off = q_off = 0
        for tpt, members in batched.buckets(lens).items():
            live_q = [q for q in members if per_q[q] > 0]
            for s0 in range(0, len(live_q), batched.GROUP):
                grp = live_q[s0:s0 + batched.GROUP]
                cnt = per_q[grp]
                m = int(cnt.max())
                k = np.minimum(np.arange(m)[None, :], cnt[:, None] - 1)
                pos_parts.append((qstart_h[grp][:, None] + k).reshape(-1))
                qid_parts.append(np.asarray(grp, np.int64))
                plan.append((tpt, len(grp), m, pos_off, q_off))
                pos_off += len(grp) * m
                q_off += len(grp)
        pos = torch.from_numpy(np.concatenate(pos_parts)).to(dev)
        lq = torch.from_numpy(np.concatenate(qid_parts)).to(dev)
        idx_all = inv[pos].to(torch.int32)
        qbuf = torch.zeros((nq, batched.MAX_QUERY), dtype=torch.uint8, device=dev)
        for j, e in enumerate(enc):
            qbuf[j, :e.numel()] = e
        qlen = torch.tensor(lens, dtype=torch.int32, device=dev)
        qrows, qls = qbuf[lq], qlen[lq]
        aff = torch.empty(n, dtype=torch.int32, device=dev)
        for tpt, G, m, po, qo in plan:
            sc = batched.sw_scan_queries(qrows[qo:qo + G], qls[qo:qo + G], tpt, packed, pdelim,
                                         affine=True, good_idx=idx_all[po:po + G * m].view(G, m),
                                         skip=1, gap_a=gap_open, gap_b=gap_extend)
            aff.index_copy_(0, pos[po:po + G * m], sc[:, :m].reshape(-1))
        del packed
        # normalised score as the exhaustive search forms it (float32 of the
        # affine score over float32 sqrt of Lq * maxlen of the hit's batch)
        den = torch.sqrt((qlen.to(torch.int64)[qid] * T["maxlen"][batch]).to(torch.float32))
        norm = aff.to(torch.float32) / den
        # rank: inside each query normalised score desc; the flat order is
        # (batch, segment) ascending, which the stable sorts keep for ties
        o = torch.sort(norm, descending=True, stable=True).indices
        o = o[torch.sort(qid[o], stable=True).indices]
        qstart = torch.from_numpy(qstart_h).to(dev)
        rank = torch.arange(n, device=dev) - qstart[qid[o]]
        o = o[rank < top]
        keep = np.minimum(per_q, top)
        h_norm, h_b = to_host(norm[o]), to_host(batch[o])
        h_s, h_a = to_host(seg[o]), to_host(aff[o])
        cuts = np.cumsum(keep)[:-1]
        return [(a_, b_.astype(np.int64), c_.astype(np.int64), d_.astype(np.int64))
                for a_, b_, c_, d_ in zip(np.split(h_norm, cuts), np.split(h_b, cuts),
                                          np.split(h_s, cuts), np.split(h_a, cuts))]

    def rescore(self, queries, cands, top: int = 4096, gap_open=11, gap_extend=1):
        """``rescore_flat`` of per-query candidate row tensors; returns per
        query the ``top`` hits as rows (normalised score, batch, segment,
        affine score) sorted by normalised score desc, then batch, then
        segment."""
        dev = self.db.device
        counts = [int(c.numel()) for c in cands]
        if sum(counts) == 0:
            return [[] for _ in queries]
        rows = torch.cat([c.to(dev, torch.int64) for c in cands])
        qid = torch.repeat_interleave(torch.arange(len(cands), device=dev),
                                      torch.tensor(counts, device=dev))
        o = torch.argsort(qid * max(self.n, 1) + rows)
        res = self.rescore_flat(queries, qid[o], rows[o], top, gap_open, gap_extend)
        return [list(zip(r[0].tolist(), r[1].tolist(), r[2].tolist(), r[3].tolist()))
                for r in res]

    def search_arrays(self, queries, n_cand: int = 32768, top: int = 4096, **kw) -> list:
        """``rescore_flat`` of the candidates of ``queries``: per query host
        arrays (norm, batch, segment, affine)."""
        codes = self.query_codes(queries)
        kq, kr, _ = self.candidates_flat(codes, n_cand, **kw)
        return self.rescore_flat(queries, kq, kr, top=top)

    def search(self, queries, n_cand: int = 32768, top: int = 4096, **kw):
        """Per query the ``top`` hits as rows (normalised score, batch,
        segment, affine score)."""
        return [list(zip(r[0].tolist(), r[1].tolist(), r[2].tolist(), r[3].tolist()))
                for r in self.search_arrays(queries, n_cand, top, **kw)]


def hit_strings(db, rows, width: int = 500) -> list:
    """First ``width`` residues of each hit (rows of ``rescore``), as the
    exhaustive search reports them (sseqs/msa.py:367-369)."""
    msa = importlib.import_module("sseqs_b200.msa")
    out = [None] * len(rows)
    by_batch: dict = {}
    for i, r in enumerate(rows):
        by_batch.setdefault(r[1], []).append(i)
    for bi, idx in by_batch.items():
        b = db.batches[bi]
        # the segment index is used as the exhaustive search uses it
        g = torch.tensor([rows[i][2] for i in idx], dtype=torch.int32, device=db.device)
        hb, hl = msa._gather_hits(b, g, len(idx))
        hb, hl = to_host(hb), to_host(hl)
        for j, i in enumerate(idx):
            out[i] = hb[j, :hl[j]].tobytes().decode("latin-1")
    return out

"""TEST AND MEASUREMENT INFRASTRUCTURE ONLY -- the reference's search loop on
the GPU, driving the reference's own CUDA kernels.

The reference's ``msa()`` (sseqs/msa.py:71-446) is Python; it does not travel
to a GPU machine here, but its kernels do (``oracle/_ref``, compiled from its
sources unmodified, bound by ``refkernels``).  ``search_chunks`` restates the
loop of sseqs/msa.py:196-405 step by step with the same torch operations --
chunk H2D copy from pinned memory on a copy stream with the reference's
synchronisations, per batch the xbit decode, the delimiter compaction, the
segment table, the fp16 FFT prefilter, ``topk``/``sort``/``[1:-1]``, linear
SW, ``topk``, affine SW, ``topk``, normalisation, the hit gather and its
copy to the host -- so that the reference path can be timed on the same B200
and inputs as this build.  The final sort and the a3m file (after the loop,
sseqs/msa.py:411-437) are not part of the timed loop, as in the reference's
own GB/s figure (its progress bar over chunks, README.md:11-12).

Only ``bench.py --impl reference`` uses it.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import refkernels

AA = "ARNDCQEGHILKMFPSTWYV"
AA_TO_POS = {a: i for i, a in enumerate(AA)}
AA_TO_POS.update({"X": 20, "-": 20, "*": 20})


def _luts(query: str, fft_rank: int):
    """sseqs/msa.py:110-145 (same numpy calls)."""
    from . import oracle as O
    return O.prefilter_luts(query, fft_rank)


def search_chunks(query: str, pinned_chunks, bs=50_000_000, fft_rank=4, top_fft=200,
                  top_sw=10, top_sw_affine=2, dlength=1e6):
    """One query through the reference loop over 1e9-byte packed chunks held
    in pinned host memory.  Returns the per-batch hit lists (normalised
    affine scores and hit strings)."""
    dev = torch.device("cuda")
    L = refkernels.lib()
    A, B = _luts(query, fft_rank)
    k = max(1, min(fft_rank, A.shape[0]))
    Ad = torch.from_numpy(np.ascontiguousarray(A[:k], np.float32)).to(dev)
    Bpad = np.zeros(max(100, (k + 1) * 21), np.float32)       # refkernels.warp_corr
    Bpad[:k * 21] = np.asarray(B[:k], np.float32).reshape(-1)
    Bd = torch.from_numpy(Bpad).to(dev)
    q_enc = torch.tensor([AA.index(c) for c in query if c in AA], dtype=torch.uint8, device=dev)
    qrev = torch.tensor([AA_TO_POS.get(c, 20) for c in query[::-1]], dtype=torch.uint8,
                        device=dev)
    arange = torch.arange(int(bs * 1.6), device=dev, dtype=torch.int32)
    pre_arange = torch.arange(500, device=dev, dtype=torch.int32)
    copy_stream = torch.cuda.Stream()
    compute_stream = torch.cuda.Stream()
    b = torch.zeros(pinned_chunks[0].numel(), dtype=torch.uint8, device=dev)
    out = []
    nxt = None
    for i, a_pin in enumerate(pinned_chunks):
        with torch.cuda.stream(copy_stream):                  # sseqs/msa.py:199-207
            if i != 0:
                b.copy_(nxt)
                torch.cuda.synchronize()
                if i + 1 < len(pinned_chunks):
                    nxt = pinned_chunks[i + 1].to(dev, non_blocking=True)
            else:
                b.copy_(a_pin.to(dev))
                torch.cuda.synchronize()
                if len(pinned_chunks) > 1:
                    nxt = pinned_chunks[i + 1].to(dev, non_blocking=True)
        with torch.cuda.stream(compute_stream):
            for j in range(math.ceil(b.numel() / bs)):
                n_sym = int(bs * 8 / 5)
                ascii = torch.empty(((n_sym + 7) // 8) * 8, dtype=torch.uint8, device=dev)
                # the reference decoder runs on the legacy default stream
                # (sseqs/xbit.cu:70); order it after this stream's work
                compute_stream.synchronize()
                L.decompress_launcher(b.data_ptr(), ascii.data_ptr(), n_sym, j * bs)
                torch.cuda.default_stream().synchronize()
                ascii = ascii[:n_sym]
                delim_pos = arange[ascii == 64]                      # :227
                starts = delim_pos + 1                               # :237-247
                starts = starts[starts < ascii.numel()]
                offsets = torch.cat([starts.to(torch.int32),
                                     torch.tensor([ascii.numel()], dtype=torch.int32, device=dev)])
                lengths = offsets - torch.cat([torch.tensor([0], dtype=torch.int32, device=dev),
                                               offsets[:-1]])
                lengths[:-1] -= 1
                if ascii[-1] == 64:
                    lengths[-1] -= 1
                max_seq_length = float(lengths.float().max().item())
                if abs(len(query) - max_seq_length) > dlength:      # :252
                    continue
                lengths = lengths[lengths != 0]
                if lengths.numel() == 0:
                    continue                     # the reference fails here (:261)
                n = 1 << (max(len(query), int(lengths.max())) - 1).bit_length()
                scores = torch.zeros(len(lengths), device=dev, dtype=torch.float16)
                maxlen = lengths.max()
                _offsets = torch.zeros(lengths.size(0) + 1, device=dev, dtype=torch.int32)
                _offsets[1:] = torch.cumsum(lengths + 1, 0)
                scratch = torch.zeros(k * (n + 2) + 64, dtype=torch.float16, device=dev)
                stats = torch.empty((len(lengths), 2), dtype=torch.float32, device=dev)
                ln32 = lengths.to(torch.int32).contiguous()
                off32 = _offsets[:-1].contiguous()
                L.launch_warp_corr(scores.data_ptr(), qrev.data_ptr(), Ad.data_ptr(),
                                   Bd.data_ptr(), ascii.data_ptr(), off32.data_ptr(),
                                   ln32.data_ptr(), stats.data_ptr(), len(lengths), 21, k,
                                   len(query), int(maxlen), n, compute_stream.cuda_stream,
                                   scratch.data_ptr())
                good_idx = torch.topk(scores, k=scores.shape[0] // top_fft)[1]   # :297
                good_idx = torch.sort(good_idx)[0][1:-1]                          # :307
                if good_idx.shape[0] == 0:
                    continue
                gi = good_idx.to(torch.int32).contiguous()
                dp = delim_pos.to(torch.int32).contiguous()
                sw_scores = torch.empty(gi.numel(), dtype=torch.int32, device=dev)
                L.launch_sw_cuda_blosum62(q_enc.data_ptr(), q_enc.numel(), gi.data_ptr(),
                                          ascii.data_ptr(), dp.data_ptr(), gi.numel(),
                                          sw_scores.data_ptr(), -1, compute_stream.cuda_stream)
                _topk = torch.topk(sw_scores, k=sw_scores.shape[0] // top_sw)          # :324
                g2 = good_idx[_topk.indices].to(torch.int32).contiguous()
                st = starts.to(torch.int32).contiguous()
                gap_sw = torch.empty(g2.numel(), dtype=torch.int32, device=dev)
                L.launch_sw_cuda_affine(q_enc.data_ptr(), q_enc.numel(), g2.data_ptr(),
                                        ascii.data_ptr(), st.data_ptr(), g2.numel(),
                                        gap_sw.data_ptr(), 11, 1, compute_stream.cuda_stream)
                if top_sw_affine > gap_sw.shape[0]:
                    continue                     # the reference's topk raises here (:335)
                __topk = torch.topk(gap_sw, k=top_sw_affine)
                gap_sw = gap_sw[__topk.indices]
                _topk_i = _topk.indices[__topk.indices]
                gap_sw = gap_sw / (len(query) * maxlen).sqrt()                      # :345
                seg_st = torch.cat((torch.zeros(1, dtype=lengths.dtype, device=dev),
                                    torch.cumsum(lengths[:-1] + 1, dim=0)))
                good_starts, good_stops = seg_st[good_idx], lengths[good_idx]
                good_starts, good_stops = good_starts[_topk_i], good_stops[_topk_i]
                _ar = (pre_arange < torch.max(good_stops)).nonzero(as_tuple=True)[0]
                idx = good_starts[:, None] + _ar
                seqs = ascii.expand(idx.size(0), -1).gather(1, idx)
                out.append((gap_sw.cpu().numpy(), seqs.cpu().numpy(), good_stops.cpu().numpy()))
    torch.cuda.synchronize()
    return out


def pinned_copies(chunks):
    """Pinned host copies of packed chunks (sseqs/msa.py:50-55)."""
    out = []
    for c in chunks:
        h = torch.empty(c.numel(), dtype=torch.uint8, pin_memory=True)
        h.copy_(c)
        out.append(h)
    return out


def kernels_one_batch(queries, packed_chunk, bs=1_000_000_000):
    """GCUPS of the reference's linear (gap -1, windows of sseqs/msa.py:313-319)
    and affine (11/1, windows of :327-332) kernels over every segment
    1 .. n-2 of the first batch of a packed chunk, per query; the batch is
    decoded by the reference's decoder."""
    dev = torch.device("cuda")
    L = refkernels.lib()
    n_sym = int(bs * 8 / 5)
    ascii = torch.empty(((n_sym + 7) // 8) * 8, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    L.decompress_launcher(packed_chunk.data_ptr(), ascii.data_ptr(), n_sym, 0)
    torch.cuda.synchronize()
    ascii = ascii[:n_sym]
    delim = torch.nonzero(ascii == 64).flatten().to(torch.int32)
    # real segments end where the padding starts: the last delimiter after a residue
    nz = torch.nonzero(ascii != 64).flatten()
    last = int(nz[-1].item()) if nz.numel() else 0
    nseg = int(torch.searchsorted(delim, torch.tensor([last], dtype=torch.int32,
                                                      device=dev)).item()) + 1
    good = torch.arange(1, nseg - 1, dtype=torch.int32, device=dev)
    residues = int((delim[1:nseg - 1] - delim[0:nseg - 2] - 1).to(torch.int64).sum().item())
    dp1 = (delim + 1).contiguous()
    stream = torch.cuda.current_stream().cuda_stream
    lin_ms, aff_ms, cells = 0.0, 0.0, 0
    for q in queries:
        if len(q) > 1024:
            continue
        qe = torch.tensor([AA.index(c) for c in q if c in AA], dtype=torch.uint8, device=dev)
        o = torch.empty(good.numel(), dtype=torch.int32, device=dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        L.launch_sw_cuda_blosum62(qe.data_ptr(), qe.numel(), good.data_ptr(), ascii.data_ptr(),
                                  delim.data_ptr(), good.numel(), o.data_ptr(), -1, stream)
        ev[1].record()
        L.launch_sw_cuda_affine(qe.data_ptr(), qe.numel(), good.data_ptr(), ascii.data_ptr(),
                                dp1.data_ptr(), good.numel(), o.data_ptr(), 11, 1, stream)
        ev[2].record()
        torch.cuda.synchronize()
        lin_ms += ev[0].elapsed_time(ev[1])
        aff_ms += ev[1].elapsed_time(ev[2])
        cells += len(q) * residues
    return {"gcups_linear": round(cells / (lin_ms * 1e-3) / 1e9, 1),
            "gcups_affine": round(cells / (aff_ms * 1e-3) / 1e9, 1),
            "segments": nseg - 2, "residues": residues,
            "queries": sum(1 for q in queries if len(q) <= 1024)}

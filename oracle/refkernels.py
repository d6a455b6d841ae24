"""ctypes binding of the reference's own CUDA kernels (test oracle only).

``oracle/Makefile`` compiles sseqs/sw.cu, sseqs/xbit.cu and sseqs/filter.cu
unmodified into ``oracle/_ref/libsseqs_ref.so``; their launchers are already
``extern "C"`` (sseqs/sw.cu:336-425, sseqs/xbit.cu:65-78,
sseqs/filter.cu:161-174).  Inputs given to them here are checked to stay
inside the reference's defined behaviour (no target index 0, whose window
reads ``starts[-1]``; query lengths <= 1024).
"""
import ctypes
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "oracle", "_ref", "libsseqs_ref.so")
_lib = None


def available():
    return os.path.exists(PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(PATH)
        P, I = ctypes.c_void_p, ctypes.c_int
        L.launch_sw_cuda_blosum62.argtypes = [P, I, P, P, P, I, P, I, P]
        L.launch_sw_cuda_blosum62.restype = None
        L.launch_sw_cuda_affine.argtypes = [P, I, P, P, P, I, P, I, I, P]
        L.launch_sw_cuda_affine.restype = None
        L.decompress_launcher.argtypes = [P, P, I, I]
        L.decompress_launcher.restype = None
        L.compress_launcher.argtypes = [P, P, I]
        L.compress_launcher.restype = None
        L.launch_warp_corr.argtypes = [P, P, P, P, P, P, P, P, I, I, I, I, I, I, P, P]
        L.launch_warp_corr.restype = None
        _lib = L
    return _lib


def sw_linear(q, good_idx, ascii, starts, gap):
    import torch
    assert q.numel() <= 1024 and int(good_idx.min()) >= 1
    out = torch.empty(good_idx.numel(), dtype=torch.int32, device="cuda")
    lib().launch_sw_cuda_blosum62(q.data_ptr(), q.numel(), good_idx.data_ptr(), ascii.data_ptr(),
                                  starts.data_ptr(), good_idx.numel(), out.data_ptr(), gap,
                                  torch.cuda.current_stream().cuda_stream)
    return out


def sw_affine(q, good_idx, ascii, starts, go, ge):
    import torch
    assert q.numel() <= 1024 and int(good_idx.min()) >= 1
    out = torch.empty(good_idx.numel(), dtype=torch.int32, device="cuda")
    lib().launch_sw_cuda_affine(q.data_ptr(), q.numel(), good_idx.data_ptr(), ascii.data_ptr(),
                                starts.data_ptr(), good_idx.numel(), out.data_ptr(), go, ge,
                                torch.cuda.current_stream().cuda_stream)
    return out


def decompress(packed, n, lo):
    """Reference decoder; writes n rounded up to 8 symbols, so pad the output."""
    import torch
    out = torch.empty(((n + 7) // 8) * 8, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    lib().decompress_launcher(packed.data_ptr(), out.data_ptr(), n, lo)
    torch.cuda.synchronize()
    return out[:n]


def warp_corr(query: str, A, B, ascii, offsets, lengths, n, k):
    """The reference prefilter (sseqs/filter.cu:161-395) on a batch.

    Two over-reads of the reference are given memory to land in: the query
    spectrum scratch holds k*(n+2) halves (the kernel writes k*(n/2+1)
    half2), and the database table holds at least 100 floats (the kernel
    stages W_db[0..99], sseqs/fft.cu:91-93), zero past the k x 21 table.
    """
    import numpy as np
    import torch
    AA = "ARNDCQEGHILKMFPSTWYV"
    pos = {a: i for i, a in enumerate(AA)}
    pos.update({"X": 20, "-": 20, "*": 20})
    qrev = torch.tensor([pos.get(c, 20) for c in query[::-1]], dtype=torch.uint8, device="cuda")
    Ad = torch.from_numpy(np.ascontiguousarray(A[:k], np.float32)).cuda()
    Bpad = np.zeros(max(100, (k + 1) * 21), np.float32)
    Bpad[:k * 21] = np.asarray(B[:k], np.float32).reshape(-1)
    Bd = torch.from_numpy(Bpad).cuda()
    nseg = lengths.numel()
    corr = torch.zeros(nseg, dtype=torch.float16, device="cuda")
    stats = torch.empty((nseg, 2), dtype=torch.float32, device="cuda")
    scratch = torch.zeros(k * (n + 2) + 64, dtype=torch.float16, device="cuda")
    off32 = offsets.to(torch.int32).contiguous()
    ln32 = lengths.to(torch.int32).contiguous()
    maxlen = int(ln32.max().item())
    torch.cuda.synchronize()
    lib().launch_warp_corr(corr.data_ptr(), qrev.data_ptr(), Ad.data_ptr(), Bd.data_ptr(),
                           ascii.data_ptr(), off32.data_ptr(), ln32.data_ptr(), stats.data_ptr(),
                           nseg, 21, k, len(query), maxlen, n,
                           torch.cuda.current_stream().cuda_stream, scratch.data_ptr())
    torch.cuda.synchronize()
    return corr

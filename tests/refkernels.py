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

"""ctypes binding of ``libsseqs_b200.so`` (the C ABI in ``include/sseqs_b200.h``).

The library is built in-tree by ``python -m sseqs_b200.build`` (or
``__graft_entry__.build()``).  There is no fallback: if the shared library is
missing, every operation raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libsseqs_b200.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_SZ = ctypes.c_size_t
_D = ctypes.c_double
_F = ctypes.c_float

# name -> (restype, argtypes)
_SIGNATURES = {
    "sseqs_status_string": (ctypes.c_char_p, [_I]),
    "sseqs_version": (_I, []),
    "sseqs_max_query_len": (_I, []),
    "sseqs_xbit_decompress": (_I, [_P, _P, _I64, _I64, _P]),
    "sseqs_xbit_compress": (_I, [_P, _P, _I64, _P]),
    "sseqs_sw_linear": (_I, [_P, _I, _P, _P, _P, _I64, _P, _I, _P]),
    "sseqs_sw_affine": (_I, [_P, _I, _P, _P, _P, _I64, _P, _I, _I, _P]),
    "sseqs_sw_scan": (_I, [_I, _P, _I, _P, ctypes.c_int32, _I64, _P, _P, _I, _P, _I, _I, _P]),
    "sseqs_sw_scan_both": (_I, [_P, _I, _P, ctypes.c_int32, _I64, _P, _P, _I, _P, _P, _I, _I, _I,
                                _P]),
    "sseqs_sw_scan_queries": (_I, [_I, _I, _I, _P, _I64, _P, _P, _I64, ctypes.c_int32, _I64,
                                   _P, _P, _I, _P, _I64, _I, _I, _P, _P]),
    "sseqs_find_delims_workspace_bytes": (_SZ, [_I64]),
    "sseqs_find_delims": (_I, [_P, _I64, _P, _I64, _P, _P, _SZ, _P]),
    "sseqs_segment_table_workspace_bytes": (_SZ, [_I64]),
    "sseqs_segment_table": (_I, [_P, _I64, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "sseqs_topk_workspace_bytes": (_SZ, [_I64]),
    "sseqs_topk": (_I, [_P, _I, _I64, _I64, _P, _P, _SZ, _P]),
    "sseqs_topk_static": (_I, [_P, _I, _I64, _I64, _P, _P]),
    "sseqs_gather_windows": (_I, [_P, _P, _P, _P, _I64, _I, _P, _P, _P]),
    "sseqs_pack_segments": (_I, [_P, _P, _P, _P, _P, _I64, _P, _P]),
    "sseqs_backtrack_workspace_bytes": (_SZ, [_I, _I, _I]),
    "sseqs_backtrack_affine": (_I, [_P, _I, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _I,
                                    _P, _I, _P, _SZ, _P]),
    "sseqs_a3m_rows": (_I, [_P, _I64, _I64, _P, _P, _P, _P, _P, _P, _I64, _P]),
    "sseqs_prefilter_workspace_bytes": (_SZ, [_I, _I]),
    "sseqs_prefilter": (_I, [_P, _P, _P, _I64, _P, _I, _P, _P, _I, _I, _P, _P, _SZ, _P]),
    "sseqs_dpx_peak": (_I, [_P, ctypes.POINTER(_D), _P]),
    "sseqs_launch_count": (_I64, []),
    "sseqs_int16x2_peak": (_I, [_P, ctypes.POINTER(_D), _P]),
    "sseqs_sw_set_variant": (_I, [_I, _I, _I]),
    "sseqs_gemm_bf16": (_I, [_I, _I, _I, _I64, _I64, _I64, _P, _I64, _P, _I64, _P, _I64, _P, _P,
                             _P, _P, _P, _P]),
    "sseqs_gemm_set_tensor_path": (_I, [_I]),
    "sseqs_gemm_error": (_I, [ctypes.POINTER(_I)]),
    "sseqs_embed_layout": (_I, [_P, _P, _P, _P, _I, _P, _P]),
    "sseqs_embed_lookup": (_I, [_P, _I64, _P, _I, _P, _P]),
    "sseqs_embed_conv1_table": (_I, [_P, _I64, _P, _P, _P, _I, _P, _P, _P]),
    "sseqs_embed_grad": (_I, [_P, _I64, _P, _I, _P, _P]),
    "sseqs_pool_normalize": (_I, [_P, _I, _P, _P, _I, _P, _P, _P, _P]),
    "sseqs_pair_loss": (_I, [_P, _I, _P, _P, _P, _P, _I64, _P, _P, _P, _P]),
    "sseqs_pool_backward": (_I, [_P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
    "sseqs_bias_grad": (_I, [_P, _I64, _I, _P, _P]),
    "sseqs_adam_conv": (_I, [_P, _P, _P, _P, _I, _I, _F, _F, _F, _F, _I, _P, _P, _P]),
    "sseqs_adam_flat": (_I, [_P, _P, _P, _P, _I64, _F, _F, _F, _F, _I, _P, _P]),
    "sseqs_quantize_e4m3": (_I, [_P, _I64, _F, _P, _P]),
    "sseqs_score_select": (_I, [_P, _I, _P, _I64, _P, _P, _P, _P, _I, _P]),
    "sseqs_score_dense": (_I, [_P, _I, _P, _I64, _P, _P]),
    "sseqs_kth_largest_rows": (_I, [_P, _I, _I, _I, _P, _P]),
    "sseqs_sw_variant_words": (_I, [_I, _I, _I]),
    "sseqs_sw_get_variant": (_I, [_I, _I]),
    "sseqs_sw_set_query_pairing": (_I, [_I, _I]),
    "sseqs_sw_get_query_pairing": (_I, [_I]),
}

_lock = threading.Lock()
_lib = None


class SseqsError(RuntimeError):
    """A libsseqs_b200 entry point returned a non-zero status."""


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        f"{LIB_PATH} is missing: build it with `python -m sseqs_b200.build` "
                        "(there is no CPU fallback)")
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in _SIGNATURES.items():
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = lib().sseqs_status_string(status).decode()
        raise SseqsError(f"{what}: {msg} (status {status})")


def stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def ptr(t) -> int | None:
    if t is None:
        return None
    return int(t.data_ptr())


def require_cuda(*tensors) -> None:
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise ValueError("sseqs_b200 operations take CUDA tensors")


# Bytes moved between host and device by the package's own transfer points
# (queries and traceback inputs in, hits and alignments out).
transfer_bytes = {"h2d": 0, "d2h": 0}


def to_device(t: torch.Tensor, device="cuda") -> torch.Tensor:
    transfer_bytes["h2d"] += t.numel() * t.element_size()
    return t.to(device)


def to_host(t: torch.Tensor):
    transfer_bytes["d2h"] += t.numel() * t.element_size()
    return t.cpu().numpy()


def workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)

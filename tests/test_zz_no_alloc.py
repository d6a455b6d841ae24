"""The allocation-free top-k entry point, checked against the ordinary one.

`sseqs_topk_static` exists for callers that may not allocate GPU memory
themselves -- code whose device memory belongs to another allocator (a
framework's caching pool, a serving process with a fixed budget), or code on
a latency-critical path that cannot take the stalls cudaMalloc / cudaFree can
cause.  It keeps its scratch in a fixed array inside the library instead of
a caller-provided workspace.  These tests call it through the C ABI and
compare its output with `sseqs_topk` (which takes a workspace), on two calls
in a row, so that anything the first call leaves in the shared array would
show up in the second.  Indices are integers: they must match exactly.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_N = 1 << 24            # SSEQS_TOPK_STATIC_MAX_N in include/sseqs_b200.h
SSEQS_ERR_CAPACITY = 5


def _static_topk(values: torch.Tensor, k: int) -> torch.Tensor:
    from sseqs_b200 import _lib
    kt = 0 if values.dtype == torch.int32 else 1
    out = torch.full((max(k, 1),), -7, dtype=torch.int32, device=values.device)
    st = _lib.lib().sseqs_topk_static(values.data_ptr(), kt, values.numel(), k, out.data_ptr(),
                                      _lib.stream_ptr())
    assert st == 0, _lib.lib().sseqs_status_string(st)
    return out[:k]


def test_static_topk_matches_workspace_topk_on_two_calls():
    from sseqs_b200 import select
    rng = np.random.default_rng(2024)
    # first call: many tiles, many ties at the cut
    a = torch.from_numpy(rng.integers(-1, 300, 3_000_000).astype(np.int32)).cuda()
    got1 = _static_topk(a, 4096)
    exp1 = select.topk_indices(a, 4096)
    torch.cuda.synchronize()
    assert torch.equal(got1, exp1)
    # second call right after: fewer tiles, other key type; stale counters of
    # the first call sit in the scratch array
    b = torch.from_numpy((rng.standard_normal(5000) * 3).astype(np.float16)).cuda()
    got2 = _static_topk(b, 17)
    exp2 = select.topk_indices(b, 17)
    torch.cuda.synchronize()
    assert torch.equal(got2, exp2)
    # and the first input once more, to see the second call left nothing behind
    assert torch.equal(_static_topk(a, 4096), exp1)


def test_static_topk_at_capacity_and_beyond():
    from sseqs_b200 import _lib, select
    rng = np.random.default_rng(7)
    a = torch.from_numpy(rng.integers(0, 1 << 20, MAX_N).astype(np.int32)).cuda()
    assert torch.equal(_static_topk(a, 1000), select.topk_indices(a, 1000))
    # one key more than the fixed scratch holds is refused before any launch
    st = _lib.lib().sseqs_topk_static(a.data_ptr(), 0, MAX_N + 1, 10, a.data_ptr(),
                                      _lib.stream_ptr())
    assert st == SSEQS_ERR_CAPACITY
    assert b"capacity" in _lib.lib().sseqs_status_string(st)

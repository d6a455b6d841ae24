"""GPU parity of the xbit codec and the selection kernels (bit-exact)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refkernels

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 8, 33, 4096, 8191, 100_003, 3_000_000])
def test_xbit_matches_oracle(n):
    from sseqs_b200 import xbit
    rng = np.random.default_rng(n)
    sym = rng.integers(64, 96, n).astype(np.uint8)
    packed = xbit.compress(torch.from_numpy(sym))
    exp_packed = O.xbit_compress(sym)
    np.testing.assert_array_equal(packed.cpu().numpy(), exp_packed)
    for lo in (0, 5, 13):
        m = max(0, (exp_packed.size - lo) * 8 // 5)
        if m == 0:
            continue
        got = xbit.decompress(packed, m, lo).cpu().numpy()
        np.testing.assert_array_equal(got, O.xbit_decompress(exp_packed, m, lo))


def test_xbit_decode_unaligned_views():
    from sseqs_b200 import xbit
    rng = np.random.default_rng(9)
    sym = rng.integers(64, 96, 50_000).astype(np.uint8)
    packed = xbit.compress(torch.from_numpy(sym))
    for off in (1, 3, 7):
        view = packed[off:]
        m = view.numel() * 8 // 5
        got = xbit.decompress(view, m, 0).cpu().numpy()
        np.testing.assert_array_equal(got, O.xbit_decompress(packed.cpu().numpy()[off:], m, 0))


def test_xbit_matches_reference_kernel():
    if not refkernels.available():
        pytest.skip("oracle/_ref/libsseqs_ref.so not built")
    from sseqs_b200 import xbit
    rng = np.random.default_rng(4)
    n = 1_600_000
    sym = rng.integers(64, 96, n).astype(np.uint8)
    packed = xbit.compress(torch.from_numpy(sym))
    padded = torch.cat([packed, torch.zeros(16, dtype=torch.uint8, device="cuda")])
    for lo in (0, 50_000):
        m = (packed.numel() - lo) * 8 // 5 // 8 * 8
        ref = refkernels.decompress(padded, m, lo)
        torch.testing.assert_close(xbit.decompress(packed, m, lo), ref, rtol=0, atol=0)


def _np_delims(a):
    return np.flatnonzero(a == 64).astype(np.int32)


@pytest.mark.parametrize("n", [1, 100, 4096, 4097, 1_000_000])
def test_find_delims_and_segment_table(n):
    from sseqs_b200 import select
    rng = np.random.default_rng(n)
    a = rng.choice(np.frombuffer(b"ACDEFGHIK@", np.uint8), size=n)
    if n > 10:
        a[-5:] = 64                                  # padding tail
    ad = torch.from_numpy(a).cuda()
    delim = select.find_delims(ad)
    np.testing.assert_array_equal(delim.cpu().numpy(), _np_delims(a))
    tab = select.segment_table(ad, delim)
    seg = O.segment(a)
    np.testing.assert_array_equal(tab["lengths"].cpu().numpy(), seg["lengths"])
    np.testing.assert_array_equal(tab["offsets"].cpu().numpy(), seg["offsets"])
    assert tab["maxlen"] == (int(seg["lengths"].max()) if seg["lengths"].size else 0)


@pytest.mark.parametrize("n,k", [(10, 3), (1000, 1000), (1000, 999), (5000, 17),
                                 (100_000, 1000), (2_000_000, 4096)])
def test_topk_int32_canonical(n, k):
    from sseqs_b200 import select
    rng = np.random.default_rng(n + k)
    v = rng.integers(-1, 60, n).astype(np.int32)     # many ties
    got = select.topk_indices(torch.from_numpy(v).cuda(), k).cpu().numpy()
    exp = np.sort(O.topk_canonical(v, k))
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("n,k", [(1000, 10), (300_000, 1500)])
def test_topk_fp16_canonical(n, k):
    from sseqs_b200 import select
    rng = np.random.default_rng(k)
    v = (rng.standard_normal(n) * 4).astype(np.float16)
    v[::7] = v[3]                                    # ties
    got = select.topk_indices(torch.from_numpy(v).cuda(), k).cpu().numpy()
    exp = np.sort(O.topk_canonical(v.astype(np.float64), k))
    np.testing.assert_array_equal(got, exp)

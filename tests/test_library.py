"""CPU checks of the C ABI library: it loads and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "sseqs_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sseqs_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def built_lib():
    from sseqs_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_library_exports_every_declared_symbol(built_lib):
    names = _declared()
    assert len(names) >= 10
    for name in names:
        assert hasattr(built_lib, name), name


def test_python_binding_covers_declared_symbols():
    from sseqs_b200 import _lib
    assert set(_declared()) <= set(_lib.exported_symbols())


def test_status_strings_and_limits(built_lib):
    from sseqs_b200 import _lib
    L = _lib.lib()
    assert L.sseqs_status_string(0) == b"ok"
    assert b"workspace" in L.sseqs_status_string(4)
    assert L.sseqs_max_query_len() == 2048
    assert L.sseqs_version() >= 1


def test_argument_errors_are_reported_without_a_gpu(built_lib):
    """Host-side argument checks run before any CUDA call."""
    from sseqs_b200 import _lib
    L = _lib.lib()
    assert L.sseqs_topk(None, 0, 10, 11, None, None, 0, None) == 1        # k > n
    assert L.sseqs_topk(None, 5, 10, 1, None, None, 0, None) == 1         # bad key type
    assert L.sseqs_xbit_decompress(None, None, -1, 0, None) == 1
    assert L.sseqs_sw_scan(1, None, 10, None, -1, 5, None, None, 0, None, 11, 1, None) == 1
    assert L.sseqs_find_delims(None, 10, None, 0, None, None, 0, None) == 1
    assert L.sseqs_backtrack_workspace_bytes(10, 20, 2) > 0


def test_fails_loudly_without_library(monkeypatch, tmp_path):
    from sseqs_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()


def test_batched_buckets_group_by_stripe_width():
    from sseqs_b200 import batched
    lengths = [300, 31, 32, 33, 2048, 64, 289, 1]
    b = batched.buckets(lengths)
    assert b == {10: [6, 0], 1: [7, 1, 2], 2: [3, 5], 64: [4]}
    for tpt, members in b.items():
        assert all((lengths[i] + 31) // 32 == tpt for i in members)


def test_score_kernel_registry_matches_dispatch_rules(built_lib):
    """The instantiated score kernels are the ones the host dispatch counts
    on: the fused pass up to width 23 (``tune.fused``), a wide layout of its
    own for the linear kernel at widths 2-29 and for the affine and fused
    kernels at 2-16 (``tune.has_wide``; at width 1 both layouts hold 16
    words per lane).  Read from the library's registry;
    no GPU needed."""
    from sseqs_b200 import _lib, tune
    L = _lib.lib()
    words = lambda mode, t, wide: L.sseqs_sw_variant_words(mode, t, wide)
    assert tune.MAX_FUSED_TPT == 23
    for t in range(1, 65):
        assert (words(2, t, 0) > 0) == (t <= 23), t
        assert tune.fused(32 * t) == (t <= 23)
        assert words(0, t, 0) > 0 and words(1, t, 0) > 0
        assert tune.has_wide(0, t) == (2 <= t <= 29), t
        assert tune.has_wide(1, t) == (2 <= t <= 16), t
        if t <= 23:
            assert tune.has_wide(2, t) == (2 <= t <= 16), t
        # the query-pair kernel (mode 3) exists at every width, with the
        # affine kernel's layouts
        assert words(3, t, 0) == words(1, t, 0) and words(3, t, 1) == words(1, t, 1), t
    assert words(0, 27, 1) == 2 and words(0, 27, 0) == 1
    assert L.sseqs_sw_variant_words(4, 5, 0) == -1 and L.sseqs_sw_variant_words(0, 65, 0) == -1


def test_variant_selection_round_trips(built_lib):
    """The lane layout chosen per (kernel, width) reads back as set; out of
    range reads -1.  Host state only, no GPU."""
    from sseqs_b200 import tune
    before = tune.get_variant(1, 9)
    try:
        for w in (1, 0, 1):
            tune.set_variant(1, 9, w)
            assert tune.get_variant(1, 9) == w
    finally:
        tune.set_variant(1, 9, before)
    L = built_lib
    assert L.sseqs_sw_get_variant(4, 1) == -1 and L.sseqs_sw_get_variant(0, 65) == -1


def test_scan_both_argument_checks_without_a_gpu(built_lib):
    """sseqs_sw_scan_both rejects bad arguments on the host, before any
    CUDA call: a window shift other than 0/1, a missing output, a negative
    query length or one above 2048, gaps outside the int16 domain; no
    targets is a no-op.  (Query length 0 fills both outputs with -1 on the
    GPU, as the separate scans do: ``test_gpu_sw``.)"""
    import ctypes
    from sseqs_b200 import _lib
    L = _lib.lib()
    fake = ctypes.c_void_p(16)              # never dereferenced: every call returns early
    assert L.sseqs_sw_scan_both(fake, 10, None, 0, 0, fake, fake, 1, fake, fake, -1, 11, 1,
                                None) == 0
    assert L.sseqs_sw_scan_both(fake, 10, None, 0, 5, fake, fake, 2, fake, fake, -1, 11, 1,
                                None) == 1
    assert L.sseqs_sw_scan_both(fake, 10, None, 0, 5, fake, fake, 1, None, fake, -1, 11, 1,
                                None) == 1
    assert L.sseqs_sw_scan_both(fake, -1, None, 0, 5, fake, fake, 1, fake, fake, -1, 11, 1,
                                None) == 1
    assert L.sseqs_sw_scan_both(fake, 2049, None, 0, 5, fake, fake, 1, fake, fake, -1, 11, 1,
                                None) == 2
    assert L.sseqs_sw_scan_both(fake, 10, None, 0, 5, fake, fake, 1, fake, fake, 1, 11, 1,
                                None) == 2
    assert L.sseqs_sw_scan_both(fake, 10, None, 0, 5, fake, fake, 1, fake, fake, -1, -3, 1,
                                None) == 2

"""GPU parity of the score kernels: CUDA vs the CPU oracle vs the reference's
own CUDA kernels, bit-exact (int32 scores)."""
import importlib
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refkernels
from tests.helpers import homolog_targets, rand_seq

pytestmark = pytest.mark.gpu
NT = os.cpu_count() or 4


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _case(seed, Lq, n_targets, extra=""):
    rng = np.random.default_rng(seed)
    query = rand_seq(rng, Lq)
    targets = homolog_targets(rng, query, n_targets, lo=1, hi=400)
    if extra:
        targets += [rand_seq(rng, int(rng.integers(1, 80)), extra=extra) for _ in range(8)]
    ascii, starts = O.pack_targets(targets)
    return query, O.encode_query(query), ascii, starts


QUERY_LENGTHS = [1, 2, 17, 32, 33, 64, 65, 100, 128, 129, 200, 256, 257, 300, 500, 511, 640,
                 777, 1000, 1024, 1025, 1500, 2048]


@pytest.mark.parametrize("Lq", QUERY_LENGTHS)
def test_sw_ops_match_oracle(Lq):
    S = importlib.import_module("sseqs_b200.sw")
    n = 600 if Lq <= 300 else (250 if Lq <= 1024 else 120)
    query, q, ascii, starts = _case(Lq, Lq, n, extra="XBZU*@")
    good = np.arange(len(starts), dtype=np.int32)
    rng = np.random.default_rng(Lq + 7)
    good = rng.permutation(good)            # arbitrary order, includes g = 0
    qd, gd, ad, sd = _dev(q), _dev(good), _dev(ascii), _dev(starts)
    lin = S.sw_cuda_blosum62(qd, gd, ad, sd, gap_penalty_param=-1).cpu().numpy()
    np.testing.assert_array_equal(lin, O.sw_linear(q, good, ascii, starts, -1, NT))
    aff = S.sw_cuda_affine(qd, gd, ad, sd, 11, 1).cpu().numpy()
    np.testing.assert_array_equal(aff, O.sw_affine(q, good, ascii, starts, 11, 1, NT))
    # the msa() affine call passes delimiter+1 so windows skip one residue and
    # end on the '@'
    sp = (starts + 1).astype(np.int32)
    aff2 = S.sw_cuda_affine(qd, gd, ad, _dev(sp), 11, 1).cpu().numpy()
    np.testing.assert_array_equal(aff2, O.sw_affine(q, good, ascii, sp, 11, 1, NT))
    # gaps other than msa()'s run the kernels that read them from the
    # arguments (msa()'s own run the twins with them built in)
    sub = good[: max(1, len(good) // 3)]
    sd3 = _dev(sub)
    lin4 = S.sw_cuda_blosum62(qd, sd3, ad, sd, gap_penalty_param=-4).cpu().numpy()
    np.testing.assert_array_equal(lin4, O.sw_linear(q, sub, ascii, starts, -4, NT))
    aff52 = S.sw_cuda_affine(qd, sd3, ad, sd, 5, 2).cpu().numpy()
    np.testing.assert_array_equal(aff52, O.sw_affine(q, sub, ascii, starts, 5, 2, NT))


# one query length per stripe width 1..32 (the reference's kernels L = 32..1024,
# sseqs/sw.cu:336-425), with varied remainders
REF_LENGTHS = [32 * t - (7 * t) % 32 for t in range(1, 33)]


class _Variants:
    """Select lane layouts for a width and put back the ones selected before."""

    def __init__(self, tpt):
        from sseqs_b200 import tune
        self.tune, self.tpt = tune, tpt
        self.before = [tune.get_variant(m, tpt) for m in (0, 1, 2)]

    def set(self, wide):
        for m in (0, 1, 2):
            self.tune.set_variant(m, self.tpt, wide)

    def restore(self):
        for m, w in enumerate(self.before):
            self.tune.set_variant(m, self.tpt, w)


@pytest.mark.parametrize("Lq", REF_LENGTHS)
def test_sw_ops_match_reference_cuda_kernels(Lq):
    """Every score kernel of this width -- linear, affine and the fused pass,
    in each lane layout the width has -- equals the reference's own kernels
    compiled from source, on both window forms msa() uses."""
    if not refkernels.available():
        pytest.skip("oracle/_ref/libsseqs_ref.so not built")
    S = importlib.import_module("sseqs_b200.sw")
    from sseqs_b200 import tune
    tpt = tune.tpt_of(Lq)
    assert tpt == REF_LENGTHS.index(Lq) + 1
    query, q, ascii, starts = _case(1000 + Lq, Lq, 500 if Lq <= 512 else 300, extra="XB")
    ascii = np.concatenate([ascii, np.full(48, 64, np.uint8)])
    delim = np.flatnonzero(ascii == 64).astype(np.int32)
    nseg = len(starts)
    good = np.arange(1, nseg, dtype=np.int32)     # g >= 1: defined windows
    qd, gd, ad, dd = _dev(q), _dev(good), _dev(ascii), _dev(delim)
    dp = _dev(delim + 1)
    ref_lin = {gap: refkernels.sw_linear(qd, gd, ad, dd, gap) for gap in (-1, -4, -11)}
    ref_aff = {p: refkernels.sw_affine(qd, gd, ad, dd, *p) for p in ((11, 1), (5, 2), (0, 0))}
    ref_shift = refkernels.sw_affine(qd, gd, ad, dp, 11, 1)
    layouts = [0] + [1 for m in (0, 1, 2) if tune.has_wide(m, tpt)][:1]
    v = _Variants(tpt)
    try:
        for wide in layouts:
            v.set(wide)
            for gap, ref in ref_lin.items():
                torch.testing.assert_close(S.sw_cuda_blosum62(qd, gd, ad, dd, gap), ref,
                                           rtol=0, atol=0)
            for (go, ge), ref in ref_aff.items():
                torch.testing.assert_close(S.sw_cuda_affine(qd, gd, ad, dd, go, ge), ref,
                                           rtol=0, atol=0)
            torch.testing.assert_close(S.sw_cuda_affine(qd, gd, ad, dp, 11, 1), ref_shift,
                                       rtol=0, atol=0)
            # scan forms: msa()'s linear call (skip 0) and affine call (delim+1 = skip 1)
            torch.testing.assert_close(
                S.sw_scan(qd, ad, dd, affine=False, g0=1, n_targets=nseg - 1, skip=0, gap_a=-1),
                ref_lin[-1], rtol=0, atol=0)
            torch.testing.assert_close(
                S.sw_scan(qd, ad, dd, affine=True, g0=1, n_targets=nseg - 1, skip=1, gap_a=11,
                          gap_b=1), ref_shift, rtol=0, atol=0)
            lin, aff = S.sw_scan_both(qd, ad, dd, g0=1, n_targets=nseg - 1, affine_skip=1)
            torch.testing.assert_close(lin, ref_lin[-1], rtol=0, atol=0)
            torch.testing.assert_close(aff, ref_shift, rtol=0, atol=0)
    finally:
        v.restore()


def test_scan_matches_reference_windows():
    """sw_scan over a decoded batch == the two window forms msa() uses."""
    S = importlib.import_module("sseqs_b200.sw")
    query, q, ascii, starts = _case(77, 333, 3000)
    pad = np.full(100, 64, np.uint8)             # '@' padding as in a packed chunk
    ascii = np.concatenate([ascii, pad])
    delim = np.flatnonzero(ascii == 64).astype(np.int32)
    nseg = len(starts)
    qd, ad, dd = _dev(q), _dev(ascii), _dev(delim)
    good = np.arange(1, nseg - 1, dtype=np.int32)
    gd = _dev(good)
    lin = S.sw_scan(qd, ad, dd, affine=False, good_idx=gd, skip=0, gap_a=-1)
    lin_ref = S.sw_cuda_blosum62(qd, gd, ad, dd, gap_penalty_param=-1)
    torch.testing.assert_close(lin, lin_ref, rtol=0, atol=0)
    sp = _dev((delim + 1).astype(np.int32))
    aff = S.sw_scan(qd, ad, dd, affine=True, good_idx=gd, skip=1, gap_a=11, gap_b=1)
    aff_ref = S.sw_cuda_affine(qd, gd, ad, sp, 11, 1)
    torch.testing.assert_close(aff, aff_ref, rtol=0, atol=0)
    # implicit target range (whole batch), g0 offset
    full = S.sw_scan(qd, ad, dd, affine=True, g0=1, n_targets=nseg - 2, skip=1, gap_a=11, gap_b=1)
    torch.testing.assert_close(full, aff_ref, rtol=0, atol=0)
    np.testing.assert_array_equal(
        full.cpu().numpy(), O.sw_affine(q, good, ascii, delim + 1, 11, 1, NT))


def test_nonstandard_gap_parameters_use_exact_generic_path():
    S = importlib.import_module("sseqs_b200.sw")
    query, q, ascii, starts = _case(5, 90, 200)
    good = np.arange(len(starts), dtype=np.int32)
    qd, gd, ad, sd = _dev(q), _dev(good), _dev(ascii), _dev(starts)
    np.testing.assert_array_equal(S.sw_cuda_blosum62(qd, gd, ad, sd, 2).cpu().numpy(),
                                  O.sw_linear(q, good, ascii, starts, 2, NT))
    np.testing.assert_array_equal(S.sw_cuda_affine(qd, gd, ad, sd, -3, 1).cpu().numpy(),
                                  O.sw_affine(q, good, ascii, starts, -3, 1, NT))


def test_degenerate_inputs():
    S = importlib.import_module("sseqs_b200.sw")
    q = _dev(O.encode_query("MKTAYIAKQRQ"))
    ascii = _dev(np.frombuffer(b"MKTAYIAK@@QRQ@W@", np.uint8).copy())
    starts = np.array([8, 9, 13, 15, 15, 3], np.int32)
    good = np.arange(6, dtype=np.int32)
    out = S.sw_cuda_affine(q, _dev(good), ascii, _dev(starts)).cpu().numpy()
    np.testing.assert_array_equal(out, O.sw_affine(O.encode_query("MKTAYIAKQRQ"), good,
                                                   ascii.cpu().numpy(), starts))
    empty = torch.zeros(0, dtype=torch.uint8, device="cuda")
    assert (S.sw_cuda_blosum62(empty, _dev(good), ascii, _dev(starts)) == -1).all()
    none = S.sw_cuda_affine(q, _dev(np.zeros(0, np.int32)), ascii, _dev(starts))
    assert none.numel() == 0
    with pytest.raises(RuntimeError):
        S.sw_cuda_affine(_dev(np.zeros(2049, np.uint8)), _dev(good), ascii, _dev(starts))


def test_sw_api_matches_oracle():
    import sseqs_b200
    rng = np.random.default_rng(3)
    query = rand_seq(rng, 150)
    targets = homolog_targets(rng, query, 50, lo=3, hi=200)
    got = sseqs_b200.sw(query, targets).cpu().numpy()
    ascii, starts = O.pack_targets(targets)
    exp = O.sw_affine(O.encode_query(query), np.arange(len(targets), dtype=np.int32),
                      ascii, starts, 11, 1)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("Lq", [17, 40, 100, 200, 300, 500, 513, 600, 700, 858, 928, 929])
def test_wide_layout_matches_oracle(Lq):
    """Both lane layouts of a stripe width give the oracle's scores."""
    S = importlib.import_module("sseqs_b200.sw")
    from sseqs_b200 import tune
    query, q, ascii, starts = _case(5000 + Lq, Lq, 400, extra="XB@")
    good = np.arange(len(starts), dtype=np.int32)
    qd, gd, ad, sd = _dev(q), _dev(good), _dev(ascii), _dev(starts)
    tpt = tune.tpt_of(Lq)
    v = _Variants(tpt)
    try:
        for wide in (0, 1):
            v.set(wide)
            np.testing.assert_array_equal(
                S.sw_cuda_blosum62(qd, gd, ad, sd, gap_penalty_param=-1).cpu().numpy(),
                O.sw_linear(q, good, ascii, starts, -1, NT))
            np.testing.assert_array_equal(
                S.sw_cuda_affine(qd, gd, ad, sd, 11, 1).cpu().numpy(),
                O.sw_affine(q, good, ascii, starts, 11, 1, NT))
    finally:
        v.restore()


@pytest.mark.parametrize("Lq", [1, 20, 33, 64, 100, 200, 287, 500, 545, 640, 672, 673, 700, 858,
                                1000, 1300, 1536, 1537, 2048])
@pytest.mark.parametrize("wide", [0, 1])
def test_scan_both_equals_two_scans(Lq, wide):
    """The fused pass gives exactly the linear (skip 0) and affine (skip 1 or
    0) scores of the two separate scans and of the oracle; widths above 48
    words run the two kernels in turn."""
    S = importlib.import_module("sseqs_b200.sw")
    from sseqs_b200 import tune
    tpt = (Lq + 31) // 32
    if wide and not any(tune.has_wide(m, tpt) for m in (0, 1, 2)):
        pytest.skip("no kernel has a wide layout at this width")
    n = 500 if Lq <= 300 else 160
    query, q, ascii, starts = _case(Lq + 3, Lq, n, extra="XBZU*")
    ascii = np.concatenate([ascii, np.full(40, 64, np.uint8)])
    delim = np.flatnonzero(ascii == 64).astype(np.int32)
    nseg = len(delim)
    qd, ad, dd = _dev(q), _dev(ascii), _dev(delim)
    v = _Variants(tpt)
    v.set(wide)
    try:
        lin, aff = S.sw_scan_both(qd, ad, dd, g0=1, n_targets=nseg - 1, affine_skip=1)
        exp_l = S.sw_scan(qd, ad, dd, affine=False, g0=1, n_targets=nseg - 1, skip=0, gap_a=-1)
        exp_a = S.sw_scan(qd, ad, dd, affine=True, g0=1, n_targets=nseg - 1, skip=1, gap_a=11,
                          gap_b=1)
        torch.testing.assert_close(lin, exp_l, rtol=0, atol=0)
        torch.testing.assert_close(aff, exp_a, rtol=0, atol=0)
        good = np.arange(1, nseg, dtype=np.int32)
        np.testing.assert_array_equal(lin.cpu().numpy(),
                                      O.sw_linear(q, good, ascii, delim, -1, NT))
        np.testing.assert_array_equal(aff.cpu().numpy(),
                                      O.sw_affine(q, good, ascii, delim + 1, 11, 1, NT))
        # explicit order with repeats, other gaps, affine windows not shifted
        rng = np.random.default_rng(Lq)
        idx = rng.integers(1, nseg, 300).astype(np.int32)
        gd = _dev(idx)
        lin2, aff2 = S.sw_scan_both(qd, ad, dd, good_idx=gd, affine_skip=0, gap=-2, gap_open=7,
                                    gap_extend=2)
        torch.testing.assert_close(lin2, S.sw_scan(qd, ad, dd, affine=False, good_idx=gd, skip=0,
                                                   gap_a=-2), rtol=0, atol=0)
        torch.testing.assert_close(aff2, S.sw_scan(qd, ad, dd, affine=True, good_idx=gd, skip=0,
                                                   gap_a=7, gap_b=2), rtol=0, atol=0)
        np.testing.assert_array_equal(lin2.cpu().numpy(),
                                      O.sw_linear(q, idx, ascii, delim, -2, NT))
        np.testing.assert_array_equal(aff2.cpu().numpy(),
                                      O.sw_affine(q, idx, ascii, delim, 7, 2, NT))
    finally:
        v.restore()


def test_scan_both_empty_query_fills_minus_one():
    """Query length 0: both outputs -1, as the two scans give (sseqs/sw.cu:73)."""
    S = importlib.import_module("sseqs_b200.sw")
    raw = np.frombuffer(b"MKTAYIAK@@QRQ@W@", np.uint8).copy()
    ascii, dd = _dev(raw), _dev(np.flatnonzero(raw == 64).astype(np.int32))
    q = torch.zeros(0, dtype=torch.uint8, device="cuda")
    lin, aff = S.sw_scan_both(q, ascii, dd, g0=1, n_targets=3, affine_skip=1)
    assert (lin == -1).all() and (aff == -1).all()
    assert (S.sw_scan(q, ascii, dd, affine=False, g0=1, n_targets=3, skip=0, gap_a=-1) == -1).all()


def test_scan_both_degenerate_windows():
    """Empty, one-residue and inverted windows (decreasing delimiters), and
    g = 0, in the fused pass."""
    S = importlib.import_module("sseqs_b200.sw")
    qs = "MKTAYIAKQRQISFVKSHFSRQ"
    q = _dev(O.encode_query(qs))
    ascii = np.frombuffer(b"MKTAYIAK@@QRQ@W@AKQRQISF@", np.uint8).copy()
    delim = np.array([8, 9, 13, 15, 15, 3, 24, 24, 0, 20], np.int32)
    ad, dd = _dev(ascii), _dev(delim)
    idx = _dev(np.arange(len(delim), dtype=np.int32))
    for skip in (0, 1):
        lin, aff = S.sw_scan_both(q, ad, dd, good_idx=idx, affine_skip=skip)
        torch.testing.assert_close(lin, S.sw_scan(q, ad, dd, affine=False, good_idx=idx, skip=0,
                                                  gap_a=-1), rtol=0, atol=0)
        torch.testing.assert_close(aff, S.sw_scan(q, ad, dd, affine=True, good_idx=idx,
                                                  skip=skip, gap_a=11, gap_b=1), rtol=0, atol=0)

"""CPU tests: the oracle against the reference's golden vectors and kernels."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import emulate_ref_kernel, homolog_targets, rand_seq

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_backtrack_matches_reference_triton_golden():
    for rec in _load("triton_backtrack.json"):
        best, al = O.sw_affine_backtrack(rec["query"], rec["targets"], rec["gap_open"],
                                         rec["gap_extend"])
        assert list(best) == rec["best"]
        assert al == rec["aligned"]


def test_a3m_matches_reference_to_a3m_golden():
    for rec in _load("to_a3m.json"):
        _, al = O.sw_affine_backtrack(rec["query"], rec["seqs"])
        assert O.to_a3m_text(rec["query"], al) == rec["a3m"]


@pytest.mark.parametrize("seed", range(6))
def test_sw_oracle_matches_lane_emulation_of_reference_kernel(seed):
    rng = np.random.default_rng(seed)
    Lq = int(rng.choice([1, 5, 31, 32, 33, 47, 64, 70, 96]))
    query = rand_seq(rng, Lq)
    q_idx = O.encode_query(query)
    targets = homolog_targets(rng, query, 6, lo=1, hi=60)
    targets.append(rand_seq(rng, 25, extra="XBZ*"))
    ascii, starts = O.pack_targets(targets)
    good = np.arange(1, len(targets), dtype=np.int32)
    lin = O.sw_linear(q_idx, good, ascii, starts, gap=-1)
    aff = O.sw_affine(q_idx, good, ascii, starts, 11, 1)
    aff2 = O.sw_affine(q_idx, good, ascii, starts, 5, 2)
    for t, g in enumerate(good):
        lo, hi = starts[g - 1] + 1, starts[g]
        tb = ascii[lo:hi].tolist()
        assert lin[t] == emulate_ref_kernel(q_idx, tb, False, -1)
        assert aff[t] == emulate_ref_kernel(q_idx, tb, True, 11, 1)
        assert aff2[t] == emulate_ref_kernel(q_idx, tb, True, 5, 2)


def test_sw_oracle_window_edge_cases():
    q = O.encode_query("MKTAYIAKQRQISFVKSHFSRQ")
    ascii = np.frombuffer(b"MKTAYIAK@@QRQ@W@", dtype=np.uint8).copy()
    # windows: g=0 exact first target; starts equal -> length -1 -> 0;
    # inverted -> -1; zero length -> -1
    starts = np.array([8, 9, 13, 15, 15, 3], dtype=np.int32)
    good = np.array([0, 1, 2, 3, 4, 5], dtype=np.int32)
    out = O.sw_affine(q, good, ascii, starts, 11, 1)
    assert out[1] == -1          # starts[1]-starts[0]-1 == 0
    assert out[4] == 0           # length -1: loop runs no row
    assert out[5] == -1          # stop < start
    assert out[0] == emulate_ref_kernel(q, ascii[0:8].tolist(), True)
    assert out[2] > 0
    empty_q = O.sw_linear(np.zeros(0, np.uint8), good, ascii, starts)
    assert (empty_q == -1).all()


def test_xbit_roundtrip_and_layout():
    rng = np.random.default_rng(1)
    for n in [1, 7, 8, 9, 40, 1001]:
        sym = rng.integers(64, 96, n).astype(np.uint8)
        packed = O.xbit_compress(sym)
        assert packed.size == (5 * n + 7) // 8
        assert (O.xbit_decompress(packed, n, 0) == sym).all()
    # layout: first symbol in the high bits of the 40-bit big-endian window
    sym = np.array([64 + 1, 64, 64, 64, 64, 64, 64, 64 + 31], np.uint8)
    p = O.xbit_compress(sym)
    w = int.from_bytes(bytes(p[:5]), "big")
    assert (w >> 35) & 31 == 1 and w & 31 == 31


def test_segmentation_matches_reference_reading():
    ascii = np.frombuffer(b"AAA@BB@@C@DDDD@@@", dtype=np.uint8).copy()
    seg = O.segment(ascii)
    assert list(seg["delim_pos"]) == [3, 6, 7, 9, 14, 15, 16]
    assert list(seg["lengths"]) == [3, 2, 1, 4]
    assert list(seg["offsets"]) == [0, 4, 7, 9]
    # no trailing delimiter: the fragment after the last '@' is a segment
    seg2 = O.segment(np.frombuffer(b"AB@CDE", dtype=np.uint8).copy())
    assert list(seg2["lengths"]) == [2, 3]


def test_topk_canonical_tie_break():
    v = np.array([5, 7, 7, 1, 7, 5])
    assert list(O.topk_canonical(v, 2)) == [1, 2]
    assert list(O.topk_canonical(v, 4)) == [1, 2, 4, 0]

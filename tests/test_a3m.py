"""The vectorised a3m writer (``a3m_text_raw``) gives exactly the text of
the string-by-string writer (``a3m_text``, sseqs/to_a3m.py:16-72) on the
same traceback results; runs on the CPU with host-built results."""
import numpy as np
import pytest
import torch

from sseqs_b200.sw import Alignments
from sseqs_b200.to_a3m import a3m_text, a3m_text_raw

AA = b"ARNDCQEGHILKMFPSTWYV"


def _results(rng, query: bytes, n_batches=3, per=40, extra=b"", dup=True):
    out = []
    for _ in range(n_batches):
        cap = len(query) + 300
        best = np.zeros(per, np.int32)
        info = np.zeros((per, 5), np.int32)
        q_al = np.zeros((per, cap), np.uint8)
        t_al = np.zeros((per, cap), np.uint8)
        prev = None
        for b in range(per):
            kind = rng.integers(0, 10)
            if kind == 0:                      # no alignment
                continue
            s = int(rng.integers(0, len(query) - 5))
            e = int(rng.integers(s + 1, min(len(query), s + 120) + 1))
            qs, ts = [], []
            for c in query[s:e]:
                r = rng.random()
                if r < 0.08:
                    qs.append(45)
                    ts.append(int(rng.choice(list(AA + extra))))
                if r > 0.92:
                    qs.append(c)
                    ts.append(45)
                    continue
                qs.append(c)
                ts.append(int(rng.choice(list(AA + b"xz" + extra))))
            if dup and prev is not None and kind == 1:
                qs, ts = prev                  # duplicate row
            prev = (qs, ts)
            n = len(qs)
            q_al[b, cap - n:] = qs
            t_al[b, cap - n:] = ts
            info[b, 0] = n
            best[b] = 0 if kind == 2 else int(rng.integers(1, 60))   # ties and zeros
        out.append(Alignments(torch.from_numpy(best), torch.from_numpy(info),
                              torch.from_numpy(q_al), torch.from_numpy(t_al), cap, None))
    return out


def _dicts(res):
    return [d for r in res for d in r.to_dicts()]


@pytest.mark.parametrize("seed", range(6))
def test_raw_writer_equals_string_writer(seed):
    rng = np.random.default_rng(seed)
    query = bytes(rng.choice(list(AA), 200).astype(np.uint8))
    query = query[:60] + query[20:50] + query[60:]      # repeats: find() picks the first
    res = _results(rng, query, extra=b"@*" if seed % 2 else b"")
    q = query.decode("ascii")
    assert a3m_text_raw(q, res) == a3m_text(q, _dicts(res))


def test_raw_writer_non_ascii_bytes_take_the_string_path():
    rng = np.random.default_rng(7)
    query = bytes(rng.choice(list(AA), 150).astype(np.uint8))
    res = _results(rng, query, extra=bytes([0xe9, 0xff, 0xb5]))
    q = query.decode("ascii")
    assert a3m_text_raw(q, res) == a3m_text(q, _dicts(res))


def test_raw_writer_empty_and_missing_fragment():
    q = "MKTAYIAKQR"
    assert a3m_text_raw(q, []) == a3m_text(q, [])
    cap = 20
    q_al = np.zeros((1, cap), np.uint8)
    t_al = np.zeros((1, cap), np.uint8)
    q_al[0, -3:] = list(b"WWW")
    t_al[0, -3:] = list(b"AAA")
    res = [Alignments(torch.tensor([5], dtype=torch.int32),
                      torch.tensor([[3, 0, 0, 0, 0]], dtype=torch.int32),
                      torch.from_numpy(q_al), torch.from_numpy(t_al), cap, None)]
    with pytest.raises(ValueError):
        a3m_text_raw(q, res)
    with pytest.raises(ValueError):
        a3m_text(q, _dicts(res))


def test_sequence_helpers_keep_the_reference_layout():
    """encode_seq / pack_targets (sseqs/sw.py:262-276): int16 character codes
    behind a leading 0; rows padded with zeros to the longest target + 1,
    lengths = sequence + 1."""
    import importlib
    S = importlib.import_module("sseqs_b200.sw")
    v = S.encode_seq("AC", device="cpu")
    assert v.dtype == torch.int16 and v.tolist() == [0, 65, 67]
    T, lens, W = S.pack_targets(["AC", "WYV", ""], device="cpu")
    assert W == 4 and T.dtype == torch.int16 and lens.dtype == torch.int32
    assert T.tolist() == [[0, 65, 67, 0], [0, 87, 89, 86], [0, 0, 0, 0]]
    assert lens.tolist() == [3, 4, 1]

"""FASTA -> .xbit packer and its sidecar segment index (CPU): the file is
byte-identical to ``write_xbit`` of the normalised sequences, decodes (oracle
decoder, sseqs/xbit.cu:8-34) to the sequences at the positions the index
records, and the index maps positions back to sequences."""
import numpy as np
import pytest

from oracle import oracle as O
from sseqs_b200 import dbtools

FASTA = """junk before the first header
>seq1 first record
MKTAYIAKQR
QISFVKSHFS
>seq2 lower case and odd characters
mktay*iak-qr12 x
>empty

>seq4
ACDEFGHIKLMNPQRSTVWY
ACDEFGHIKLMNPQRSTVWY
ACDEFGHIKLMNPQRSTVWY
>seq5
BZUOJ
"""


def _write(tmp_path, text, extra=0, seed=0):
    rng = np.random.default_rng(seed)
    text += "".join(f">r{i}\n{dbtools.random_query(int(rng.integers(1, 120)), i)}\n"
                    for i in range(extra))
    p = tmp_path / "in.fasta"
    p.write_text(text)
    return str(p)


def test_read_fasta_and_normalise(tmp_path):
    recs = list(dbtools.read_fasta(_write(tmp_path, FASTA)))
    assert [r[0] for r in recs] == ["seq1 first record", "seq2 lower case and odd characters",
                                    "empty", "seq4", "seq5"]
    assert recs[0][1] == "MKTAYIAKQRQISFVKSHFS"
    assert dbtools.normalise_residues(recs[1][1]) == b"MKTAYXIAKXQRXXX"
    assert recs[2][1] == ""
    assert dbtools.normalise_residues(recs[4][1]) == b"BZUOJ"


@pytest.mark.parametrize("chunk_bytes", [100, 200, 1000])
def test_fasta_to_xbit_layout_and_index(tmp_path, chunk_bytes):
    fa = _write(tmp_path, FASTA, extra=40, seed=chunk_bytes)
    xb = str(tmp_path / "db.xbit")
    idx = dbtools.fasta_to_xbit(fa, xb, chunk_bytes=chunk_bytes)
    seqs = [dbtools.normalise_residues(s) for _, s in dbtools.read_fasta(fa)]
    ref = str(tmp_path / "ref.xbit")
    n_ref = dbtools.write_xbit(ref, [s.decode() for s in seqs], chunk_bytes=chunk_bytes)
    data = open(xb, "rb").read()
    assert data == open(ref, "rb").read()
    assert idx.n_chunks == n_ref and len(data) == n_ref * chunk_bytes
    cap = chunk_bytes * 8 // 5
    chunks = [O.xbit_decompress(np.frombuffer(data[c * chunk_bytes:(c + 1) * chunk_bytes],
                                              np.uint8), cap) for c in range(n_ref)]
    for k, s in enumerate(seqs):
        a = chunks[idx.chunk_of[k]]
        st, ln = int(idx.start[k]), int(idx.length[k])
        assert ln == len(s) and a[st:st + ln].tobytes() == s and a[st + ln] == 64
        assert idx.locate(int(idx.chunk_of[k]), st) == k
        assert idx.locate(int(idx.chunk_of[k]), st + ln) == k          # its '@'
        if ln > 1:
            assert idx.locate(int(idx.chunk_of[k]), st + ln // 2) == k
    last = len(seqs) - 1
    end = int(idx.start[last] + idx.length[last]) + 1
    if end < cap:
        assert idx.locate(int(idx.chunk_of[last]), end) == -1           # chunk padding
    back = dbtools.SeqIndex.load(dbtools.index_path(xb))
    assert back.names == idx.names and back.chunk_bytes == chunk_bytes
    assert np.array_equal(back.start, idx.start) and np.array_equal(back.chunk_of, idx.chunk_of)


def test_fasta_to_xbit_rejects_a_sequence_longer_than_a_chunk(tmp_path):
    fa = _write(tmp_path, ">long\n" + "A" * 200 + "\n")
    with pytest.raises(ValueError):
        dbtools.fasta_to_xbit(fa, str(tmp_path / "x.xbit"), chunk_bytes=100)


def test_empty_fasta_writes_no_chunk(tmp_path):
    fa = _write(tmp_path, "")
    idx = dbtools.fasta_to_xbit(fa, str(tmp_path / "e.xbit"), chunk_bytes=100)
    assert idx.n_chunks == 0 and (tmp_path / "e.xbit").stat().st_size == 0

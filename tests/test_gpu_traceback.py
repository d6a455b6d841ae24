"""GPU parity of the CUDA traceback and the a3m writer against the
reference's Triton kernels (golden vectors) and the CPU oracle."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import homolog_targets, rand_seq

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_backtrack_matches_triton_golden():
    from sseqs_b200.sw import sw_affine_backtrack
    for rec in _load("triton_backtrack.json"):
        M, best, al = sw_affine_backtrack(rec["query"], rec["targets"], rec["gap_open"],
                                          rec["gap_extend"])
        assert best.cpu().tolist() == rec["best"]
        assert al == rec["aligned"]
        assert M.shape == (len(rec["targets"]), len(rec["query"]) + 1,
                           max(map(len, rec["targets"])) + 1)


def test_backtrack_matrix_matches_definition():
    """M_full holds M(i,j) = s + H(i-1,j-1) on the valid cells, 0 elsewhere."""
    from sseqs_b200.sw import sw_affine_backtrack
    q, ts = "HEAGAWGHEE", ["PAWHEAE", "AW"]
    M, best, al = sw_affine_backtrack(q, ts)
    M = M.cpu().numpy()
    assert M[0, 0].sum() == 0 and M[:, :, 0].sum() == 0
    assert M[1, 1:, len(ts[1]) + 1:].sum() == 0
    B62 = O.BLOSUM62
    i, j = q.index("W") + 1, ts[0].index("W") + 1
    assert M[0, i, j] >= B62[17, 17]


@pytest.mark.parametrize("seed", range(4))
def test_backtrack_matches_oracle_random(seed):
    from sseqs_b200.sw import backtrack
    rng = np.random.default_rng(seed)
    Lq = int(rng.choice([5, 31, 33, 64, 150, 400]))
    query = rand_seq(rng, Lq)
    targets = homolog_targets(rng, query, 60, lo=1, hi=500)
    targets += ["", "X", rand_seq(rng, 40, extra="XBZ*")]
    got = backtrack(query, targets).to_dicts()
    best, exp = O.sw_affine_backtrack(query, targets)
    assert got == exp


@pytest.mark.parametrize("Lq", [1000, 1500, 2048])
def test_backtrack_matches_oracle_long_queries(Lq):
    """Queries up to the longest the search takes (2048) against hit-length
    targets (the search keeps 500 residues of a hit, sseqs/msa.py:183):
    planted homologs of query pieces, random targets, and non-standard
    letters."""
    from sseqs_b200.sw import backtrack
    rng = np.random.default_rng(Lq)
    query = rand_seq(rng, Lq)
    targets = []
    for i in range(24):
        a = int(rng.integers(0, Lq - 400))
        piece = query[a:a + int(rng.integers(200, 400))]
        targets.append(homolog_targets(rng, piece, 1, lo=150, hi=500, frac=1.0)[0][:500])
    targets += [rand_seq(rng, 500), rand_seq(rng, 499, extra="XBZ*"), query[-500:], query[:500]]
    got = backtrack(query, targets).to_dicts()
    best, exp = O.sw_affine_backtrack(query, targets)
    assert got == exp
    assert max(best) > 300


def test_to_a3m_matches_reference_golden(tmp_path):
    from sseqs_b200.to_a3m import to_a3m
    for k, rec in enumerate(_load("to_a3m.json")):
        path = tmp_path / f"{k}.a3m"
        to_a3m(rec["query"], rec["seqs"], str(path))
        assert path.read_text() == rec["a3m"]


def test_to_a3m_matches_oracle_large(tmp_path):
    from sseqs_b200.to_a3m import to_a3m
    rng = np.random.default_rng(11)
    query = rand_seq(rng, 300)
    seqs = homolog_targets(rng, query, 1500, lo=20, hi=500, frac=0.7)
    text = to_a3m(query, seqs, str(tmp_path / "x.a3m"))
    _, al = O.sw_affine_backtrack(query, seqs)
    assert text == O.to_a3m_text(query, al)

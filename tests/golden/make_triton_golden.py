"""Generate golden vectors from the reference's own traceback and a3m writer.

Runs in the build container only (it reads the reference sources), on the CPU:
the reference's Triton DP/traceback kernels (sseqs/sw.py:27-219, :408-768)
execute under ``TRITON_INTERPRET=1`` with ``device="cpu"``, and its
``to_a3m`` (sseqs/to_a3m.py:5-72) runs unmodified on top of them.  The only
change to the reference source is that the module-level JIT build of the
CUDA extension (sseqs/sw.py:9) is skipped, since nothing here calls it.

Usage:  python tests/golden/make_triton_golden.py REF_DIR
        (or SSEQS_REF=REF_DIR python tests/golden/make_triton_golden.py)
REF_DIR is the reference's sseqs/ source directory.
Writes: tests/golden/triton_backtrack.json, tests/golden/to_a3m.json
"""
import functools
import json
import os
import sys

os.environ["TRITON_INTERPRET"] = "1"

import numpy as np  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SSEQS_REF", "")
OUT = os.path.dirname(os.path.abspath(__file__))
AA = "ARNDCQEGHILKMFPSTWYV"


def load_reference():
    src = open(os.path.join(REF, "sw.py")).read()
    stub = "sseqs_sw_ext = load("
    assert stub in src
    src = src.replace(stub, "sseqs_sw_ext = None and load(")
    ns = {"__name__": "ref_sw", "__file__": os.path.join(REF, "sw.py")}
    exec(compile(src, os.path.join(REF, "sw.py"), "exec"), ns)
    bt = functools.partial(ns["sw_affine_backtrack"], device="cpu")
    a3m_src = open(os.path.join(REF, "to_a3m.py")).read()
    a3m_src = a3m_src.replace("from sseqs.sw import sw_affine_backtrack", "")
    ns2 = {"__name__": "ref_a3m", "sw_affine_backtrack": bt}
    exec(compile(a3m_src, os.path.join(REF, "to_a3m.py"), "exec"), ns2)
    return bt, ns2["to_a3m"]


def mutate(rng, s, ident, indel=0.05):
    out = []
    for c in s:
        r = rng.random()
        if r < indel / 2:
            continue                                   # deletion
        if r < indel:
            out.append(AA[rng.integers(20)])           # insertion
        out.append(c if rng.random() < ident else AA[rng.integers(20)])
    return "".join(out)


def rand_seq(rng, n):
    return "".join(AA[i] for i in rng.integers(0, 20, n))


def cases(rng):
    out = []
    # planted homologs of assorted identities and lengths
    for b in range(4):
        q = rand_seq(rng, int(rng.integers(12, 48)))
        ts = []
        for _ in range(10):
            kind = rng.random()
            if kind < 0.6:
                core = q[int(rng.integers(0, len(q) // 3)):]
                t = rand_seq(rng, int(rng.integers(0, 8))) + mutate(rng, core, rng.uniform(0.3, 0.95)) \
                    + rand_seq(rng, int(rng.integers(0, 8)))
            else:
                t = rand_seq(rng, int(rng.integers(1, 50)))
            ts.append(t)
        out.append((q, ts, 11, 1))
    # non-standard letters in query and targets, lower case, tiny targets
    q = "MKTAYIAKQRQISFVKSHFSRQX" + "LEDRW"
    ts = ["MKTAYIAKQRQISFVKSHF", "MKTAXIAKBRQZSFVKSHFSRQ", "mktayiakqrq",
          "A", "W", "KTAYIAK@QRQISF", "QQQQQQQQQQ", "MKTAYIAKQRQISFVKSHFSRQXLEDRW"]
    out.append((q, ts, 11, 1))
    # other gap parameters
    q = rand_seq(rng, 30)
    ts = [mutate(rng, q, 0.6, 0.1) for _ in range(6)]
    out.append((q, ts, 5, 2))
    out.append((q, ts, 1, 1))
    return out


def main():
    if not os.path.isfile(os.path.join(REF, "sw.py")):
        sys.exit("give the reference's sseqs/ directory (argument or SSEQS_REF)")
    bt, to_a3m = load_reference()
    rng = np.random.default_rng(20240601)
    records = []
    for q, ts, go, ge in cases(rng):
        M, best, aligned = bt(q, ts, gap_open=go, gap_extend=ge)
        records.append({"query": q, "targets": ts, "gap_open": go,
                        "gap_extend": ge, "best": [int(x) for x in best],
                        "aligned": aligned})
    with open(os.path.join(OUT, "triton_backtrack.json"), "w") as f:
        json.dump(records, f, indent=0)

    # to_a3m on hit lists, including a duplicate row and a weak hit.
    a3m = []
    for r in range(3):
        q = rand_seq(rng, int(rng.integers(25, 45)))
        seqs = []
        for _ in range(12):
            core = q[int(rng.integers(0, 8)):int(rng.integers(len(q) - 8, len(q)))]
            seqs.append(rand_seq(rng, int(rng.integers(0, 5))) + mutate(rng, core, rng.uniform(0.4, 1.0))
                        + rand_seq(rng, int(rng.integers(0, 5))))
        seqs.append(seqs[0])                      # duplicate row -> deduped
        seqs.append(rand_seq(rng, 6))             # weak hit
        path = os.path.join(OUT, f"_tmp_{r}.a3m")
        to_a3m(q, seqs, path)
        text = open(path).read()
        os.remove(path)
        a3m.append({"query": q, "seqs": seqs, "a3m": text})
    with open(os.path.join(OUT, "to_a3m.json"), "w") as f:
        json.dump(a3m, f, indent=0)
    print("wrote", len(records), "backtrack cases and", len(a3m), "a3m cases")


if __name__ == "__main__":
    main()

"""Generate end-to-end golden outputs by running the reference's own ``msa()``.

Runs in the build container only (it reads the reference sources), on the
CPU, one case of ``msa_cases.py`` per subprocess.  The reference's Python --
``sseqs/msa.py`` (module body and ``msa()``), ``sseqs/to_a3m.py`` and
``sseqs/sw.py`` -- executes unmodified; what cannot run without a GPU is
replaced underneath it:

* the ``torch.utils.cpp_extension.load`` calls of sseqs/msa.py:33-35 and
  sseqs/sw.py:9 return stand-ins for the three CUDA extensions, each the CPU
  oracle's restatement of the reference kernel (``oracle/oracle.py``):
  ``xbit.decompress`` (sseqs/xbit.cu:8-34), ``sw.sw_cuda_blosum62`` and
  ``sw.sw_cuda_affine`` (sseqs/sw.cu:55-325; these two are checked bit for
  bit against the reference kernels compiled from source, on the GPU, by
  ``tests/test_gpu_sw.py``) and ``conv.warp_corr`` (sseqs/fft.cu:17-415,
  restated in float64 and rounded to fp16 as the reference stores it;
  not bit-exact with the fp16 FFT, so the prefiltered case is compared by
  agreement only);
* ``sw_affine_backtrack`` (the Triton DP and traceback, sseqs/sw.py:27-219)
  is the oracle's C restatement, which reproduces the reference's own
  Triton outputs (``triton_backtrack.json``); the Triton interpreter takes
  about half a minute per target on this CPU;
* tensors the reference puts on 'cuda' are made on the CPU (a torch function
  mode), pinned memory is plain memory, and ``torch.cuda`` streams,
  ``device`` contexts and ``synchronize`` do nothing;
* ``torch.topk`` breaks ties by position (equal values: lower index first),
  one instance of the order torch leaves unspecified, so that the per-batch
  cuts (sseqs/msa.py:297, 324, 335) are reproducible: parity is defined on
  this order.

The database file is the case's 1e9-byte chunk; the reference reads it with
``CHUNKS=1`` and searches it with the default ``bs`` (5e7, 20 batches).

Usage:  SSEQS_REF=<reference sseqs/ directory> python tests/golden/make_msa_golden.py [case ...]
Writes: tests/golden/msa_<case>.json.gz
"""
import contextlib
import gzip
import json
import os
import pickle
import subprocess
import sys
import tempfile
import time
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _ref_dir():
    ref = os.environ.get("SSEQS_REF")
    if not ref or not os.path.isfile(os.path.join(ref, "msa.py")):
        sys.exit("set SSEQS_REF to the reference's sseqs/ source directory")
    return ref


def _stand_ins():
    import numpy as np
    import torch

    from oracle import oracle as O

    def decompress(b, n, lo):
        return torch.from_numpy(O.xbit_decompress(b.numpy(), int(n), int(lo)))

    def warp_corr(corr, qrev, A, B, flat, offsets, lengths, k, La, maxlen, n, rfft):
        codes = qrev.numpy().astype(np.int64)
        s = O.prefilter_scores_codes(codes, A.numpy(), B.numpy(), flat.numpy(),
                                     offsets.numpy(), lengths.numpy(), int(n), int(k))
        corr.copy_(torch.from_numpy(s.astype(np.float16)))
        return torch.empty((lengths.numel(), 2), dtype=torch.float32)

    nt = os.cpu_count()

    def sw_linear(q, good_idx, ascii, starts, gap_penalty_param=-10):
        return torch.from_numpy(O.sw_linear(q.numpy(), good_idx.numpy(), ascii.numpy(),
                                            starts.numpy(), int(gap_penalty_param), nt))

    def sw_affine(q, good_idx, ascii, starts, gap_open=11, gap_extend=1):
        return torch.from_numpy(O.sw_affine(q.numpy(), good_idx.numpy(), ascii.numpy(),
                                            starts.numpy(), int(gap_open), int(gap_extend), nt))

    mods = {"xbit": types.SimpleNamespace(decompress=decompress),
            "conv": types.SimpleNamespace(warp_corr=warp_corr),
            "sw": types.SimpleNamespace(sw_cuda_blosum62=sw_linear, sw_cuda_affine=sw_affine)}
    mods["sseqs_sw_ext"] = mods["sw"]

    def load(name, sources=None, **kw):
        return mods[name]

    def backtrack(query, targets, gap_open=11, gap_extend=1, device="cuda", scores=False):
        best, aligned = O.sw_affine_backtrack(query, [str(t) for t in targets], gap_open,
                                              gap_extend)
        best = torch.from_numpy(best)
        return best if scores else (None, best, aligned)

    return load, backtrack


def _stable_topk(input, k, dim=-1, largest=True, sorted=True):
    """torch.topk with ties to the lower index (1-D inputs, as msa() has)."""
    import torch
    assert input.dim() == 1 and largest
    order = torch.sort(input, descending=True, stable=True).indices[:k]
    return torch.return_types.topk((input[order], order))


def _cpu_mode():
    """Torch function mode: 'cuda' tensors on the CPU, no pinning, ties of
    torch.topk to the lower index."""
    import torch
    from torch.overrides import TorchFunctionMode

    class Mode(TorchFunctionMode):
        def __torch_function__(self, func, types_, args=(), kwargs=None):
            kwargs = dict(kwargs or {})
            dev = kwargs.get("device")
            if dev is not None and "cuda" in str(dev):
                kwargs["device"] = "cpu"
            if kwargs.get("pin_memory"):
                kwargs["pin_memory"] = False
            name = getattr(func, "__name__", "")
            if func is torch.topk:
                return _stable_topk(*args, **kwargs)
            if name == "cuda":
                return args[0]
            if name == "is_pinned":
                return True
            return func(*args, **kwargs)
    return Mode()


def _patch_torch_cuda():
    import torch

    class _Stream:
        def __init__(self, *a, **k):
            pass

    torch.cuda.device = lambda *a, **k: contextlib.nullcontext()
    torch.cuda.Stream = _Stream
    torch.cuda.stream = lambda *a, **k: contextlib.nullcontext()
    torch.cuda.synchronize = lambda *a, **k: None
    torch.cuda.empty_cache = lambda *a, **k: None


def _exec_module(name, path):
    mod = types.ModuleType(name)
    mod.__file__ = path
    sys.modules[name] = mod
    exec(compile(open(path).read(), path, "exec"), mod.__dict__)
    return mod


def run_case(name):
    """Child process: write the case database, run the reference msa()."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    import numpy as np
    import torch.utils.cpp_extension as cpp

    import msa_cases as C

    ref = _ref_dir()
    case = C.CASES[name]
    query, chunk, sha = C.case_chunk(name)
    tmp = tempfile.mkdtemp(prefix="msa_golden_")
    db_path = os.path.join(tmp, "db.xbit")
    chunk.tofile(db_path)
    del chunk
    os.environ["CHUNKS"] = "1"
    os.environ["DBPATH"] = db_path

    load, backtrack = _stand_ins()
    cpp.load = load
    _patch_torch_cuda()
    pkg = types.ModuleType("sseqs")
    pkg.__path__ = [ref]
    sys.modules["sseqs"] = pkg
    with _cpu_mode():
        sw_mod = _exec_module("sseqs.sw", os.path.join(ref, "sw.py"))
        sw_mod.sw_affine_backtrack = backtrack
        _exec_module("sseqs.to_a3m", os.path.join(ref, "to_a3m.py"))
        msa_mod = _exec_module("sseqs.msa", os.path.join(ref, "msa.py"))
        a3m_path = os.path.join(tmp, "out.a3m")
        raw_path = os.path.join(tmp, "raw.pkl")
        p = case["params"]
        t0 = time.time()
        msa_mod.msa(query, a3m_path, num_msas=p["num_msas"], save_raw=raw_path, verbose=False,
                    bs=C.BS, top_fft=p["top_fft"], top_sw=p["top_sw"],
                    top_sw_affine=p["top_sw_affine"])
        dt = time.time() - t0
    with open(raw_path, "rb") as fh:
        q, matches, lin, fft, norm = pickle.load(fh)
    assert q == query
    hits = [[str(s), int(a), float(np.float32(g))] for s, a, g in zip(matches, lin, norm)]
    out = {"case": name, "query": query, "db_sha256": sha, "params": p, "bs": C.BS,
           "hits": hits, "a3m": open(a3m_path).read(),
           "generated_by": "reference sseqs/msa.py msa() on the CPU, kernels replaced by the "
                           "oracle's restatements (make_msa_golden.py)",
           "reference_seconds": round(dt, 1)}
    with gzip.open(os.path.join(HERE, f"msa_{name}.json.gz"), "wt") as f:
        json.dump(out, f)
    for fn in (db_path, a3m_path, raw_path):
        os.remove(fn)
    os.rmdir(tmp)
    print(f"{name}: {len(hits)} hits, {out['a3m'].count(chr(10)) // 2 - 1} a3m rows, "
          f"{dt:.0f} s, db {sha[:12]}")


def main():
    _ref_dir()
    if len(sys.argv) > 2 and sys.argv[1] == "--child":
        run_case(sys.argv[2])
        return
    sys.path.insert(0, HERE)
    import msa_cases as C
    names = sys.argv[1:] or list(C.CASES)
    for n in names:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--child", n], check=True,
                       cwd=ROOT)


if __name__ == "__main__":
    main()

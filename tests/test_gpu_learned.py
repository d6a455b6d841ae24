"""GPU tests of the learned prefilter's kernels against plain PyTorch fp32
references of the same operations (tolerances stated per test), and of the
search's contract: every reported score is the exact SW score."""
import importlib
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bf(x):
    return x.to(torch.bfloat16)


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (300, 200, 160), (1000, 256, 1280),
                                   (77, 32, 64)])
@pytest.mark.parametrize("epi", [0, 1, 2, 3])
def test_gemm_nt_matches_fp32(M, N, K, epi):
    from sseqs_b200 import learned
    g = torch.Generator(device="cpu")
    g.manual_seed(M + N + K + epi)
    A = _bf(torch.randn(M, K, generator=g)).cuda()
    B = _bf(torch.randn(N, K, generator=g)).cuda()
    bias = torch.randn(N, generator=g).cuda()
    aux = _bf(torch.randn(M, N, generator=g)).cuda()
    mask = (torch.rand(M, generator=g) > 0.2).to(torch.uint8).cuda()
    ref = A.float() @ B.float().T
    C = torch.zeros((M, N), dtype=torch.float32 if epi == 0 else torch.bfloat16, device="cuda")
    C2 = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
    learned._gemm(0, 0, epi, M, N, K, A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), N,
                  C2.data_ptr(), bias, aux.data_ptr(), mask if epi else None)
    m = mask.bool()[:, None]
    if epi == 0:
        exp = ref
    elif epi == 1:
        exp = torch.where(m, ref, 0)
    elif epi == 2:
        z = _bf(ref + bias).float()
        assert torch.allclose(C2.float(), torch.where(m, z, 0), rtol=1e-2, atol=1e-2)
        exp = torch.where(m, torch.nn.functional.gelu(z, approximate="tanh"), 0)
    else:
        zf = aux.float()
        t = torch.tanh(0.7978845608 * (zf + 0.044715 * zf ** 3))
        gp = 0.5 * (1 + t) + 0.5 * zf * (1 - t * t) * 0.7978845608 * (1 + 0.134145 * zf * zf)
        exp = torch.where(m, ref * gp, 0)
    # fp32 accumulation of exact bf16 products; bf16 output rounding
    tol = 1e-3 if epi == 0 else 1e-2
    err = (C.float() - exp).abs().max().item()
    assert err <= tol * max(1.0, exp.abs().max().item()), err


def _gemm_error():
    import ctypes
    from sseqs_b200 import _lib
    v = ctypes.c_int(-1)
    _lib.check(_lib.lib().sseqs_gemm_error(ctypes.byref(v)), "gemm_error")
    return v.value


@pytest.mark.parametrize("M", [1, 131, 5000])
@pytest.mark.parametrize("epi", [1, 2, 3, 5, 6])
@pytest.mark.parametrize("K", [64, 1280])
def test_tcgen05_gemm_matches_mma_sync_and_fp32(M, epi, K):
    """N = 256 GEMMs take the tcgen05 kernel; the same call on the mma.sync
    kernel and an fp32 reference must agree (fp32 accumulation of exact
    bf16 products in both; outputs rounded to bf16)."""
    from sseqs_b200 import _lib, learned
    g = torch.Generator(device="cpu")
    g.manual_seed(M * 7 + epi * 3 + K)
    N = 256
    A = _bf(torch.randn(M, K, generator=g)).cuda()
    B = _bf(torch.randn(N, K, generator=g)).cuda()
    bias = torch.randn(N, generator=g).cuda()
    aux = _bf(torch.randn(M, N, generator=g)).cuda()
    res = _bf(torch.randn(M, N, generator=g)).cuda()
    mask = (torch.rand(M, generator=g) > 0.2).to(torch.uint8).cuda()
    outs = []
    for path in (1, 0):
        _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(path), "path")
        C = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
        C2 = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
        learned._gemm(0, 0, epi, M, N, K, A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), N,
                      C2.data_ptr(), bias, aux.data_ptr(), mask, res.data_ptr())
        torch.cuda.synchronize()
        outs.append((C.float(), C2.float()))
    _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(1), "path")
    assert _gemm_error() == 0
    ref = A.float() @ B.float().T
    m = mask.bool()[:, None]
    if epi == 1:
        exp = torch.where(m, ref, 0)
    elif epi in (2, 5):
        z = _bf(ref + bias).float()
        exp = torch.where(m, torch.nn.functional.gelu(z, approximate="tanh") +
                          (res.float() if epi == 5 else 0), 0)
    else:
        gg = _bf(ref + res.float()).float() if epi == 6 else ref
        zf = aux.float()
        t = torch.tanh(0.7978845608 * (zf + 0.044715 * zf ** 3))
        gp = 0.5 * (1 + t) + 0.5 * zf * (1 - t * t) * 0.7978845608 * (1 + 0.134145 * zf * zf)
        exp = torch.where(m, gg * gp, 0)
    scale = max(1.0, exp.abs().max().item())
    for C, C2 in outs:
        assert (C - exp).abs().max().item() <= 2e-2 * scale
    # the two kernels agree up to the bf16 rounding of their outputs
    assert (outs[0][0] - outs[1][0]).abs().max().item() <= 2e-2 * scale


@pytest.mark.parametrize("M", [5, 128, 1000, 40000])
def test_tcgen05_gemm_overlapping_rows(M):
    """The conv form: row m of A starts lda = 256 elements after row m - 1
    and spans K = 5 * 256 (im2col without a buffer); the TMA-fed tcgen05
    kernel loads each K tile as a box of the lda-wide rows.  Same result as
    the mma.sync kernel and an fp32 reference."""
    from sseqs_b200 import _lib, learned
    g = torch.Generator(device="cpu")
    g.manual_seed(M)
    C_, K, N = 256, 1280, 256
    X = _bf(torch.randn(M + 4, C_, generator=g)).cuda()
    B = _bf(torch.randn(N, K, generator=g)).cuda()
    outs = []
    for path in (1, 0):
        _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(path), "path")
        C = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
        learned._gemm(0, 0, 1, M, N, K, X.data_ptr(), C_, B.data_ptr(), K, C.data_ptr(), N,
                      0, None, 0, None, 0)
        torch.cuda.synchronize()
        outs.append(C.float())
    _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(1), "path")
    assert _gemm_error() == 0
    A = X.float().unfold(0, 5, 1).permute(0, 2, 1).reshape(M, K)    # row m = X[m .. m+4]
    ref = A @ B.float().T
    scale = max(1.0, ref.abs().max().item())
    for C in outs:
        assert (C - ref).abs().max().item() <= 2e-2 * scale
    assert (outs[0] - outs[1]).abs().max().item() <= 2e-2 * scale


@pytest.mark.parametrize("M,N,K", [(160, 256, 96), (1280, 256, 4096), (40, 24, 32)])
def test_gemm_tn_matches_fp32(M, N, K):
    from sseqs_b200 import learned
    g = torch.Generator(device="cpu")
    g.manual_seed(M * N + K)
    A = _bf(torch.randn(K, M, generator=g)).cuda()      # stored [K][M]
    B = _bf(torch.randn(K, N, generator=g)).cuda()      # stored [K][N]
    C = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    learned._gemm(1, 1, 0, M, N, K, A.data_ptr(), M, B.data_ptr(), N, C.data_ptr(), N)
    ref = A.float().T @ B.float()
    assert (C - ref).abs().max().item() <= 1e-3 * ref.abs().max().item()


def _ref_embed(model, seqs):
    """fp32 reference: per sequence conv1d (padding 2) + GELU(tanh), mean,
    L2 normalise, with the model's bf16-rounded parameters."""
    from sseqs_b200 import sw as _unused  # noqa: F401
    AA = "ARNDCQEGHILKMFPSTWYV"
    E = model.emb_b.float()
    outs = []
    for s in seqs:
        cls = torch.tensor([AA.index(c) if c in AA else 20 for c in s], device="cuda")
        x = E[cls].T[None]                                  # [1, 32, L]
        for l in range(4):
            w = model.Wb[l].float().reshape(256, 5, -1).permute(0, 2, 1)   # [co, ci, 5]
            y = torch.nn.functional.conv1d(x, w, model.b[l], padding=2)
            y = torch.nn.functional.gelu(y, approximate="tanh")
            x = y + x if (l > 0 and model.residual) else y
        p = x[0].mean(1)
        outs.append(p / p.norm())
    return torch.stack(outs)


def _layout_of(seqs):
    from sseqs_b200 import learned
    buf = "".join(s + "@" for s in seqs).encode()
    ascii = torch.from_numpy(np.frombuffer(buf, np.uint8).copy()).cuda()
    lens = torch.tensor([len(s) for s in seqs], dtype=torch.int64, device="cuda")
    offs = torch.cumsum(lens + 1, 0) - (lens + 1)
    return learned.make_layout(ascii, offs, lens)


@pytest.mark.parametrize("residual", [True, False])
def test_embedder_forward_matches_fp32_conv(residual):
    from sseqs_b200 import dbtools, learned
    model = learned.Embedder(seed=3, residual=residual)
    seqs = [dbtools.random_query(int(n), 40 + i) for i, n in enumerate([1, 5, 37, 300, 1000])]
    seqs[3] = seqs[3][:20] + "XBZU" + seqs[3][24:]
    got = model.forward(_layout_of(seqs))
    exp = _ref_embed(model, seqs)
    # bf16 activations between layers: cosine of the unit vectors >= 0.999
    cos = (got * exp).sum(1)
    assert bool((cos > 0.999).all()), cos


@pytest.mark.parametrize("residual", [True, False])
def test_embedder_backward_matches_autograd(residual):
    from sseqs_b200 import dbtools, learned
    model = learned.Embedder(seed=5, residual=residual)
    seqs = [dbtools.random_query(int(n), 60 + i) for i, n in enumerate([50, 120, 80, 200])]
    lay = _layout_of(seqs)
    emb = model.forward(lay, train=True)
    # loss = sum_s <emb_s, r_s> for a fixed random r: dE = r
    g = torch.Generator(device="cpu")
    g.manual_seed(9)
    r = torch.randn(emb.shape, generator=g).cuda()
    grads = model.backward(r.contiguous())
    # reference with autograd on fp32 copies of the bf16 parameters
    AA = "ARNDCQEGHILKMFPSTWYV"
    Ep = model.emb_b.float().clone().requires_grad_()
    Ws = [model.Wb[l].float().reshape(256, 5, -1).clone().requires_grad_() for l in range(4)]
    bs = [model.b[l].clone().requires_grad_() for l in range(4)]
    tot = 0
    for si, s in enumerate(seqs):
        cls = torch.tensor([AA.index(c) if c in AA else 20 for c in s], device="cuda")
        x = Ep[cls].T[None]
        for l in range(4):
            y = torch.nn.functional.conv1d(x, Ws[l].permute(0, 2, 1), bs[l], padding=2)
            y = torch.nn.functional.gelu(y, approximate="tanh")
            x = y + x if (l > 0 and model.residual) else y
        p = x[0].mean(1)
        tot = tot + ((p / p.norm()) * r[si]).sum()
    tot.backward()

    def close(a, b):   # bf16 forward/backward activations: cosine >= 0.99
        a, b = a.flatten().float(), b.flatten().float()
        return (a @ b / (a.norm() * b.norm() + 1e-30)).item()

    for l in range(4):
        cin = model.cin[l]
        dW = grads["W"][l].reshape(5, cin, 256).permute(2, 0, 1)     # [co, t, ci]
        assert close(dW, Ws[l].grad) > 0.99, l
        assert close(grads["b"][l], bs[l].grad) > 0.99, l
    assert close(grads["emb"], Ep.grad) > 0.99


def _codes(nq, n, seed=1):
    from sseqs_b200 import _lib
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    q = torch.randn(nq, 256, generator=g)
    d = torch.randn(n, 256, generator=g)
    q = (q / q.norm(dim=1, keepdim=True)).cuda()
    d = (d / d.norm(dim=1, keepdim=True)).cuda()
    L = _lib.lib()
    qc = torch.empty((nq, 256), dtype=torch.uint8, device="cuda")
    dc = torch.empty((n, 256), dtype=torch.uint8, device="cuda")
    _lib.check(L.sseqs_quantize_e4m3(q.data_ptr(), q.numel(), 16.0, qc.data_ptr(), 0), "q")
    _lib.check(L.sseqs_quantize_e4m3(d.data_ptr(), d.numel(), 16.0, dc.data_ptr(), 0), "q")
    return qc, dc


def _select(qc, dc, tau, cap):
    from sseqs_b200 import _lib
    nq, n = qc.shape[0], dc.shape[0]
    cnt = torch.zeros(nq, dtype=torch.int32, device="cuda")
    cand = torch.empty((nq, cap), dtype=torch.int64, device="cuda")
    cs = torch.empty((nq, cap), dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().sseqs_score_select(qc.data_ptr(), nq, dc.data_ptr(), n, tau.data_ptr(),
                                             cnt.data_ptr(), cand.data_ptr(), cs.data_ptr(), cap,
                                             0), "select")
    return cnt, cand, cs


def test_score_select_and_threshold():
    from sseqs_b200 import _lib
    nq, n = 130, 5000
    qc, dc = _codes(nq, n)
    L = _lib.lib()
    qf = qc.view(torch.float8_e4m3fn).float()
    df = dc.view(torch.float8_e4m3fn).float()
    ref = qf @ df.T                                             # fp32 reference
    dense = torch.empty((nq, n), dtype=torch.float32, device="cuda")
    _lib.check(L.sseqs_score_dense(qc.data_ptr(), nq, dc.data_ptr(), n, dense.data_ptr(), 0), "d")
    assert (dense - ref).abs().max().item() < 1e-3
    k = 7
    kth = torch.empty(nq, dtype=torch.float32, device="cuda")
    sub = ref[:, :4000].contiguous()
    _lib.check(L.sseqs_kth_largest_rows(sub.data_ptr(), nq, 4000, k, kth.data_ptr(), 0), "k")
    assert torch.equal(kth, torch.topk(sub, k, dim=1).values[:, -1])


# batch sizes: one query, a partial 16-column tile, exactly 256 (one full
# tcgen05 query tile), 300 (two tiles, the second ragged); database sizes
# with and without a partial 128-row tile
@pytest.mark.parametrize("nq,n", [(1, 5000), (8, 4096), (37, 5000), (130, 5000),
                                  (256, 3000), (300, 2000)])
@pytest.mark.parametrize("path", [1, 0])    # 1: tcgen05 kind::f8f6f4, 0: mma.sync
def test_score_select_paths(nq, n, path):
    """Every (query, row) at least 1e-3 above the query's threshold is
    selected and none more than 1e-3 below it (fp32 reference of the FP8
    dot products); the scores reported are the reference's within 1e-3;
    both paths select the same sets apart from rows within 1e-3 of a
    threshold."""
    from sseqs_b200 import _lib
    qc, dc = _codes(nq, n, seed=nq + n)
    qf = qc.view(torch.float8_e4m3fn).float()
    df = dc.view(torch.float8_e4m3fn).float()
    ref = qf @ df.T
    tau = torch.quantile(ref, 0.99, dim=1).contiguous()
    cap = 200
    _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(path), "path")
    try:
        cnt, cand, cs = _select(qc, dc, tau, cap)
        torch.cuda.synchronize()
    finally:
        _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(1), "path")
    assert _gemm_error() == 0
    for i in range(nq):
        c = int(cnt[i])
        assert c <= cap
        rows = cand[i, :c]
        got = set(rows.tolist())
        assert len(got) == c
        sure_in = set(torch.nonzero(ref[i] >= tau[i] + 1e-3).flatten().tolist())
        maybe = set(torch.nonzero(ref[i] >= tau[i] - 1e-3).flatten().tolist())
        assert sure_in <= got <= maybe
        if c:
            assert (cs[i, :c] - ref[i, rows]).abs().max().item() < 1e-3


@pytest.mark.parametrize("dim", [256, 128])
def test_learned_search_reports_exact_scores(dim):
    from sseqs_b200 import dbtools, learned, select
    from sseqs_b200.database import Database
    sw = importlib.import_module("sseqs_b200.sw")
    pairs = learned.training_pairs(24, 32, seed=2)
    model = learned.Embedder(seed=2)
    hist = learned.train(model, pairs, queries_per_step=8, targets_per_query=16, epochs=2)
    assert hist["losses"][-1][1] < hist["losses"][0][1]
    q0 = dbtools.random_query(220, 11)
    syn = dbtools.synthetic_db([q0], 4000, 0.02, (0.5, 0.95), seed=11, device="cpu",
                               chunk_bytes=150_000)
    db = Database(syn.chunks, bs=150_000)
    idx = learned.LearnedIndex(model, db, chunk=1000, dim=dim)
    assert idx.codes.shape[1] == dim
    hits = idx.search([q0], n_cand=300, top=50)[0]
    assert hits
    enc = sw.encode_query(q0)
    for norm, bi, g, score in hits:
        b = db.batches[bi]
        exp = sw.sw_scan(enc, b.ascii, b.delim, affine=True,
                         good_idx=torch.tensor([g], dtype=torch.int32, device="cuda"),
                         skip=1, gap_a=11, gap_b=1)
        assert int(exp[0]) == score
        assert abs(norm - score / math.sqrt(len(q0) * b.maxlen)) < 1e-5


def _ragged_db(n_seqs=3000, chunk_bytes=100_000, seed=3):
    """Several batches with empty segments ('@@') among the sequences."""
    from sseqs_b200 import dbtools
    from sseqs_b200.database import Database
    rng = np.random.default_rng(seed)
    seqs = ["" if rng.random() < 0.03 else dbtools.random_query(int(rng.integers(20, 400)),
                                                                90000 + i)
            for i in range(n_seqs)]
    raw = b"".join(s.encode() + b"@" for s in seqs)
    stream = torch.from_numpy(np.frombuffer(raw, np.uint8).copy())
    lengths = torch.tensor([len(s) for s in seqs], dtype=torch.int64)
    chunks, _, _ = dbtools.assemble_stream(stream, lengths, chunk_bytes)
    return Database(chunks, bs=chunk_bytes)


def test_rescore_matches_direct_scoring():
    """Rescoring of explicit candidate lists (random rows plus the first and
    last row of every batch, which are not scored) on a multi-batch database
    with empty segments, queries of several stripe widths: the same hits, in
    the same order, as scoring every candidate directly and ranking by
    normalised score desc, then batch, then segment."""
    from sseqs_b200 import dbtools, learned
    sw = importlib.import_module("sseqs_b200.sw")
    db = _ragged_db()
    assert len(db.batches) >= 4
    idx = learned.LearnedIndex(learned.Embedder(seed=4), db, chunk=1000)
    rng = np.random.default_rng(5)
    queries = [dbtools.random_query(L, 500 + j)
               for j, L in enumerate([40, 150, 151, 300, 700, 33, 1000])]
    edges = np.concatenate([idx.cum[:-1], idx.cum[1:] - 1])
    cands = [torch.from_numpy(np.unique(np.concatenate(
        [rng.choice(idx.n, size=min(idx.n, 400), replace=False), edges]))).cuda()
        for _ in queries]
    top = 150
    got = idx.rescore(queries, cands, top=top)
    # the same with the packed buffer limited so that the queries are scored
    # in several parts
    idx.PACK_LIMIT = 150_000
    assert idx.rescore(queries, cands, top=top) == got
    del idx.PACK_LIMIT
    for j, q in enumerate(queries):
        enc = sw.encode_query(q)
        rows = cands[j].cpu().numpy()
        bat = np.searchsorted(idx.cum[1:], rows, side="right")
        loc = rows - idx.cum[bat]
        S, B, G, A = [], [], [], []
        for bi in np.unique(bat):
            b = db.batches[bi]
            sel = (bat == bi) & (loc >= 1) & (loc <= b.n_segments - 2)
            if not sel.any():
                continue
            g = b.seg_index[torch.from_numpy(loc[sel]).cuda()].to(torch.int32)
            sc = sw.sw_scan(enc, b.ascii, b.delim, affine=True, good_idx=g, skip=1, gap_a=11,
                            gap_b=1).cpu().numpy().astype(np.int64)
            A.append(sc)
            G.append(g.cpu().numpy().astype(np.int64))
            B.append(np.full(sc.size, bi, np.int64))
            S.append((sc.astype(np.float32) / np.sqrt(np.float32(len(q) * b.maxlen)))
                     .astype(np.float32))
        S, B, G, A = (np.concatenate(x) for x in (S, B, G, A))
        o = np.lexsort((G, B, -S.astype(np.float64)))[:top]
        want = list(zip(S[o].tolist(), B[o].tolist(), G[o].tolist(), A[o].tolist()))
        assert got[j] == want


def test_candidates_take_top_keys_with_lower_rows_at_ties():
    """The per-query cut of the selection: the n_cand largest fp16 keys,
    ties at the cut to the lower rows (against the raw selection lists)."""
    from sseqs_b200 import dbtools, learned
    db = _ragged_db(seed=6)
    idx = learned.LearnedIndex(learned.Embedder(seed=6), db, chunk=1000)
    queries = [dbtools.random_query(L, 700 + j) for j, L in enumerate([60, 250, 512])]
    codes = idx.query_codes(queries)
    n_cand = 50
    cand, cs, cnt, cap = idx._select(codes, n_cand, 8192, 2.5, 8)
    kq, kr, counts = idx.candidates_flat(codes, n_cand)
    kq, kr = kq.cpu().numpy(), kr.cpu().numpy()
    for j in range(len(queries)):
        c = int(min(cnt[j], cap))
        assert c > n_cand                  # the cut is exercised
        rows = cand[j, :c].cpu().numpy()
        keys = cs[j, :c].to(torch.float16).float().cpu().numpy()
        want = np.sort(rows[np.lexsort((rows, -keys.astype(np.float64)))[:n_cand]])
        mine = kr[kq == j]
        assert counts[j] == n_cand
        assert np.array_equal(mine, want)


def test_pack_segments_copies_every_window():
    """sseqs_pack_segments against a host copy: windows of 0..70 bytes from
    three buffers at every source/destination alignment (the 4-byte-word and
    the byte-by-byte paths), each followed by one '@'."""
    from sseqs_b200 import _lib
    rng = np.random.default_rng(9)
    bufs = [torch.from_numpy(rng.integers(65, 90, size=n, dtype=np.uint8)).cuda()
            for n in (1000, 777, 4096)]
    n = 600
    part = rng.integers(0, 3, n)
    ln = rng.integers(0, 71, n)
    ln[:6] = [0, 1, 2, 3, 4, 5]
    src = np.array([rng.integers(0, bufs[p].numel() - l + 1) for p, l in zip(part, ln)])
    dst = np.cumsum(ln + 1) - (ln + 1)
    total = int(dst[-1] + ln[-1] + 1)
    out = torch.full((total,), 0, dtype=torch.uint8, device="cuda")
    bases = torch.tensor([b.data_ptr() for b in bufs], dtype=torch.int64, device="cuda")
    part_d = torch.from_numpy(part.astype(np.int32)).cuda()
    src_d = torch.from_numpy(src.astype(np.int64)).cuda()
    len_d = torch.from_numpy(ln.astype(np.int32)).cuda()
    dst_d = torch.from_numpy(dst.astype(np.int64)).cuda()
    _lib.check(_lib.lib().sseqs_pack_segments(bases.data_ptr(), part_d.data_ptr(),
                                              src_d.data_ptr(), len_d.data_ptr(),
                                              dst_d.data_ptr(), n, out.data_ptr(), 0), "pack")
    host = [b.cpu().numpy() for b in bufs]
    want = np.concatenate([np.concatenate([host[p][s:s + l], [64]]).astype(np.uint8)
                           for p, s, l in zip(part, src, ln)])
    assert np.array_equal(out.cpu().numpy(), want)


@pytest.mark.parametrize("path", [1, 0])    # 1: tcgen05 kind::f8f6f4, 0: mma.sync
def test_half_width_index_selects_by_its_codes(path):
    """A 128-wide index (read by the selection kernel as 256-byte rows of two
    codes, against [q, 0] and [0, q]): every returned row is a real code row
    (the spare zero row never), reported once, with the fp32 dot product of
    the query's and the row's 128-byte codes within 1e-3, and every row more
    than 1e-3 above the lowest reported score is returned."""
    from sseqs_b200 import _lib, dbtools, learned
    db = _ragged_db(seed=8)
    idx = learned.LearnedIndex(learned.Embedder(seed=8), db, chunk=1000, dim=128)
    n = idx.n
    assert idx.codes.shape == (n + (n & 1), 128)
    assert not idx.codes[n:].any()
    queries = [dbtools.random_query(L, 800 + j) for j, L in enumerate([60, 250, 512, 999])]
    codes = idx.query_codes(queries)
    assert codes.shape == (len(queries), 128)
    qf = codes.view(torch.float8_e4m3fn).float()
    df = idx.codes[:n].view(torch.float8_e4m3fn).float()
    ref = qf @ df.T
    _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(path), "path")
    try:
        cand, cs, cnt, cap = idx._select(codes, 50, 8192, 2.5, 8)
        torch.cuda.synchronize()
    finally:
        _lib.check(_lib.lib().sseqs_gemm_set_tensor_path(1), "path")
    assert _gemm_error() == 0
    for j in range(len(queries)):
        c = int(min(cnt[j], cap))
        assert c > 50
        rows = cand[j, :c]
        got = set(rows.tolist())
        assert len(got) == c and max(got) < n
        assert (cs[j, :c] - ref[j, rows]).abs().max().item() < 1e-3
        low = float(cs[j, :c].min())
        assert set(torch.nonzero(ref[j] >= low + 1e-3).flatten().tolist()) <= got

"""Seeded test inputs and a literal emulation of the reference warp kernels."""
from __future__ import annotations

import numpy as np

AA = "ARNDCQEGHILKMFPSTWYV"
# Robinson & Robinson (1991) background amino-acid frequencies, order AA.
BACKGROUND = np.array([0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295,
                       0.07377, 0.02199, 0.05142, 0.09019, 0.05744, 0.02243, 0.03856,
                       0.05203, 0.07120, 0.05841, 0.01330, 0.03216, 0.06441])
BACKGROUND = BACKGROUND / BACKGROUND.sum()


def rand_seq(rng, n, extra=""):
    alphabet = AA + extra
    p = None if extra else BACKGROUND
    return "".join(rng.choice(list(alphabet), size=n, p=p))


def mutate(rng, s, ident, indel=0.02):
    out = []
    for c in s:
        r = rng.random()
        if r < indel / 2:
            continue
        if r < indel:
            out.append(AA[rng.integers(20)])
        out.append(c if rng.random() < ident else AA[rng.integers(20)])
    return "".join(out)


def homolog_targets(rng, query, n, lo=5, hi=300, frac=0.5):
    ts = []
    for _ in range(n):
        if rng.random() < frac and len(query) > 4:
            a = int(rng.integers(0, len(query) // 2))
            b = int(rng.integers(a + 2, len(query) + 1))
            t = rand_seq(rng, int(rng.integers(0, 20))) + mutate(rng, query[a:b], rng.uniform(0.3, 0.95)) \
                + rand_seq(rng, int(rng.integers(0, 20)))
        else:
            t = rand_seq(rng, int(rng.integers(lo, hi)))
        ts.append(t)
    return ts


# ---------------------------------------------------------------------------
# Literal emulation of the reference kernels sseqs/sw.cu:55-179 and :182-325:
# 32 lanes, each holding TPT = roundup32(Lq)/32 columns in prev/curr arrays,
# advancing row by row, diagonal values passed by __shfl_up_sync.  Used to pin
# the row-major C oracle on small cases.
_CLS = {c: i for i, c in enumerate(AA)}


def _b62():
    import oracle.oracle as O
    return O.BLOSUM62


def emulate_ref_kernel(q_idx, t_bytes, affine, p0=11, p1=1):
    B62 = _b62()
    Lq = len(q_idx)
    if Lq == 0 or len(t_bytes) == 0:
        return -1
    TPT = ((Lq + 31) >> 5 << 5) // 32
    if affine:
        prevM = [[0] * TPT for _ in range(32)]
        prevX = [[0] * TPT for _ in range(32)]
        prevY = [[0] * TPT for _ in range(32)]
        currM = [[0] * TPT for _ in range(32)]
        currX = [[0] * TPT for _ in range(32)]
        currY = [[0] * TPT for _ in range(32)]
    else:
        prev = [[0] * TPT for _ in range(32)]
        curr = [[0] * TPT for _ in range(32)]
    best = [0] * 32

    def i16(v):
        v &= 0xFFFF
        return v - 0x10000 if v >= 0x8000 else v

    for ch in t_bytes:
        c = _CLS.get(chr(ch), -1) if ch < 128 else -1
        if affine:
            up_last = [(prevM[l][TPT - 1], prevX[l][TPT - 1], prevY[l][TPT - 1]) for l in range(32)]
        else:
            up_last = [prev[l][TPT - 1] for l in range(32)]
        for lane in range(32):
            jb = lane * TPT
            if affine:
                dM, dX, dY = (0, 0, 0) if lane == 0 else up_last[lane - 1]
                lM = lX = 0
            else:
                diag = 0 if lane == 0 else up_last[lane - 1]
                left = 0
            for k in range(TPT):
                j = jb + k
                if j >= Lq:
                    break
                s = -4 if c < 0 else int(B62[c][q_idx[j]])
                if affine:
                    uM, uX, uY = prevM[lane][k], prevX[lane][k], prevY[lane][k]
                    m = i16(max(0, max(dM + s, max(dX + s, dY + s))))
                    x = i16(max(0, max(lM - p0, lX - p1)))
                    y = i16(max(0, max(uM - p0, uY - p1)))
                    currM[lane][k], currX[lane][k], currY[lane][k] = m, x, y
                    best[lane] = max(best[lane], max(m, max(x, y)))
                    dM, dX, dY = uM, uX, uY
                    lM, lX = m, x
                else:
                    up = prev[lane][k]
                    h = max(0, max(diag + s, max(up + p0, left + p0))) & 0xFFFF
                    curr[lane][k] = h
                    best[lane] = max(best[lane], h)
                    diag = up
                    left = h
        for lane in range(32):
            for k in range(TPT):
                if affine:
                    prevM[lane][k], prevX[lane][k], prevY[lane][k] = currM[lane][k], currX[lane][k], currY[lane][k]
                else:
                    prev[lane][k] = curr[lane][k]
    return max(best)

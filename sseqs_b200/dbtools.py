"""Database tooling: the .xbit packer (from sequences or a FASTA file, with a
sidecar segment index) and a seeded synthetic database generator.

File layout (as read by sseqs/msa.py:50-55 and decoded by sseqs/xbit.cu:8-34):
a raw, header-less 5-bit stream of ``S0@S1@...@`` in chunks of ``chunk_bytes``
packed bytes (1e9 in the reference).  Each chunk here holds whole sequences
only and is zero-padded to exactly ``chunk_bytes`` (zero symbols decode to
'@', i.e. empty segments, which the search drops), so no sequence straddles a
chunk and every chunk starts with a sequence.

The synthetic generator follows the shapes of the benchmark configurations:
residues iid from the Robinson & Robinson (1991) background composition of
the 20 amino acids, lengths log-normal (median 250, sigma 0.6) clipped to
30..1000, and planted homologs of given queries with a target identity drawn
uniformly from a range, indels at rate 0.02 per position with geometric
(p = 0.5) lengths.  It runs with torch on the CPU or on CUDA (the two devices
draw different random streams for the same seed).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

AA = "ARNDCQEGHILKMFPSTWYV"
AA_BYTES = torch.tensor(list(AA.encode()), dtype=torch.uint8)
# Robinson & Robinson (1991) amino-acid background frequencies, order AA.
BACKGROUND = [0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295, 0.07377,
              0.02199, 0.05142, 0.09019, 0.05744, 0.02243, 0.03856, 0.05203, 0.07120,
              0.05841, 0.01330, 0.03216, 0.06441]
CHUNK_BYTES = 1_000_000_000


def _cdf(device):
    p = torch.tensor(BACKGROUND, dtype=torch.float64)
    c = torch.cumsum(p / p.sum(), 0)
    c[-1] = 1.0
    return c.to(torch.float32).to(device)


def random_residues(n: int, gen: torch.Generator, device, cdf=None) -> torch.Tensor:
    """n residues (ASCII bytes) iid from the background composition."""
    cdf = _cdf(device) if cdf is None else cdf
    out = torch.empty(n, dtype=torch.uint8, device=device)
    step = 1 << 27
    aa = AA_BYTES.to(device)
    for s in range(0, n, step):
        m = min(step, n - s)
        u = torch.rand(m, generator=gen, device=device)
        idx = torch.bucketize(u, cdf, right=True).clamp_(max=19)
        out[s:s + m] = aa[idx]
    return out


def random_query(length: int, seed: int = 0) -> str:
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    return random_residues(length, g, "cpu").numpy().tobytes().decode()


def lognormal_lengths(n, gen, device, median=250.0, sigma=0.6, lo=30, hi=1000):
    z = torch.randn(n, generator=gen, device=device, dtype=torch.float32)
    return torch.exp(z * sigma + math.log(median)).round_().clamp_(lo, hi).to(torch.int64)


def _geometric(shape, gen, device, p=0.5):
    u = torch.rand(shape, generator=gen, device=device).clamp_(min=1e-12)
    return (torch.floor(torch.log(u) / math.log(1.0 - p)) + 1).to(torch.int64)


def plant_homologs(query: str, n: int, ident_lo: float, ident_hi: float, gen, device,
                   indel_rate: float = 0.02, cdf=None, with_identity: bool = False):
    """``n`` mutated copies of ``query``: per copy an identity u ~ U(lo, hi);
    each residue is replaced by a background residue with probability 1-u;
    at each position a deletion (rate/2) or insertion (rate/2) event of
    geometric length starts.  Returns (residue bytes, lengths), and with
    ``with_identity`` also the u of every copy (float32)."""
    q = torch.tensor(list(query.encode()), dtype=torch.uint8, device=device)
    L = q.numel()
    if n == 0:
        out = (torch.empty(0, dtype=torch.uint8, device=device),
               torch.empty(0, dtype=torch.int64, device=device))
        return out + (torch.empty(0, dtype=torch.float32, device=device),) if with_identity else out
    ident = ident_lo + (ident_hi - ident_lo) * torch.rand(n, 1, generator=gen, device=device)
    sub = torch.rand(n, L, generator=gen, device=device) >= ident
    sub_res = random_residues(n * L, gen, device, cdf).view(n, L)
    base = torch.where(sub, sub_res, q.expand(n, L))
    ev = torch.rand(n, L, generator=gen, device=device)
    is_del = ev < indel_rate / 2
    is_ins = (ev >= indel_rate / 2) & (ev < indel_rate)
    ln = _geometric((n, L), gen, device)
    # deletions cover [p, p + len): difference array + running sum
    diff = torch.zeros(n, L + 1, dtype=torch.int64, device=device)
    starts = torch.nonzero(is_del, as_tuple=False)
    if starts.numel():
        r, c = starts[:, 0], starts[:, 1]
        e = torch.clamp(c + ln[r, c], max=L)
        diff.index_put_((r, c), torch.ones_like(c), accumulate=True)
        diff.index_put_((r, e), -torch.ones_like(c), accumulate=True)
    deleted = torch.cumsum(diff[:, :L], 1) > 0
    keep = (~deleted).to(torch.int64)
    ins = torch.where(is_ins, ln, torch.zeros_like(ln))
    emit = keep + ins                                   # residues emitted at p
    lengths = emit.sum(1)
    total = int(lengths.sum().item())
    # slot -> (copy, position); first `keep` slots of a position carry base
    flat_emit = emit.flatten()
    src = torch.repeat_interleave(torch.arange(n * L, device=device), flat_emit)
    first = torch.cumsum(flat_emit, 0) - flat_emit
    rank = torch.arange(total, device=device) - first[src]
    is_base = rank < keep.flatten()[src]
    ins_res = random_residues(total, gen, device, cdf)
    res = torch.where(is_base, base.flatten()[src], ins_res)
    if with_identity:
        return res, lengths, ident.flatten().to(torch.float32)
    return res, lengths


@dataclass
class SyntheticDB:
    chunks: list                       # packed chunks (uint8 tensors of chunk_bytes)
    n_seqs: int
    n_residues: int
    planted: dict = field(default_factory=dict)   # query index -> db sequence ids
    planted_identity: dict = field(default_factory=dict)   # query index -> identity u of each
    seq_chunk: torch.Tensor | None = None          # chunk of every sequence
    seq_rank: torch.Tensor | None = None           # position inside its chunk


def _pack(sym: torch.Tensor) -> torch.Tensor:
    from . import xbit
    if sym.device.type == "cuda":
        return xbit.compress(sym)
    return torch.from_numpy(pack_symbols_host(sym.numpy()))


def assemble_stream(stream: torch.Tensor, lengths: torch.Tensor, chunk_bytes: int = CHUNK_BYTES):
    """Cut an ``S0@S1@...@`` stream (sequence lengths given) into packed
    chunks of ``chunk_bytes``, each holding whole sequences and '@' padding.

    Returns (chunks, chunk of every sequence, rank of every sequence inside
    its chunk)."""
    device = stream.device
    cap = chunk_bytes * 8 // 5                        # symbols per chunk
    sizes = lengths + 1
    cum = torch.cumsum(sizes, 0)
    n = lengths.numel()
    chunks = []
    seq_chunk = torch.empty(n, dtype=torch.int64, device=device)
    seq_rank = torch.empty(n, dtype=torch.int64, device=device)
    first, base = 0, 0
    while first < n:
        if int(sizes[first].item()) > cap:
            raise ValueError("a sequence is longer than a chunk")
        last = int(torch.searchsorted(cum, torch.tensor([base + cap], device=device),
                                      right=True).item())
        end = int(cum[last - 1].item())
        sym = torch.full((cap,), 64, dtype=torch.uint8, device=device)
        sym[: end - base] = stream[base:end]
        chunks.append(_pack(sym))
        del sym
        seq_chunk[first:last] = len(chunks) - 1
        seq_rank[first:last] = torch.arange(last - first, device=device)
        base, first = end, last
    return chunks, seq_chunk, seq_rank


def synthetic_db(queries: list[str], n_seqs: int, homolog_frac: float, ident: tuple,
                 seed: int = 0, device="cuda", chunk_bytes: int = CHUNK_BYTES) -> SyntheticDB:
    """Seeded synthetic database with ``round(homolog_frac * n_seqs)``
    planted homologs per query at random positions; every other sequence is
    iid background with log-normal length."""
    device = torch.device(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    cdf = _cdf(device)
    n_h = int(round(homolog_frac * n_seqs))
    if n_h * len(queries) > n_seqs:
        raise ValueError("more planted homologs than sequences")
    owner = torch.full((n_seqs,), -1, dtype=torch.int64, device=device)
    for qi in range(len(queries)):
        owner[qi * n_h:(qi + 1) * n_h] = qi
    owner = owner[torch.randperm(n_seqs, generator=gen, device=device)]
    lengths = lognormal_lengths(n_seqs, gen, device)
    homologs = []
    identity = {}
    for qi, q in enumerate(queries):
        hb, hl, hu = plant_homologs(q, n_h, ident[0], ident[1], gen, device, cdf=cdf,
                                    with_identity=True)
        slots = torch.nonzero(owner == qi).flatten()
        lengths[slots] = hl
        homologs.append((slots, hb, hl))
        identity[qi] = hu
    sizes = lengths + 1
    ends = torch.cumsum(sizes, 0)
    total = int(ends[-1].item())
    stream = random_residues(total, gen, device, cdf)
    stream[ends - 1] = 64                                   # '@' after every sequence
    starts = ends - sizes
    for slots, hb, hl in homologs:
        if hb.numel() == 0:
            continue
        first = torch.cumsum(hl, 0) - hl
        dst = torch.repeat_interleave(starts[slots] - first, hl) + torch.arange(
            hb.numel(), device=device)
        stream[dst] = hb
        del dst
    del homologs
    n_res = int(lengths.sum().item())
    chunks, seq_chunk, seq_rank = assemble_stream(stream, lengths, chunk_bytes)
    planted = {qi: torch.nonzero(owner == qi).flatten() for qi in range(len(queries))}
    return SyntheticDB(chunks, n_seqs, n_res, planted, identity, seq_chunk, seq_rank)


def pack_symbols_host(sym: np.ndarray) -> np.ndarray:
    """Host xbit packer (layout of sseqs/xbit.cu:36-62), for building files."""
    sym = np.asarray(sym, dtype=np.uint8).reshape(-1)
    n = sym.size
    g = (n + 7) // 8
    out = np.empty((g, 5), np.uint8)
    step = 1 << 22                       # groups per block
    for g0 in range(0, g, step):
        g1 = min(g, g0 + step)
        blk = np.full((g1 - g0) * 8, 64, np.uint8)
        part = sym[g0 * 8:min(n, g1 * 8)]
        blk[:part.size] = part
        blk -= 64
        blk &= 31
        # a group's 8 symbols as one little-endian word: symbol k in byte k;
        # place symbol k at bit 59 - 5k, so the 40-bit group fills the top
        # of the word, and byte-swap: its first 5 bytes are the big-endian
        # packed group
        x = blk.view("<u8")
        w = np.zeros_like(x)
        for k in range(8):
            w |= ((x >> np.uint64(8 * k)) & np.uint64(31)) << np.uint64(59 - 5 * k)
        out[g0:g1] = w.byteswap().view(np.uint8).reshape(-1, 8)[:, :5]
    return out.reshape(-1)[: (5 * n + 7) // 8]


def write_xbit(path: str, sequences, chunk_bytes: int = CHUNK_BYTES) -> int:
    """Write sequences (iterable of str) as a chunk-aligned .xbit file;
    returns the number of chunks."""
    seqs = [s.encode() for s in sequences]
    lengths = torch.tensor([len(s) for s in seqs], dtype=torch.int64)
    stream = torch.from_numpy(np.frombuffer(b"".join(s + b"@" for s in seqs), np.uint8).copy())
    chunks, _, _ = assemble_stream(stream, lengths, chunk_bytes)
    with open(path, "wb") as f:
        for c in chunks:
            f.write(c.cpu().numpy().tobytes())
    return len(chunks)


# --------------------------------------------------------- FASTA -> .xbit
def read_fasta(path: str):
    """(name, sequence) of every record of a FASTA file: the name is the
    header line after '>' (stripped), the sequence its following lines with
    whitespace removed; text before the first header is ignored."""
    name, parts = None, []
    with open(path, "r", encoding="latin-1") as fh:
        for line in fh:
            if line.startswith(">"):
                if name is not None:
                    yield name, "".join(parts)
                name, parts = line[1:].strip(), []
            elif name is not None:
                parts.append("".join(line.split()))
    if name is not None:
        yield name, "".join(parts)


_RESIDUE_MAP = np.full(256, ord("X"), np.uint8)
_RESIDUE_MAP[ord("A"):ord("Z") + 1] = np.arange(ord("A"), ord("Z") + 1)
_RESIDUE_MAP[ord("a"):ord("z") + 1] = np.arange(ord("A"), ord("Z") + 1)


def normalise_residues(seq: str) -> bytes:
    """The bytes a sequence is stored as: letters upper-cased, every other
    character 'X'.  (The 5-bit alphabet holds '@'..'_'; the reference's
    packer, sseqs/xbit.cu:47-49, keeps the low 5 bits of byte - 64, which
    would turn '*' into 'J' and '-' into 'M'.)"""
    return _RESIDUE_MAP[np.frombuffer(seq.encode("latin-1"), np.uint8)].tobytes()


@dataclass
class SeqIndex:
    """Sidecar segment index of an .xbit file: for sequence k (file order),
    its chunk, its first symbol inside that chunk, its length and its name."""
    chunk_bytes: int
    n_chunks: int
    chunk_of: np.ndarray       # int32[n]
    start: np.ndarray          # int64[n] symbol position inside the chunk
    length: np.ndarray         # int32[n]
    names: list

    def save(self, path: str) -> None:
        blob = "\n".join(self.names).encode("latin-1") if self.names else b""
        with open(path, "wb") as fh:
            np.savez(fh, chunk_bytes=np.int64(self.chunk_bytes), n_chunks=np.int64(self.n_chunks),
                     chunk_of=self.chunk_of, start=self.start, length=self.length,
                     names=np.frombuffer(blob, np.uint8), n=np.int64(len(self.names)))

    @classmethod
    def load(cls, path: str) -> "SeqIndex":
        z = np.load(path)
        n = int(z["n"])
        names = z["names"].tobytes().decode("latin-1").split("\n") if n else []
        return cls(int(z["chunk_bytes"]), int(z["n_chunks"]), z["chunk_of"], z["start"],
                   z["length"], names)

    def locate(self, chunk: int, pos: int) -> int:
        """Sequence whose bytes or closing '@' hold symbol ``pos`` of
        ``chunk`` (-1 for chunk padding)."""
        lo = int(np.searchsorted(self.chunk_of, chunk, side="left"))
        hi = int(np.searchsorted(self.chunk_of, chunk, side="right"))
        if lo == hi:
            return -1
        k = lo + int(np.searchsorted(self.start[lo:hi], pos, side="right")) - 1
        if k < lo or pos > self.start[k] + self.length[k]:
            return -1
        return k


def index_path(xbit_path: str) -> str:
    """Where the sidecar index of an .xbit file lives."""
    return xbit_path + ".idx.npz"


def fasta_to_xbit(fasta_path: str, xbit_path: str, chunk_bytes: int = CHUNK_BYTES,
                  sidecar: str | None = None) -> SeqIndex:
    """Pack a FASTA file into a chunk-aligned .xbit file (the layout
    ``write_xbit`` writes, byte for byte, for the normalised sequences) and
    write its sidecar segment index (``index_path(xbit_path)`` unless given).

    Streams the input: one chunk of symbols is held at a time.  A sequence
    longer than a chunk raises ValueError."""
    cap = chunk_bytes * 8 // 5                       # symbols per chunk
    chunk_of, start, length, names = [], [], [], []
    buf = np.full(cap, 64, np.uint8)
    used, ci = 0, 0

    def flush(fh):
        packed = pack_symbols_host(buf)
        fh.write(packed.tobytes())
        if packed.size < chunk_bytes:
            fh.write(bytes(chunk_bytes - packed.size))

    with open(xbit_path, "wb") as fh:
        for name, seq in read_fasta(fasta_path):
            s = np.frombuffer(normalise_residues(seq), np.uint8)
            if s.size + 1 > cap:
                raise ValueError(f"sequence {name!r} ({s.size} residues) is longer than a chunk")
            if used + s.size + 1 > cap:
                flush(fh)
                buf[:] = 64
                used, ci = 0, ci + 1
            buf[used:used + s.size] = s
            chunk_of.append(ci)
            start.append(used)
            length.append(s.size)
            names.append(name.replace("\n", " "))
            used += s.size + 1
        if used:
            flush(fh)
            ci += 1
    idx = SeqIndex(chunk_bytes, ci, np.asarray(chunk_of, np.int32), np.asarray(start, np.int64),
                   np.asarray(length, np.int32), names)
    idx.save(sidecar or index_path(xbit_path))
    return idx

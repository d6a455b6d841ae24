"""sseqs_b200 -- the sseqs database-search path on NVIDIA B200 (sm_100a).

Drop-in for the reference's public calls: ``msa(query, "out.a3m")`` and
``sw(query, targets)``; ``sseqs_b200.sw`` also holds ``sw_affine_backtrack``
and the extension operators ``sw_cuda_blosum62`` / ``sw_cuda_affine``,
``sseqs_b200.xbit`` the codec and ``sseqs_b200.to_a3m`` the a3m writer.
"""
from .sw import sw  # noqa: F401


def __getattr__(name):
    if name in ("msa", "Database"):
        from . import msa as _m
        return getattr(_m, name)
    raise AttributeError(name)

"""sseqs_b200 -- the sseqs database-search path on NVIDIA B200 (sm_100a).

Drop-in for the reference's public calls (sseqs/__init__.py:1-2):
``msa(query, "out.a3m")`` and ``sw(query, targets)``.  As in the reference,
the package attributes ``msa`` and ``sw`` are the functions; the modules
``sseqs_b200.sw`` (``sw_affine_backtrack``, ``sw_cuda_blosum62``,
``sw_cuda_affine``), ``sseqs_b200.xbit``, ``sseqs_b200.conv`` and
``sseqs_b200.to_a3m`` hold the rest.
"""
from .msa import msa  # noqa: F401
from .sw import sw  # noqa: F401
from .database import Database  # noqa: F401

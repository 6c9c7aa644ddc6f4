"""physxcoopa_b200: B200 (sm_100a) XPBD cloth and hair-strand substep behind physxcoopa's
`cloth::solve_cloth` / `hair::solve_strands` boundary.

The product is the C-ABI shared library built from `physxcoopa_b200/csrc` (declared in
`include/physxcoopa_b200.h`). This Python package is a thin ctypes host over it: `runtime`
loads the library (and fails loudly if it is missing), `arrays` holds cloths and strand sets in
the reference's memory layout, `scenes` generates the seeded synthetic workloads.
"""
from . import _abi  # noqa: F401
from .arrays import ClothArrays, StrandArrays  # noqa: F401

__all__ = ["ClothArrays", "StrandArrays"]

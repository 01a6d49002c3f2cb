"""B200-native statFEM forward-and-conditioning path.

The product is the C-ABI library ``libstatfem_cuda.so`` (CUDA for sm_100a,
declared in include/statfem_cuda.h) plus the header-only C++ drop-ins in
include/corlib/.  ``statfem_b200.api`` is the Python mirror of the reference
interface bound to that library; ``statfem_b200.meshgen`` generates seeded
synthetic inputs; ``statfem_b200.build`` compiles the library in-tree.
"""
__all__ = ["api", "meshgen", "build"]

"""anukulan_b200 - a B200-native (sm_100a) PDHG / PDLP engine for linear
programming, a drop-in for the first-order LP path of anukulan.

The engine is ``libanu_pdhg.so`` (hand-written CUDA kernels behind the C ABI
declared in include/anu_pdhg.h). This package is the host-side mirror of the
reference's interface: ``PdhgOptions``-compatible options, ``solve_pdhg``,
``evaluate_residual``, ``estimate_matrix_norm``, the batched case stack, and
the data model and workload generators.
"""
from .model import Csr, Model, StandardLp, to_standard_form  # noqa: F401

__version__ = "0.1.0"

"""stenpy_b200 — a B200-native (sm_100a) fused executor for Stenpy-style stencil graphs.

Public API (same names and contracts as the reference's ``stenpy`` /
``stenpy_engine`` modules for the expression → graph → executor path):

* ``compile_expression``, ``parse_expression`` (+ ``compile_expressions``)
* ``Graph``, ``GraphNode``
* ``register_operator``, ``OP_REGISTRY``, ``OP_METADATA``
* ``Runtime`` (``run(graph, seed=None)``), ``MemoryManager``
* ``Pipeline`` / attribute dispatch (``stenpy_b200.laplacian("f")``) and the
  ``stenpy`` command line (``python -m stenpy_b200``)
* ``LazyPipeline`` / ``run_chunked`` — out-of-core execution of fields held in
  pinned host memory
* ``run_batch`` / ``BatchJob`` — many graphs over uneven fields in one persistent
  launch (``stenpy_b200.batch``)

Kernels are generated per graph and compiled with NVRTC for sm_100a; the C ABI is
``include/stenpy_b200.h`` (``libstenpy_b200.so``). There is no CPU execution path.
"""
from __future__ import annotations

from .graph import Graph, GraphNode, _uid
from .registry import OP_METADATA, OP_REGISTRY, register_operator
from . import spectral  # noqa: F401  (registers the FFT operators, run outside the fused passes)
from . import geometry  # noqa: F401  (registers distance_transform)
from .frontend import compile_expression, compile_expressions, parse_expression
from .memory_manager import MemoryManager
from .runtime import Runtime, run_single_op
from .codegen import PassConfig
from .pipeline import OperatorDispatch, PerfStats, Pipeline, load_tensor, save_tensor

__all__ = [
    "Graph", "GraphNode", "register_operator", "OP_REGISTRY", "OP_METADATA",
    "compile_expression", "compile_expressions", "parse_expression",
    "MemoryManager", "Runtime", "run_single_op", "PassConfig",
    "Pipeline", "PerfStats", "load_tensor", "save_tensor", "LazyPipeline", "run_chunked",
    "run_batch", "BatchJob",
]


def __getattr__(name: str):
    """``stenpy_b200.<op>(expr)`` → Pipeline, as the reference's module-level dispatch
    (stenpy.py:979-984); lazy imports for the heavier submodules."""
    if name in ("LazyPipeline", "run_chunked"):
        from . import lazy
        return getattr(lazy, name)
    if name in ("run_batch", "BatchJob"):
        from . import batch
        return getattr(batch, name)
    if name in OP_REGISTRY:
        return OperatorDispatch(name)
    raise AttributeError(f"module 'stenpy_b200' has no attribute {name!r}")

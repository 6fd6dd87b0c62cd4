"""Operator registry: ``register_operator`` / ``OP_REGISTRY`` / ``OP_METADATA``.

Same plugin contract as the reference (stenpy_engine.py:1184-1212): a name maps to a
callable taking tensors positionally plus params as keyword arguments (optionally
``alloc=`` and ``mm=``, injected by signature), and to a metadata dict with the
keys ``stencil_radius, halo_left, halo_right, cost, exchange_dims,
flops_per_element, bytes_read_per_element, bytes_written_per_element,
supports_fp64_fusion``.

Built-in operators are registered with callables that run a one-node graph
through the fused CUDA executor, so ``OP_REGISTRY["laplacian"](x, dx=1.0)`` works
on a CUDA tensor exactly like the reference's per-op call. Operators registered
by users are opaque to the code generator: the executor materialises their
inputs, calls them on the GPU tensors (as the reference's ``NormalNodeTask``,
fused_compiler.py:581-588, 683-703) and feeds their outputs to later passes.

``KNOWN_OPS`` is the code generator's catalogue: for each built-in, its kind
(pointwise / stencil / reduction / scan), the component shape it takes and
returns, and its interior stencil radius.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable, Dict, List, Optional, Tuple

OP_REGISTRY: Dict[str, Callable] = {}
OP_METADATA: Dict[str, dict] = {}


def register_operator(
    name: str,
    func: Callable,
    radius: int = 0,
    halo_l: int = 0,
    halo_r: int = 0,
    cost: str = "low",
    exchange_dims: Optional[List[int]] = None,
    flops: int = 0,
    bytes_in: int = 0,
    bytes_out: int = 0,
    fp64_fusion: bool = True,
) -> None:
    """Register ``func`` under ``name`` (signature of stenpy_engine.py:1188-1212)."""
    OP_REGISTRY[name] = func
    OP_METADATA[name] = {
        "stencil_radius": radius,
        "halo_left": halo_l if halo_l else radius,
        "halo_right": halo_r if halo_r else radius,
        "cost": cost,
        "exchange_dims": exchange_dims,
        "flops_per_element": flops,
        "bytes_read_per_element": bytes_in,
        "bytes_written_per_element": bytes_out,
        "supports_fp64_fusion": fp64_fusion,
    }


@dataclass(frozen=True)
class OpSpec:
    kind: str            # "const" | "pointwise" | "stencil" | "reduction" | "scan"
    radius: int = 0      # interior stencil radius
    onesided: bool = False  # uses torch.gradient-style one-sided edges somewhere


KNOWN_OPS: Dict[str, OpSpec] = {
    "_constant": OpSpec("const"),
    # elementwise (stenpy_engine.py:1228-1367)
    "add": OpSpec("pointwise"), "sub": OpSpec("pointwise"), "mul": OpSpec("pointwise"),
    "div": OpSpec("pointwise"), "neg": OpSpec("pointwise"), "clamp": OpSpec("pointwise"),
    "exp": OpSpec("pointwise"), "log": OpSpec("pointwise"), "sqrt": OpSpec("pointwise"),
    "sin": OpSpec("pointwise"), "cos": OpSpec("pointwise"), "tanh": OpSpec("pointwise"),
    "abs": OpSpec("pointwise"),
    # tensor epilogues (stenpy_engine.py:2674-2721, 2256-2259)
    "trace": OpSpec("pointwise"), "eigenvalues": OpSpec("pointwise"),
    "select_component": OpSpec("pointwise"),
    # per-voxel tensor and vector helpers (stenpy_engine.py:2247-2313, 2683-2730, 2852-2869)
    "determinant": OpSpec("pointwise"), "inverse": OpSpec("pointwise"), "deviatoric": OpSpec("pointwise"),
    "stack_components": OpSpec("pointwise"), "norm_last": OpSpec("pointwise"), "div_last": OpSpec("pointwise"),
    "neg_stack3": OpSpec("pointwise"), "scale_eye": OpSpec("pointwise"), "velocity_dot_grad": OpSpec("pointwise"),
    "matmul_batched_custom": OpSpec("pointwise"),
    # stencils (stenpy_engine.py:1466-2197)
    "laplacian": OpSpec("stencil", 1), "gradient": OpSpec("stencil", 1, True),
    "divergence": OpSpec("stencil", 1, True), "curl": OpSpec("stencil", 1, True),
    "hessian": OpSpec("stencil", 2, True), "mean_curvature": OpSpec("stencil", 2, True),
    "grad_mag": OpSpec("stencil", 1, True), "jacobian": OpSpec("stencil", 1, True),
    "material_derivative": OpSpec("stencil", 1, True), "surface_normals": OpSpec("stencil", 1, True),
    "gradient_nd": OpSpec("stencil", 1, True),
    # box and Gaussian smoothing (stenpy_engine.py:2385-2408, 2755-2860); the reach of
    # moving_average is window // 2
    "moving_average": OpSpec("stencil", 1), "conv3d_spectral": OpSpec("stencil", 1),
    # global reductions (stenpy_engine.py:2340-2459, 2546-2667)
    "sum": OpSpec("reduction"), "mean": OpSpec("reduction"), "norm_l2": OpSpec("reduction"),
    "variance": OpSpec("reduction"), "entropy": OpSpec("reduction"),
    "integrate": OpSpec("reduction"), "min_max": OpSpec("reduction"),
    "entropy_hist": OpSpec("reduction"), "surface_integral": OpSpec("reduction"),
    "covariance": OpSpec("reduction"), "correlation": OpSpec("reduction"),
    # running trapezoid along dim 0 (stenpy_engine.py:2462-2483)
    "cumulative_integral": OpSpec("scan"),
}

# Ops that take no dx/boundary parameters when compiled from an expression
# (stenpy_engine.py:3476-3484), extended with this executor's added ops.
NO_STENCIL_OPS = {
    "add", "sub", "mul", "div", "neg", "clamp", "exp", "log", "sqrt", "sin", "tanh",
    "sum", "mean", "norm_l2", "min_max", "variance", "entropy", "trace", "determinant",
    "eigenvalues", "inverse", "deviatoric", "fft", "ifft", "covariance", "correlation",
    "moving_average", "surface_integral", "distance_transform", "stack_components",
    "select_component", "norm_last", "div_last", "neg_stack3", "scale_eye",
    "velocity_dot_grad", "integrate", "cumulative_integral", "spectral_gradient",
    "spectral_laplacian",
    # added (conv3d_spectral accepts no dx: the reference's expression path passes one
    # and fails, here the op is reachable from expressions)
    "cos", "abs", "entropy_hist", "conv3d_spectral", "matmul_batched_custom",
}


def _gpu_op(name: str) -> Callable:
    """Callable for a built-in op: runs a one-node graph on the fused executor."""
    def op(*inputs: Any, alloc=None, mm=None, **params: Any):
        from .runtime import run_single_op
        return run_single_op(name, inputs, params)
    op.__name__ = name
    op.__qualname__ = name
    op.__doc__ = f"Built-in '{name}' run through the fused CUDA executor."
    return op


# name, radius, cost, flops, bytes_in, bytes_out (metadata values follow the
# reference's register_operator calls where it has the op)
_BUILTINS: List[Tuple[str, int, str, int, int, int]] = [
    ("add", 0, "low", 1, 16, 8), ("sub", 0, "low", 1, 16, 8), ("mul", 0, "low", 1, 16, 8),
    ("div", 0, "low", 1, 16, 8), ("neg", 0, "low", 1, 8, 8), ("clamp", 0, "low", 2, 8, 8),
    ("exp", 0, "medium", 8, 8, 8), ("log", 0, "medium", 8, 8, 8), ("sqrt", 0, "medium", 8, 8, 8),
    ("sin", 0, "medium", 8, 8, 8), ("cos", 0, "medium", 8, 8, 8), ("tanh", 0, "medium", 8, 8, 8),
    ("abs", 0, "low", 1, 8, 8),
    ("laplacian", 1, "high", 8, 56, 8), ("gradient", 1, "medium", 0, 0, 0),
    ("divergence", 1, "medium", 0, 0, 0), ("curl", 1, "high", 0, 0, 0),
    ("hessian", 2, "very_high", 0, 0, 0), ("mean_curvature", 2, "very_high", 0, 0, 0),
    ("grad_mag", 1, "medium", 0, 0, 0), ("jacobian", 1, "high", 0, 0, 0),
    ("material_derivative", 1, "high", 0, 0, 0), ("moving_average", 0, "medium", 0, 0, 0),
    ("conv3d_spectral", 0, "very_high", 2, 8, 8), ("surface_normals", 1, "high", 0, 0, 0),
    ("gradient_nd", 1, "high", 0, 0, 0), ("determinant", 0, "high", 0, 0, 0), ("inverse", 0, "very_high", 0, 0, 0),
    ("deviatoric", 0, "medium", 0, 0, 0), ("stack_components", 0, "low", 0, 0, 0), ("norm_last", 0, "low", 0, 0, 0),
    ("div_last", 0, "low", 0, 0, 0), ("neg_stack3", 0, "low", 0, 0, 0), ("scale_eye", 0, "low", 0, 0, 0),
    ("velocity_dot_grad", 0, "low", 0, 0, 0), ("surface_integral", 0, "medium", 0, 0, 0),
    ("matmul_batched_custom", 0, "high", 2, 8, 8), ("covariance", 0, "medium", 0, 0, 0),
    ("correlation", 0, "medium", 0, 0, 0),
    ("trace", 0, "low", 0, 0, 0), ("eigenvalues", 0, "very_high", 0, 0, 0),
    ("select_component", 0, "low", 0, 0, 0),
    ("sum", 0, "low", 0, 0, 0), ("mean", 0, "low", 0, 0, 0), ("norm_l2", 0, "low", 0, 0, 0),
    ("variance", 0, "low", 0, 0, 0), ("entropy", 0, "medium", 0, 0, 0),
    ("integrate", 0, "medium", 0, 0, 0), ("min_max", 0, "low", 0, 0, 0),
    ("entropy_hist", 0, "medium", 0, 0, 0),
    ("cumulative_integral", 0, "low", 0, 0, 0),
]

_EXCHANGE_DIMS = {"laplacian": [0], "gradient": [0], "divergence": [0]}


def _register_builtins() -> None:
    from .ops_constant import constant
    register_operator("_constant", constant, cost="low", flops=0, bytes_in=0, bytes_out=8)
    for name, r, cost, fl, bi, bo in _BUILTINS:
        register_operator(name, _gpu_op(name), radius=r, cost=cost,
                          exchange_dims=_EXCHANGE_DIMS.get(name), flops=fl,
                          bytes_in=bi, bytes_out=bo)


_register_builtins()

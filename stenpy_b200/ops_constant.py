"""The ``_constant`` leaf operator.

The reference upcasts every constant to FP64 (stenpy_engine.py:1218-1223). Here a
tensor keeps its storage dtype (FP32 / BF16 / FP16 / FP64): the fused executor
reads it in that dtype and computes in FP32. Plain numbers become 0-d FP64
tensors, as in the reference.
"""
from __future__ import annotations

import torch


def constant(*, value):
    if isinstance(value, bool):
        raise TypeError("_constant: bool is not a numeric field value")
    if isinstance(value, (int, float)):
        return torch.tensor(float(value), dtype=torch.float64)
    if not isinstance(value, torch.Tensor):
        raise TypeError(f"_constant: expected torch.Tensor or number, got {type(value).__name__}")
    return value

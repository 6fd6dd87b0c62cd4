"""Allocation contract of the reference's ``MemoryManager`` (memory_manager.py:219-568).

Operators may take ``alloc=`` (``mm.allocate(shape, device, key=..., dtype=...)``)
and ``mm=``; the runtime injects them by signature (stenpy_engine.py:1074-1080). This
class keeps that contract on top of PyTorch's caching allocator, with a small
per-(shape, dtype, device) reuse pool like the reference's. The reference's zict
host/disk spill tiers are not part of the GPU hot path and are not reproduced;
fields larger than a device budget go through the lazy chunk pipeline instead
(``stenpy_b200.lazy``). ``halo_exchange`` / ``all_reduce_sum`` are identities: the
executor runs on one GPU.
"""
from __future__ import annotations

import collections
import math
import threading
from typing import Dict, List, Optional, Tuple

import torch

from .graph import _uid


class MemoryManager:
    def __init__(self, pool_depth: int = 4, pool_max_mb: float = 256.0, budget_bytes: Optional[int] = None):
        self._lock = threading.RLock()
        self._live: Dict[str, torch.Tensor] = {}
        self._pool: Dict[Tuple, List[torch.Tensor]] = collections.defaultdict(list)
        self._pool_depth = pool_depth
        self._pool_max_bytes = pool_max_mb * 1024 ** 2
        self.budget_bytes = budget_bytes

    def should_manage(self, shape) -> bool:
        return math.prod(tuple(shape)) >= 1024

    def get_buffer(self, shape, dtype=torch.float64, device=torch.device("cpu"), key=None,
                   layout=torch.contiguous_format) -> torch.Tensor:
        shape = tuple(shape)
        key = key or _uid("buf")
        with self._lock:
            if key in self._live:
                t = self._live[key]
                if tuple(t.shape) != shape or t.dtype != dtype:
                    raise KeyError(f"get_buffer: key '{key}' is live with shape {tuple(t.shape)} {t.dtype}")
                return t
            pool = self._pool.get((shape, str(device), dtype))
            t = pool.pop().zero_() if pool else None
        if t is None:
            nbytes = math.prod(shape) * torch.empty((), dtype=dtype).element_size()
            if self.budget_bytes is not None and nbytes > self.budget_bytes:
                raise MemoryError(f"Refusing to allocate {nbytes / 1e9:.3f} GB: budget is "
                                  f"{self.budget_bytes / 1e9:.3f} GB")
            t = torch.zeros(shape, dtype=dtype, device=device)
        with self._lock:
            self._live[key] = t
        t._mm_key = key
        return t

    def allocate(self, shape, device, key=None, layout=torch.contiguous_format, dtype=torch.float64):
        return self.get_buffer(shape, dtype=dtype, device=torch.device(device), key=key, layout=layout)

    def adopt(self, tensor: torch.Tensor, key: Optional[str] = None) -> torch.Tensor:
        k = key or _uid("adopt")
        with self._lock:
            self._live[k] = tensor
        tensor._mm_key = k
        return tensor

    def owns(self, tensor) -> bool:
        key = getattr(tensor, "_mm_key", None)
        return key is not None and key in self._live

    def release(self, tensor: torch.Tensor, key: Optional[str] = None) -> None:
        key = getattr(tensor, "_mm_key", key)
        with self._lock:
            t = self._live.pop(key, None)
            if t is None:
                return
            nbytes = t.numel() * t.element_size()
            if t.is_contiguous() and nbytes <= self._pool_max_bytes:
                pool = self._pool[(tuple(t.shape), str(t.device), t.dtype)]
                if len(pool) < self._pool_depth:
                    pool.append(t)

    def clear_pool(self, full: bool = False) -> None:
        with self._lock:
            self._pool.clear()
            if full:
                self._live.clear()

    def halo_exchange(self, tensor, radius, dims=None):
        return tensor

    def all_reduce_sum(self, tensor):
        return tensor

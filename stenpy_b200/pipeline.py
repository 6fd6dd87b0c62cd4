"""User API: ``Pipeline``, per-operator dispatch, field I/O and the perf report.

Mirrors the reference's ``stenpy`` module surface (stenpy.py:621-984):

* ``Pipeline(op_name, expr)`` is configured by attribute assignment — settings
  ``stream_i, stream_o, device, log, perf_report, output, boundary, dx, chunk_mb``;
  other string attributes are field paths, other values are constants — and
  setting ``.output`` runs it (stenpy.py:657-669); ``.value`` / ``run()`` return
  the result. Boundary defaults to periodic as in the reference Pipeline.
* ``stenpy_b200.<op>(expr, **settings)`` returns a Pipeline (the op name is a
  label, the expression is what runs), like ``_OperatorDispatch`` (stenpy.py:955-984).
* ``load_tensor`` / ``save_tensor`` read and write ``.npy`` / ``.npz`` / ``.pt``
  files (field + spacing + origin). The reference's HDF5 format needs h5py,
  which is not part of this environment; ``.h5`` paths raise a clear error.

Differences: the device defaults to ``cuda`` and there is no CPU execution path;
``stream_i``/``stream_o`` select the lazy chunk pipeline (``LazyPipeline``) over
pinned host memory instead of HDF5 streaming.
"""
from __future__ import annotations

import math
import os
import time
from typing import Any, Dict, Optional, Tuple

import numpy as np
import torch

from .frontend import compile_expression
from .graph import Graph
from .registry import OP_REGISTRY
from .runtime import Runtime

_KNOWN_SETTINGS = {"stream_i", "stream_o", "device", "log", "perf_report", "output", "boundary", "dx",
                   "chunk_mb", "dtype"}


def load_tensor(path: str, device: Any = "cpu", return_mode: str = "eager",
                dtype: Optional[torch.dtype] = None) -> Tuple[torch.Tensor, Tuple[float, ...], Tuple[float, ...]]:
    """Load ``(field, spacing, origin)``. ``.npy``: array only; ``.npz``: keys
    ``field`` (or ``data``), optional ``spacing``/``origin``; ``.pt``: a tensor or a
    dict with the same keys. The file's dtype is kept unless ``dtype`` is given
    (the reference forces FP64)."""
    ext = os.path.splitext(path)[1].lower()
    spacing = origin = None
    if ext in (".h5", ".hdf5"):
        raise RuntimeError(f"{path}: HDF5 needs h5py, which is not installed here; "
                           "convert the field to .npy/.npz/.pt")
    if ext == ".npy":
        arr = torch.from_numpy(np.load(path))
    elif ext == ".npz":
        z = np.load(path)
        key = "field" if "field" in z else ("data" if "data" in z else list(z.keys())[0])
        arr = torch.from_numpy(z[key])
        spacing = tuple(float(v) for v in z["spacing"]) if "spacing" in z else None
        origin = tuple(float(v) for v in z["origin"]) if "origin" in z else None
    elif ext in (".pt", ".pth"):
        obj = torch.load(path, map_location="cpu", weights_only=True)
        if isinstance(obj, dict):
            arr = obj.get("field", obj.get("data"))
            spacing = tuple(float(v) for v in obj["spacing"]) if "spacing" in obj else None
            origin = tuple(float(v) for v in obj["origin"]) if "origin" in obj else None
        else:
            arr = obj
    else:
        raise ValueError(f"{path}: unsupported field file type '{ext}' (use .npy, .npz or .pt)")
    if dtype is not None:
        arr = arr.to(dtype)
    nd = max(1, min(arr.ndim, 3))
    spacing = spacing or (1.0,) * nd
    origin = origin or (0.0,) * len(spacing)
    if return_mode == "lazy":
        return arr.pin_memory(), spacing, origin
    dev = torch.device(device)
    return (arr.to(dev) if dev.type == "cuda" else arr), spacing, origin


def save_tensor(tensor: torch.Tensor, spacing, origin, path: str) -> None:
    """Write ``field``/``spacing``/``origin`` (``.npz``) or the bare array (``.npy``/``.pt``)."""
    t = tensor.detach().cpu()
    ext = os.path.splitext(path)[1].lower()
    if ext == ".npz":
        np.savez(path, field=t.float().numpy() if t.dtype == torch.bfloat16 else t.numpy(),
                 spacing=np.asarray(spacing, dtype=np.float64), origin=np.asarray(origin, dtype=np.float64))
    elif ext == ".npy":
        np.save(path, t.float().numpy() if t.dtype == torch.bfloat16 else t.numpy())
    elif ext in (".pt", ".pth"):
        torch.save({"field": t, "spacing": list(spacing), "origin": list(origin)}, path)
    else:
        raise ValueError(f"{path}: unsupported output type '{ext}'")


class PerfStats:
    """Wall-clock timing plus bytes moved (stenpy.py:355-380)."""

    def __init__(self) -> None:
        self.t0 = self.t1 = None
        self.bytes_read = 0
        self.bytes_written = 0
        self.n_chunks = 0

    def start(self) -> None:
        self.t0 = time.perf_counter()

    def stop(self) -> None:
        self.t1 = time.perf_counter()

    @property
    def elapsed_s(self) -> float:
        if self.t0 is None:
            return 0.0
        return (self.t1 or time.perf_counter()) - self.t0

    def bandwidth_gbps(self) -> float:
        return (self.bytes_read + self.bytes_written) / 1024 ** 3 / max(self.elapsed_s, 1e-9)


def print_perf_report(stats: PerfStats, op_name: str, device: str) -> None:
    print("--- stenpy_b200 perf report ---\n"
          f"  op        : {op_name}\n  device    : {device}\n  elapsed   : {stats.elapsed_s:.4f} s\n"
          f"  bandwidth : {stats.bandwidth_gbps():.3f} GiB/s\n  chunks    : {stats.n_chunks}")


class Pipeline:
    def __init__(self, op_name: str, expr_str: str) -> None:
        object.__setattr__(self, "_op_name", op_name)
        object.__setattr__(self, "_expr_str", expr_str)
        for k, v in dict(stream_i=False, stream_o=False, device="cuda", chunk_mb=None, log=True,
                         perf_report=False, boundary="periodic", dx=1.0, dtype=None, output=None,
                         result=None, ran=False, field_paths={}, constants={}).items():
            object.__setattr__(self, f"_{k}", v if not isinstance(v, dict) else dict(v))

    def __setattr__(self, name: str, value: Any) -> None:
        if name in _KNOWN_SETTINGS:
            object.__setattr__(self, f"_{name}", value)
            if name == "output":
                self.run()
            return
        if name.startswith("_"):
            object.__setattr__(self, name, value)
            return
        if isinstance(value, str):
            self._field_paths[name] = value
        elif isinstance(value, torch.Tensor) and value.ndim >= 3:
            self._field_paths[name] = value
        else:
            self._constants[name] = value

    def set(self, **kwargs) -> "Pipeline":
        for k, v in kwargs.items():
            setattr(self, k, v)
        return self

    def run(self) -> Any:
        if self._ran:
            return self._result
        object.__setattr__(self, "_ran", True)
        stats = PerfStats()
        stats.start()
        dev = torch.device(self._device)
        lazy = bool(self._stream_i or self._stream_o)
        fmap: Dict[str, Any] = {}
        spacing, origin = (1.0,) * 3, (0.0,) * 3
        for name, src in self._field_paths.items():
            if isinstance(src, torch.Tensor):
                t = src
            else:
                t, spacing, origin = load_tensor(src, device="cpu" if lazy else dev,
                                                 return_mode="lazy" if lazy else "eager", dtype=self._dtype)
            fmap[name] = t
            stats.bytes_read += t.numel() * t.element_size()
        for name, val in self._constants.items():
            fmap.setdefault(name, torch.tensor(float(val), dtype=torch.float64))
        g, sink, warns, _, _ = compile_expression(self._expr_str, dx=self._dx, boundary=self._boundary,
                                                  field_map=fmap)
        out_dtype = self._dtype or torch.float32
        if lazy:
            from .lazy import LazyPipeline
            budget = int(self._chunk_mb * 1024 ** 2 * 6) if self._chunk_mb else 8 << 30
            lp = LazyPipeline(g, [sink], dev, budget_bytes=budget, out_dtype=out_dtype)
            out = lp.run()[sink]
            stats.n_chunks = len(lp.passes[0]["chunks"]) if lp.passes else 0
        else:
            out = Runtime(device=dev, out_dtype=out_dtype).run(g, wanted=[sink])[sink]
        if isinstance(out, torch.Tensor):
            stats.bytes_written += out.numel() * out.element_size()
        if self._output:
            save_tensor(out, spacing, origin, self._output)
        object.__setattr__(self, "_result", out)
        stats.stop()
        if self._perf_report:
            print_perf_report(stats, self._op_name, str(dev))
        return out

    @property
    def value(self) -> Any:
        return self.run()

    def __getitem__(self, idx):
        return self.run()[idx]

    def __repr__(self) -> str:
        if self._ran:
            return f"Pipeline({self._op_name}, result={type(self._result).__name__})"
        return f"Pipeline({self._op_name}({self._expr_str}), unconfigured)"


class OperatorDispatch:
    """``stenpy_b200.<op>(expr, **settings)`` → Pipeline (stenpy.py:955-966)."""

    def __init__(self, op_name: str) -> None:
        self._op_name = op_name

    def __call__(self, expr, *args, **kwargs) -> Pipeline:
        p = Pipeline(self._op_name, expr if isinstance(expr, str) else str(expr))
        if kwargs:
            p.set(**kwargs)
        return p

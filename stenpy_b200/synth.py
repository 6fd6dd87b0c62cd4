"""Seeded synthetic fields with the shapes and value distributions of the
reference's benchmark configurations (the reference ships no datasets).

* ``sinusoid_field``: sum of 3 sinusoids, each wavevector component drawn
  uniformly from [1, 8]·2π/128 per axis, random phase in [0, 2π), plus Gaussian
  noise of standard deviation 0.01.
* ``uniform_field``: U[lo, hi].
* ``smoothed_vector``: 3 components, each N(0, 1) smoothed by a 5-point box filter
  (a 5-tap mean along each axis in turn, periodic wrap), stored channels-last
  ``(*shape, 3)`` as the reference's vector layout.
* ``batch_specs`` / ``batch_fields``: the batched workload — independent fields,
  each dimension uniform in [lo, hi], a seeded 60/40 FP32/BF16 split, each field
  with one of eight expressions (field i gets expression i mod 8); the curl
  expression takes a 3-component field whose components are sinusoid fields.

Generation runs with torch on the requested device (FP64 on the CPU, FP32 on a
GPU, where 512³ fields would take minutes with numpy); parameters come from
``numpy.random.default_rng(seed)`` so both agree to FP32 rounding.
"""
from __future__ import annotations

import math
from typing import Sequence, Tuple

import numpy as np
import torch


def _grid_axes(shape: Sequence[int], device, dtype):
    n0, n1, n2 = shape
    i = torch.arange(n0, device=device, dtype=dtype).view(-1, 1, 1)
    j = torch.arange(n1, device=device, dtype=dtype).view(1, -1, 1)
    k = torch.arange(n2, device=device, dtype=dtype).view(1, 1, -1)
    return i, j, k


def sinusoid_field(shape: Sequence[int], seed: int = 0, device="cpu",
                   dtype: torch.dtype = torch.float32, noise: float = 0.01) -> torch.Tensor:
    rng = np.random.default_rng(seed)
    dev = torch.device(device)
    work = torch.float64 if dev.type == "cpu" else torch.float32
    i, j, k = _grid_axes(shape, dev, work)
    out = torch.zeros(tuple(shape), device=dev, dtype=work)
    for _ in range(3):
        kv = rng.uniform(1.0, 8.0, size=3) * (2.0 * math.pi / 128.0)
        phi = rng.uniform(0.0, 2.0 * math.pi)
        out += torch.sin(float(kv[0]) * i + float(kv[1]) * j + float(kv[2]) * k + float(phi))
    gen = torch.Generator(device=dev).manual_seed(int(rng.integers(0, 2**31 - 1)))
    out += noise * torch.randn(tuple(shape), generator=gen, device=dev, dtype=work)
    return out.to(dtype)


def uniform_field(shape: Sequence[int], seed: int = 1, device="cpu",
                  dtype: torch.dtype = torch.float32, lo: float = -1.0, hi: float = 1.0) -> torch.Tensor:
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(int(seed))
    work = torch.float64 if dev.type == "cpu" else torch.float32
    out = torch.rand(tuple(shape), generator=gen, device=dev, dtype=work)
    return (lo + (hi - lo) * out).to(dtype)


def _box5_periodic(x: torch.Tensor, axis: int) -> torch.Tensor:
    acc = torch.zeros_like(x)
    for s in (-2, -1, 0, 1, 2):
        acc += torch.roll(x, s, axis)
    return acc / 5.0


def smoothed_vector(shape: Sequence[int], seed: int = 2, device="cpu",
                    dtype: torch.dtype = torch.float32) -> torch.Tensor:
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(int(seed))
    work = torch.float64 if dev.type == "cpu" else torch.float32
    out = torch.empty(tuple(shape) + (3,), device=dev, dtype=dtype)
    for c in range(3):
        comp = torch.randn(tuple(shape), generator=gen, device=dev, dtype=work)
        for ax in range(3):
            comp = _box5_periodic(comp, ax)
        out[..., c] = comp.to(dtype)
        del comp
    return out


BATCH_EXPRESSIONS = (
    "laplacian(f)", "grad_mag(f)", "curl(f)", "f**2 + tanh(f)*exp(f)", "clamp(log(abs(f) + 1), 0, 2)",
    "trace(hessian(f))", "integrate(f)", "entropy_hist(f, bins=256)",
)


def batch_specs(n: int = 256, seed: int = 0, lo: int = 32, hi: int = 320,
                bf16_frac: float = 0.4) -> list:
    """[(expression, storage dtype, shape, field seed)] for ``n`` independent fields."""
    rng = np.random.default_rng(seed)
    dims = rng.integers(lo, hi + 1, size=(n, 3))
    n_bf16 = int(round(bf16_frac * n))
    is_bf16 = np.zeros(n, dtype=bool)
    is_bf16[rng.permutation(n)[:n_bf16]] = True
    out = []
    for i in range(n):
        dt = torch.bfloat16 if is_bf16[i] else torch.float32
        out.append((BATCH_EXPRESSIONS[i % len(BATCH_EXPRESSIONS)], dt, tuple(int(d) for d in dims[i]),
                    int(seed) * 100003 + i))
    return out


def batch_field(expr: str, dtype: torch.dtype, shape: Sequence[int], seed: int, device="cpu") -> torch.Tensor:
    """The input field of one batched job (3 components for the curl expression)."""
    if expr.startswith("curl"):
        comps = [sinusoid_field(shape, seed=seed * 3 + c, device=device, dtype=torch.float32) for c in range(3)]
        return torch.stack(comps, dim=-1).to(dtype).contiguous()
    return sinusoid_field(shape, seed=seed, device=device, dtype=dtype)

"""Spectral operators: FFTs and Fourier-space derivatives, on the GPU (cuFFT through
``torch.fft``), outside the fused stencil passes.

Same names, signatures and results as the reference's spectral operators
(stenpy_engine.py:2875-3012): ``fft`` / ``ifft`` (n-D transforms of the whole field;
``fft`` returns complex128, ``ifft`` the real part in FP64), ``fft_complex`` /
``ifft_complex`` (complex in, complex out), ``spectral_gradient`` (∂/∂x_dim as
ifft(i·k_dim·fft(t)), real part) and ``spectral_laplacian`` (ifft(−|k|²·fft(t))),
with k = 2π·fftfreq(n, dx) per axis — periodic by construction. Like the reference
they compute in FP64 (complex128): inputs stored in FP32, FP16 or BF16 are widened
first. The graph runtime treats them as opaque nodes: their inputs come from the
fused executor, their outputs feed later fused passes as FP64 fields. CUDA tensors
only; there is no CPU path.
"""
from __future__ import annotations

import math
from typing import Any, Sequence, Tuple, Union

import torch

from .registry import register_operator


def _cuda(t: Any, op: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise ValueError(f"{op}: needs a CUDA tensor (there is no CPU path)")
    return t


def _real64(t: torch.Tensor) -> torch.Tensor:
    return t if t.dtype == torch.float64 else t.to(torch.float64)


def _spacing(dx: Union[float, Sequence[float]], ndim: int, op: str) -> Tuple[float, ...]:
    if isinstance(dx, (int, float)):
        return (float(dx),) * ndim
    d = tuple(float(v) for v in dx)
    if len(d) != ndim:
        raise ValueError(f"{op}: dx needs {ndim} values, got {len(d)}")
    return d


def _wavenumbers(shape: Sequence[int], dx: Tuple[float, ...], device: torch.device):
    """Angular wavenumbers 2π·fftfreq(n, dx) per axis, shaped to broadcast. The
    frequencies are rounded to FP32 before widening, as the reference forms them
    (fftfreq in torch's default dtype), so results agree to FP64 rounding."""
    ks = []
    for d, (n, h) in enumerate(zip(shape, dx)):
        k = torch.fft.fftfreq(n, d=h, device=device, dtype=torch.float32).to(torch.float64) * (2.0 * math.pi)
        sh = [1] * len(shape)
        sh[d] = -1
        ks.append(k.view(sh))
    return ks


def fft(t: torch.Tensor, norm: str = "backward", alloc=None) -> torch.Tensor:
    """n-D FFT of the whole field, complex128 (stenpy_engine.py:2875-2885). Called with
    ``alloc`` — as the graph runtime calls it — the reference copies the transform into
    the real FP64 buffer ``alloc`` returns, which keeps the real part only; that is the
    value a graph node gets there, and here."""
    t = _cuda(t, "fft")
    out = torch.fft.fftn(t if t.is_complex() else t.to(torch.complex128), norm=norm)
    return out.real.to(torch.float64).contiguous() if alloc is not None else out


def ifft(t: torch.Tensor, norm: str = "backward", alloc=None) -> torch.Tensor:
    """Real part of the n-D inverse FFT, FP64 (stenpy_engine.py:2887-2896)."""
    t = _cuda(t, "ifft")
    x = t.to(torch.complex128) if t.is_complex() else torch.complex(_real64(t), torch.zeros_like(_real64(t)))
    return torch.fft.ifftn(x, norm=norm).real.contiguous()


def fft_complex(t: torch.Tensor, norm: str = "backward", alloc=None) -> torch.Tensor:
    """n-D FFT, complex out; ``numpy_compatible`` means ``backward``
    (stenpy_engine.py:2901-2908)."""
    t = _cuda(t, "fft_complex")
    return torch.fft.fftn(t if t.is_complex() else _real64(t), norm="backward" if norm == "numpy_compatible" else norm)


def ifft_complex(t: torch.Tensor, norm: str = "backward", alloc=None) -> torch.Tensor:
    """n-D inverse FFT, complex out (stenpy_engine.py:2910-2918)."""
    t = _cuda(t, "ifft_complex")
    x = t if t.is_complex() else torch.complex(_real64(t), torch.zeros_like(_real64(t)))
    return torch.fft.ifftn(x, norm="backward" if norm == "numpy_compatible" else norm)


def spectral_gradient(t: torch.Tensor, dx: Union[float, Sequence[float]] = 1.0, dim: int = 0,
                      norm: str = "backward", alloc=None) -> torch.Tensor:
    """∂t/∂x_dim = Re ifft(i·k_dim·fft(t)), FP64 (stenpy_engine.py:2980-2993)."""
    t = _real64(_cuda(t, "spectral_gradient"))
    k = _wavenumbers(t.shape, _spacing(dx, t.ndim, "spectral_gradient"), t.device)
    th = torch.fft.fftn(t, norm=norm)
    return torch.fft.ifftn(1j * k[int(dim)] * th, norm=norm).real.contiguous()


def spectral_laplacian(t: torch.Tensor, dx: Union[float, Sequence[float]] = 1.0, norm: str = "backward",
                       alloc=None) -> torch.Tensor:
    """∇²t = Re ifft(−|k|²·fft(t)), FP64 (stenpy_engine.py:2998-3010)."""
    t = _real64(_cuda(t, "spectral_laplacian"))
    k = _wavenumbers(t.shape, _spacing(dx, t.ndim, "spectral_laplacian"), t.device)
    k2 = sum(kk * kk for kk in k)
    th = torch.fft.fftn(t, norm=norm)
    return torch.fft.ifftn(-k2 * th, norm=norm).real.contiguous()


for _name, _fn in (("fft", fft), ("ifft", ifft), ("fft_complex", fft_complex), ("ifft_complex", ifft_complex),
                   ("spectral_gradient", spectral_gradient), ("spectral_laplacian", spectral_laplacian)):
    register_operator(_name, _fn, cost="high")

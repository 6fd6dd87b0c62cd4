"""CPU FP64 oracle for the fused stencil-graph executor — TEST INFRASTRUCTURE ONLY.

This module is the correctness checker. Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / ``--impl reference`` leg may import it; the
product package (``stenpy_b200``) never imports or calls it and has no CPU
fallback.

It restates, in float64 on the CPU with the same torch primitives, the
reference's eager CPU path (``Runtime._run_original`` with ``device="cpu"``,
stenpy_engine.py:983-1146) for every operator on the hot path. Each function
cites the reference lines it follows. It is pinned against golden vectors that
``tests/golden/make_golden.py`` generated by running the reference itself
(``tests/test_oracle_golden.py``).

Operators the reference does not have (``abs``, ``grad_mag``, ``entropy_hist``)
are restated from their definitions here; their parity is unpinned by the
reference.

Graphs are duck-typed: anything with ``topological_sort()`` returning nodes with
``id, op_name, input_ids, params`` (the ``Graph`` of either implementation).
"""
from __future__ import annotations

import math
from typing import Any, Callable, Dict, Iterable, Optional, Sequence, Tuple, Union

import torch
import torch.nn.functional as F

F64 = torch.float64


def _f64(x: Any) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.detach().to("cpu", F64)
    return torch.tensor(float(x), dtype=F64)


def _dx_tuple(dx: Any, n: int) -> Tuple[float, ...]:
    if isinstance(dx, (int, float)):
        return (float(dx),) * n
    dx = tuple(float(v) for v in dx)
    if len(dx) != n:
        raise ValueError(f"dx must have {n} entries, got {len(dx)}")
    return dx


# ---------------------------------------------------------------- elementwise
# stenpy_engine.py:1228-1367
def add(a, b): return a + b
def sub(a, b): return a - b
def neg(a): return -a


def mul(a, b=None, scalar=None):
    if b is None:
        if scalar is None:
            raise ValueError("mul: need b or scalar")
        b = torch.full_like(a, float(scalar))
    return a * b


def div(a, b, eps: float = 1e-15):
    """Divisor with |b| < eps replaced by ±eps (stenpy_engine.py:1263-1279)."""
    e = torch.as_tensor(eps, dtype=F64)
    b_safe = torch.where(b.abs() < e, torch.where(b < 0, -e, e), b)
    return a / b_safe


def clamp(a, lo=0.0, hi=1.0):
    """torch.clamp with defaults lo=0, hi=1 (stenpy_engine.py:1292-1302)."""
    return torch.clamp(a, lo, hi)


def exp(a): return torch.exp(a)
def log(a, eps: float = 1e-15): return torch.log(a.clamp(min=eps))      # :1321-1326
def sqrt(a, eps: float = 0.0): return torch.sqrt(a.clamp(min=eps))      # :1331-1336
def sin(a): return torch.sin(a)
def cos(a): return torch.cos(a)
def tanh(a): return torch.tanh(a)
def abs_(a): return a.abs()  # not in the reference


# ---------------------------------------------------------------- stencils
def _pad1d(t: torch.Tensor, dim: int, r: int, bc: str) -> torch.Tensor:
    """Pad ``r`` cells on both sides of ``dim`` (stenpy_engine.py:1374-1416):
    neumann → replicate, dirichlet → zeros, periodic → wrap, reflect → mirror
    without repeating the edge; any other name pads with zeros."""
    n = t.shape[dim]
    idx = torch.arange(-r, n + r)
    if bc == "neumann":
        src = idx.clamp(0, n - 1)
    elif bc == "periodic":
        src = idx % n
    elif bc == "reflect" and n > 1:
        # the reference's r=1 mirror: index -1 → 1, n → n-2
        src = torch.where(idx < 0, (-idx).clamp(max=n - 1), idx)
        src = torch.where(src > n - 1, (2 * (n - 1) - src).clamp(min=0), src)
    else:
        out_shape = list(t.shape)
        out_shape[dim] = n + 2 * r
        out = torch.zeros(out_shape, dtype=t.dtype)
        out.narrow(dim, r, n).copy_(t)
        return out
    return t.index_select(dim, src)


def laplacian(x, dx=1.0, boundary="periodic"):
    """Compact 7-point Laplacian, Σ_d (x₊ + x₋ − 2x)/dx_d² (stenpy_engine.py:1466-1519):
    periodic uses torch.roll; other modes pad by ``_pad1d``."""
    d = _dx_tuple(dx, x.ndim)
    out = torch.zeros_like(x)
    for ax in range(x.ndim):
        if boundary == "periodic":
            xp, xm = torch.roll(x, -1, ax), torch.roll(x, 1, ax)
        else:
            p = _pad1d(x, ax, 1, boundary)
            n = x.shape[ax]
            xp, xm = p.narrow(ax, 2, n), p.narrow(ax, 0, n)
        out += (xp + xm - 2.0 * x) / (d[ax] ** 2)
    return out


def _tgrad(t: torch.Tensor, h: float, ax: int, order: int = 2) -> torch.Tensor:
    return torch.gradient(t, spacing=h, dim=ax, edge_order=order)[0]


def gradient(t, dx=1.0, boundary="neumann", dim=None):
    """Central differences; periodic via torch.roll, otherwise torch.gradient with
    second-order one-sided edges (first order below 3 points)
    (stenpy_engine.py:1780-1867, CPU branch)."""
    h = _dx_tuple(dx, t.ndim)

    def one(ax):
        if t.shape[ax] == 1:
            return torch.zeros_like(t)
        if boundary == "periodic":
            return (torch.roll(t, -1, ax) - torch.roll(t, 1, ax)) / (2.0 * h[ax])
        return _tgrad(t, h[ax], ax, 2 if t.shape[ax] >= 3 else 1)

    if dim is not None:
        return one(int(dim))
    return torch.stack([one(ax) for ax in range(t.ndim)], dim=-1)


def divergence(t, dx=1.0, boundary="neumann"):
    """Σ_d ∂_d t[..., d] with gradient's conventions, but always edge order 2 off
    the periodic branch (stenpy_engine.py:1870-1933, CPU branch)."""
    D = t.shape[-1]
    h = _dx_tuple(dx, D)
    out = torch.zeros_like(t[..., 0])
    for ax in range(D):
        c = t[..., ax]
        if boundary == "periodic":
            out += (torch.roll(c, -1, ax) - torch.roll(c, 1, ax)) / (2.0 * h[ax])
        else:
            out += _tgrad(c, h[ax], ax, 2)
    return out


def curl(t, dx=1.0, boundary="neumann"):
    """3-D curl from torch.gradient (edge order 2) of each component; the boundary
    argument is ignored on this path (stenpy_engine.py:1936-2034, CPU branch)."""
    D = t.ndim - 1
    h = _dx_tuple(dx, D)
    if D == 3:
        g = [torch.gradient(t[..., c], spacing=h, edge_order=2) for c in range(3)]
        return torch.stack([g[2][1] - g[1][2], g[0][2] - g[2][0], g[1][0] - g[0][1]], dim=-1)
    if D == 2:
        g0 = torch.gradient(t[..., 0], spacing=h, edge_order=2)
        g1 = torch.gradient(t[..., 1], spacing=h, edge_order=2)
        return g1[0] - g0[1]
    raise ValueError("curl: only 2-D or 3-D vector fields")


def gradient_nd(t, dx=1.0, boundary="neumann", dim=None):
    """torch.gradient over all axes, edge order 2 when every axis has ≥3 points,
    boundary ignored (stenpy_engine.py:2037-2083)."""
    order = 2 if min(t.shape) >= 3 else 1
    h = _dx_tuple(dx, t.ndim)
    return torch.stack(torch.gradient(t, spacing=h, edge_order=order), dim=-1)


def hessian(t, dx=1.0, boundary="neumann"):
    """H[..., i, :] = gradient_nd(gradient_nd(t)[..., i]) (stenpy_engine.py:2086-2130):
    the diagonal is the wide (f₊₂ − 2f + f₋₂)/(4dx²) stencil in the interior."""
    g = gradient_nd(t, dx)
    return torch.stack([gradient_nd(g[..., i], dx) for i in range(t.ndim)], dim=-2)


def jacobian(t, dx=1.0, boundary="neumann"):
    """J[..., i, d] = ∂_d t[..., i] via gradient_nd (stenpy_engine.py:2133-2177)."""
    return torch.stack([gradient_nd(t[..., i], dx) for i in range(t.shape[-1])], dim=-2)


def mean_curvature(t, dx=1.0, boundary="neumann", eps: float = 1e-15):
    """div(∇f / max(|∇f|, eps)) with ∇ = gradient_nd and the divergence honouring
    ``boundary`` (stenpy_engine.py:2180-2197)."""
    h = _dx_tuple(dx, t.ndim)
    g = gradient_nd(t, h)
    mag = torch.linalg.norm(g, dim=-1, keepdim=True).clamp(min=eps)
    return divergence(g / mag, dx=h, boundary=boundary)


def material_derivative(t, velocity, dx=1.0, boundary="neumann"):
    """Σ_d velocity[..., d] · ∂_d t with ∂ = gradient_nd, accumulated from zero in
    axis order (stenpy_engine.py:2223-2244)."""
    g = gradient_nd(t, dx)
    out = torch.zeros_like(t)
    for d in range(t.ndim):
        out = out + velocity[..., d] * g[..., d]
    return out


def moving_average(t, window: int = 3, boundary: str = "neumann"):
    """Mean over ``window`` cells along each axis in turn (axis 0 first), each axis
    padded by ``window // 2`` cells with ``_pad1d``'s rule (stenpy_engine.py:2385-2408).
    Even windows change the length and the reference fails; so does this."""
    if t.ndim > 3:
        raise NotImplementedError("moving_average: only 1-D/2-D/3-D supported")
    window = int(window)
    r = window // 2
    out = t
    for d in range(t.ndim):
        n = out.shape[d]
        p = _pad1d(out, d, r, boundary)
        if p.shape[d] - window + 1 != n:
            raise RuntimeError(f"moving_average: window {window} changes the length of axis {d}")
        acc = torch.zeros_like(out)
        for s in range(window):
            acc = acc + p.narrow(d, s, n)
        out = acc / window
    return out


def surface_normals(t, dx=1.0, boundary="neumann"):
    """Unit normals (−∂₀t, −∂₁t, 1)/max(|·|, 1e-15) of a 2-D height field with
    torch.gradient's edge order 2, boundary ignored (stenpy_engine.py:2199-2220)."""
    if t.ndim != 2:
        raise ValueError(f"surface_normals: expected 2D field, got {t.ndim}D")
    h = (float(dx),) * 2 if isinstance(dx, (int, float)) else tuple(float(v) for v in dx)
    gx, gy = torch.gradient(t, spacing=h, edge_order=2)
    n = torch.stack([-gx, -gy, torch.ones_like(gx)], dim=-1)
    return n / torch.linalg.norm(n, dim=-1, keepdim=True).clamp(min=1e-15)


def conv3d_spectral(a, boundary: str = "periodic"):
    """The 27-point Gaussian (1,2,1)⊗(1,2,1)⊗(1,2,1)/64 as a circular convolution,
    whatever ``boundary`` says: the reference's CPU path multiplies FFTs
    (stenpy_engine.py:2800-2860). Restated as a direct sum of rolled copies (equal up
    to FP64 rounding); every axis needs ≥ 3 points, as the reference's kernel
    placement requires."""
    if a.ndim != 3 or min(a.shape) < 3:
        raise ValueError(f"conv3d_spectral: needs a 3-D field with >= 3 points per axis, got {tuple(a.shape)}")
    w1 = {-1: 1.0, 0: 2.0, 1: 1.0}
    out = torch.zeros_like(a)
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                out = out + (w1[di] * w1[dj] * w1[dk]) * torch.roll(a, (-di, -dj, -dk), (0, 1, 2))
    return out / 64.0


# ---------------------------------------------------------------- tensor and vector helpers
def determinant(t):
    """det of each (3, 3), the diagonal lifted by 1e-12 everywhere when any |diagonal|
    entry of the field is below 1e-12; NaN → 0, ±inf and beyond → ±1e30
    (stenpy_engine.py:2683-2710)."""
    eye = torch.eye(t.shape[-1], dtype=F64)
    diag = torch.diagonal(t, dim1=-2, dim2=-1)
    tr = t + 1e-12 * eye if bool((diag.abs() < 1e-12).any()) else t
    det = torch.linalg.det(tr)
    return torch.nan_to_num(det, nan=0.0, posinf=1e30, neginf=-1e30).clamp(-1e30, 1e30)


def inverse(t):
    """torch.linalg.inv of each matrix (stenpy_engine.py:2724-2728)."""
    return torch.linalg.inv(t)


def deviatoric(t):
    """t − tr(t)/D · I with NaN and ±inf → 0 (stenpy_engine.py:2852-2867)."""
    d = t.shape[-1]
    tr = torch.diagonal(t, dim1=-2, dim2=-1).sum(-1, keepdim=True).unsqueeze(-1)
    out = t - (tr / max(d, 1e-15)) * torch.eye(d, dtype=F64)
    return torch.nan_to_num(out, nan=0.0, posinf=0.0, neginf=0.0)


def stack_components(*ts, dim=-1):
    """torch.stack of the fields (stenpy_engine.py:2247-2250)."""
    return torch.stack(list(ts), dim=dim)


def norm_last(t, eps: float = 1e-15):
    """‖t‖ over the last axis, kept as an axis of 1, at least eps (stenpy_engine.py:2262-2264)."""
    return torch.linalg.norm(t, dim=-1, keepdim=True).clamp(min=eps)


def div_last(a, b):
    """a / b, b given a trailing axis when it has one fewer (stenpy_engine.py:2269-2274)."""
    return a / (b.unsqueeze(-1) if b.ndim == a.ndim - 1 else b)


def neg_stack3(gx, gy):
    """(−gx, −gy, 1) / max(‖·‖, 1e-15) (stenpy_engine.py:2279-2288)."""
    n = torch.stack([-gx, -gy, torch.ones_like(gx)], dim=-1)
    return n / torch.linalg.norm(n, dim=-1, keepdim=True).clamp(min=1e-15)


def scale_eye(scalar_field, D):
    """s · I_D per voxel (stenpy_engine.py:2293-2300)."""
    return scalar_field.unsqueeze(-1).unsqueeze(-1) * torch.eye(int(D), dtype=F64)


def velocity_dot_grad(v, g):
    """v · g elementwise (stenpy_engine.py:2305-2311)."""
    return v * g


def covariance(a, b):
    """Centred dot product over max(n − 1, 1) (stenpy_engine.py:2575-2590, CPU branch)."""
    if a.shape != b.shape:
        raise ValueError(f"covariance: shape mismatch {a.shape} vs {b.shape}")
    af, bf = (a - a.mean()).flatten(), (b - b.mean()).flatten()
    return torch.dot(af, bf) / max(af.numel() - 1, 1)


def correlation(a, b):
    """Centred dot product over the product of the centred norms + 1e-15
    (stenpy_engine.py:2595-2613, CPU branch)."""
    if a.shape != b.shape:
        raise ValueError(f"correlation: shape mismatch {a.shape} vs {b.shape}")
    af, bf = (a - a.mean()).flatten(), (b - b.mean()).flatten()
    return torch.dot(af, bf) / (af.norm() * bf.norm() + 1e-15)


def matmul_batched_custom(a):
    """A·Aᵀ per matrix (stenpy_engine.py:2735-2742)."""
    n = a.shape[-1]
    b = a.reshape(-1, n, n)
    return (b @ b.transpose(-1, -2)).reshape(*a.shape[:-2], n, n)


def surface_integral(t, normals, area_weights):
    """Σ (t · normals) · area_weights (stenpy_engine.py:2486-2494)."""
    return ((t * normals).sum(dim=-1) * area_weights).sum()


# ---------------------------------------------------------------- geometry
def distance_transform(t, dx=1.0, method="auto"):
    """The reference's CPU path (stenpy_engine.py:3146-3152): SciPy's
    ``ndimage.distance_transform_edt`` (SciPy 1.18.1 here; no version is pinned by the
    reference) of ``t == 0`` with ``sampling`` = dx — for each voxel with t == 0 the
    Euclidean distance to the nearest voxel with t != 0, else 0."""
    import numpy as np
    from scipy.ndimage import distance_transform_edt
    dxs = _dx_tuple(dx, t.ndim)
    out = distance_transform_edt((t == 0).numpy(), sampling=list(dxs))
    return torch.from_numpy(np.asarray(out, dtype=np.float64))


# ---------------------------------------------------------------- spectral
def _k(shape, dx):
    """Angular wavenumbers 2π·fftfreq(n, dx) per axis (stenpy_engine.py:2934-2948): the
    frequencies are formed in FP32 (torch's default dtype) and widened, as there."""
    ks = []
    for d, (n, h) in enumerate(zip(shape, dx)):
        sh = [1] * len(shape)
        sh[d] = -1
        ks.append((torch.fft.fftfreq(n, d=h, dtype=torch.float32).to(F64) * (2 * math.pi)).view(sh))
    return ks


def fft(t, norm="backward"):
    """fftn of the field as complex128 (stenpy_engine.py:2875-2885), as a graph node sees
    it: the reference's runtime passes ``alloc`` and the op copies its result into that
    real FP64 buffer (stenpy_engine.py:2881-2884), keeping the real part."""
    return torch.fft.fftn(t if t.is_complex() else t.to(torch.complex128), norm=norm).real


def ifft(t, norm="backward"):
    """Real part of ifftn (stenpy_engine.py:2887-2896)."""
    x = t if t.is_complex() else torch.complex(t, torch.zeros_like(t))
    return torch.fft.ifftn(x, norm=norm).real


def spectral_gradient(t, dx=1.0, dim=0, norm="backward"):
    """Re ifftn(i·k_dim·fftn(t)) (stenpy_engine.py:2980-2993)."""
    k = _k(t.shape, _dx_tuple(dx, t.ndim))
    return torch.fft.ifftn(1j * k[int(dim)] * torch.fft.fftn(t, norm=norm), norm=norm).real


def spectral_laplacian(t, dx=1.0, norm="backward"):
    """Re ifftn(−|k|²·fftn(t)) (stenpy_engine.py:2998-3010)."""
    k = _k(t.shape, _dx_tuple(dx, t.ndim))
    return torch.fft.ifftn(-sum(kk * kk for kk in k) * torch.fft.fftn(t, norm=norm), norm=norm).real


def grad_mag(t, dx=1.0, boundary="neumann"):
    """|gradient(t)| with gradient's boundary conventions (not in the reference)."""
    return torch.linalg.norm(gradient(t, dx, boundary), dim=-1)


# ---------------------------------------------------------------- tensor ops
def trace(t):
    """Σ diagonal (stenpy_engine.py:2674-2680)."""
    return torch.diagonal(t, dim1=-2, dim2=-1).sum(-1)


def eigenvalues(t):
    """torch.linalg.eigvalsh: ascending, lower triangle (stenpy_engine.py:2715-2721)."""
    return torch.linalg.eigvalsh(t)


def select_component(t, index):
    """t[..., index] (stenpy_engine.py:2256-2259)."""
    return t[..., int(index)].contiguous()


# ---------------------------------------------------------------- reductions
def sum_(t, dim=None, keepdim=False):
    return t.sum() if dim is None else t.sum(dim=dim, keepdim=keepdim)   # :2340-2349


def mean(t, dim=None, keepdim=False):
    return t.mean() if dim is None else t.mean(dim=dim, keepdim=keepdim)  # :2352-2363


def norm_l2(t):
    return t.norm()                                                      # :2366-2373


def variance(t, dim=None, unbiased=True, keepdim=False):
    """torch.var, unbiased by default (stenpy_engine.py:2546-2572, CPU branch)."""
    return torch.var(t, dim=dim, unbiased=bool(unbiased), keepdim=keepdim)


def entropy(t, dim=None, eps: float = 1e-15):
    """p = |x| / (Σ|x| + eps); −Σ p log(p + eps) (stenpy_engine.py:2638-2667, CPU)."""
    p = t.abs()
    if dim is None:
        p = p / (p.sum() + eps)
        return -(p * (p + eps).log()).sum()
    p = p / (p.sum(dim=dim, keepdim=True) + eps)
    return -(p * (p + eps).log()).sum(dim=dim)


def min_max(t):
    return torch.stack([t.min(), t.max()])                               # :2376-2380


def simpson_weights(n: int, h: float) -> torch.Tensor:
    """Quadrature weights of ``_simpson_1d`` (stenpy_engine.py:2415-2437): composite
    Simpson for odd n; for even n Simpson on the first n−1 points plus a trapezoid
    on the last interval; trapezoid below 3 points."""
    w = torch.zeros(n, dtype=F64)
    if n < 3:
        if n == 2:
            w[:] = 0.5 * h
        return w
    m = n if n % 2 == 1 else n - 1
    w[0] += 1.0
    w[m - 1] += 1.0
    w[1:m - 1:2] += 4.0
    w[2:m - 1:2] += 2.0
    w *= h / 3.0
    if n % 2 == 0:
        w[n - 2] += 0.5 * h
        w[n - 1] += 0.5 * h
    return w


def _simpson_1d(y: torch.Tensor, h: float, dim: int) -> torch.Tensor:
    w = simpson_weights(y.shape[dim], h)
    shape = [1] * y.ndim
    shape[dim] = -1
    if y.shape[dim] < 3:
        return torch.trapezoid(y, dx=h, dim=dim)
    return (y * w.view(shape)).sum(dim)


def integrate(t, dx=1.0, dims=None, method="simpson"):
    """Simpson (or trapezoid) along each requested dim, last to first
    (stenpy_engine.py:2440-2459)."""
    h = (float(dx),) * t.ndim if isinstance(dx, (int, float)) else tuple(dx)
    seq = tuple(range(t.ndim)) if dims is None else ((dims,) if isinstance(dims, int) else tuple(dims))
    out = t
    for d in sorted(seq, reverse=True):
        out = _simpson_1d(out, h[d], d) if method == "simpson" else torch.trapezoid(out, dx=h[d], dim=d)
    return out


def cumulative_integral(t, dx=1.0, dim=0):
    """Running trapezoid with a leading zero slice (stenpy_engine.py:2462-2483)."""
    n = t.shape[dim]
    if n < 2:
        return torch.zeros_like(t)
    a = t.narrow(dim, 0, n - 1)
    b = t.narrow(dim, 1, n - 1)
    z_shape = list(t.shape)
    z_shape[dim] = 1
    return torch.cat([torch.zeros(z_shape, dtype=F64), torch.cumsum((a + b) * (dx * 0.5), dim=dim)], dim=dim)


def entropy_hist(t, bins=256):
    """Shannon entropy (nats) of a ``bins``-bin histogram spanning [min, max], last
    bin closed (numpy.histogram convention); 0 for a constant field. Not in the
    reference."""
    x = t.reshape(-1)
    lo, hi = float(x.min()), float(x.max())
    n = x.numel()
    if hi <= lo:
        return torch.tensor(0.0, dtype=F64)
    b = int(bins)
    idx = torch.floor((x - lo) / (hi - lo) * b).clamp(0, b - 1).to(torch.int64)
    counts = torch.bincount(idx, minlength=b).to(F64)
    p = counts[counts > 0] / n
    return -(p * p.log()).sum()


OPS: Dict[str, Callable] = {
    "add": add, "sub": sub, "mul": mul, "div": div, "neg": neg, "clamp": clamp,
    "exp": exp, "log": log, "sqrt": sqrt, "sin": sin, "cos": cos, "tanh": tanh, "abs": abs_,
    "laplacian": laplacian, "gradient": gradient, "divergence": divergence, "curl": curl,
    "hessian": hessian, "jacobian": jacobian, "mean_curvature": mean_curvature,
    "grad_mag": grad_mag, "gradient_nd": gradient_nd, "material_derivative": material_derivative,
    "moving_average": moving_average, "conv3d_spectral": conv3d_spectral,
    "surface_normals": surface_normals, "fft": fft, "ifft": ifft,
    "spectral_gradient": spectral_gradient, "spectral_laplacian": spectral_laplacian,
    "distance_transform": distance_transform, "determinant": determinant, "inverse": inverse,
    "deviatoric": deviatoric, "stack_components": stack_components, "norm_last": norm_last,
    "div_last": div_last, "neg_stack3": neg_stack3, "scale_eye": scale_eye,
    "velocity_dot_grad": velocity_dot_grad, "surface_integral": surface_integral,
    "matmul_batched_custom": matmul_batched_custom, "covariance": covariance, "correlation": correlation,
    "trace": trace, "eigenvalues": eigenvalues, "select_component": select_component,
    "sum": sum_, "mean": mean, "norm_l2": norm_l2, "variance": variance, "entropy": entropy,
    "min_max": min_max, "integrate": integrate, "cumulative_integral": cumulative_integral,
    "entropy_hist": entropy_hist,
}


def evaluate(graph: Any, wanted: Optional[Iterable[str]] = None) -> Dict[str, torch.Tensor]:
    """Evaluate ``graph`` node by node in topological order, FP64 on the CPU
    (the structure of stenpy_engine.py:983-1146 without the memory manager).
    Returns every node's value (or only ``wanted``)."""
    values: Dict[str, torch.Tensor] = {}
    for node in graph.topological_sort():
        if node.op_name == "_constant":
            values[node.id] = _f64(node.params["value"])
            continue
        fn = OPS[node.op_name]
        args = [values[i] for i in node.input_ids]
        values[node.id] = fn(*args, **node.params)
    if wanted is None:
        return values
    return {k: values[k] for k in wanted}

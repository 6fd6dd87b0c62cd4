"""Lowering of graph operators onto per-voxel primitives (``codegen.PNode``).

Each operator keeps the reference CPU path's boundary conventions:

* ``laplacian`` — compact 7-point, periodic via torch.roll, otherwise the
  ``_pad1d`` rule: neumann → replicate, dirichlet → zeros, reflect → mirror, any
  other name → zeros (stenpy_engine.py:1374-1416, 1500-1519);
* ``gradient`` — periodic wrapped central differences, otherwise torch.gradient
  with second-order one-sided edges (first order on length-2 axes, zero on
  length-1 axes) (stenpy_engine.py:1816-1867);
* ``divergence`` — the same, always edge order 2 off the periodic branch
  (stenpy_engine.py:1910-1933);
* ``curl`` — torch.gradient edge order 2 on every axis, whatever the boundary
  (stenpy_engine.py:1983-2000);
* ``hessian`` / ``jacobian`` — gradient_nd applied twice / once: torch.gradient
  with edge order 2 when every axis has ≥ 3 points, else 1, boundary ignored
  (stenpy_engine.py:2037-2130, 2133-2177);
* ``mean_curvature`` — gradient_nd, normalise by max(|∇f|, eps), then
  ``divergence`` with the requested boundary (stenpy_engine.py:2180-2197);
* ``material_derivative`` — Σ_d v[..., d] · gradient_nd(f)[..., d]
  (stenpy_engine.py:2223-2244);
* ``moving_average`` — a window³ box mean, the per-axis 1-D means of the
  reference composed, each axis padded by the ``_pad1d`` rule (default neumann)
  (stenpy_engine.py:2385-2408);
* ``surface_normals`` — 2-D fields only: (−∂₀f, −∂₁f, 1)/|·| with torch.gradient's
  edge order 2 on both axes, boundary ignored (stenpy_engine.py:2199-2220);
* ``conv3d_spectral`` — the 27-point Gaussian (1-2-1)⊗(1-2-1)⊗(1-2-1)/64 as a
  circular convolution, whatever the boundary: the reference's CPU path multiplies
  FFTs (stenpy_engine.py:2800-2860).
"""
from __future__ import annotations

from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

from .codegen import PGraph


class LoweringError(ValueError):
    pass


MAX_TAP_REACH = 4   # widest weighted-tap stencil (window 9): the plane ring holds 2R+1+P slots


def dx3(dx: Any) -> Tuple[float, float, float]:
    if isinstance(dx, (int, float)):
        return (float(dx),) * 3
    t = tuple(float(v) for v in dx)
    if len(t) != 3:
        raise LoweringError(f"dx must be a number or 3 values, got {dx!r}")
    return t


def _gradient_mode(boundary: str, n: int) -> str:
    if boundary == "periodic":
        return "periodic"
    if n >= 3:
        return "edge2"
    if n == 2:
        return "edge1"
    return "zero"


def _strict_edge2(boundary: str, n: int, op: str) -> str:
    if boundary == "periodic":
        return "periodic"
    if n < 3:
        raise LoweringError(f"{op}: torch.gradient edge_order=2 needs >= 3 points per axis, got {n}")
    return "edge2"


def _gnd_mode(shape: Sequence[int], op: str) -> str:
    if min(shape) < 2:
        raise LoweringError(f"{op}: axes of length 1 are not supported (got {tuple(shape)})")
    return "edge2" if min(shape) >= 3 else "edge1"


def _pad_mode(boundary: str) -> str:
    return {"periodic": "periodic", "neumann": "replicate", "reflect": "reflect"}.get(boundary, "zero")


class OpLowerer:
    """Lower one graph op given already-lowered inputs. ``shape`` = (n0, n1, n2)."""

    def __init__(self, pg: PGraph, shape: Tuple[int, int, int], dims2: bool = False):
        self.pg = pg
        self.shape = shape
        self.dims2 = dims2   # the fields are 2-D: shape is (1, n0, n1)

    def nc(self, nid: int) -> int:
        return self.pg.nodes[nid].nc

    def r(self, *nids: int) -> int:
        return max([self.pg.nodes[n].radius for n in nids] + [0])

    def component(self, x: int, c: int) -> Optional[int]:
        """The scalar node holding component ``c`` of ``x`` when ``x`` is built by
        stacking (so a consumer of one component does not evaluate the others)."""
        n = self.pg.nodes[x]
        if n.nc == 1 and c == 0:
            return x
        if n.op != "stack":
            return None
        for y in n.ins:
            k = self.nc(y)
            if c < k:
                return self.component(y, c)
            c -= k
        return None

    def d1(self, x: int, axis: int, mode: str, h: float, comp: Optional[int] = None) -> int:
        if comp is not None:
            y = self.component(x, comp)
            if y is not None:          # derivative of one stacked component: that component alone
                x, comp = y, None
        nc = 1 if comp is not None else self.nc(x)
        rad = self.r(x) + (0 if mode == "zero" else 1)
        return self.pg.add("d1", (x,), nc, rad, axis=axis, mode=mode, comp=comp,
                           inv2h=1.0 / (2.0 * h), invh=1.0 / h)

    def taps(self, x: int, reach: int, taps: Sequence[Tuple[int, int, int, float]], scale: float,
             pad: str) -> int:
        """Weighted sum of ``x`` at offsets (di, dj, dk) within ``reach`` of the voxel,
        times ``scale``; out-of-range offsets follow the padding rule ``pad``."""
        return self.pg.add("taps", (x,), self.nc(x), self.r(x) + reach, taps=tuple(taps),
                           scale=float(scale), pad=pad, reach=reach)

    def stack(self, xs: Sequence[int]) -> int:
        return self.pg.add("stack", tuple(xs), sum(self.nc(x) for x in xs), self.r(*xs))

    def binop(self, op: str, a: int, b: int, **attrs) -> int:
        na, nb = self.nc(a), self.nc(b)
        if na != nb and 1 not in (na, nb):
            raise LoweringError(f"{op}: component mismatch {na} vs {nb}")
        return self.pg.add(op, (a, b), max(na, nb), self.r(a, b), **attrs)

    def unop(self, op: str, a: int, **attrs) -> int:
        return self.pg.add(op, (a,), self.nc(a), self.r(a), **attrs)

    # ---- the operators
    def lower(self, op: str, ins: List[int], params: Dict[str, Any],
              is_scalar: Callable[[int], bool]) -> int:
        p = dict(params)
        p.pop("alloc", None)
        p.pop("mm", None)
        n0, n1, n2 = self.shape

        def need(k: int):
            if len(ins) != k:
                raise LoweringError(f"{op}: expected {k} inputs, got {len(ins)}")

        def no_extra(*allowed):
            extra = set(p) - set(allowed)
            if extra:
                raise LoweringError(f"{op}: unexpected parameters {sorted(extra)}")

        if op in ("add", "sub"):
            need(2); no_extra()
            return self.binop(op, ins[0], ins[1])
        if op == "mul":
            no_extra("scalar")
            if len(ins) == 1 and "scalar" in p:
                return self.pg.add("mulk", (ins[0],), self.nc(ins[0]), self.r(ins[0]), k=float(p["scalar"]))
            need(2)
            return self.binop("mul", ins[0], ins[1])
        if op == "div":
            need(2); no_extra("eps")
            return self.binop("div", ins[0], ins[1], eps=float(p.get("eps", 1e-15)))
        if op in ("neg", "exp", "sin", "cos", "tanh", "abs"):
            need(1); no_extra()
            return self.unop(op, ins[0])
        if op == "log":
            need(1); no_extra("eps")
            return self.unop("log", ins[0], eps=float(p.get("eps", 1e-15)))
        if op == "sqrt":
            need(1); no_extra("eps")
            return self.unop("sqrt", ins[0], eps=float(p.get("eps", 0.0)))
        if op == "clamp":
            no_extra("lo", "hi")
            if not 1 <= len(ins) <= 3:
                raise LoweringError("clamp: 1 to 3 inputs")
            for extra in ins[1:]:
                if self.nc(extra) != 1:
                    raise LoweringError("clamp: bounds must be scalar-valued")
            return self.pg.add("clamp", tuple(ins), self.nc(ins[0]), self.r(*ins),
                               lo=float(p.get("lo", 0.0)), hi=float(p.get("hi", 1.0)))
        if op == "trace":
            need(1); no_extra()
            if self.nc(ins[0]) != 9:
                raise LoweringError("trace: needs (*, 3, 3) input")
            diag = [self.component(ins[0], c) for c in (0, 4, 8)]
            if all(d is not None for d in diag):   # only the diagonal is evaluated
                return self.binop("add", self.binop("add", diag[0], diag[1]), diag[2])
            return self.pg.add("trace", (ins[0],), 1, self.r(ins[0]))
        if op == "eigenvalues":
            need(1); no_extra()
            if self.nc(ins[0]) != 9:
                raise LoweringError("eigenvalues: needs (*, 3, 3) input")
            return self.pg.add("eig", (ins[0],), 3, self.r(ins[0]))
        if op == "select_component":
            need(1); no_extra("index")
            nc = self.nc(ins[0])
            idx = int(p["index"])
            if nc == 3 and 0 <= idx < 3:
                y = self.component(ins[0], idx)
                if y is not None:
                    return y
                return self.pg.add("select", (ins[0],), 1, self.r(ins[0]), index=idx)
            if nc == 9 and 0 <= idx < 3:
                row = [self.component(ins[0], 3 * idx + c) for c in range(3)]
                if all(y is not None for y in row):
                    return self.stack(row)
                return self.pg.add("select", (ins[0],), 3, self.r(ins[0]), index=idx)
            raise LoweringError("select_component: index out of range")

        if op in ("determinant", "inverse", "deviatoric"):
            need(1); no_extra()
            if self.nc(ins[0]) != 9:
                raise LoweringError(f"{op}: needs a (*, 3, 3) input")
            prim = {"determinant": "det3", "inverse": "inv3", "deviatoric": "dev3"}[op]
            return self.pg.add(prim, (ins[0],), 1 if op == "determinant" else 9, self.r(ins[0]))
        if op == "stack_components":
            no_extra("dim")
            if int(p.get("dim", -1)) not in (-1, 3) or len(ins) != 3 or any(self.nc(x) != 1 for x in ins):
                raise LoweringError("stack_components: three scalar fields stacked along the last axis")
            return self.stack(ins)
        if op == "norm_last":
            need(1); no_extra("eps")
            if self.nc(ins[0]) != 3:
                raise LoweringError("norm_last: (*, 3) vector fields")
            return self.pg.add("norm", (ins[0],), 1, self.r(ins[0]), eps=float(p.get("eps", 1e-15)))
        if op == "div_last":
            need(2); no_extra()
            if self.nc(ins[1]) not in (1, self.nc(ins[0])):
                raise LoweringError("div_last: divisor must be scalar or match the components")
            return self.binop("div", ins[0], ins[1], eps=0.0)
        if op == "neg_stack3":
            need(2); no_extra()
            if self.nc(ins[0]) != 1 or self.nc(ins[1]) != 1:
                raise LoweringError("neg_stack3: two scalar fields")
            return self.pg.add("surfnorm", (ins[0], ins[1]), 3, self.r(*ins))
        if op == "scale_eye":
            need(1); no_extra("D")
            if int(p.get("D", 3)) != 3 or self.nc(ins[0]) != 1:
                raise LoweringError("scale_eye: a scalar field and D=3")
            s = ins[0]
            z = self.pg.add("mulk", (s,), 1, self.r(s), k=0.0)   # s·0, as the reference's s·I entries
            return self.stack([s, z, z, z, s, z, z, z, s])
        if op == "matmul_batched_custom":
            need(1); no_extra()
            if self.nc(ins[0]) != 9:
                raise LoweringError("matmul_batched_custom: needs a (*, 3, 3) input")
            return self.pg.add("aat3", (ins[0],), 9, self.r(ins[0]))
        if op == "velocity_dot_grad":
            need(2); no_extra()
            return self.binop("mul", ins[0], ins[1])

        # ---- stencils
        bnd = str(p.get("boundary", "neumann"))
        if op == "laplacian":
            need(1); no_extra("dx", "boundary")
            bnd = str(p.get("boundary", "periodic"))
            x = ins[0]
            if self.nc(x) != 1:
                raise LoweringError("laplacian: scalar fields only")
            h = dx3(p.get("dx", 1.0))
            return self.pg.add("lap", (x,), 1, self.r(x) + 1, pad=_pad_mode(bnd),
                               invh2=tuple(1.0 / (v * v) for v in h))
        if op in ("gradient", "grad_mag"):
            need(1); no_extra("dx", "boundary", "dim")
            x = ins[0]
            if self.nc(x) != 1:
                raise LoweringError(f"{op}: scalar fields only")
            h = dx3(p.get("dx", 1.0))
            dim = p.get("dim")
            if dim is not None:
                a = int(dim) % 3
                return self.d1(x, a, "zero" if self.shape[a] == 1 else _gradient_mode(bnd, self.shape[a]), h[a])
            g = self.stack([self.d1(x, a, _gradient_mode(bnd, self.shape[a]), h[a]) for a in range(3)])
            if op == "grad_mag":
                return self.pg.add("norm", (g,), 1, self.r(g))
            return g
        if op == "divergence":
            need(1); no_extra("dx", "boundary")
            v = ins[0]
            if self.nc(v) != 3:
                raise LoweringError("divergence: needs a (*, 3) vector field")
            h = dx3(p.get("dx", 1.0))
            t = [self.d1(v, a, _strict_edge2(bnd, self.shape[a], op), h[a], comp=a) for a in range(3)]
            return self.binop("add", self.binop("add", t[0], t[1]), t[2])
        if op == "curl":
            need(1); no_extra("dx", "boundary")
            v = ins[0]
            if self.nc(v) != 3:
                raise LoweringError("curl: needs a (*, 3) vector field")
            h = dx3(p.get("dx", 1.0))
            m = [_strict_edge2("neumann", self.shape[a], op) for a in range(3)]

            def d(c, a):
                return self.d1(v, a, m[a], h[a], comp=c)

            return self.stack([self.binop("sub", d(2, 1), d(1, 2)),
                               self.binop("sub", d(0, 2), d(2, 0)),
                               self.binop("sub", d(1, 0), d(0, 1))])
        if op == "gradient_nd":
            need(1); no_extra("dx", "boundary", "dim")   # dim is accepted and ignored, as there
            x = ins[0]
            if self.nc(x) != 1:
                raise LoweringError("gradient_nd: scalar fields only")
            h = dx3(p.get("dx", 1.0))
            mode = _gnd_mode(self.shape, op)
            return self.stack([self.d1(x, a, mode, h[a]) for a in range(3)])
        if op in ("hessian", "jacobian", "mean_curvature"):
            no_extra("dx", "boundary", "eps")
            need(1)
            x = ins[0]
            h = dx3(p.get("dx", 1.0))
            mode = _gnd_mode(self.shape, op)
            if op == "jacobian":
                if self.nc(x) != 3:
                    raise LoweringError("jacobian: needs a (*, 3) vector field")
                return self.stack([self.d1(x, d, mode, h[d], comp=c) for c in range(3) for d in range(3)])
            if self.nc(x) != 1:
                raise LoweringError(f"{op}: scalar fields only")
            g = self.stack([self.d1(x, a, mode, h[a]) for a in range(3)])
            if op == "hessian":
                return self.stack([self.d1(g, j, mode, h[j], comp=i) for i in range(3) for j in range(3)])
            nh = self.pg.add("normalize", (g,), 3, self.r(g), eps=float(p.get("eps", 1e-15)))
            t = [self.d1(nh, a, _strict_edge2(bnd, self.shape[a], op), h[a], comp=a) for a in range(3)]
            return self.binop("add", self.binop("add", t[0], t[1]), t[2])
        if op == "material_derivative":
            need(2); no_extra("dx", "boundary")
            f, v = ins
            if self.nc(f) != 1 or self.nc(v) != 3:
                raise LoweringError("material_derivative: needs a scalar field and a (*, 3) velocity")
            h = dx3(p.get("dx", 1.0))
            mode = _gnd_mode(self.shape, op)
            t = []
            for d in range(3):
                vd = self.component(v, d)
                if vd is None:
                    vd = self.pg.add("select", (v,), 1, self.r(v), index=d)
                t.append(self.binop("mul", vd, self.d1(f, d, mode, h[d])))
            return self.binop("add", self.binop("add", t[0], t[1]), t[2])
        if op == "moving_average":
            need(1); no_extra("window", "boundary")
            x = ins[0]
            if self.nc(x) != 1:
                raise LoweringError("moving_average: scalar fields only")
            w = int(p.get("window", 3))
            if w < 1 or w % 2 == 0:
                raise LoweringError(f"moving_average: window must be odd and positive, got {w}")
            rr = w // 2
            if rr > MAX_TAP_REACH:
                raise LoweringError(f"moving_average: window {w} exceeds {2 * MAX_TAP_REACH + 1}")
            bnd = str(p.get("boundary", "neumann"))
            pad = _pad_mode(bnd)
            for n in self.shape:
                if pad == "periodic" and rr > n:
                    raise LoweringError(f"moving_average: circular padding of {rr} wider than an axis of {n}")
                if pad == "reflect" and rr >= n:
                    raise LoweringError(f"moving_average: reflect padding of {rr} needs axes longer than {rr}")
            if rr == 0:    # window 1: the field itself
                return self.pg.add("mulk", (x,), 1, self.r(x), k=1.0)
            rng = range(-rr, rr + 1)
            return self.taps(x, rr, [(a, b, c, 1.0) for a in rng for b in rng for c in rng],
                             (1.0 / w) ** 3, pad)
        if op == "surface_normals":
            need(1); no_extra("dx", "boundary")
            x = ins[0]
            if not self.dims2:
                raise LoweringError("surface_normals: expected a 2-D field, got a 3-D one")
            if self.nc(x) != 1:
                raise LoweringError("surface_normals: scalar fields only")
            dx = p.get("dx", 1.0)
            h = (float(dx),) * 2 if isinstance(dx, (int, float)) else tuple(float(v) for v in dx)
            if len(h) != 2:
                raise LoweringError(f"surface_normals: dx must be a number or 2 values, got {dx!r}")
            if min(self.shape[1:]) < 3:
                raise LoweringError(f"surface_normals: torch.gradient edge_order=2 needs >= 3 points per axis, "
                                    f"got {self.shape[1:]}")
            gx = self.d1(x, 1, "edge2", h[0])
            gy = self.d1(x, 2, "edge2", h[1])
            return self.pg.add("surfnorm", (gx, gy), 3, self.r(gx, gy))
        if op == "conv3d_spectral":
            need(1); no_extra("dx", "boundary")
            x = ins[0]
            if self.nc(x) != 1:
                raise LoweringError("conv3d_spectral: scalar fields only")
            if min(self.shape) < 3:
                raise LoweringError(f"conv3d_spectral: axes need >= 3 points, got {self.shape}")
            rng = (-1, 0, 1)
            return self.taps(x, 1, [(a, b, c, float(2 ** (3 - abs(a) - abs(b) - abs(c))))
                                    for a in rng for b in rng for c in rng], 1.0 / 64.0, "periodic")
        raise LoweringError(f"no lowering for operator '{op}'")

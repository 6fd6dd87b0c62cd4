"""Expression front end: string → SymPy tree → CSE'd ``Graph``.

Behaviour follows the reference front end (stenpy_engine.py:3462-3778):

* operator names resolve through an alias table (stenpy_engine.py:3462-3475);
* ops outside the "no-stencil" set get ``dx`` and ``boundary`` params
  (stenpy_engine.py:3613-3615);
* ``name=value`` arguments are carried through SymPy as encoded symbols and
  decoded as int, then float, then string (stenpy_engine.py:3515-3543, 3596-3610);
* every node is common-subexpression cached on ``(op, child ids, scalar params)``
  (stenpy_engine.py:3618-3759);
* ``divergence(gradient(f))`` is rewritten to ``laplacian(f)``
  (stenpy_engine.py:3494-3496, 3683-3688); the orphaned ``gradient`` node stays in
  the graph as in the reference, and the executor drops it as dead code;
* ``Add``/``Mul`` become left folds in SymPy's argument order, ``-1*x`` becomes
  ``neg``; ``Pow`` lowers 0.5 → sqrt, small integer powers → multiply chains,
  negative powers → ``div(1, ·)``, others → ``exp(log(·) * c)``
  (stenpy_engine.py:3697-3755).

Differences, all additive: ``hessian(...)`` parses (the reference only accepts
``_hessian``, because SymPy's own ``hessian`` shadows the name), ``l2norm`` is an
alias of ``norm_l2``, ``cos``/``abs``/``grad_mag``/``jacobian``/``entropy_hist``/
``select_component`` are reachable, and ``abs(x)`` (SymPy ``Abs``) maps to the
``abs`` op.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field as dc_field
from typing import Any, Dict, List, Optional, Set, Tuple

import sympy as sp
import torch

from .graph import Graph
from .registry import NO_STENCIL_OPS, OP_REGISTRY

ALIAS: Dict[str, str] = {
    "gradient": "gradient", "grad": "gradient", "divergence": "divergence", "div": "divergence",
    "laplacian": "laplacian", "laplace": "laplacian", "lap": "laplacian", "curl": "curl",
    "spectral_gradient": "spectral_gradient", "spectral_laplacian": "spectral_laplacian",
    "fft": "fft", "ifft": "ifft", "add": "add", "sub": "sub", "mul": "mul", "div_op": "div",
    "neg": "neg", "clamp": "clamp", "exp": "exp", "log": "log", "sqrt": "sqrt", "sin": "sin",
    "tanh": "tanh", "sum": "sum", "mean": "mean", "norm_l2": "norm_l2", "variance": "variance",
    "entropy": "entropy", "integrate": "integrate", "cumulative_integral": "cumulative_integral",
    "trace": "trace", "determinant": "determinant", "eigenvalues": "eigenvalues", "inverse": "inverse",
    "deviatoric": "deviatoric", "var": "variance", "moving_average": "moving_average",
    "min_max": "min_max", "minmax": "min_max", "covariance": "covariance", "cov": "covariance",
    "correlation": "correlation", "corr": "correlation", "surface_integral": "surface_integral",
    "distance_transform": "distance_transform",
    # additions
    "cos": "cos", "hessian": "hessian", "_hessian": "hessian", "l2norm": "norm_l2",
    "mean_curvature": "mean_curvature", "grad_mag": "grad_mag", "jacobian": "jacobian",
    "entropy_hist": "entropy_hist", "select_component": "select_component",
}

SIMPLIFY_RULES: Dict[Tuple[str, str], str] = {("divergence", "gradient"): "laplacian"}
RESERVED_SYMBOLS = frozenset({"x", "y", "z", "t"})
_PRIMARY_FALLBACK = ("f", "g", "h", "u", "v")
_KW_PREFIX = "_kw_"
_CALL_RE = re.compile(r"(\w+)\s*\(([^()]*?)\)", re.DOTALL)


def _kw_token(key: str, value: str) -> str:
    return f"{_KW_PREFIX}{key}__{value.encode().hex()}"


def _decode_kw_value(enc: str) -> Any:
    try:
        text = bytes.fromhex(enc).decode()
    except ValueError:
        text = enc
    for conv in (int, float):
        try:
            return conv(text)
        except ValueError:
            pass
    return text


def _encode_kwargs(s: str) -> str:
    """Rewrite ``f(a, k=v)`` into ``f(a, _kw_k__<hex v>)`` innermost-first until stable."""
    def repl(m: re.Match) -> str:
        positional, keyword = [], []
        for part in m.group(2).split(","):
            part = part.strip()
            if "=" in part and not part.startswith(_KW_PREFIX):
                k, v = part.split("=", 1)
                keyword.append(_kw_token(k.strip(), v.strip().strip("'\"")))
            else:
                positional.append(part)
        return f"{m.group(1)}({', '.join(positional + keyword)})"
    while True:
        new = _CALL_RE.sub(repl, s)
        if new == s:
            return s
        s = new


def _namespace(field_names: Set[str]) -> Dict[str, Any]:
    ns: Dict[str, Any] = {}
    for sym in RESERVED_SYMBOLS - field_names:
        ns[sym] = sp.Symbol(sym)
    for name in field_names:
        ns[name] = sp.Symbol(name)
    for alias, canonical in ALIAS.items():
        ns.setdefault(alias, sp.Function(alias))
        ns.setdefault(canonical, sp.Function(canonical))
    ns["pi"] = sp.pi
    ns["E"] = sp.E
    return ns


def parse_expression(expr_str: str, field_names: Optional[Set[str]] = None) -> sp.Expr:
    """Parse ``expr_str`` with SymPy (stenpy_engine.py:3576-3582)."""
    names = set(field_names or ())
    cleaned = _encode_kwargs(expr_str.strip())
    ns = _namespace(names)
    for token in re.findall(r"_kw_\w+", cleaned):
        ns[token] = sp.Symbol(token)
    try:
        return sp.sympify(cleaned, locals=ns)
    except Exception as exc:  # SymPy raises many types
        raise ValueError(f"Could not parse '{expr_str}': {exc}\nProcessed form: '{cleaned}'") from exc


@dataclass
class _Ctx:
    graph: Graph
    dx: Any
    boundary: str
    cse: Dict[Tuple, str] = dc_field(default_factory=dict)
    src_id: str = ""
    warnings: List[str] = dc_field(default_factory=list)
    field_map: Dict[str, str] = dc_field(default_factory=dict)
    bypassed: set = dc_field(default_factory=set)

    def cached(self, key: Tuple, op: str, inputs: Tuple[str, ...], params: Dict[str, Any]) -> str:
        nid = self.cse.get(key)
        if nid is None:
            nid = self.graph.add(op, inputs, params)
            self.cse[key] = nid
        return nid

    def const(self, value: float) -> str:
        key = ("_scalar", float(value))
        nid = self.cse.get(key)
        if nid is None:
            nid = self.graph.add("_constant", (), {"value": torch.tensor(float(value), dtype=torch.float64)})
            self.cse[key] = nid
        return nid


def _scalar_items(params: Dict[str, Any]) -> Tuple:
    return tuple(sorted((k, v) for k, v in params.items() if isinstance(v, (int, float, str, bool))))


def _split_kwargs(args: Tuple) -> Tuple[Dict[str, Any], List[sp.Expr]]:
    kwargs: Dict[str, Any] = {}
    positional: List[sp.Expr] = []
    for a in args:
        s = str(a)
        if isinstance(a, sp.Symbol) and s.startswith(_KW_PREFIX):
            key, enc = s[len(_KW_PREFIX):].split("__", 1)
            kwargs[key] = _decode_kw_value(enc)
        else:
            positional.append(a)
    return kwargs, positional


def _stencil_params(op: str, ctx: _Ctx) -> Dict[str, Any]:
    return {} if op in NO_STENCIL_OPS else {"dx": ctx.dx, "boundary": ctx.boundary}


def _fold(op: str, ids: List[str], ctx: _Ctx) -> str:
    acc = ids[0]
    for nxt in ids[1:]:
        acc = ctx.cached((op, (acc, nxt), ()), op, (acc, nxt), {})
    return acc


def _compile(expr: sp.Expr, ctx: _Ctx) -> str:
    if isinstance(expr, sp.Symbol):
        name = str(expr)
        if name in ctx.field_map:
            return ctx.field_map[name]
        if name not in _PRIMARY_FALLBACK:
            ctx.warnings.append(f"Unknown symbol '{name}' — falling back to primary field.")
        return ctx.src_id

    if isinstance(expr, sp.Number):
        return ctx.const(float(expr))

    if isinstance(expr, sp.NumberSymbol):  # pi, E
        return ctx.const(float(expr))

    if isinstance(expr, sp.Abs):
        child = _compile(expr.args[0], ctx)
        return ctx.cached(("abs", (child,), ()), "abs", (child,), {})

    if isinstance(expr, sp.core.function.AppliedUndef):
        fname = type(expr).__name__
        kwargs, positional = _split_kwargs(expr.args)
        op = ALIAS.get(fname.lower(), fname.lower())
        if fname == "_hessian":
            op = "hessian"
        children = tuple(_compile(a, ctx) for a in positional)
        params = _stencil_params(op, ctx)
        params.update(kwargs)
        if len(children) == 1:
            child = ctx.graph._nodes.get(children[0])
            if child is not None and (op, child.op_name) in SIMPLIFY_RULES:
                new_op = SIMPLIFY_RULES[(op, child.op_name)]
                ctx.warnings.append(f"Simplified {op}({child.op_name}(f)) → {new_op}(f)")
                ctx.bypassed.add(children[0])
                op, children = new_op, child.input_ids
        if op not in OP_REGISTRY:
            raise ValueError(f"Unknown operator '{op}' (from '{fname}').\n"
                             f"Available: {sorted(OP_REGISTRY.keys())}")
        return ctx.cached((op, children, _scalar_items(params)), op, children, params)

    if isinstance(expr, sp.Add):
        return _fold("add", [_compile(a, ctx) for a in expr.args], ctx)

    if isinstance(expr, sp.Mul):
        args = list(expr.args)
        if len(args) == 2 and sp.Integer(-1) in args:
            other = args[1] if args[0] == sp.Integer(-1) else args[0]
            child = _compile(other, ctx)
            return ctx.cached(("neg", (child,), ()), "neg", (child,), {})
        return _fold("mul", [_compile(a, ctx) for a in args], ctx)

    if isinstance(expr, sp.Pow):
        base = _compile(expr.args[0], ctx)
        try:
            e = float(expr.args[1])
        except TypeError as exc:
            raise ValueError(f"Non-numeric exponent in {expr}") from exc
        if abs(e - 0.5) < 1e-9:
            return ctx.cached(("sqrt", (base,), ()), "sqrt", (base,), {})
        n = int(e)
        if abs(e - n) < 1e-9 and abs(n) <= 16:
            g = ctx.graph
            if n == 0:
                return g.add("_constant", (), {"value": torch.tensor(1.0, dtype=torch.float64)})
            if n < 0:
                pos = _compile(sp.Pow(expr.args[0], sp.Integer(-n)), ctx)
                one = g.add("_constant", (), {"value": torch.tensor(1.0, dtype=torch.float64)})
                return g.add("div", (one, pos), {})
            acc = base
            for _ in range(n - 1):
                acc = ctx.cached(("mul", (acc, base), ()), "mul", (acc, base), {})
            return acc
        g = ctx.graph
        lg = g.add("log", (base,), {})
        c = _compile(sp.Float(e), ctx)
        m = g.add("mul", (lg, c), {})
        return g.add("exp", (m,), {})

    raise ValueError(f"Unsupported SymPy node {type(expr).__name__}: {expr}\n"
                     "Use recognised operators and arithmetic (+, *, **).")


def _mark_orphans(g: Graph, ctx: _Ctx) -> None:
    """Record nodes left unconsumed by a rewrite (e.g. the ``gradient`` under a
    div∘grad → laplacian rewrite). The reference keeps and executes them; the
    runtime here excludes them from the default outputs."""
    consumed = set()
    for node in g._nodes.values():
        consumed.update(node.input_ids)
    g._orphans = {n for n in ctx.bypassed if n not in consumed}


def compile_expression(
    expr_str: str,
    dx: Any = 1.0,
    boundary: str = "neumann",
    field_map: Optional[Dict[str, Any]] = None,
) -> Tuple[Graph, str, List[str], Dict[str, str], sp.Expr]:
    """Compile ``expr_str`` into ``(graph, sink_id, warnings, field ids, sympy expr)``
    (stenpy_engine.py:3762-3778). Fields become ``_constant`` nodes holding the
    given tensors; ``f`` (else the first field) is the primary field."""
    if field_map is None:
        field_map = {"f": torch.zeros(1, dtype=torch.float64)}
    sym = parse_expression(expr_str, field_names=set(field_map))
    g = Graph()
    ctx = _Ctx(graph=g, dx=dx, boundary=boundary)
    for name, value in field_map.items():
        ctx.field_map[name] = g.add("_constant", (), {"value": value})
    ctx.src_id = ctx.field_map.get("f", next(iter(ctx.field_map.values())))
    sink = _compile(sym, ctx)
    _mark_orphans(g, ctx)
    return g, sink, ctx.warnings, dict(ctx.field_map), sym


def compile_expressions(
    exprs: Dict[str, str],
    dx: Any = 1.0,
    boundary: str = "neumann",
    field_map: Optional[Dict[str, Any]] = None,
) -> Tuple[Graph, Dict[str, str], List[str], Dict[str, str]]:
    """Compile several named expressions into ONE graph sharing fields and the CSE
    cache, so a fused executor can evaluate them in shared passes. Returns
    ``(graph, {name: sink_id}, warnings, field ids)``. Not in the reference."""
    if field_map is None:
        field_map = {"f": torch.zeros(1, dtype=torch.float64)}
    g = Graph()
    ctx = _Ctx(graph=g, dx=dx, boundary=boundary)
    for name, value in field_map.items():
        ctx.field_map[name] = g.add("_constant", (), {"value": value})
    ctx.src_id = ctx.field_map.get("f", next(iter(ctx.field_map.values())))
    sinks = {}
    for name, text in exprs.items():
        sinks[name] = _compile(parse_expression(text, field_names=set(field_map)), ctx)
    _mark_orphans(g, ctx)
    return g, sinks, ctx.warnings, dict(ctx.field_map)

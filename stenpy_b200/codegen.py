"""CUDA C++ generation for one fused pass over a 3-D grid.

A *pass* is one launch of a z-marching stencil kernel over an (n0, n1, n2) grid
(C order, dim 2 contiguous). It evaluates a DAG of primitive per-voxel nodes
(``PNode``) whose leaves are fields in HBM and scalars from the device scalar
table, and for every voxel delivers its *roots*: values stored to output fields,
values folded into FP64 reduction partials, and running (scan) integrals.

Primitives (every graph operator is lowered onto these, see ``lowering.py``):

* ``field`` / ``scalar`` leaves;
* pointwise math: add sub mul div neg exp log sqrt sin cos tanh abs clamp, trace,
  eig (3×3 symmetric eigenvalues), select, stack, normalize, norm, surfnorm
  ((−a, −b, 1)/|·|);
* ``d1``: first derivative of (one component of) a node along one axis, with the
  edge rule of the operator that produced it — ``periodic`` (wrapped central
  difference, torch.roll semantics), ``edge2`` / ``edge1`` (torch.gradient's
  one-sided second/first-order edges), ``zero`` (axis of length 1);
* ``lap``: compact 7-point Laplacian with a padding rule (periodic, replicate,
  zero, reflect);
* ``taps``: weighted sum of a node at compile-time offsets within a reach (box
  and Gaussian smoothing), out-of-range offsets remapped by a padding rule.

Kernel shape (``emit_pass``): a CTA owns a TJ × TK tile of the (dim1, dim2) plane
and marches along dim 0 over a segment of planes. Every field read at an offset
is staged plane by plane into a shared-memory ring of 2R+1+P slots (R = the
pass's stencil reach, P = prefetch depth), by TMA (``cp.async.bulk.tensor``, one
elected thread, mbarrier completion) when the layout allows it, else by row staging
(16-byte ``cp.async`` copies of the units covering each row, shifted into place in
shared memory). Voxels at least R away from every face take the *fast* path:
central formulas reading the ring at compile-time offsets. Voxels within R of a
face take the *slow* path: the same DAG evaluated from global memory with each
operator's own boundary rule. Compute is FP32; reductions accumulate in FP64.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field as dc_field
from typing import Dict, List, Optional, Sequence, Tuple

HEADER_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "include", "sten_device.cuh")

CTYPE = {"f32": "float", "f64": "double", "bf16": "bf16_t", "f16": "f16_t"}
ESIZE = {"f32": 4, "f64": 8, "bf16": 2, "f16": 2}


# ----------------------------------------------------------------------------- IR
@dataclass
class PNode:
    id: int
    op: str
    ins: Tuple[int, ...]
    nc: int
    attrs: Tuple[Tuple[str, object], ...] = ()
    radius: int = 0

    def a(self, key, default=None):
        for k, v in self.attrs:
            if k == key:
                return v
        return default


class PGraph:
    """Hash-consed DAG of primitive nodes for one pass."""

    def __init__(self) -> None:
        self.nodes: List[PNode] = []
        self._memo: Dict[Tuple, int] = {}

    def add(self, op: str, ins: Sequence[int], nc: int, radius: int = 0, **attrs) -> int:
        items = tuple(sorted(attrs.items()))
        key = (op, tuple(ins), nc, items)
        hit = self._memo.get(key)
        if hit is not None:
            return hit
        nid = len(self.nodes)
        self.nodes.append(PNode(nid, op, tuple(ins), nc, items, radius))
        self._memo[key] = nid
        return nid

    def radius_of(self, nid: int) -> int:
        return self.nodes[nid].radius


@dataclass
class FieldSpec:
    slot: int           # index into Params::fld
    dtype: str          # f32 / bf16 / f16 / f64
    nc: int             # interleaved components per voxel (1, 3, 9)
    staged: bool = False  # held in a shared-memory plane ring
    tma: bool = False     # ring filled by TMA (else by row staging)
    halo: int = 0         # j/k halo of the staged tile (0 for fields read only at the voxel)
    wrap_k: bool = False  # periodic ghosts along dim 2 come from extra TMA strips
    wrap_j: bool = False  # periodic ghosts along dim 1 come from extra TMA strips


@dataclass
class RootSpec:
    kind: str           # "out" | "red" | "scan" | "hist"
    node: int           # PNode id
    out_slot: int = -1  # for out/scan: index into Params::out
    out_dtype: str = "f32"
    red: str = ""       # sum | sumsq | var | entropy | integrate | minmax | hist
    slot: int = -1      # first partial slot (red) / histogram base (hist)
    bins: int = 0
    lohi_index: int = -1  # hist: scalar-table index of (min, max)
    table_index: int = -1  # hist: scalar-table index of the entropy
    dx: Tuple[float, float, float] = (1.0, 1.0, 1.0)  # integrate / scan spacing
    method: str = "simpson"


@dataclass
class PassConfig:
    tj: int = 8
    tk: int = 64
    threads: int = 128
    prefetch: int = 2
    seg_len: int = 64
    min_blocks: int = 1
    ghost: bool = True   # evaluate dim-1/dim-2 faces in the z-march (else in the shell kernel)
    kv: int = 1          # k-adjacent voxels per thread (one vector chunk per row in shared memory)


@dataclass
class PassSpec:
    graph: PGraph
    fields: List[FieldSpec]
    roots: List[RootSpec]
    n_scalars: int
    nslots: int                 # FP64 partial slots per CTA
    radius: int
    cfg: PassConfig = dc_field(default_factory=PassConfig)
    has_scan: bool = False
    # ghost-cell mode: {(field slot, axis): rule}; None when some stencil is nested
    ghosts: Optional[Dict[Tuple[int, int], str]] = None
    i_periodic: bool = False   # every tap along dim 0 wraps: planes are loaded wrapped
    nested_ok: bool = False    # dims 1 and 2 have >= 4 points (two-layer extrapolation)
    idx32: bool = False        # every element offset of every array, plus one stride of
                               # the shell launch, fits in an int: the boundary (shell)
                               # code indexes in 32-bit arithmetic

    def hk(self, f: FieldSpec) -> int:
        """k-halo in elements. TMA-staged fields: rounded so TMA x-coordinates stay
        16-byte aligned. Row-staged fields: the least halo >= f.halo that keeps each
        thread's vector chunk aligned in the ring and the box row a whole number of
        16-byte units."""
        if f.halo == 0:
            return 0
        es = ESIZE[f.dtype]
        if f.tma:
            a = 16 // es
            return ((f.halo + a - 1) // a) * a
        cw = self.cfg.kv * f.nc * es
        vec = 16 if cw % 16 == 0 else (8 if cw % 8 == 0 else (4 if cw % 4 == 0 else es))
        hk = f.halo
        # an extrapolated ghost at the last column reads the 3 (two layers: 4) columns
        # before it, which a tile holding only that column has in its halo only
        rk = (self.ghosts or {}).get((f.slot, 2))
        if rk in ("edge2", "edge2x2"):
            hk = max(hk, 3 if rk == "edge2x2" else 2)
        while (hk * f.nc * es) % vec or ((self.cfg.tk + 2 * hk) * f.nc * es) % 16:
            hk += 1
            assert hk <= f.halo + 64, "no k-halo keeps row-staged chunks aligned"
        return hk

    def box(self, f: FieldSpec) -> Tuple[int, int]:
        """(row width in elements, rows) of one staged plane tile."""
        return ((self.cfg.tk + 2 * self.hk(f)) * f.nc, self.cfg.tj + 2 * f.halo)


_REMAP_RULES = ("periodic", "replicate", "reflect")
STENCIL_PRIMS = ("d1", "lap", "taps")   # primitives that read their input at offsets
RED_SCRATCH_DOUBLES = 6 * 32   # block-reduction scratch: six values per warp (co-moments)
_EXTRAPOLATED = ("edge2", "edge1", "edge2x2")  # ghost rules that compute a value, not copy one


def analyse_ghosts(spec: "PassSpec") -> None:
    """Decide whether the z-march can evaluate the dim-1/dim-2 faces itself.

    It can when every stencil is single-level (no d1/lap below another): then each
    boundary rule is reproduced by a ghost cell next to the face — periodic wrap,
    replicate, reflect and zero padding by the value they read; torch.gradient's
    one-sided edges by extrapolation (quadratic for edge order 2: with
    f[-1] = 3f0 - 3f1 + f2 the central difference equals (-3f0 + 4f1 - f2)/2h;
    linear for edge order 1). Index-remap rules commute with pointwise ops, so they
    also apply through pointwise subexpressions; zero padding and extrapolation only
    when the stencil reads the field directly. Each (field, axis) must get one rule.
    Extrapolated ghosts are only written into FP32/FP64 rings: a 16-bit ring would
    round them.
    """
    g = spec.graph
    spec.ghosts = None
    spec.i_periodic = False
    for f in spec.fields:
        f.wrap_k = f.wrap_j = False
    if spec.radius == 0 or spec.has_scan or not spec.cfg.ghost:
        return

    def subtree(nid, acc):
        n = g.nodes[nid]
        acc.add(nid)
        for x in n.ins:
            subtree(x, acc)
        return acc

    rules: Dict[Tuple[int, int], str] = {}
    i_periodic = True

    def second_derivative(n) -> bool:
        """d1(d1(field, a), a), both with edge order 2: reproduced by two ghost layers."""
        inner = g.nodes[n.ins[0]]
        return (spec.nested_ok and n.op == "d1" and n.a("mode") == "edge2" and inner.op == "d1"
                and inner.a("mode") == "edge2" and inner.a("axis") == n.a("axis")
                and g.nodes[inner.ins[0]].op == "field")

    live: set = set()
    for r in spec.roots:
        subtree(r.node, live)
    for n in g.nodes:
        if n.op not in STENCIL_PRIMS or n.id not in live:
            continue
        if n.op == "taps":
            # diagonal taps read the tile's corner cells, which the ghost fill does not
            # write: every face goes to the shell kernel
            return
        sub = subtree(n.ins[0], set())
        nested = any(g.nodes[x].op in STENCIL_PRIMS for x in sub)
        if nested and not second_derivative(n):
            return
        direct = g.nodes[n.ins[0]].op == "field" or nested
        if n.op == "lap":
            rule, axes = n.a("pad"), (0, 1, 2)
        else:
            rule, axes = n.a("mode"), (n.a("axis"),)
            if rule == "zero":
                continue
            if nested:
                rule = "edge2x2"
        if rule not in _REMAP_RULES and not direct:
            return
        for x in sub:
            if g.nodes[x].op != "field":
                continue
            slot = g.nodes[x].a("field")
            if rule in _EXTRAPOLATED and spec.fields[slot].dtype in ("bf16", "f16"):
                # the ring stores the field's own dtype: an extrapolated ghost would be
                # rounded to 16 bits, so these faces are left to the shell kernel
                return
            for ax in axes:
                have = rules.setdefault((slot, ax), rule)
                if have != rule:
                    # the two-layer rule's first layer is the edge-order-2 ghost
                    if {have, rule} == {"edge2", "edge2x2"}:
                        rules[(slot, ax)] = "edge2x2"
                        continue
                    return
                if ax == 0 and rule != "periodic":
                    i_periodic = False
    spec.ghosts = rules
    spec.i_periodic = i_periodic
    for f in spec.fields:
        f.wrap_k = f.tma and f.halo > 0 and rules.get((f.slot, 2)) == "periodic"
        f.wrap_j = f.tma and f.halo > 0 and rules.get((f.slot, 1)) == "periodic"


def valid_shape(cfg: "PassConfig") -> bool:
    """Thread mapping: TK/KV threads along k (each KV adjacent voxels), the block's
    other threads along j, VPT = TJ / (threads / (TK/KV)) rows each."""
    if cfg.kv not in (1, 2, 4, 8) or cfg.tk % 32 or cfg.tk % cfg.kv or cfg.prefetch < 1:
        return False
    tkt = cfg.tk // cfg.kv
    if cfg.threads % tkt:
        return False
    rows = cfg.threads // tkt
    return cfg.tj % rows == 0 and cfg.tj // rows >= 1


FLAT_V = 4       # voxels per thread per step of a flat (stencil-free) pass
FLAT_ITER = 32   # steps per work item: an item covers threads x FLAT_V x FLAT_ITER voxels


def is_flat(spec: "PassSpec") -> bool:
    """A pass without stencils or scans runs flat: its voxels as one linear range,
    each thread FLAT_V consecutive voxels per step with vector loads, no staging."""
    return spec.radius == 0 and not spec.has_scan


def pass_grid(spec: "PassSpec", n1: int, n2: int, n_out: int) -> Tuple[int, int]:
    """(tiles or chunks, z-segments) of one launch covering ``n_out`` planes."""
    cfg = spec.cfg
    if is_flat(spec):
        ch = cfg.threads * FLAT_V * FLAT_ITER
        return max(1, -(-(n_out * n1 * n2) // ch)), 1
    return -(-n1 // cfg.tj) * -(-n2 // cfg.tk), max(1, -(-n_out // cfg.seg_len))


def with_config(spec: "PassSpec", cfg: "PassConfig") -> "PassSpec":
    """Copy of ``spec`` under another schedule (fields copied, ghost plan redone)."""
    import dataclasses
    out = dataclasses.replace(spec, cfg=cfg, fields=[dataclasses.replace(f) for f in spec.fields])
    analyse_ghosts(out)
    return out


def shell_regions(spec: "PassSpec") -> str:
    """Which boundary regions the shell kernel evaluates: all faces ("ABC"), only the
    dim-0 faces ("A", ghost mode), or none."""
    if spec.radius == 0 or spec.has_scan:
        return ""
    if spec.ghosts is None:
        return "ABC"
    return "" if spec.i_periodic else "A"


def _lit(x: float) -> str:
    if x != x:
        return "__int_as_float(0x7fc00000)"
    if math.isinf(x):
        return "__int_as_float(0x7f800000)" if x > 0 else "__int_as_float(0xff800000)"
    return repr(float(x)) + "f"


# ----------------------------------------------------------------------------- emitter
class _Emitter:
    def __init__(self, spec: PassSpec):
        self.s = spec
        self.flat = is_flat(spec)
        self.g = spec.graph
        self.R = spec.radius
        self.lines: List[str] = []
        self.tmp = 0
        # which nodes need offset (fast) / point (slow) functions (live nodes only:
        # lowering may leave unused components behind)
        live: set = set()
        stack = [r.node for r in spec.roots]
        while stack:
            x = stack.pop()
            if x not in live:
                live.add(x)
                stack += list(self.g.nodes[x].ins)
        self.need_fn = set()
        for n in self.g.nodes:
            if n.op in STENCIL_PRIMS and n.id in live:
                self._mark(n.ins[0])

    def _mark(self, nid: int) -> None:
        if nid in self.need_fn:
            return
        self.need_fn.add(nid)
        for i in self.g.nodes[nid].ins:
            self._mark(i)

    def t(self) -> str:
        self.tmp += 1
        return f"t{self.tmp}"

    # -- pointwise op body: inputs are C array names, output array name o
    def pointwise(self, n: PNode, ins: List[str], o: str, out: List[str]) -> None:
        op = n.op
        g = self.g

        def comp(arr, nid, c):
            return f"{arr}[{0 if g.nodes[nid].nc == 1 else c}]"

        if op in ("add", "sub", "mul", "div"):
            a, b = ins
            for c in range(n.nc):
                x, y = comp(a, n.ins[0], c), comp(b, n.ins[1], c)
                if op == "div":
                    out.append(f"{o}[{c}] = sten_div({x}, {y}, {_lit(n.a('eps', 1e-15))});")
                else:
                    sym = {"add": "+", "sub": "-", "mul": "*"}[op]
                    out.append(f"{o}[{c}] = {x} {sym} {y};")
        elif op == "mulk":
            for c in range(n.nc):
                out.append(f"{o}[{c}] = {ins[0]}[{c}] * {_lit(n.a('k'))};")
        elif op in ("neg", "exp", "sin", "cos", "tanh", "abs"):
            fn = {"neg": "-", "exp": "expf", "sin": "sinf", "cos": "cosf", "tanh": "tanhf", "abs": "fabsf"}[op]
            for c in range(n.nc):
                out.append(f"{o}[{c}] = {fn}({ins[0]}[{c}]);")
        elif op == "log":
            for c in range(n.nc):
                out.append(f"{o}[{c}] = sten_log({ins[0]}[{c}], {_lit(n.a('eps', 1e-15))});")
        elif op == "sqrt":
            for c in range(n.nc):
                out.append(f"{o}[{c}] = sten_sqrt({ins[0]}[{c}], {_lit(n.a('eps', 0.0))});")
        elif op == "clamp":
            lo = comp(ins[1], n.ins[1], 0) if len(ins) > 1 else _lit(n.a("lo", 0.0))
            hi = comp(ins[2], n.ins[2], 0) if len(ins) > 2 else _lit(n.a("hi", 1.0))
            for c in range(n.nc):
                lo_c = comp(ins[1], n.ins[1], c) if len(ins) > 1 else lo
                hi_c = comp(ins[2], n.ins[2], c) if len(ins) > 2 else hi
                out.append(f"{o}[{c}] = sten_clamp({ins[0]}[{c}], {lo_c}, {hi_c});")
        elif op == "trace":
            out.append(f"{o}[0] = {ins[0]}[0] + {ins[0]}[4] + {ins[0]}[8];")
        elif op == "eig":
            out.append(f"eig3_sym({ins[0]}, {o});")
        elif op == "select":
            k = int(n.a("index"))
            for c in range(n.nc):
                out.append(f"{o}[{c}] = {ins[0]}[{k * n.nc + c}];")
        elif op == "stack":
            c = 0
            for arr, nid in zip(ins, n.ins):
                for cc in range(g.nodes[nid].nc):
                    out.append(f"{o}[{c}] = {arr}[{cc}];")
                    c += 1
        elif op == "normalize":
            a = ins[0]
            m = self.t()
            out.append(f"float {m} = sqrtf({a}[0]*{a}[0] + {a}[1]*{a}[1] + {a}[2]*{a}[2]);")
            out.append(f"{m} = fmaxf({m}, {_lit(n.a('eps', 1e-15))});")
            for c in range(3):
                out.append(f"{o}[{c}] = {a}[{c}] / {m};")
        elif op == "surfnorm":
            gx, gy = ins[0] + "[0]", ins[1] + "[0]"
            m = self.t()
            out.append(f"const float {m} = fmaxf(sqrtf({gx}*{gx} + {gy}*{gy} + 1.0f), 1e-15f);")
            out.append(f"{o}[0] = -{gx} / {m};")
            out.append(f"{o}[1] = -{gy} / {m};")
            out.append(f"{o}[2] = 1.0f / {m};")
        elif op == "norm":
            a = ins[0]
            nrm = f"sqrtf({' + '.join(f'{a}[{c}]*{a}[{c}]' for c in range(self.g.nodes[n.ins[0]].nc))})"
            eps = n.a("eps")
            out.append(f"{o}[0] = {nrm};" if eps is None else f"{o}[0] = fmaxf({nrm}, {_lit(eps)});")
        elif op == "det3":
            a = ins[0]
            d = self.t()
            out.append(f"float {d} = {a}[0] * ({a}[4] * {a}[8] - {a}[5] * {a}[7]) - {a}[1] * ({a}[3] * {a}[8] - {a}[5] * {a}[6])"
                       f" + {a}[2] * ({a}[3] * {a}[7] - {a}[4] * {a}[6]);")
            # nan -> 0, then clamped to +-1e30 (infinities included)
            out.append(f"{o}[0] = ({d} != {d}) ? 0.0f : fminf(fmaxf({d}, -1e30f), 1e30f);")
        elif op == "inv3":
            a = ins[0]
            c = [f"({a}[4] * {a}[8] - {a}[5] * {a}[7])", f"({a}[5] * {a}[6] - {a}[3] * {a}[8])",
                 f"({a}[3] * {a}[7] - {a}[4] * {a}[6])", f"({a}[2] * {a}[7] - {a}[1] * {a}[8])",
                 f"({a}[0] * {a}[8] - {a}[2] * {a}[6])", f"({a}[1] * {a}[6] - {a}[0] * {a}[7])",
                 f"({a}[1] * {a}[5] - {a}[2] * {a}[4])", f"({a}[2] * {a}[3] - {a}[0] * {a}[5])",
                 f"({a}[0] * {a}[4] - {a}[1] * {a}[3])"]
            cof = self.t()
            out.append(f"float {cof}[9] = {{{', '.join(c)}}};")   # cofactor matrix, row-major
            det = self.t()
            out.append(f"const float {det} = {a}[0] * {cof}[0] + {a}[1] * {cof}[1] + {a}[2] * {cof}[2];")
            for i in range(3):
                for j in range(3):
                    out.append(f"{o}[{3 * i + j}] = {cof}[{3 * j + i}] / {det};")
        elif op == "aat3":
            a = ins[0]   # A·Aᵀ: entry (i, j) = row i · row j
            for i in range(3):
                for j in range(3):
                    out.append(f"{o}[{3 * i + j}] = ({a}[{3 * i}] * {a}[{3 * j}] + {a}[{3 * i + 1}] * {a}[{3 * j + 1}])"
                               f" + {a}[{3 * i + 2}] * {a}[{3 * j + 2}];")
        elif op == "dev3":
            a = ins[0]
            q = self.t()
            out.append(f"const float {q} = ({a}[0] + {a}[4] + {a}[8]) / 3.0f;")
            for i in range(3):
                for j in range(3):
                    v = f"{a}[{3 * i + j}] - {q} * {'1.0f' if i == j else '0.0f'}"
                    out.append(f"{{ const float v_ = {v}; {o}[{3 * i + j}] = isfinite(v_) ? v_ : 0.0f; }}")
        else:
            raise NotImplementedError(f"codegen: pointwise op {op}")

    # -- fast (interior) functions: template offsets
    def emit_fast_fns(self) -> None:
        for n in self.g.nodes:
            if n.id not in self.need_fn:
                continue
            body: List[str] = []
            self.fast_value(n, "DI", "DJ", "DK", "o", body)
            self.lines.append(f"template <int DI, int DJ, int DK> __device__ __forceinline__ void "
                              f"FF{n.id}(const FCtx& x, float* o) {{")
            self.lines += ["  " + b for b in body]
            self.lines.append("}")

    def fast_call(self, nid: int, di: str, dj: str, dk: str, body: List[str]) -> str:
        arr = self.t()
        body.append(f"float {arr}[{self.g.nodes[nid].nc}];")
        n = self.g.nodes[nid]
        if n.op == "field":
            self.field_fast(n, di, dj, dk, arr, body)
        elif n.op == "scalar":
            body.append(f"{arr}[0] = x.sc[{n.a('index')}];")
        else:
            body.append(f"FF{nid}<{di}, {dj}, {dk}>(x, {arr});")
        return arr

    def field_fast(self, n: PNode, di, dj, dk, arr, body):
        f = self.s.fields[n.a("field")]
        if f.staged:
            for c in range(n.nc):
                body.append(f"{arr}[{c}] = LDF{f.slot}<{di}, {dj}, ({dk}) * {f.nc} + {c}>(x);")
        elif di != "0" or dj not in ("0", "M") or dk not in ("0", "KK"):
            raise AssertionError("unstaged field read at an offset")
        elif self.flat:
            for c in range(n.nc):
                body.append(f"{arr}[{c}] = x.fv{f.slot}[({dk}) * {f.nc} + {c}];")
        else:
            for c in range(n.nc):
                body.append(f"{arr}[{c}] = ldg_as_f32(x.gp{f.slot} + {c});")

    def central_diffs(self, d: PNode, di: str, dj: str, dk: str, body: List[str]) -> List[str]:
        """Per component, the unscaled central difference f(+1) - f(-1) of the d1 node d
        along its axis at offset (di, dj, dk). From a 16-bit staged field the minuend
        is not converted: one mixed-precision subtraction (LDS) takes it as stored
        and the subtrahend as FP32 (the same rounding as the FP32 difference)."""
        off = [di, dj, dk]
        ax, comp = d.a("axis"), d.a("comp")
        plus = list(off); plus[ax] = f"({off[ax]}) + 1"
        minus = list(off); minus[ax] = f"({off[ax]}) - 1"
        src = self.g.nodes[d.ins[0]]
        b = self.fast_call(d.ins[0], *minus, body)
        cs = [c if comp is None else comp for c in range(d.nc)]
        if src.op == "field":
            f = self.s.fields[src.a("field")]
            if f.staged and ESIZE[f.dtype] == 2:
                return [f"LDS{f.slot}<{plus[0]}, {plus[1]}, ({plus[2]}) * {f.nc} + {c}>(x, {b}[{c}])" for c in cs]
        a = self.fast_call(d.ins[0], *plus, body)
        return [f"({a}[{c}] - {b}[{c}])" for c in cs]

    def fast_value(self, n: PNode, di: str, dj: str, dk: str, o: str, body: List[str]) -> None:
        """Statements computing node n at offset (di,dj,dk) into array o (interior)."""
        if n.op == "field":
            self.field_fast(n, di, dj, dk, o, body)
            return
        if n.op == "scalar":
            body.append(f"{o}[0] = x.sc[{n.a('index')}];")
            return
        if n.op == "d1":
            ax = n.a("axis")
            comp = n.a("comp")
            mode = n.a("mode")
            if mode == "zero":
                for c in range(n.nc):
                    body.append(f"{o}[{c}] = 0.0f;")
                return
            s = _lit(n.a("inv2h"))
            for c, dv in enumerate(self.central_diffs(n, di, dj, dk, body)):
                body.append(f"{o}[{c}] = {dv} * {s};")
            return
        if n.op == "lap":
            off = [di, dj, dk]
            ctr = self.fast_call(n.ins[0], di, dj, dk, body)
            terms = []
            for ax in range(3):
                plus = list(off); plus[ax] = f"({off[ax]}) + 1"
                minus = list(off); minus[ax] = f"({off[ax]}) - 1"
                a = self.fast_call(n.ins[0], *plus, body)
                b = self.fast_call(n.ins[0], *minus, body)
                terms.append((a, b, _lit(n.a("invh2")[ax])))
            h2 = n.a("invh2")
            src = self.g.nodes[n.ins[0]]
            f16 = None
            if src.op == "field":
                fs = self.s.fields[src.a("field")]
                f16 = fs if fs.staged and ESIZE[fs.dtype] == 2 else None
            for c in range(n.nc):
                if h2[0] == h2[1] == h2[2]:
                    # equal spacing: the six neighbours summed, then one fused -6 c; from a
                    # 16-bit staged field each pair's first value is added as stored
                    # (add.f32.f16: the rounding of the FP32 sum, without its conversion)
                    if f16 is not None:
                        pairs = []
                        for ax in range(3):
                            q = list(off); q[ax] = f"({off[ax]}) + 1"
                            pairs.append(f"LDA{f16.slot}<{q[0]}, {q[1]}, ({q[2]}) * {f16.nc} + {c}>(x, {terms[ax][1]}[{c}])")
                        ssum = " + ".join(f"({t})" for t in pairs)
                    else:
                        ssum = " + ".join(f"({a}[{c}] + {b}[{c}])" for a, b, _ in terms)
                    v = f"fmaf(-6.0f, {ctr}[{c}], {ssum})"
                    body.append(f"{o}[{c}] = {v if h2[0] == 1.0 else f'{v} * {terms[0][2]}'};")
                    continue
                parts = [f"(({a}[{c}] + {b}[{c}]) - 2.0f * {ctr}[{c}]) * {s}" for a, b, s in terms]
                body.append(f"{o}[{c}] = ({parts[0]} + {parts[1]}) + {parts[2]};")
            return
        if n.op == "taps":
            off = [di, dj, dk]
            vals = []
            for tap in n.a("taps"):
                q = [off[ax] if not tap[ax] else
                     (f"({off[ax]}) + {tap[ax]}" if tap[ax] > 0 else f"({off[ax]}) - {-tap[ax]}")
                     for ax in range(3)]
                vals.append((self.fast_call(n.ins[0], *q, body), tap[3]))
            self._tap_sum(n, vals, o, body)
            return
        if self.d1_pair(n):
            self.d1_pair_value(n, di, dj, dk, o, body)
            return
        ins = [self.fast_call(i, di, dj, dk, body) for i in n.ins]
        self.pointwise(n, ins, o, body)

    def d1_pair(self, n: PNode) -> bool:
        """A sum or difference of two central first differences with one spacing (the
        curl's components): scaled once, after the difference of the differences."""
        if n.op not in ("add", "sub") or len(n.ins) != 2:
            return False
        a, b = (self.g.nodes[i] for i in n.ins)
        return (a.op == b.op == "d1" and a.a("mode") != "zero" and b.a("mode") != "zero"
                and a.a("inv2h") == b.a("inv2h") and a.nc == b.nc == n.nc)

    def d1_pair_value(self, n: PNode, di: str, dj: str, dk: str, o: str, body: List[str]) -> None:
        """o = ((a1 - b1) +/- (a2 - b2)) * inv2h for the two d1 inputs of n (the same
        value as scaling each difference first when inv2h is a power of two)."""
        raws = [self.central_diffs(self.g.nodes[nid], di, dj, dk, body) for nid in n.ins]
        sym = "+" if n.op == "add" else "-"
        s = _lit(self.g.nodes[n.ins[0]].a("inv2h"))
        for c in range(n.nc):
            body.append(f"{o}[{c}] = ({raws[0][c]} {sym} {raws[1][c]}) * {s};")

    def point_raw(self, nid: int, body: List[str]) -> str:
        """Interior value of node nid (``raw_scale(graph, nid)`` is not None) at the
        thread's voxel (0, M, KK) without its spacing factor: central differences
        and stacks of them left unscaled."""
        n = self.g.nodes[nid]
        arr = self.t()
        if n.op == "stack":
            parts = [self.point_raw(i, body) for i in n.ins]
            body.append(f"float {arr}[{n.nc}];")
            self.pointwise(n, parts, arr, body)
            return arr
        body.append(f"float {arr}[{n.nc}];")
        pair = n.op != "d1"
        raws = [self.central_diffs(d, "0", "M", "KK", body)
                for d in ([self.g.nodes[i] for i in n.ins] if pair else [n])]
        for c in range(n.nc):
            v = raws[0][c] if not pair else f"{raws[0][c]} {'+' if n.op == 'add' else '-'} {raws[1][c]}"
            body.append(f"{arr}[{c}] = {v};")
        return arr

    def _tap_sum(self, n: PNode, vals, o: str, body: List[str]) -> None:
        """o = scale * Σ w·v over (array, weight) pairs, accumulated in tap order."""
        for c in range(n.nc):
            acc = None
            for arr, w in vals:
                term = f"{arr}[{c}]" if w == 1.0 else f"{arr}[{c}] * {_lit(w)}"
                if acc is None:
                    acc = self.t()
                    body.append(f"float {acc} = {term};")
                elif w == 1.0:
                    body.append(f"{acc} += {arr}[{c}];")
                else:
                    body.append(f"{acc} = fmaf({arr}[{c}], {_lit(w)}, {acc});")
            body.append(f"{o}[{c}] = {acc} * {_lit(n.a('scale'))};")

    # -- slow (boundary) functions: runtime global coordinates
    def emit_slow_fns(self) -> None:
        order = sorted(self.need_fn)
        for nid in order:
            self.lines.append(f"__device__ __noinline__ void SS{nid}(const Params& p, "
                              f"int i, int j, int k, float* o);")
        for nid in order:
            n = self.g.nodes[nid]
            body: List[str] = []
            self.slow_value(n, "i", "j", "k", "o", body)
            self.lines.append(f"__device__ __noinline__ void SS{nid}(const Params& p, "
                              f"int i, int j, int k, float* o) {{")
            self.lines += ["  " + b for b in body]
            self.lines.append("}")

    def slow_call(self, nid: int, i: str, j: str, k: str, body: List[str]) -> str:
        arr = self.t()
        n = self.g.nodes[nid]
        body.append(f"float {arr}[{n.nc}];")
        if n.op == "field":
            self.field_slow(n, i, j, k, arr, body)
        elif n.op == "scalar":
            body.append(f"{arr}[0] = (float)__ldcg(p.scal + {n.a('index')});")
        elif nid in self.need_fn:
            body.append(f"SS{nid}(p, {i}, {j}, {k}, {arr});")
        else:
            self.slow_value(n, i, j, k, arr, body)
        return arr

    def field_slow(self, n: PNode, i, j, k, arr, body):
        f = self.s.fields[n.a("field")]
        ct = CTYPE[f.dtype]
        base = self.t()
        if self.s.idx32:
            body.append(f"const {ct}* {base} = (const {ct}*)p.fld[{f.slot}] + "
                        f"((sten_plane(p, {i}) * p.n1 + ({j})) * p.n2 + ({k})) * {f.nc};")
        else:
            body.append(f"const {ct}* {base} = (const {ct}*)p.fld[{f.slot}] + "
                        f"(((size_t)sten_plane(p, {i}) * p.n1 + ({j})) * p.n2 + ({k})) * {f.nc};")
        for c in range(n.nc):
            body.append(f"{arr}[{c}] = ldg_as_f32({base} + {c});")

    def slow_value(self, n: PNode, i: str, j: str, k: str, o: str, body: List[str]) -> None:
        if n.op == "field":
            self.field_slow(n, i, j, k, o, body)
            return
        if n.op == "scalar":
            body.append(f"{o}[0] = (float)__ldcg(p.scal + {n.a('index')});")
            return
        if n.op == "d1":
            self.slow_d1(n, i, j, k, o, body)
            return
        if n.op == "lap":
            self.slow_lap(n, i, j, k, o, body)
            return
        if n.op == "taps":
            self.slow_taps(n, i, j, k, o, body)
            return
        ins = [self.slow_call(x, i, j, k, body) for x in n.ins]
        self.pointwise(n, ins, o, body)

    def slow_d1(self, n: PNode, i, j, k, o, body):
        ax = n.a("axis")
        mode = n.a("mode")
        comp = n.a("comp")
        nn = ["p.n0g", "p.n1", "p.n2"][ax]
        crd = [i, j, k]
        cc = (lambda c: c) if comp is None else (lambda c: comp)
        if mode == "zero":
            for c in range(n.nc):
                body.append(f"{o}[{c}] = 0.0f;")
            return

        def at(expr):
            q = list(crd)
            q[ax] = expr
            return q

        x = crd[ax]
        s2 = _lit(n.a("inv2h"))
        if mode == "periodic":
            a = self.slow_call(n.ins[0], *at(f"wrap_idx(({x}) + 1, {nn})"), body)
            b = self.slow_call(n.ins[0], *at(f"wrap_idx(({x}) - 1, {nn})"), body)
            for c in range(n.nc):
                body.append(f"{o}[{c}] = ({a}[{cc(c)}] - {b}[{cc(c)}]) * {s2};")
            return
        # torch.gradient edges, second order (edge2: (-3f0 + 4f1 - f2) / 2h) or first
        # order (edge1: (f1 - f0) / h), both faces in one branch: the face point x
        # and the inward step d (+1 at 0, -1 at n - 1); the last face's formula is the
        # first's mirrored, (3f0 - 4f1 + f2) / 2h = -(first at d = -1), so the scale
        # takes d's sign (an exact negation). One branch keeps a warp whose lanes
        # hold both faces' voxels (a row's first and last columns) from running both.
        body.append(f"if (({x}) > 0 && ({x}) < {nn} - 1) {{")
        sub: List[str] = []
        a = self.slow_call(n.ins[0], *at(f"({x}) + 1"), sub)
        b = self.slow_call(n.ins[0], *at(f"({x}) - 1"), sub)
        for c in range(n.nc):
            sub.append(f"{o}[{c}] = ({a}[{cc(c)}] - {b}[{cc(c)}]) * {s2};")
        body += ["  " + s for s in sub]
        body.append("} else {")
        dd = self.t()
        sub = [f"const int {dd} = ({x}) == 0 ? 1 : -1;"]
        e0 = self.slow_call(n.ins[0], *at(f"({x})"), sub)
        e1 = self.slow_call(n.ins[0], *at(f"({x}) + {dd}"), sub)
        if mode == "edge2":
            e2 = self.slow_call(n.ins[0], *at(f"({x}) + 2 * {dd}"), sub)
            sc = self.t()
            sub.append(f"const float {sc} = {dd} > 0 ? {s2} : -{s2};")
            for c in range(n.nc):
                sub.append(f"{o}[{c}] = ((-3.0f * {e0}[{cc(c)}] + 4.0f * {e1}[{cc(c)}]) - {e2}[{cc(c)}]) * {sc};")
        else:
            s1 = _lit(n.a("invh"))
            sc = self.t()
            sub.append(f"const float {sc} = {dd} > 0 ? {s1} : -{s1};")
            for c in range(n.nc):
                sub.append(f"{o}[{c}] = ({e1}[{cc(c)}] - {e0}[{cc(c)}]) * {sc};")
        body += ["  " + s for s in sub]
        body.append("}")

    def slow_lap(self, n: PNode, i, j, k, o, body):
        pad = n.a("pad")
        crd = [i, j, k]
        dims = ["p.n0g", "p.n1", "p.n2"]
        ctr = self.slow_call(n.ins[0], i, j, k, body)
        terms = []
        for ax in range(3):
            nn = dims[ax]
            x = crd[ax]
            vals = []
            for sgn in ("+ 1", "- 1"):
                q = list(crd)
                arr = self.t()
                body.append(f"float {arr}[{n.nc}];")
                if pad == "periodic":
                    q[ax] = f"wrap_idx(({x}) {sgn}, {nn})"
                    got = self.slow_call(n.ins[0], *q, body)
                    body.append(f"for (int c = 0; c < {n.nc}; ++c) {arr}[c] = {got}[c];")
                elif pad == "replicate":
                    q[ax] = f"clamp_idx(({x}) {sgn}, {nn})"
                    got = self.slow_call(n.ins[0], *q, body)
                    body.append(f"for (int c = 0; c < {n.nc}; ++c) {arr}[c] = {got}[c];")
                elif pad == "reflect":
                    q[ax] = f"reflect_idx(({x}) {sgn}, {nn})"
                    body.append(f"if ({nn} > 1) {{")
                    sub: List[str] = []
                    got = self.slow_call(n.ins[0], *q, sub)
                    sub.append(f"for (int c = 0; c < {n.nc}; ++c) {arr}[c] = {got}[c];")
                    body += ["  " + s for s in sub]
                    body.append(f"}} else {{ for (int c = 0; c < {n.nc}; ++c) {arr}[c] = 0.0f; }}")
                else:  # zero padding
                    q[ax] = f"(({x}) {sgn})"
                    body.append(f"if (({x}) {sgn} >= 0 && ({x}) {sgn} < {nn}) {{")
                    sub = []
                    got = self.slow_call(n.ins[0], *q, sub)
                    sub.append(f"for (int c = 0; c < {n.nc}; ++c) {arr}[c] = {got}[c];")
                    body += ["  " + s for s in sub]
                    body.append(f"}} else {{ for (int c = 0; c < {n.nc}; ++c) {arr}[c] = 0.0f; }}")
                vals.append(arr)
            terms.append((vals[0], vals[1], _lit(n.a("invh2")[ax])))
        for c in range(n.nc):
            parts = [f"(({a}[{c}] + {b}[{c}]) - 2.0f * {ctr}[{c}]) * {s}" for a, b, s in terms]
            body.append(f"{o}[{c}] = ({parts[0]} + {parts[1]}) + {parts[2]};")

    def slow_taps(self, n: PNode, i, j, k, o, body):
        """Taps at runtime coordinates: remapped by the padding rule, or skipped
        (zero padding) when they fall outside the grid."""
        pad = n.a("pad")
        crd = [i, j, k]
        dims = ["p.n0g", "p.n1", "p.n2"]
        remap = {"periodic": "wrap_idx", "replicate": "clamp_idx", "reflect": "reflect_idx"}.get(pad)
        acc = self.t()
        body.append(f"float {acc}[{n.nc}];")
        body.append(f"for (int c = 0; c < {n.nc}; ++c) {acc}[c] = 0.0f;")
        for tap in n.a("taps"):
            q, conds = [], []
            for ax in range(3):
                d = tap[ax]
                if not d:
                    q.append(crd[ax])
                    continue
                e = f"({crd[ax]}) + {d}" if d > 0 else f"({crd[ax]}) - {-d}"
                if remap:
                    q.append(f"{remap}({e}, {dims[ax]})")
                else:
                    q.append(f"({e})")
                    conds.append(f"({e}) >= 0 && ({e}) < {dims[ax]}")
            sub: List[str] = []
            arr = self.slow_call(n.ins[0], *q, sub)
            w = tap[3]
            for c in range(n.nc):
                sub.append(f"{acc}[{c}] += {arr}[{c}]" + ("" if w == 1.0 else f" * {_lit(w)}") + ";")
            if conds:
                body.append(f"if ({' && '.join(conds)}) {{")
                body += ["  " + x for x in sub]
                body.append("}")
            else:
                body.append("{")
                body += ["  " + x for x in sub]
                body.append("}")
        for c in range(n.nc):
            body.append(f"{o}[{c}] = {acc}[{c}] * {_lit(n.a('scale'))};")

    # -- per-voxel root evaluation
    def emit_eval(self) -> None:
        roots = self.s.roots
        widths = [self.g.nodes[r.node].nc for r in roots]
        self.offsets = []
        acc = 0
        for w in widths:
            self.offsets.append(acc)
            acc += w
        self.nroot = max(acc, 1)
        # fast
        body: List[str] = []
        memo: Dict[int, str] = {}

        def point(nid: int) -> str:
            if nid in memo:
                return memo[nid]
            n = self.g.nodes[nid]
            if n.op in STENCIL_PRIMS or n.op == "field" or n.op == "scalar":
                arr = self.t()
                body.append(f"float {arr}[{n.nc}];")
                self.fast_value(n, "0", "M", "KK", arr, body)
            else:
                arr = self.t()
                if self.d1_pair(n):
                    body.append(f"float {arr}[{n.nc}];")
                    self.d1_pair_value(n, "0", "M", "KK", arr, body)
                    memo[nid] = arr
                    return arr
                ins = [point(i) for i in n.ins]
                body.append(f"float {arr}[{n.nc}];")
                self.pointwise(n, ins, arr, body)
            memo[nid] = arr
            return arr

        for r, off in zip(roots, self.offsets):
            arr = self.point_raw(r.node, body) if deferred_scale(self.s, r) else point(r.node)
            for c in range(self.g.nodes[r.node].nc):
                body.append(f"rv[{off + c}] = {arr}[{c}];")
        self.lines.append("template <int M, int KK> __device__ __forceinline__ void eval_fast(const FCtx& x, float* rv) {")
        self.lines += ["  " + b for b in body]
        self.lines.append("}")
        # slow
        body = []
        memo_s: Dict[int, str] = {}

        def spoint(nid: int) -> str:
            if nid in memo_s:
                return memo_s[nid]
            n = self.g.nodes[nid]
            if nid in self.need_fn or n.op in STENCIL_PRIMS or n.op in ("field", "scalar"):
                arr = self.t()
                body.append(f"float {arr}[{n.nc}];")
                self.slow_value(n, "i", "j", "k", arr, body)
            else:
                ins = [spoint(i) for i in n.ins]
                arr = self.t()
                body.append(f"float {arr}[{n.nc}];")
                self.pointwise(n, ins, arr, body)
            memo_s[nid] = arr
            return arr

        for r, off in zip(roots, self.offsets):
            arr = spoint(r.node)
            for c in range(self.g.nodes[r.node].nc):
                body.append(f"rv[{off + c}] = {arr}[{c}];")
        self.lines.append("__device__ __forceinline__ void eval_slow(const Params& p, "
                          "int i, int j, int k, float* rv) {")
        self.lines += ["  " + b for b in body]
        self.lines.append("}")


# ----------------------------------------------------------------------------- params layout
@dataclass
class ParamLayout:
    size: int
    offsets: Dict[str, int]


def param_layout(spec: PassSpec) -> ParamLayout:
    """Byte layout of ``struct Params`` (mirrors C++ alignment rules)."""
    off = 0
    offs: Dict[str, int] = {}

    def put(name, size, align):
        nonlocal off
        off = (off + align - 1) // align * align
        offs[name] = off
        off += size

    ntma = len(tmap_specs(spec))
    if ntma:
        put("tmap", 128 * ntma, 64)
    put("fld", 8 * max(len(spec.fields), 1), 8)
    nout = sum(1 for r in spec.roots if r.kind in ("out", "scan"))
    put("out", 8 * max(nout, 1), 8)
    put("scal", 8, 8)
    put("part", 8, 8)
    put("hist", 8, 8)
    put("err", 8, 8)
    for name in ("n0g", "n1", "n2", "nl", "i_base", "out_lo", "n_out", "seg_len", "tiles_k", "cta_off"):
        put(name, 4, 4)
    size = (off + 63) // 64 * 64
    return ParamLayout(size, offs)


# ----------------------------------------------------------------------------- kernel
def smem_layout(spec: PassSpec) -> Tuple[int, Dict[int, int], int]:
    """(total bytes, byte offset of each staged field's ring, offset of the
    block-reduction scratch). Ring slots are 128-byte aligned (TMA destinations)."""
    nslot = 2 * spec.radius + 1 + spec.cfg.prefetch
    off = 128  # mbarriers: up to 16 slots
    rings: Dict[int, int] = {}
    for f in spec.fields:
        if f.staged:
            rings[f.slot] = off
            off += plane_bytes(spec, f) * nslot
    off = (off + 127) // 128 * 128
    red_off = off
    off += RED_SCRATCH_DOUBLES * 8
    off += sum(4 * r.bins for r in spec.roots if r.kind == "red" and r.red == "hist")
    return off, rings, red_off


def _a128(x: int) -> int:
    return (x + 127) // 128 * 128


def strip_boxes(spec: PassSpec, f: FieldSpec) -> Tuple[Tuple[int, int], Tuple[int, int]]:
    """TMA boxes (elements wide, rows) of the periodic wrap strips: a dim-2 strip of
    hk columns for the tile's rows, and a dim-1 strip of ``halo`` rows across the
    tile's (haloed) width."""
    hk = spec.hk(f)
    return (hk * f.nc, spec.cfg.tj), ((spec.cfg.tk + 2 * hk) * f.nc, f.halo)


def slot_layout(spec: PassSpec, f: FieldSpec) -> Dict[str, int]:
    """Byte offsets inside one ring slot: the plane box, then wrap strips
    (left/right along dim 2, top/bottom along dim 1) when the field has them."""
    h = spec.box(f)[1]
    es = ESIZE[f.dtype]
    off = {"box": 0}
    o = _a128(ring_w(spec, f) * h * es)
    rule, ns = rs_strip(spec, f)
    if rule:                              # row-staged dim-2 strips: 2 faces x box rows
        off["rs_strip"] = ring_w(spec, f) * h * es
        o = _a128(off["rs_strip"] + 2 * h * ns * 16)
    (kw, kh), (jw, jh) = strip_boxes(spec, f)
    if f.wrap_k:
        off["kl"], off["kr"] = o, o + _a128(kw * kh * es)
        o += 2 * _a128(kw * kh * es)
    if f.wrap_j:
        off["jt"], off["jb"] = o, o + _a128(jw * jh * es)
        o += 2 * _a128(jw * jh * es)
    off["size"] = o
    return off


def plane_bytes(spec: PassSpec, f: FieldSpec) -> int:
    return slot_layout(spec, f)["size"]


def tmap_specs(spec: PassSpec) -> List[Tuple[int, str, Tuple[int, int]]]:
    """Ordered TMA descriptors of a pass: (field slot, "box" | "kstrip" | "jstrip", box)."""
    out = []
    for f in spec.fields:
        if not f.tma:
            continue
        out.append((f.slot, "box", spec.box(f)))
        ks, js = strip_boxes(spec, f)
        if f.wrap_k:
            out.append((f.slot, "kstrip", ks))
        if f.wrap_j:
            out.append((f.slot, "jstrip", js))
    return out


def _simpson_fn() -> str:
    return r"""
__device__ __forceinline__ double sten_simpson_w(int idx, int n, double h, int simpson) {
  // weight of sample idx in _simpson_1d's composite rule (or the trapezoid rule)
  if (!simpson || n < 3) {
    if (n < 2) return 0.0;
    return (idx == 0 || idx == n - 1) ? 0.5 * h : h;
  }
  const int m = (n % 2 == 1) ? n : n - 1;   // Simpson over the first m points
  double w = 0.0;
  if (idx < m) {
    w = (idx == 0 || idx == m - 1) ? 1.0 : ((idx % 2 == 1) ? 4.0 : 2.0);
    w *= h / 3.0;
  }
  if (n % 2 == 0 && (idx == n - 2 || idx == n - 1)) w += 0.5 * h;
  return w;
}
"""


def _epilogue(spec: PassSpec, e: "_Emitter", scan_ok: bool, skip: Sequence[RootSpec] = (),
              where: str = "main", m: int = 0, kk: int = 0, plane: bool = False) -> List[str]:
    """Per-voxel root handling (stores, reduction accumulation, scans). Expects
    ``rv`` (root values), ``vox`` (linear voxel index), ``gi, j, k`` and, for scans,
    the register slot ``mq``. Roots in ``skip`` are stored by the caller. With
    ``plane`` the roots of ``plane_roots`` accumulate per plane (``_plane_open`` /
    ``_plane_close``)."""
    K: List[str] = []
    pr = {id(r) for _, r in plane_roots(spec)} if plane else set()
    ri = si = 0
    for r, off in zip(spec.roots, e.offsets):  # noqa: C901
        nc = e.g.nodes[r.node].nc
        if any(r is x for x in skip):
            continue
        # z-march: per-plane row pointers advanced by the march (no 64-bit index math per voxel)
        tile_ptr = where == "main" and not is_flat(spec)
        if r.kind == "out":
            ct = CTYPE[r.out_dtype]
            if tile_ptr:
                K.append(f"{{ {ct}* o_ = orow{r.out_slot} + ro_[{{M}}] * {nc} + {{KK}} * {nc};")
            else:
                K.append(f"{{ {ct}* o_ = ({ct}*)p.out[{r.out_slot}] + (vox - out_base) * {nc};")
            for c in range(nc):
                K.append(f"  st_from_f32(o_ + {c}, rv[{off + c}]);")
            K.append("}")
        elif r.kind == "scan":
            assert scan_ok
            ct = CTYPE[r.out_dtype]
            half = repr(0.5 * float(r.dx[0]))
            if tile_ptr:
                K.append(f"{{ {ct}* o_ = orow{r.out_slot} + ro_[{{M}}] * {nc} + {{KK}} * {nc};")
            else:
                K.append(f"{{ {ct}* o_ = ({ct}*)p.out[{r.out_slot}] + (vox - out_base) * {nc};")
            for c in range(nc):
                q = f"mq * {nc} + {c}"
                K.append(f"  if (gi > 0) sc{si}_acc[{q}] += ((double)sc{si}_prev[{q}] + (double)rv[{off + c}]) * {half};")
                K.append(f"  sc{si}_prev[{q}] = rv[{off + c}];")
                K.append(f"  st_from_f64(o_ + {c}, sc{si}_acc[{q}]);")
            K.append("}")
            si += 1
        elif r.kind == "red":
            ri_here = ri
            ri += 1
            if r.red == "sum" and _sum_from_var(spec, r) is not None:
                continue  # derived from the variance accumulator of the same value
            if id(r) in pr:
                for c in range(nc):
                    v = f"rv[{off + c}]"
                    if r.red == "var" and _exact_value(spec, r):
                        K.append(f"{{ const double d_ = (double){v} - rv{ri_here}_piv; rv{ri_here}_s1 += d_;"
                                 f" rv{ri_here}_s2 = fma(d_, d_, rv{ri_here}_s2); }}")
                    elif r.red == "var":
                        K.append(f"{{ const float d_ = {v} - rv{ri_here}_p32; pp{ri_here}_s1 += d_;"
                                 f" pp{ri_here}_s2 = fmaf(d_, d_, pp{ri_here}_s2); }}")
                    elif r.red == "sumsq":
                        K.append(f"pp{ri_here}_a = fmaf({v}, {v}, pp{ri_here}_a);")
                    else:
                        K.append(f"pp{ri_here}_a += {v};")
                continue
            if r.red == "cov":
                h = f"rv{ri_here}"
                for c in range(nc // 2):
                    a_, b_ = f"(double)rv[{off + c}]", f"(double)rv[{off + nc // 2 + c}]"
                    K.append(f"{{ const double a_ = {a_}, b_ = {b_}; if (!{h}_h) {{ {h}_pa = a_; {h}_pb = b_; {h}_h = true; }}"
                             f" const double da_ = a_ - {h}_pa, db_ = b_ - {h}_pb; {h}_sa += da_; {h}_sb += db_;"
                             f" {h}_sab = fma(da_, db_, {h}_sab); {h}_saa = fma(da_, da_, {h}_saa);"
                             f" {h}_sbb = fma(db_, db_, {h}_sbb); ++{h}_n; }}")
                continue
            if r.red == "sumsq" and nc > 1 and e.g.nodes[r.node].op != "field":
                # a computed vector (FP32 rounding already in each component): the
                # squared norm in FP32, accumulated in FP64
                terms = " + ".join(f"rv[{off + c}] * rv[{off + c}]" for c in range(nc))
                K.append(f"rv{ri_here}_a += (double)({terms});")
                continue
            for c in range(nc):
                val = f"(double)rv[{off + c}]"
                if r.red == "sum":
                    K.append(f"rv{ri_here}_a += {val};")
                elif r.red == "sumsq":
                    K.append(f"{{ const double t_ = {val}; rv{ri_here}_a = fma(t_, t_, rv{ri_here}_a); }}")
                elif r.red == "var":
                    K.append(f"{{ const double t_ = {val}; rv{ri_here}_piv = rv{ri_here}_h ? rv{ri_here}_piv : t_; rv{ri_here}_h = true;"
                             f" const double d_ = t_ - rv{ri_here}_piv; rv{ri_here}_s1 += d_; rv{ri_here}_s2 = fma(d_, d_, rv{ri_here}_s2);"
                             f" ++rv{ri_here}_n; }}")
                elif r.red == "entropy":
                    K.append(f"{{ const double a_ = fabs({val}); rv{ri_here}_a += a_; if (a_ > 0.0) rv{ri_here}_b += a_ * log(a_); }}")
                elif r.red == "minmax":
                    K.append(f"{{ const double t_ = {val}; rv{ri_here}_a = fmin(rv{ri_here}_a, t_); rv{ri_here}_b = fmax(rv{ri_here}_b, t_); }}")
                elif r.red == "hist":
                    # bin index as the oracle forms it: floor((x - lo) / (hi - lo) * bins) in
                    # FP64. FP32 first when its error bound (rv_f32) keeps it within 2.5e-4 of
                    # the exact t and t is more than 1e-3 from an integer (then both floors
                    # agree); else the FP64 product, and within 1e-9 of an edge the FP64
                    # quotient. Counts are run-length merged per thread (smooth data puts
                    # consecutive voxels in one bin) before the shared-memory atomic.
                    h = f"rv{ri_here}"
                    K.append(f"if ({h}_hh > {h}_hl) {{ int b_;"
                             f" const float t32_ = (rv[{off + c}] - {h}_hl32) * {h}_hi32;"
                             f" if ({h}_f32 && fabsf(t32_ - rintf(t32_)) > 1e-3f) b_ = (int)floorf(t32_);"
                             f" else {{ const double d_ = {val} - {h}_hl; double t_ = d_ * {h}_hinv;"
                             f" if (fabs(t_ - rint(t_)) <= 1e-9) t_ = d_ / ({h}_hh - {h}_hl) * {float(r.bins)!r};"
                             f" b_ = (int)floor(t_); }}"
                             f" b_ = b_ < 0 ? 0 : (b_ > {r.bins - 1} ? {r.bins - 1} : b_);"
                             f" if (b_ == {h}_hb) ++{h}_hn;"
                             f" else {{ if ({h}_hn) atomicAdd({h}_hs + {h}_hb, ({h}_cnt_t){h}_hn); {h}_hb = b_; {h}_hn = 1u; }} }}")
                elif r.red == "integrate":
                    sm = 1 if r.method == "simpson" else 0
                    if where == "main" and not is_flat(spec):
                        # per-plane and per-column weights computed outside the voxel loop
                        K.append(f"rv{ri_here}_a += {val} * rv{ri_here}_wi * rv{ri_here}_wj[{{M}}] * rv{ri_here}_wk[{{KK}}];")
                    elif where == "flat":
                        K.append(f"rv{ri_here}_a += {val} * rv{ri_here}_wi * rv{ri_here}_wj"
                                 f" * sten_simpson_w(k, p.n2, {r.dx[2]!r}, {sm});")
                    else:
                        K.append(f"rv{ri_here}_a += {val} * sten_simpson_w(gi, p.n0g, {r.dx[0]!r}, {sm})"
                                 f" * sten_simpson_w(j, p.n1, {r.dx[1]!r}, {sm}) * sten_simpson_w(k, p.n2, {r.dx[2]!r}, {sm});")
                else:
                    raise NotImplementedError(r.red)
        else:
            raise NotImplementedError(r.kind)
    return [k.replace("{M}", str(m)).replace("{KK}", str(kk)) for k in K]


def plane_roots(spec: PassSpec) -> List[Tuple[int, RootSpec]]:
    """Reduction roots (index among reductions, root) that the z-march accumulates
    per plane: the variances of any value, and the sums and sums of squares of
    COMPUTED values. A thread's voxels of one plane (VPT x KV of them) are summed in
    FP32 and the plane sums added to its FP64 accumulators; for a variance the
    pivot of the pivot-shifted sums is the thread's first valid voxel value, taken
    once. A computed value already carries FP32 rounding, and the FP32 plane sums
    add errors of that order per voxel, random in sign; against the FP64 oracle the
    scalars keep their accuracy, and between schedules (which group voxels into
    threads differently) they agree to FP32 rounding of the plane sums (about 1e-7
    relative), while per-voxel results stay bit-identical. Variances and sums of stored field values (exact in FP32)
    are accumulated in FP64 per voxel (plane sums only move the pivot and count)."""
    out = []
    for ri, r in enumerate([x for x in spec.roots if x.kind == "red"]):
        if r.red == "var" or (r.red in ("sum", "sumsq") and spec.graph.nodes[r.node].op != "field"
                              and _sum_from_var(spec, r) is None):
            out.append((ri, r))
    return out


def _exact_value(spec: PassSpec, r: RootSpec) -> bool:
    return spec.graph.nodes[r.node].op == "field"


def _plane_open(spec: PassSpec, e: "_Emitter") -> List[str]:
    """Before a plane's voxels: FP32 plane partials and, for variances, the
    thread's pivot if it has none yet."""
    K: List[str] = []
    for ri, r in plane_roots(spec):
        if r.red == "var":
            off = e.offsets[spec.roots.index(r)]
            if not _exact_value(spec, r):
                K.append(f"float pp{ri}_s1 = 0.0f, pp{ri}_s2 = 0.0f;")
            K.append(f"if (!rv{ri}_h) {{")
            K.append("  #pragma unroll")
            K.append("  for (int m = 0; m < VPT; ++m) {")
            K.append("    #pragma unroll")
            K.append("    for (int q = 0; q < KV; ++q) "
                     f"if (!rv{ri}_h && m_ok[m] && k_ok[q]) {{ rv{ri}_p32 = rvk[m][q][{off}];"
                     f" rv{ri}_piv = (double)rv{ri}_p32; rv{ri}_h = true; }}")
            K.append("  }")
            K.append("}")
        else:
            K.append(f"float pp{ri}_a = 0.0f;")
    return K


def _plane_close(spec: PassSpec, e: "_Emitter") -> List[str]:
    """After a plane's voxels: plane partials into the FP64 accumulators, and the
    plane's valid voxels into the variance counts."""
    K: List[str] = []
    for ri, r in plane_roots(spec):
        nc = e.g.nodes[r.node].nc
        if r.red == "var":
            if not _exact_value(spec, r):
                K.append(f"rv{ri}_s1 += (double)pp{ri}_s1; rv{ri}_s2 += (double)pp{ri}_s2;")
            K.append(f"rv{ri}_n += {nc}u * nvalid_;")
        else:
            K.append(f"rv{ri}_a += (double)pp{ri}_a;")
    return K


def hist_offsets(spec: PassSpec, red_off: int) -> Tuple[Dict[int, int], int]:
    """Shared-memory byte offsets of the per-CTA histograms (by reduction-root
    index) placed after the block-reduction scratch, and the end of the region."""
    off = red_off + RED_SCRATCH_DOUBLES * 8
    offs: Dict[int, int] = {}
    for ri, r in enumerate([r for r in spec.roots if r.kind == "red"]):
        if r.red == "hist":
            offs[ri] = off
            off += 4 * r.bins
    return offs, off


def _red_decls(spec: PassSpec, where: str = "main") -> List[str]:
    K: List[str] = []
    hoffs = hist_offsets(spec, smem_layout(spec)[2])[0] if where == "main" else {}
    for ri, r in enumerate([r for r in spec.roots if r.kind == "red"]):
        if r.red == "hist":
            K.append(f"const double rv{ri}_hl = __ldcg(p.scal + {r.lohi_index}), "
                     f"rv{ri}_hh = __ldcg(p.scal + {r.lohi_index + 1});")
            K.append(f"const double rv{ri}_hinv = rv{ri}_hh > rv{ri}_hl ? {float(r.bins)!r} / (rv{ri}_hh - rv{ri}_hl) : 0.0;")
            # FP32 binning is exact-floor-safe when bins·(4·max|lo,hi|/(hi-lo) + 2)·2^-23,
            # twice its worst-case error of t, is at most 2.5e-4
            K.append(f"const float rv{ri}_hl32 = (float)rv{ri}_hl, rv{ri}_hi32 = (float)rv{ri}_hinv;")
            K.append(f"const bool rv{ri}_f32 = rv{ri}_hh > rv{ri}_hl && {float(r.bins)!r} * (4.0 * fmax(fabs(rv{ri}_hl), "
                     f"fabs(rv{ri}_hh)) / (rv{ri}_hh - rv{ri}_hl) + 2.0) * 1.1920928955078125e-07 <= 2.5e-4;")
            K.append(f"int rv{ri}_hb = 0; unsigned int rv{ri}_hn = 0u;")
            if where == "main":
                K.append(f"typedef unsigned int rv{ri}_cnt_t;")
                K.append(f"unsigned int* rv{ri}_hs = (unsigned int*)(smem + {hoffs[ri]});")
                K.append(f"for (int b_ = tid; b_ < {r.bins}; b_ += NT) rv{ri}_hs[b_] = 0u;")
            else:
                K.append(f"typedef unsigned long long rv{ri}_cnt_t;")
                K.append(f"unsigned long long* rv{ri}_hs = p.hist + {r.slot};")
        elif r.red == "var":
            K.append(f"double rv{ri}_piv = 0.0, rv{ri}_s1 = 0.0, rv{ri}_s2 = 0.0; unsigned int rv{ri}_n = 0u; bool rv{ri}_h = false;")
            K.append(f"float rv{ri}_p32 = 0.0f;")
        elif r.red == "cov":
            # pivot-shifted sums of the pairs (a, b): n, Σda, Σdb, Σda·db, Σda², Σdb²
            K.append(f"double rv{ri}_pa = 0.0, rv{ri}_pb = 0.0, rv{ri}_sa = 0.0, rv{ri}_sb = 0.0, rv{ri}_sab = 0.0, "
                     f"rv{ri}_saa = 0.0, rv{ri}_sbb = 0.0; unsigned int rv{ri}_n = 0u; bool rv{ri}_h = false;")
        elif r.red in ("entropy",):
            K.append(f"double rv{ri}_a = 0.0, rv{ri}_b = 0.0;")
        elif r.red == "minmax":
            K.append(f"double rv{ri}_a = __longlong_as_double(0x7ff0000000000000ll), "
                     f"rv{ri}_b = __longlong_as_double(0xfff0000000000000ll);")
        else:
            K.append(f"double rv{ri}_a = 0.0;")
    return K


def _sum_from_var(spec: PassSpec, r: RootSpec) -> Optional[int]:
    """Index (among reduction roots) of a variance root over the same value as the
    sum root ``r``: the sum then comes from its (n, mean) instead of a second
    accumulator."""
    reds = [x for x in spec.roots if x.kind == "red"]
    for i, x in enumerate(reds):
        if x.red == "var" and x.node == r.node:
            return i
    return None


def raw_scale(g: "PGraph", nid: int) -> Optional[float]:
    """s when node nid's interior value is s times an unscaled expression that
    ``_Emitter.point_raw`` gives: a central difference (s = 1/2h), a sum or
    difference of two central differences with one spacing, or a stack of those
    with one s."""
    n = g.nodes[nid]
    if n.op == "d1":
        return None if n.a("mode") == "zero" else float(n.a("inv2h"))
    if n.op in ("add", "sub") and len(n.ins) == 2:
        a, b = (g.nodes[i] for i in n.ins)
        if (a.op == b.op == "d1" and a.a("mode") != "zero" and b.a("mode") != "zero"
                and a.a("inv2h") == b.a("inv2h") and a.nc == b.nc == n.nc):
            return float(a.a("inv2h"))
        return None
    if n.op == "stack":
        got = {raw_scale(g, i) for i in n.ins}
        return got.pop() if len(got) == 1 and None not in got else None
    return None


def deferred_scale(spec: PassSpec, r: RootSpec) -> Optional[float]:
    """Factor s^2 applied once to the main z-march's FP64 accumulator of the sum of
    squares ``r``, whose voxels then accumulate unscaled (three multiplies fewer per
    voxel for a curl's norm). Only where every voxel of that kernel is an interior
    evaluation (faces in the shell kernel, which keeps its own scaled partial rows,
    or in ghost cells) and s is a power of two: scaling by 2^e commutes with every
    FP32 and FP64 rounding, so the sums are bit for bit those of scaled values
    (outside the exponent range's ends)."""
    if r.kind != "red" or r.red != "sumsq" or spec.radius == 0 or spec.has_scan:
        return None
    s = raw_scale(spec.graph, r.node)
    if s is None or s == 1.0 or s <= 0.0 or math.frexp(s)[0] != 0.5:
        return None
    return s * s


def _red_flush(spec: PassSpec, cta: str, where: str = "main") -> List[str]:
    """Block-reduce each accumulator and write this CTA's partial row; add the
    CTA's histogram counts to the global (integer, order-free) histogram."""
    K: List[str] = []
    reds = [r for r in spec.roots if r.kind == "red"]
    for ri, r in enumerate(reds):
        base = f"p.part[(size_t)({cta}) * NSLOTS_RED + {r.slot}"
        if r.red == "hist":
            K.append(f"if (rv{ri}_hn) atomicAdd(rv{ri}_hs + rv{ri}_hb, (rv{ri}_cnt_t)rv{ri}_hn);")
            if where == "main":
                K.append("__syncthreads();")
                K.append(f"for (int b_ = tid; b_ < {r.bins}; b_ += NT) {{ const unsigned int c_ = rv{ri}_hs[b_];"
                         f" if (c_) atomicAdd(p.hist + {r.slot} + b_, (unsigned long long)c_); }}")
        elif r.red == "cov":
            h = f"rv{ri}"
            K.append(f"{{ const double n_ = (double){h}_n; double x_[6] = {{n_, 0.0, 0.0, 0.0, 0.0, 0.0}};")
            K.append(f"  if (n_ > 0.0) {{ x_[1] = {h}_pa + {h}_sa / n_; x_[2] = {h}_pb + {h}_sb / n_;"
                     f" x_[3] = {h}_sab - {h}_sa * {h}_sb / n_; x_[4] = fmax({h}_saa - {h}_sa * {h}_sa / n_, 0.0);"
                     f" x_[5] = fmax({h}_sbb - {h}_sb * {h}_sb / n_, 0.0); }}")
            K.append("  block_co(x_, red_scratch);")
            K.append(f"  if (tid == 0) for (int i_ = 0; i_ < 6; ++i_) {base} + i_] = x_[i_]; }}")
        elif r.red == "var":
            K.append(f"{{ double n_ = (double)rv{ri}_n, mu_ = 0.0, q_ = 0.0;")
            K.append(f"  if (n_ > 0.0) {{ mu_ = rv{ri}_piv + rv{ri}_s1 / n_; q_ = rv{ri}_s2 - rv{ri}_s1 * rv{ri}_s1 / n_; if (q_ < 0.0) q_ = 0.0; }}")
            K.append("  block_chan(n_, mu_, q_, red_scratch);")
            K.append(f"  if (tid == 0) {{ {base}] = n_; {base} + 1] = mu_; {base} + 2] = q_;")
            for r2 in reds:
                if r2.red == "sum" and r2.node == r.node:
                    K.append(f"    p.part[(size_t)({cta}) * NSLOTS_RED + {r2.slot}] = n_ * mu_;")
            K.append("  } }")
        elif r.red == "sum" and _sum_from_var(spec, r) is not None:
            continue
        elif r.red == "entropy":
            K.append(f"{{ const double a_ = block_sum(rv{ri}_a, red_scratch); const double b_ = block_sum(rv{ri}_b, red_scratch);")
            K.append(f"  if (tid == 0) {{ {base}] = a_; {base} + 1] = b_; }} }}")
        elif r.red == "minmax":
            K.append(f"{{ const double a_ = block_min(rv{ri}_a, red_scratch); const double b_ = block_max(rv{ri}_b, red_scratch);")
            K.append(f"  if (tid == 0) {{ {base}] = a_; {base} + 1] = b_; }} }}")
        else:
            ds = deferred_scale(spec, r) if where == "main" else None
            acc = f"rv{ri}_a" if ds is None else f"rv{ri}_a * {ds!r}"
            K.append(f"{{ const double a_ = block_sum({acc}, red_scratch); if (tid == 0) {base}] = a_; }}")
    return K


def _remap_line(var: str, n: str, rule: Optional[str], indent: str) -> List[str]:
    if rule == "periodic":
        return [f"{indent}{var} = wrap_idx({var}, {n});"]
    if rule == "replicate":
        return [f"{indent}{var} = clamp_idx({var}, {n});"]
    if rule == "reflect":
        return [f"{indent}if ({n} > 1) {var} = reflect_idx({var}, {n});"]
    return []


def _lsu_elem(spec: "PassSpec", f: "FieldSpec", x: str, rule: Optional[str], ind: str, tag: str) -> List[str]:
    """Global column of box column ``x`` (an element index inside the row): kg{tag},
    component c{tag}, validity ok{tag}, byte offset off{tag} inside the row."""
    es = ESIZE[f.dtype]
    L = [f"{ind}const int xr{tag} = {x} - {spec.hk(f)} * {f.nc};",
         f"{ind}int kg{tag} = tk0 + (xr{tag} >= 0 ? xr{tag} / {f.nc} : -((-xr{tag} + {f.nc} - 1) / {f.nc}));",
         f"{ind}const int c{tag} = xr{tag} - (kg{tag} - tk0) * {f.nc};"]
    L += _remap_line(f"kg{tag}", "p.n2", rule, ind)
    L.append(f"{ind}const bool ok{tag} = kg{tag} >= 0 && kg{tag} < p.n2;")
    L.append(f"{ind}const u32 off{tag} = ok{tag} ? (u32)((kg{tag} * {f.nc} + c{tag}) * {es}) : 0u;")
    return L


RS_SHIFT = 13                       # chunk table: slot offset / 16 below, row offset mod 16 from here
RS_VALID, RS_ROWOK, RS_KX = 1 << 17, 1 << 18, 1 << 19


def ring_w(spec: "PassSpec", f: "FieldSpec") -> int:
    """Row pitch of a staged field's ring slot, in elements: the box row, plus one
    16-byte unit for row-staged fields (a row lands there as the 16-byte units that
    cover it, and is shifted into place within that pitch)."""
    w = spec.box(f)[0]
    return w if f.tma else w + 16 // ESIZE[f.dtype]


def rs_geometry(spec: "PassSpec", f: "FieldSpec", cfg: "PassConfig") -> Tuple[int, int, int, int, int, int, int, int]:
    """Row staging of a field whose rows TMA cannot describe: (box width w and height h
    in elements, element size es, box row bytes RB (a multiple of 16), 16-byte chunks
    C per box row, ring row pitch SR = RB + 16 bytes, box rows per warp, chunks per
    thread). Box row r lands in ring row r as the C + 1 16-byte units that cover it
    (unit q of the slot, q = r (C + 1) + u, copied by thread q % NT); warp
    r % (NT / 32) then shifts it into place, 32 chunks at a time."""
    w, h = spec.box(f)
    es = ESIZE[f.dtype]
    rb = w * es
    assert rb % 16 == 0, "box rows are whole 16-byte chunks"
    c = rb // 16
    assert h * (c + 1) < 1 << RS_SHIFT, "slot offsets are packed in 13 bits of 16-byte units"
    rpw = -(-h // (cfg.threads // 32))
    return w, h, es, rb, c, rb + 16, rpw, -(-(rpw * c) // 32)


def rs_units(spec: "PassSpec", f: "FieldSpec", cfg: "PassConfig") -> Tuple[int, int]:
    """(16-byte copy units of one row-staged plane, units per thread)."""
    _, h, _, _, c, _, _, _ = rs_geometry(spec, f, cfg)
    return h * (c + 1), -(-(h * (c + 1)) // cfg.threads)


def rs_strip(spec: "PassSpec", f: "FieldSpec") -> Tuple[Optional[str], int]:
    """(dim-2 rule that copies values across a dim-2 face, or None; 16-byte units per
    strip). Under such a rule a tile at a dim-2 face copies, per box row and face, the
    ``halo`` grid columns its ghost layers take their values from (a strip) next to
    the plane; the shift fills the ghost layers from it."""
    rk = (spec.ghosts or {}).get((f.slot, 2))
    if f.tma or rk not in _REMAP_RULES or f.halo == 0:
        return None, 0
    es = ESIZE[f.dtype]
    return rk, -(-(16 - es + f.halo * f.nc * es) // 16)


def _rs_window(rule: str, side: int, halo: int) -> str:
    """First grid column of the strip of face ``side`` (0: column 0, 1: column n2 - 1)
    under ``rule``: the columns [ws, ws + halo) hold every column the rule maps the
    ghost layers to."""
    ws = {("periodic", 0): f"p.n2 - {halo}", ("periodic", 1): "0",
          ("replicate", 0): "0", ("replicate", 1): f"p.n2 - {halo}",
          ("reflect", 0): "1", ("reflect", 1): f"p.n2 - 1 - {halo}"}[(rule, side)]
    return f"min(max({ws}, 0), max(p.n2 - {halo}, 0))"


def _rs_plan(spec: "PassSpec", f: "FieldSpec", cfg: "PassConfig", ghost: bool) -> List[str]:
    """Per-thread tables of a row-staged field, fixed for the whole march. Copy units:
    for unit q = tid + i NT (unit u of box row r), its byte offset from a plane's start
    (row start at column tk0 - hk, plus 16 u; the rows' dim-1 rule applied) and a bit
    for rows inside the grid. Shift chunks: one word per chunk — its 16-byte unit in
    the ring slot, the row's byte offset mod 16, and flags: chunk exists / row inside
    the grid / chunk crosses a dim-2 face. Warp v owns box rows v, v + NT/32, ...; its
    lanes take that list's chunks in order, 32 at a time."""
    sl = f.slot
    w, h, es, rb, c, sr, rpw, ni = rs_geometry(spec, f, cfg)
    units, nu = rs_units(spec, f, cfg)
    epc = 16 // es
    hkn = spec.hk(f) * f.nc
    rj = (spec.ghosts or {}).get((f.slot, 1)) if ghost else None
    L = [f"// row staging of field {sl}: {h} box rows of {c} chunks; {nu} copy units and {ni} chunks per thread",
         f"const u32 rsB{sl}_ = (u32)p.n2 * {f.nc * es}u;  // bytes of a grid row (mod 2^32)",
         f"int rsw{sl}_[{nu}];",
         f"u32 rsok{sl}_ = 0u, rsex{sl}_ = 0u;  // unit's row inside the grid / unit exists",
         f"#pragma unroll\nfor (int i = 0; i < {nu}; ++i) {{",
         f"  const int q = tid + i * NT, r = q / {c + 1}, u = q - r * {c + 1};",
         f"  int jg = tj0 - {f.halo} + r;"]
    L += _remap_line("jg", "p.n1", rj, "  ")
    L += [f"  rsw{sl}_[i] = (int)((u32)jg * rsB{sl}_ + (u32)((tk0 - {spec.hk(f)}) * {f.nc * es}) + 16u * (u32)u);",
          f"  if (q < {units}) rsex{sl}_ |= 1u << i;",
          f"  if (q < {units} && jg >= 0 && jg < p.n1) rsok{sl}_ |= 1u << i;",
          "}",
          f"u32 rsit{sl}_[{ni}];",
          f"#pragma unroll\nfor (int i = 0; i < {ni}; ++i) {{",
          f"  const int ix = i * 32 + (tid & 31), m = ix / {c}, cc = ix - m * {c}, r = (tid >> 5) + m * (NT / 32);",
          f"  int jg = tj0 - {f.halo} + r;"]
    L += _remap_line("jg", "p.n1", rj, "  ")
    L += [f"  const int x0 = cc * {epc} - {hkn};  // box element of the chunk's first element, from column tk0",
          f"  const bool kx = x0 < -tk0 * {f.nc} || x0 + {epc} > (p.n2 - tk0) * {f.nc};",
          f"  rsit{sl}_[i] = (m < {rpw} && r < {h}) ? ((u32)(r * {c + 1} + cc) | ((((u32)jg * rsB{sl}_) & 15u) << {RS_SHIFT})"
          f" | {RS_VALID}u | (jg >= 0 && jg < p.n1 ? {RS_ROWOK}u : 0u) | (kx ? {RS_KX}u : 0u)) : 0u;",
          "}"]
    return L


def _rs_request(spec: "PassSpec", f: "FieldSpec", cfg: "PassConfig", rings: Dict[int, int]) -> List[str]:
    """Copies of plane ``zq`` into ring slot ``s`` by every thread, its units only: 16
    bytes from the aligned address at or below the unit's offset from the plane
    start; units of rows outside the grid, of planes outside the field and (in the
    field's first and last planes) outside the field are zero. Under a dim-2 rule
    that copies values, tiles at a dim-2 face also copy strips."""
    w, h, es, rb, c, sr, rpw, ni = rs_geometry(spec, f, cfg)
    units, nu = rs_units(spec, f, cfg)
    sl = f.slot
    L = ["{",
         f"  const unsigned long long fb_ = (unsigned long long)p.fld[{sl}];",
         f"  const unsigned long long bz_ = fb_ + (unsigned long long)zq * p.n1 * rsB{sl}_;   // plane start",
         f"  const u32 dst_ = smem_u32(smem + {rings[f.slot]} + s * {plane_bytes(spec, f)}) + (u32)tid * 16u;",
         "  if (zok && zq > 0 && zq < p.nl - 1) {   // every unit lies inside the field",
         "    // rows outside the grid are zero (nothing read): the shift needs no test"]
    for i in range(nu):
        L.append(f"    if (rsex{sl}_ & {1 << i}u) {{ const int w_ = rsw{sl}_[{i}];"
                 f" cp_async16_cg(dst_ + {i * cfg.threads * 16}u, (const void*)(bz_ + (long long)(w_ - (int)(((u32)bz_ + (u32)w_) & 15u))),"
                 f" (rsok{sl}_ >> {i}) << 4 & 16u); }}")
    L += ["  } else {   // the field's first and last planes, and planes outside it",
          f"    const unsigned long long lo_ = fb_ & ~15ull, hi_ = (fb_ + (unsigned long long)p.nl * p.n1 * rsB{sl}_ + 15ull) & ~15ull;"]
    for i in range(nu):
        L += [f"    if (rsex{sl}_ & {1 << i}u) {{ const int w_ = rsw{sl}_[{i}];",
              f"      const unsigned long long g_ = bz_ + (long long)(w_ - (int)(((u32)bz_ + (u32)w_) & 15u));",
              f"      const bool in_ = zok && (rsok{sl}_ & {1 << i}u) && g_ >= lo_ && g_ < hi_;",
              f"      cp_async16_cg(dst_ + {i * cfg.threads * 16}u, (const void*)(in_ ? g_ : lo_), in_ ? 16u : 0u); }}"]
    L.append("  }")
    rule, ns = rs_strip(spec, f)
    if rule:
        # tiles at a dim-2 face: per box row and face, the strip of grid columns the
        # ghost layers map to (only the units that hold its bytes)
        hb = f.halo * f.nc * es
        lay = slot_layout(spec, f)
        rj = (spec.ghosts or {}).get((f.slot, 1))
        L += [f"  if (zok && (tk0 == 0 || tk0 + TK + {spec.hk(f)} > p.n2)) {{",
              f"    const u32 sdst_ = smem_u32(smem + {rings[f.slot]} + s * {plane_bytes(spec, f)} + {lay['rs_strip']});",
              f"    #pragma unroll 1\n    for (int t = tid; t < {2 * h * ns}; t += NT) {{",
              f"      const int rs2 = t / {ns}, sd = rs2 & 1, r = rs2 >> 1, u = t - rs2 * {ns};",
              f"      if (sd == 0 ? tk0 != 0 : tk0 + TK + {spec.hk(f)} <= p.n2) continue;",
              f"      int jg = tj0 - {f.halo} + r;"]
        L += _remap_line("jg", "p.n1", rj, "      ")
        L += ["      if (jg < 0 || jg >= p.n1) continue;",
              f"      const int ws = sd ? {_rs_window(rule, 1, f.halo)} : {_rs_window(rule, 0, f.halo)};",
              f"      const unsigned long long g0 = bz_ + (unsigned long long)((long long)jg * rsB{sl}_ + (long long)ws * {f.nc * es});",
              "      const unsigned long long al = g0 & ~15ull;",
              f"      if ((u32)(g0 - al) + {hb}u > 16u * (u32)u) cp_async16_cg(sdst_ + (u32)t * 16u, (const void*)(al + 16ull * u), 16u);",
              "    }",
              "  }"]
    L.append("}")
    return L


def _rs_shift(spec: "PassSpec", f: "FieldSpec", cfg: "PassConfig", rings: Dict[int, int], ghost: bool,
              zexpr: str) -> List[str]:
    """``rs_shift{slot}(q)``, once plane q's copies landed in its ring slot: each ring
    chunk becomes the 16 bytes that start ``shift`` bytes into it (the row's byte
    offset mod 16), in place — per chunk, every lane of a warp reads before any
    writes; a warp's rows are its own and a row's chunks come in order; rows outside
    the grid arrive as zeros.
    Elements of chunks at a dim-2 face that lie outside the grid are then fetched from
    global memory under a dim-2 rule that copies values, or zeroed under the zero rule
    (one loop after the shift keeps that code out of the unrolled chunks); otherwise
    they stay as copied: they feed only voxels that are not kept, or ghost layers that
    the ghost fill writes."""
    w, h, es, rb, c, sr, rpw, ni = rs_geometry(spec, f, cfg)
    sl = f.slot
    ct = CTYPE[f.dtype]
    epc = 16 // es
    rj = (spec.ghosts or {}).get((f.slot, 1)) if ghost else None
    rk = (spec.ghosts or {}).get((f.slot, 2)) if ghost else None
    gather = rk in _REMAP_RULES
    # without a dim-2 rule that copies values or asks for zeros, columns outside the
    # grid feed only voxels that are not kept (and ghost layers the ghost fill writes)
    face = gather or rk == "zero"
    L = [f"auto rs_shift{sl} = [&](int q) {{",
         f"  const int zq = {zexpr};",
         "  const bool zok_ = zq >= 0 && zq < p.nl;",
         f"  const u32 sz_ = (u32)(unsigned long long)p.fld[{sl}] + (u32)zq * ((u32)p.n1 * rsB{sl}_)"
         f" + (u32)((tk0 - {spec.hk(f)}) * {f.nc * es});",
         f"  unsigned char* slot_ = smem + {rings[f.slot]} + ((q - p_first) % NSLOT) * {plane_bytes(spec, f)};"]
    if face:
        L.append("  u32 kx_ = 0u;   // chunks at a dim-2 face")
    # per chunk, every lane of the warp reads before any lane writes (a warp barrier):
    # a chunk's second unit is the next chunk's first, written by the next lane; a
    # warp's rows are its own and a row's chunks come in order. Rows outside the grid
    # (and planes outside the field) were copied as zeros, so every chunk takes the
    # same path; only chunks past a warp's last row are skipped.
    nw = cfg.threads // 32
    full_chunks = (h // nw) * c        # chunks of the warp with the fewest rows
    L.append(f"  const u32 slot32_ = smem_u32(slot_);")
    for i in range(ni):
        a = f"slot32_ + ((rsit{sl}_[{i}] & {(1 << RS_SHIFT) - 1}u) << 4)"
        st = f"st_shared_v4({a}, v_);"
        L += [f"  {{ const uint4 v_ = shifted16s<{es}>({a}, (sz_ + (rsit{sl}_[{i}] >> {RS_SHIFT})) & 15u);",
              "    __syncwarp();",
              f"    {st}" if (i + 1) * 32 <= full_chunks else f"    if (rsit{sl}_[{i}] & {RS_VALID}u) {st}"]
        if face:
            L.append(f"    if (zok_ && (rsit{sl}_[{i}] & {RS_ROWOK}u) && (rsit{sl}_[{i}] & {RS_KX}u)) kx_ |= {1 << i}u;")
        L.append("  }")
    if not face:
        L.append("};")
        return L
    L += ["  #pragma unroll 1",
          "  for (; kx_ != 0u; kx_ &= kx_ - 1u) {",
          "    const int ix = (__ffs(kx_) - 1) * 32 + (tid & 31);",
          f"    const int m = ix / {c}, cc = ix - m * {c}, r = (tid >> 5) + m * (NT / 32);",
          f"    unsigned char* d_ = slot_ + r * {sr} + cc * 16;"]
    if gather:
        # ghost layers only (columns within halo of a face): from the strip, or from
        # global memory where the rule leaves the strip (grids narrower than 2 halo)
        _, ns = rs_strip(spec, f)
        lay = slot_layout(spec, f)
        L += [f"    int jg = tj0 - {f.halo} + r;"]
        L += _remap_line("jg", "p.n1", rj, "    ")
        L += [f"    const char* rowb = (const char*)p.fld[{sl}] + ((size_t)zq * p.n1 + jg) * ((size_t)p.n2 * {f.nc * es});",
              f"    const u32 rlo_ = (u32)(unsigned long long)rowb;",
              f"    {ct}* d = ({ct}*)d_;",
              f"    #pragma unroll 1\n    for (int e = 0; e < {epc}; ++e) {{",
              f"      const int x0_ = cc * {epc} + e - {spec.hk(f) * f.nc};",
              f"      const int k0_ = tk0 + (x0_ >= 0 ? x0_ / {f.nc} : -((-x0_ + {f.nc - 1}) / {f.nc}));",
              f"      if ((k0_ >= 0 && k0_ < p.n2) || k0_ < -{f.halo} || k0_ >= p.n2 + {f.halo}) continue;",
              f"      const int cm = x0_ - (k0_ - tk0) * {f.nc}, sd = k0_ < 0 ? 0 : 1;",
              "      int kr = k0_;"]
        L += _remap_line("kr", "p.n2", rk, "      ")
        L += [f"      const int ws = sd ? {_rs_window(rk, 1, f.halo)} : {_rs_window(rk, 0, f.halo)};",
              f"      {ct} v_; " + ("v_.bits = 0;" if es == 2 else f"v_ = ({ct})0;"),
              f"      if (kr >= ws && kr < ws + {f.halo}) {{",
              f"        const u32 b_ = ((rlo_ + (u32)ws * {f.nc * es}u) & 15u) + (u32)(((kr - ws) * {f.nc} + cm) * {es});",
              f"        v_ = *(const {ct}*)(slot_ + {lay['rs_strip']} + (r * 2 + sd) * {ns * 16} + b_);",
              f"      }} else if (kr >= 0 && kr < p.n2) v_ = ldg_raw((const {ct}*)(rowb + (size_t)(kr * {f.nc} + cm) * {es}));",
              "      d[e] = v_;",
              "    }"]
    else:
        L += [f"    const int x0 = cc * {epc} - {spec.hk(f) * f.nc};",
              f"    const int elo = min(max(-tk0 * {f.nc} - x0, 0), {epc}), ehi = min(max((p.n2 - tk0) * {f.nc} - x0, 0), {epc});",
              f"    *(uint4*)d_ = keep_bytes16(*(const uint4*)d_, (u32)elo * {es}u, (u32)ehi * {es}u);"]
    L += ["  }", "};"]
    return L


def _ghost_expr2(at, n: str, side: str) -> str:
    """Second ghost layer of a second derivative with edge order 2 on both levels:
    f[-2] = 7f0 - 11f1 + 6f2 - f3 makes the inner central difference at -1 equal
    3g0 - 3g1 + g2 (g the inner derivative), so the outer central difference at 0 is
    torch.gradient's one-sided (-3g0 + 4g1 - g2)/2h of the one-sided inner values."""
    if side == "lo":
        return f"(7.0f * {at('0')} - 11.0f * {at('1')} + 6.0f * {at('2')} - {at('3')})"
    return (f"(7.0f * {at(n + ' - 1')} - 11.0f * {at(n + ' - 2')} + 6.0f * {at(n + ' - 3')}"
            f" - {at(n + ' - 4')})")


def _ghost_expr(rule: str, at, n: str, side: str) -> Optional[str]:
    """Ghost value next to a face for ``rule``; ``at(idx)`` reads the field at an
    in-domain index along the axis (fp32). None: nothing to write."""
    if rule == "edge2x2":
        rule = "edge2"
    if side == "lo":
        v = {"replicate": f"{at('0')}",
             "reflect": f"({n} > 1 ? {at('1')} : 0.0f)",
             "edge2": f"(3.0f * {at('0')} - 3.0f * {at('1')} + {at('2')})",
             "edge1": f"(2.0f * {at('0')} - {at('1')})"}
    else:
        v = {"replicate": f"{at(n + ' - 1')}",
             "reflect": f"({n} > 1 ? {at(n + ' - 2')} : 0.0f)",
             "edge2": f"(3.0f * {at(n + ' - 1')} - 3.0f * {at(n + ' - 2')} + {at(n + ' - 3')})",
             "edge1": f"(2.0f * {at(n + ' - 1')} - {at(n + ' - 2')})"}
    return v.get(rule)


def _ghost_fill(spec: PassSpec, rings: Dict[int, int]) -> List[str]:
    """``ghost_fill(q)``: write the ghost cells next to the dim-1/dim-2 faces of the
    tile in the ring slot of plane q (edge tiles only). Sources: the tile itself
    (replicate / reflect / extrapolation; along dim 1 the tile may be too thin at the
    last face, then global memory), the TMA wrap strips (periodic), or nothing when
    the row staging already applied the rule (remap rules without TMA)."""
    K = ["auto ghost_fill = [&](int q) {",
         "  const int s = (q - p_first) % NSLOT;",
         "  const int zq = sten_plane(p, q + p.i_base);",
         "  if (zq < 0 || zq >= p.nl) return;"]
    for f in spec.fields:
        if not f.staged or f.halo == 0:
            continue
        rk = spec.ghosts.get((f.slot, 2))
        rj = spec.ghosts.get((f.slot, 1))
        lsu_done = ("periodic", "replicate", "reflect", "zero")
        todo_k = rk is not None and rk != "zero" and (f.tma or rk not in lsu_done)
        todo_j = rj is not None and rj != "zero" and (f.tma or rj not in lsu_done)
        if not (todo_k or todo_j):
            continue
        ct = CTYPE[f.dtype]
        w = ring_w(spec, f)
        hk = spec.hk(f)
        nc = f.nc
        lay = slot_layout(spec, f)
        (kw, _), (jw, _) = strip_boxes(spec, f)
        K.append("  {")
        K.append(f"    unsigned char* slot_ = smem + {rings[f.slot]} + s * {plane_bytes(spec, f)};")
        K.append(f"    {ct}* dst = ({ct}*)slot_;")
        if todo_k:
            layers = 2 if rk == "edge2x2" else 1
            for layer in range(1, layers + 1):
                # periodic strips exist only for tiles at the face; extrapolated ghosts also
                # for tiles whose halo crosses it (kept inside the box)
                hi_k = ("tk0 + TK >= p.n2" if rk == "periodic" else
                        f"tk0 + TK + RAD > p.n2 && p.n2 - tk0 + {layer - 1} < TK + {hk}")
                for side, cond, col in (("lo", "tk0 == 0", f"{hk} - {layer}"),
                                        ("hi", hi_k, f"p.n2 - tk0 + {hk} + {layer - 1}")):
                    K.append(f"    if ({cond}) for (int e = tid; e < TJ * {nc}; e += NT) {{")
                    K.append(f"      const int yy = e / {nc}, c = e - yy * {nc};")
                    K.append("      if (tj0 + yy < p.n1) {")
                    if rk == "periodic":
                        buf = "kl" if side == "lo" else "kr"
                        scol = f"{hk} - 1" if side == "lo" else "0"
                        K.append(f"        const {ct}* st = ({ct}*)(slot_ + {lay[buf]});")
                        K.append(f"        dst[(yy + {f.halo}) * {w} + ({col}) * {nc} + c] = st[yy * {kw} + ({scol}) * {nc} + c];")
                    else:
                        rowp = f"dst + (yy + {f.halo}) * {w}"

                        def at_k(ix, rowp=rowp, hk=hk, nc=nc):
                            return f"ld_as_f32({rowp} + (({ix}) - tk0 + {hk}) * {nc} + c)"
                        expr = (_ghost_expr(rk, at_k, "p.n2", side) if layer == 1 else
                                _ghost_expr2(at_k, "p.n2", side))
                        K.append(f"        st_from_f32(dst + (yy + {f.halo}) * {w} + ({col}) * {nc} + c, {expr});")
                    K.append("      }")
                    K.append("    }")
        if todo_j:
            layers = 2 if rj == "edge2x2" else 1
            for layer in range(1, layers + 1):
                hi_j = ("tj0 + TJ >= p.n1" if rj == "periodic" else
                        f"tj0 + TJ + RAD > p.n1 && p.n1 - tj0 + {layer - 1} < TJ + {f.halo}")
                for side, cond, row in (("lo", "tj0 == 0", f"{f.halo} - {layer}"),
                                        ("hi", hi_j, f"p.n1 - tj0 + {f.halo} + {layer - 1}")):
                    K.append(f"    if ({cond}) for (int e = tid; e < TK * {nc}; e += NT) {{")
                    K.append(f"      const int xx = e / {nc}, c = e - xx * {nc};")
                    K.append("      if (tk0 + xx < p.n2) {")
                    if rj == "periodic":
                        buf = "jt" if side == "lo" else "jb"
                        srow = f"{f.halo} - 1" if side == "lo" else "0"
                        K.append(f"        const {ct}* st = ({ct}*)(slot_ + {lay[buf]});")
                        K.append(f"        dst[({row}) * {w} + (xx + {hk}) * {nc} + c] = st[({srow}) * {jw} + (xx + {hk}) * {nc} + c];")
                    else:
                        def at_s(ix, f=f, w=w, hk=hk, nc=nc):
                            return f"ld_as_f32(dst + (({ix}) - tj0 + {f.halo}) * {w} + (xx + {hk}) * {nc} + c)"

                        def at_g(ix, ct=ct, nc=nc, f=f):
                            return (f"ldg_as_f32((const {ct}*)p.fld[{f.slot}] + (((size_t)zq * p.n1 + ({ix})) * p.n2"
                                    f" + tk0 + xx) * {nc} + c)")
                        mk = (lambda at, side=side: _ghost_expr(rj, at, "p.n1", side)) if layer == 1 else \
                             (lambda at, side=side: _ghost_expr2(at, "p.n1", side))
                        es_ = mk(at_s)
                        if side == "hi":
                            # the rows n1-1 .. n1-need may lie above a thin last tile: read them globally
                            need = 3 if layer == 1 else 4
                            es_ = f"((p.n1 - tj0 >= {need} - {f.halo}) ? {es_} : {mk(at_g)})"
                        K.append(f"        st_from_f32(dst + ({row}) * {w} + (xx + {hk}) * {nc} + c, {es_});")
                    K.append("      }")
                    K.append("    }")
        K.append("  }")
    K.append("};")
    return K


def shell_count(shape: Tuple[int, int, int], R: int, g_lo: int = 0, g_hi: Optional[int] = None,
                regions: str = "ABC") -> int:
    """Voxels of global planes [g_lo, g_hi) that lie within R of a face (the shell
    kernel's domain); mirrors the decode in ``sten_shell``."""
    n0, n1, n2 = shape
    g_hi = n0 if g_hi is None else g_hi
    a1, a2 = max(n1 - 2 * R, 0), max(n2 - 2 * R, 0)
    c_low = max(0, min(g_hi, R) - g_lo)
    hs = max(g_lo, max(n0 - R, R))
    c_high = max(0, g_hi - hs)
    ii0 = max(g_lo, R)
    n_int = max(0, min(g_hi, n0 - R) - ii0)
    if regions == "":
        return 0
    if regions == "A":
        return (c_low + c_high) * n1 * n2
    return (c_low + c_high) * n1 * n2 + n_int * (n1 - a1) * n2 + n_int * a1 * (n2 - a2)


SHELL_THREADS = 256
SHELL_MAX_CTAS = 148 * 8   # blocks of the shell launch: 8 resident per SM on 148 SMs


def shell_ctas(n_shell: int) -> int:
    """Blocks of a ``sten_shell`` launch over ``n_shell`` voxels (the kernel strides
    over the rest); each writes one partial row."""
    return min(-(-n_shell // SHELL_THREADS), SHELL_MAX_CTAS)


def _flat_body(spec: PassSpec, e: "_Emitter", red_off: int, batch: bool) -> List[str]:
    """Kernel body of a flat pass: work item ``bx`` covers voxels
    [out_base + bx*CH, out_base + (bx+1)*CH) of the planes [out_lo, out_lo + n_out)."""
    K: List[str] = []
    nroot = e.nroot
    reds = [r for r in spec.roots if r.kind == "red"]
    K.append("  unsigned char* smem = sten_smem;")
    K.append(f"  double* red_scratch = (double*)(smem + {red_off});")
    K.append("  const int tid = threadIdx.x;")
    K.append("  const size_t plane_n = (size_t)p.n1 * p.n2;")
    K.append("  const size_t out_base = (size_t)p.out_lo * plane_n;")
    K.append("  const size_t vhi = out_base + (size_t)p.n_out * plane_n;")
    K.append("  const size_t c0 = out_base + (size_t)bx * (NT * FV * FITER);")
    K.append("  const int cta = p.cta_off + bx;")
    K.append("  FCtx x;")
    K.append(f"  #pragma unroll\n  for (int s = 0; s < {max(spec.n_scalars, 1)}; ++s) "
             f"x.sc[s] = (s < {spec.n_scalars}) ? (float)__ldcg(p.scal + s) : 0.0f;")
    K += ["  " + k for k in _red_decls(spec)]
    if any(r.red == "hist" for r in reds):
        K.append("  __syncthreads();  // histogram cleared")
    need_idx = any(r.red == "integrate" for r in reds)
    vec_outs = [r for r in spec.roots if r.kind == "out" and e.g.nodes[r.node].nc == 1
                and r.out_dtype in ("f32", "f16", "bf16")]
    K.append("  #pragma unroll 1")
    K.append("  for (int it = 0; it < FITER; ++it) {")
    K.append("    const size_t base = c0 + ((size_t)it * NT + tid) * FV;")
    K.append("    if (base >= vhi) break;")
    K.append("    const int nv = (int)min((size_t)FV, vhi - base);")
    K.append("    const bool full = nv == FV;")
    for f in spec.fields:
        ct, es = CTYPE[f.dtype], ESIZE[f.dtype]
        nb = FLAT_V * f.nc * es
        va = 16 if nb % 16 == 0 else (8 if nb % 8 == 0 else (4 if nb % 4 == 0 else 0))
        K.append(f"    {{ const {ct}* fp_ = (const {ct}*)p.fld[{f.slot}] + base * {f.nc};")
        if va and es in (2, 4):
            K.append(f"      if (full && (((size_t)fp_) & {va - 1}) == 0) ld_vec_f32<{ct}, FV * {f.nc}>(fp_, x.fv{f.slot});")
            K.append(f"      else ld_part_f32<{ct}, FV * {f.nc}>(fp_, nv * {f.nc}, x.fv{f.slot}); }}")
        else:
            K.append(f"      ld_part_f32<{ct}, FV * {f.nc}>(fp_, nv * {f.nc}, x.fv{f.slot}); }}")
    if need_idx:
        K.append("    size_t i_ = base / plane_n; const size_t r_ = base - i_ * plane_n;")
        K.append("    int jq = (int)(r_ / (size_t)p.n2), kq = (int)(r_ - (size_t)jq * p.n2);")
        for ri, r in enumerate(reds):
            if r.red == "integrate":
                sm = 1 if r.method == "simpson" else 0
                # plane and row weights change only when the voxel run wraps a row
                K.append(f"    double rv{ri}_wi = sten_simpson_w((int)i_ + p.i_base, p.n0g, {r.dx[0]!r}, {sm}), "
                         f"rv{ri}_wj = sten_simpson_w(jq, p.n1, {r.dx[1]!r}, {sm});")
    K.append(f"    float rvk[FV][{nroot}];")
    for v in range(FLAT_V):
        K.append(f"    if ({v} < nv) {{")
        if need_idx:
            K.append("      const int gi = (int)i_ + p.i_base, j = jq, k = kq;")
        K.append(f"      const size_t vox = base + {v};")
        K.append(f"      float* rv = rvk[{v}];")
        K.append(f"      eval_fast<0, {v}>(x, rv);")
        K += ["      " + k for k in _epilogue(spec, e, scan_ok=False, skip=vec_outs, where="flat", m=0, kk=v)]
        K.append("    }")
        if need_idx and v + 1 < FLAT_V:
            upd = []
            for ri, r in enumerate(reds):
                if r.red == "integrate":
                    sm = 1 if r.method == "simpson" else 0
                    upd.append(f"rv{ri}_wi = sten_simpson_w((int)i_ + p.i_base, p.n0g, {r.dx[0]!r}, {sm}); "
                               f"rv{ri}_wj = sten_simpson_w(jq, p.n1, {r.dx[1]!r}, {sm});")
            K.append("    if (++kq == p.n2) { kq = 0; if (++jq == p.n1) { jq = 0; ++i_; } " + " ".join(upd) + " }")
    for r in vec_outs:
        ct = CTYPE[r.out_dtype]
        off = e.offsets[spec.roots.index(r)]
        sa = FLAT_V * ESIZE[r.out_dtype]
        vals = ", ".join(f"rvk[{q}][{off}]" for q in range(FLAT_V))
        K.append(f"    {{ {ct}* o_ = ({ct}*)p.out[{r.out_slot}] + (base - out_base);")
        K.append(f"      if (full && (((size_t)o_) & {sa - 1}) == 0) {{ const float v_[FV] = {{{vals}}}; st_vec<FV>(o_, v_); }}")
        K.append("      else {")
        for q in range(FLAT_V):
            K.append(f"        if ({q} < nv) st_from_f32(o_ + {q}, rvk[{q}][{off}]);")
        K.append("      }")
        K.append("    }")
    K.append("  }")
    K += ["  " + k for k in _red_flush(spec, "cta")]
    if batch:
        K.append("  return true;")
    return K


def emit_pass(spec: PassSpec, batch_ns: Optional[str] = None, batch_threads: int = 0) -> str:
    """Source of the pass: ``sten_kernel`` (z-march over the tile grid) and, when the
    pass has a stencil reach R > 0 and no scan, ``sten_shell`` (the voxels within R
    of a face, one per thread per stride of the grid, evaluated from global memory
    with boundary rules); with
    histogram roots also ``sten_hist_final`` (entropy from the counts).

    With ``batch_ns`` the same code is emitted as device functions in that
    namespace for the persistent batch kernel (``run_item``: one z-march tile or
    one block of shell voxels per call, parameters read from global memory), without
    the shared header; ``batch_threads`` is the batch kernel's block size."""
    batch = batch_ns is not None
    flat = is_flat(spec)
    header = ""
    if not batch:
        with open(HEADER_PATH) as fh:
            header = fh.read()
    e = _Emitter(spec)
    cfg = spec.cfg
    R = spec.radius
    regions = shell_regions(spec)
    ghost = spec.ghosts is not None
    split = R > 0 and not spec.has_scan          # main kernel never takes the slow path
    nslot = 2 * R + 1 + cfg.prefetch
    assert nslot <= 16, "too many ring slots"
    assert valid_shape(cfg), f"invalid tile shape {cfg}"
    vpt = cfg.tj * cfg.tk // (cfg.threads * cfg.kv)
    L = e.lines
    if batch:
        assert cfg.threads == batch_threads, "batch programs share the block size"
        assert not spec.has_scan, "scans are not batched"
    else:
        L.append(header)
    L.append(f"#define TJ {cfg.tj}\n#define TK {cfg.tk}\n#define NT {cfg.threads}\n#define RAD {R}"
             f"\n#define NSLOT {nslot}\n#define VPT {vpt}\n#define NSLOTS_RED {max(spec.nslots, 1)}"
             f"\n#define KV {cfg.kv}\n#define TKT {cfg.tk // cfg.kv}\n#define FV {FLAT_V}\n#define FITER {FLAT_ITER}")
    if batch:
        L.append(f"namespace {batch_ns} {{")
    ntma = len(tmap_specs(spec))
    nout = sum(1 for r in spec.roots if r.kind in ("out", "scan"))
    L.append("struct __align__(64) Params {")
    if ntma:
        L.append(f"  TmaDesc tmap[{ntma}];")
    L.append(f"  const void* fld[{max(len(spec.fields), 1)}];")
    L.append(f"  void* out[{max(nout, 1)}];")
    L.append("  const double* scal; double* part; unsigned long long* hist; int* err;")
    L.append("  int n0g, n1, n2, nl, i_base, out_lo, n_out, seg_len, tiles_k, cta_off;")
    L.append("};")
    if batch:
        # register copy of the scalar parameters; TMA descriptors stay in global memory
        L.append("struct PView {")
        if ntma:
            L.append("  const TmaDesc* tmap;")
        L.append(f"  const void* fld[{max(len(spec.fields), 1)}];")
        L.append(f"  void* out[{max(nout, 1)}];")
        L.append("  const double* scal; double* part; unsigned long long* hist; int* err;")
        L.append("  int n0g, n1, n2, nl, i_base, out_lo, n_out, seg_len, tiles_k, cta_off;")
        L.append("};")
        L.append("__device__ __forceinline__ PView make_view(const Params& g) {")
        L.append("  PView v;")
        if ntma:
            L.append("  v.tmap = g.tmap;")
        L.append(f"  #pragma unroll\n  for (int i = 0; i < {max(len(spec.fields), 1)}; ++i) v.fld[i] = g.fld[i];")
        L.append(f"  #pragma unroll\n  for (int i = 0; i < {max(nout, 1)}; ++i) v.out[i] = g.out[i];")
        L.append("  v.scal = g.scal; v.part = g.part; v.hist = g.hist; v.err = g.err;")
        L.append("  v.n0g = g.n0g; v.n1 = g.n1; v.n2 = g.n2; v.nl = g.nl; v.i_base = g.i_base; v.out_lo = g.out_lo;")
        L.append("  v.n_out = g.n_out; v.seg_len = g.seg_len; v.tiles_k = g.tiles_k; v.cta_off = g.cta_off;")
        L.append("  return v;")
        L.append("}")
    L.append("template <class P> __device__ __forceinline__ int sten_plane(const P& p, int gi) {")
    L.append("  // global plane index -> plane of the (possibly chunked) arrays")
    L.append("  int l = gi - p.i_base;")
    L.append("  if (l < 0) l += p.n0g; else if (l >= p.nl) l -= p.n0g;")
    L.append("  return l;")
    L.append("}")
    if not batch:
        L.append("extern __shared__ __align__(128) unsigned char sten_smem[];")
    L.append("struct FCtx {")
    for f in spec.fields:
        ct = CTYPE[f.dtype]
        if f.staged:
            # byte offset of this thread's chunk (row 0, first k) in each ring slot in use
            L.append(f"  unsigned int sb{f.slot}[2 * RAD + 1];")
        elif is_flat(spec):
            L.append(f"  float fv{f.slot}[FV * {f.nc}];")
        else:
            L.append(f"  const {ct}* gp{f.slot};")
    L.append(f"  float sc[{max(spec.n_scalars, 1)}];")
    L.append("};")
    for f in spec.fields:
        if not f.staged:
            continue
        ct, es = CTYPE[f.dtype], ESIZE[f.dtype]
        cw = cfg.kv * f.nc * es
        chunk = es in (2, 4) and cw % 4 == 0
        L.append(f"template <int DI, int DJ, int E> __device__ __forceinline__ float LDF{f.slot}(const FCtx& x) {{")
        L.append(f"  // element E of row DJ (relative to the thread's chunk) in the plane at offset DI")
        L.append(f"  const unsigned char* row_ = sten_smem + x.sb{f.slot}[DI + RAD] + DJ * {ring_w(spec, f) * es};")
        if chunk:
            L.append(f"  if constexpr (E >= 0 && E < {cfg.kv * f.nc}) return chunk_elem<{ct}, {cw}, E * {es}>(row_);")
            L.append(f"  else return ld_as_f32((const {ct}*)row_ + E);")
        else:
            L.append(f"  return ld_as_f32((const {ct}*)row_ + E);")
        L.append("}")
        if es == 2:
            # the same element minus an FP32 value, in one mixed-precision subtraction
            L.append(f"template <int DI, int DJ, int E> __device__ __forceinline__ float LDS{f.slot}(const FCtx& x, float c) {{")
            L.append(f"  const unsigned char* row_ = sten_smem + x.sb{f.slot}[DI + RAD] + DJ * {ring_w(spec, f) * es};")
            if chunk:
                L.append(f"  if constexpr (E >= 0 && E < {cfg.kv * f.nc}) return chunk_sub<{ct}, {cw}, E * {es}>(row_, c);")
                L.append(f"  else return sub_as_f32((const {ct}*)row_ + E, c);")
            else:
                L.append(f"  return sub_as_f32((const {ct}*)row_ + E, c);")
            L.append("}")
            # ... and plus an FP32 value
            L.append(f"template <int DI, int DJ, int E> __device__ __forceinline__ float LDA{f.slot}(const FCtx& x, float c) {{")
            L.append(f"  const unsigned char* row_ = sten_smem + x.sb{f.slot}[DI + RAD] + DJ * {ring_w(spec, f) * es};")
            if chunk:
                L.append(f"  if constexpr (E >= 0 && E < {cfg.kv * f.nc}) return chunk_sub<{ct}, {cw}, E * {es}, true>(row_, c);")
                L.append(f"  else return add_as_f32((const {ct}*)row_ + E, c);")
            else:
                L.append(f"  return add_as_f32((const {ct}*)row_ + E, c);")
            L.append("}")
    e.emit_fast_fns()
    e.emit_slow_fns()
    e.emit_eval()
    nroot = e.nroot
    L.append(_simpson_fn())
    tma_fields = [f for f in spec.fields if f.tma]
    lsu_fields = [f for f in spec.fields if f.staged and not f.tma]
    total_smem, rings, red_off = smem_layout(spec)
    tma_bytes = sum(spec.box(f)[0] * spec.box(f)[1] * ESIZE[f.dtype] for f in tma_fields)
    reds = [r for r in spec.roots if r.kind == "red"]
    scans = [r for r in spec.roots if r.kind == "scan"]

    K: List[str] = []
    if batch:
        K.append("__device__ __forceinline__ bool run_tile(const PView& p, const Params& pg, int bx, int by, int gdx) {")
    else:
        K.append(f'extern "C" __global__ void __launch_bounds__(NT, {cfg.min_blocks}) '
                 f"sten_kernel(const __grid_constant__ Params p) {{")
        K.append("  const Params& pg = p;")
        K.append("  const int bx = blockIdx.x, by = blockIdx.y, gdx = gridDim.x;")
    if flat:
        K += _flat_body(spec, e, red_off, batch)
    else:
        K.append("  unsigned char* smem = sten_smem;")
        K.append("  u64* bars = (u64*)smem;")
        K.append(f"  double* red_scratch = (double*)(smem + {red_off});")
        K.append("  const int tid = threadIdx.x;")
        K.append("  const int tile = bx;")
        K.append("  const int tk0 = (tile % p.tiles_k) * TK;")
        K.append("  const int tj0 = (tile / p.tiles_k) * TJ;")
        K.append("  const int ib = p.out_lo + by * p.seg_len;")
        K.append("  const int ie = min(ib + p.seg_len, p.out_lo + p.n_out);")
        K.append("  const int cta = p.cta_off + by * gdx + bx;")
        # a tile whose halo reaches past a face (reach RAD) needs ghost cells there
        K.append("  const bool edge_cta = tk0 == 0 || tk0 + TK + RAD > p.n2 || tj0 == 0 || tj0 + TJ + RAD > p.n1;")
        K.append("  FCtx x;")
        K.append(f"  #pragma unroll\n  for (int s = 0; s < {max(spec.n_scalars, 1)}; ++s) "
                 f"x.sc[s] = (s < {spec.n_scalars}) ? (float)__ldcg(p.scal + s) : 0.0f;")
        K += ["  " + k for k in _red_decls(spec)]
        if any(r.red == "hist" for r in reds):
            K.append("  __syncthreads();  // histogram cleared")
        for si, r in enumerate(scans):
            nc = e.g.nodes[r.node].nc
            K.append(f"  double sc{si}_acc[VPT * KV * {nc}]; float sc{si}_prev[VPT * KV * {nc}];")
            K.append(f"  #pragma unroll\n  for (int q = 0; q < VPT * KV * {nc}; ++q) {{ sc{si}_acc[q] = 0.0; sc{si}_prev[q] = 0.0f; }}")
        staged = tma_fields or lsu_fields
        tmaps = tmap_specs(spec)
        tidx = {(sl, kind): i for i, (sl, kind, _) in enumerate(tmaps)}
        K.append("  const int p_first = ib - RAD;")
        zexpr = ("(q < 0 || q >= p.nl) ? sten_plane(p, q + p.i_base) : q" if ghost and spec.i_periodic else "q")
        if staged:
            K.append("  if (tid == 0) {")
            # with row-staged fields every thread arrives once per plane (its copies),
            # thread 0 once more with the TMA boxes
            cnt = ("NT + 1" if tma_fields else "NT") if lsu_fields else "1"
            K.append(f"    for (int s = 0; s < NSLOT; ++s) mbar_init(&bars[s], {cnt});")
            K.append("    fence_mbar_init();")
            for ti in range(len(tmaps)):
                K.append(f"    tma_prefetch_desc(&p.tmap[{ti}]);")
            K.append("  }")
            K.append("  __syncthreads();")
        for f in lsu_fields:
            K += ["  " + x for x in _rs_plan(spec, f, cfg, ghost)]
            K += ["  " + x for x in _rs_shift(spec, f, cfg, rings, ghost, zexpr)]
        if staged:
            K.append("  auto request = [&](int q) {")
            K.append("    const int s = (q - p_first) % NSLOT;")
            K.append(f"    const int zq = {zexpr};")
            tma_issue = []
            for f in tma_fields:
                base = f"smem + {rings[f.slot]} + s * {plane_bytes(spec, f)}"
                lay = slot_layout(spec, f)
                hk = spec.hk(f)
                tma_issue.append(f"tma_load_3d({base}, &p.tmap[{tidx[(f.slot, 'box')]}], &bars[s], "
                                 f"(tk0 - {hk}) * {f.nc}, tj0 - {f.halo}, zq);")
                if f.wrap_k:
                    ti = tidx[(f.slot, "kstrip")]
                    tma_issue.append(f"if (tk0 == 0) tma_load_3d({base} + {lay['kl']}, &p.tmap[{ti}], &bars[s], "
                                     f"(p.n2 - {hk}) * {f.nc}, tj0, zq);")
                    tma_issue.append(f"if (tk0 + TK >= p.n2) tma_load_3d({base} + {lay['kr']}, &p.tmap[{ti}], &bars[s], "
                                     f"0, tj0, zq);")
                if f.wrap_j:
                    ti = tidx[(f.slot, "jstrip")]
                    tma_issue.append(f"if (tj0 == 0) tma_load_3d({base} + {lay['jt']}, &p.tmap[{ti}], &bars[s], "
                                     f"(tk0 - {hk}) * {f.nc}, p.n1 - {f.halo}, zq);")
                    tma_issue.append(f"if (tj0 + TJ >= p.n1) tma_load_3d({base} + {lay['jb']}, &p.tmap[{ti}], &bars[s], "
                                     f"(tk0 - {hk}) * {f.nc}, 0, zq);")
            tma_size = []
            for f in tma_fields:
                (kw, kh), (jw, jh) = strip_boxes(spec, f)
                es = ESIZE[f.dtype]
                if f.wrap_k:
                    tma_size.append(f"if (tk0 == 0) bytes_ += {kw * kh * es}u;")
                    tma_size.append(f"if (tk0 + TK >= p.n2) bytes_ += {kw * kh * es}u;")
                if f.wrap_j:
                    tma_size.append(f"if (tj0 == 0) bytes_ += {jw * jh * es}u;")
                    tma_size.append(f"if (tj0 + TJ >= p.n1) bytes_ += {jw * jh * es}u;")
            if lsu_fields:
                # every thread copies its units and arrives once they landed; thread 0
                # also arrives with the TMA boxes' bytes
                K.append("    const bool zok = zq >= 0 && zq < p.nl;")
                for f in lsu_fields:
                    K += ["    " + x for x in _rs_request(spec, f, cfg, rings)]
                K.append("    cp_async_mbar_arrive(&bars[s]);")
                if tma_fields:
                    K.append("    if (tid == 0) {")
                    K.append("      fence_proxy_async();")
                    K.append(f"      unsigned int bytes_ = {tma_bytes}u;")
                    K += ["      " + x for x in tma_size]
                    K.append("      mbar_arrive_expect_tx(&bars[s], bytes_);")
                    K += ["      " + x for x in tma_issue]
                    K.append("    }")
            else:
                K.append("    if (tid == 0) {")
                K.append("      fence_proxy_async();")
                K.append(f"      unsigned int bytes_ = {tma_bytes}u;")
                K += ["      " + x for x in tma_size]
                K.append("      mbar_arrive_expect_tx(&bars[s], bytes_);")
                K += ["      " + x for x in tma_issue]
                K.append("    }")
            K.append("  };")
            if lsu_fields:
                K.append("  // plane q resident: its row-staged fields shifted into place (published by the")
                K.append("  // barrier that follows)")
                K.append("  auto shift_rows = [&](int q) { " + " ".join(f"rs_shift{f.slot}(q);" for f in lsu_fields) + " };")
            if ghost:
                K += ["  " + x for x in _ghost_fill(spec, rings)]
            K.append("  for (int q = p_first; q < p_first + NSLOT && q < ie + RAD; ++q) request(q);")
        K.append("  bool ok = true;")
        # planes p_first .. ib+RAD must be resident (and ghosted) before the first plane
        if staged:
            K.append("  for (int q = p_first; q <= ib + RAD && q < ie + RAD; ++q) {")
            K.append("    const int rel = q - p_first;")
            K.append("    ok = ok && mbar_wait_bounded(&bars[rel % NSLOT], (rel / NSLOT) & 1, STEN_WAIT_LIMIT_NS);")
            if lsu_fields:
                K.append("    shift_rows(q);")
            K.append("  }")
        if ghost and staged:
            if lsu_fields:
                K.append("  __syncthreads();  // shifted rows visible to the ghost fill")
            K.append("  if (edge_cta) { for (int q = p_first; q <= ib + RAD && q < ie + RAD; ++q) ghost_fill(q); }")
        if staged:
            K.append("  __syncthreads();")
        # each thread owns KV adjacent columns (kt0 ..) of the tile and VPT consecutive rows;
        # everything that does not depend on the plane is computed once, before the march
        kvn = cfg.kv
        K.append("  const int tk = (tid % TKT) * KV, tjb = (tid / TKT) * VPT;")
        K.append("  const int kt0 = tk0 + tk;")
        K.append("  bool k_ok[KV];")
        K.append("  #pragma unroll")
        if split and not ghost:
            K.append("  for (int q = 0; q < KV; ++q) k_ok[q] = kt0 + q >= RAD && kt0 + q < p.n2 - RAD;")
        else:
            K.append("  for (int q = 0; q < KV; ++q) k_ok[q] = kt0 + q < p.n2;")
        K.append("  const bool k_all = " + " && ".join(f"k_ok[{q}]" for q in range(kvn)) + ";")
        K.append("  bool m_ok[VPT];")
        K.append("  #pragma unroll")
        K.append("  for (int m = 0; m < VPT; ++m) {")
        K.append("    const int j = tj0 + tjb + m;")
        if split and not ghost:
            K.append("    m_ok[m] = j >= RAD && j < p.n1 - RAD;")
        else:
            K.append("    m_ok[m] = j < p.n1;")
        K.append("  }")
        for f in spec.fields:
            if f.staged:
                K.append(f"  const unsigned int ob{f.slot} = ((tjb + {f.halo}) * {ring_w(spec, f)} + (tk + {spec.hk(f)}) * {f.nc})"
                         f" * {ESIZE[f.dtype]};")
        for ri, r in enumerate(reds):
            if r.red == "integrate":
                sm = 1 if r.method == "simpson" else 0
                K.append(f"  double rv{ri}_wj[VPT], rv{ri}_wk[KV];")
                K.append(f"  #pragma unroll\n  for (int m = 0; m < VPT; ++m) rv{ri}_wj[m] = sten_simpson_w(tj0 + tjb + m, p.n1, {r.dx[1]!r}, {sm});")
                K.append(f"  #pragma unroll\n  for (int q = 0; q < KV; ++q) rv{ri}_wk[q] = sten_simpson_w(kt0 + q, p.n2, {r.dx[2]!r}, {sm});")
        K.append("  const bool full_ = k_all" + "".join(f" && m_ok[{m}]" for m in range(vpt)) + ";")
        K.append("  unsigned int nvalid_ = 0u;  // voxels of a plane this thread owns inside the grid")
        K.append("  #pragma unroll\n  for (int m = 0; m < VPT; ++m) {\n    #pragma unroll\n"
                 "    for (int q = 0; q < KV; ++q) nvalid_ += (m_ok[m] && k_ok[q]) ? 1u : 0u;\n  }")
        K.append("  const size_t col = (size_t)(tj0 + tjb) * p.n2 + kt0;")
        K.append("  const size_t plane_n = (size_t)p.n1 * p.n2;")
        K.append("  const size_t out_base = (size_t)p.out_lo * plane_n;")
        K.append("  int ro_[VPT];  // element offset of row m from row 0")
        K.append("  #pragma unroll\n  for (int m = 0; m < VPT; ++m) ro_[m] = m * p.n2;")
        for r in spec.roots:
            if r.kind in ("out", "scan"):
                ct, nc = CTYPE[r.out_dtype], e.g.nodes[r.node].nc
                K.append(f"  {ct}* orow{r.out_slot} = ({ct}*)p.out[{r.out_slot}] + ((size_t)(ib - p.out_lo) * plane_n + col) * {nc};")
        for f in spec.fields:
            if not f.staged:
                K.append(f"  const {CTYPE[f.dtype]}* frow{f.slot} = (const {CTYPE[f.dtype]}*)p.fld[{f.slot}] + "
                         f"((size_t)ib * plane_n + col) * {f.nc};")
        # ring slots of planes i-RAD .. i+RAD: shifted by one each plane, the newcomer is
        # the slot of plane i+RAD+1 (snext)
        for f in spec.fields:
            if f.staged:
                K.append(f"  #pragma unroll\n  for (int d = 0; d < 2 * RAD + 1; ++d) "
                         f"x.sb{f.slot}[d] = {rings[f.slot]}u + (unsigned)d * {plane_bytes(spec, f)}u + ob{f.slot};")
        K.append("  int snext = (2 * RAD + 1) % NSLOT;")
        # computed outside any plane: whether the pass evaluates whole planes before stores
        eager = (split or R == 0) and all(f.staged for f in spec.fields)
        def plane_body() -> List[str]:
            B: List[str] = []
            B.append("    const int gi = i + p.i_base;")
            if ghost and spec.i_periodic:
                B.append("    const bool i_in = true;")
            else:
                B.append("    const bool i_in = (gi >= RAD) && (gi < p.n0g - RAD);")
            B.append("    const size_t pbase = (size_t)i * plane_n + col;")
            for ri, r in enumerate(reds):
                if r.red == "integrate":
                    sm = 1 if r.method == "simpson" else 0
                    B.append(f"    const double rv{ri}_wi = sten_simpson_w(gi, p.n0g, {r.dx[0]!r}, {sm});")
            if split:
                B.append("    if (i_in) {")
            # KV-wide stores for single-component outputs
            vec_outs = [r for r in spec.roots if r.kind == "out" and e.g.nodes[r.node].nc == 1 and kvn > 1
                        and r.out_dtype in ("f32", "f16", "bf16")]
            # all voxels of the plane first, stores and accumulation after: with every field
            # staged the reads stay inside the ring even for voxels beyond the grid, so the
            # evaluation is unconditional and taps shared by neighbouring voxels load once
            eager = (split or R == 0) and all(f.staged for f in spec.fields)
            if eager:
                B.append(f"    float rvk[VPT][KV][{nroot}];")
                for m in range(vpt):
                    for kk in range(kvn):
                        B.append(f"    eval_fast<{m}, {kk}>(x, rvk[{m}][{kk}]);")
                B += ["    " + k for k in _plane_open(spec, e)]
            def voxel_loop(pred: bool) -> List[str]:
                V: List[str] = []
                for m in range(vpt):
                    V.append(f"    if (m_ok[{m}]) {{" if pred else "    {")
                    V.append(f"      const int j = tj0 + tjb + {m};")
                    V.append(f"      const size_t rowvox = pbase + (size_t){m} * p.n2;")
                    if not eager:
                        V.append(f"      float rvm[KV][{nroot}];")
                    arr = f"rvk[{m}]" if eager else "rvm"
                    for kk in range(kvn):
                        V.append(f"      if (k_ok[{kk}]) {{" if pred else "      {")
                        V.append(f"        const int k = kt0 + {kk}, mq = {m * kvn + kk};")
                        V.append(f"        const size_t vox = rowvox + {kk};")
                        V.append(f"        float* rv = {arr}[{kk}];")
                        if not eager:
                            for f in spec.fields:
                                if not f.staged:
                                    V.append(f"        x.gp{f.slot} = frow{f.slot} + ro_[{m}] * {f.nc} + {kk * f.nc};")
                            if split or R == 0:
                                V.append(f"        eval_fast<{m}, {kk}>(x, rv);")
                            else:
                                V.append("        const bool inter = i_in && j >= RAD && j < p.n1 - RAD && k >= RAD && k < p.n2 - RAD;")
                                V.append(f"        if (inter) eval_fast<{m}, {kk}>(x, rv); else eval_slow(pg, gi, j, k, rv);")
                        V += ["        " + k for k in _epilogue(spec, e, scan_ok=True, skip=vec_outs, m=m, kk=kk,
                                                             plane=eager)]
                        V.append("      }")
                    for r in vec_outs:
                        ct = CTYPE[r.out_dtype]
                        off = e.offsets[spec.roots.index(r)]
                        vals = ", ".join(f"{arr}[{q}][{off}]" for q in range(kvn))
                        allk = "k_all && " if pred else ""
                        V.append(f"      {{ {ct}* o_ = orow{r.out_slot} + ro_[{m}];")
                        V.append(f"        if ({allk}(((size_t)o_) & {kvn * ESIZE[r.out_dtype] - 1}) == 0) {{ const float v_[KV] = {{{vals}}}; st_vec<KV>(o_, v_); }}")
                        V.append("        else {")
                        for q in range(kvn):
                            cond = f"if (k_ok[{q}]) " if pred else ""
                            V.append(f"          {cond}st_from_f32(o_ + {q}, {arr}[{q}][{off}]);")
                        V.append("        }")
                        V.append("      }")
                    V.append("    }")
                return V

            if eager:
                # tiles whose voxels all lie inside the grid skip the per-voxel predicates
                B.append("    if (full_) {")
                B += ["  " + v for v in voxel_loop(False)]
                B.append("    } else {")
                B += ["  " + v for v in voxel_loop(True)]
                B.append("    }")
            else:
                B += voxel_loop(True)
            if eager:
                B += ["    " + k for k in _plane_close(spec, e)]
            if split:
                B.append("    }")
            for r in spec.roots:
                if r.kind in ("out", "scan"):
                    B.append(f"    orow{r.out_slot} += plane_n * {e.g.nodes[r.node].nc};")
            for f in spec.fields:
                if not f.staged:
                    B.append(f"    frow{f.slot} += plane_n * {f.nc};")
            # the next plane (i+1+RAD) must be resident and ghosted before the barrier;
            # ghosts derived from row-staged rows wait for every warp's shift: an extra
            # barrier, in edge tiles only
            lsu_ghost = ghost and any(
                (spec.ghosts or {}).get((f.slot, ax)) in _EXTRAPOLATED for f in lsu_fields for ax in (1, 2))
            if staged:
                B.append("    if (i + 1 < ie) {")
                B.append("      const int rel = i + 1 + RAD - p_first;")
                B.append("      ok = ok && mbar_wait_bounded(&bars[rel % NSLOT], (rel / NSLOT) & 1, STEN_WAIT_LIMIT_NS);")
                if lsu_fields:
                    B.append("      shift_rows(i + 1 + RAD);")
                if ghost and not lsu_ghost:
                    B.append("      if (edge_cta) ghost_fill(i + 1 + RAD);")
                B.append("    }")
            if lsu_ghost:
                B.append("    if (edge_cta) { __syncthreads(); if (i + 1 < ie) ghost_fill(i + 1 + RAD); }")
            if staged:
                # the ring slot of plane i - RAD is refilled next: every thread must be done with it
                B.append("    ok = __syncthreads_and(ok);")
                B.append("    if (!ok) break;")
            for f in spec.fields:
                if f.staged:
                    B.append(f"    #pragma unroll\n    for (int d = 0; d < 2 * RAD; ++d) x.sb{f.slot}[d] = x.sb{f.slot}[d + 1];")
                    B.append(f"    x.sb{f.slot}[2 * RAD] = {rings[f.slot]}u + (unsigned)snext * {plane_bytes(spec, f)}u + ob{f.slot};")
            B.append("    snext = (snext + 1 == NSLOT) ? 0 : snext + 1;")
            if staged:
                B.append(f"    if (i + RAD + 1 + {cfg.prefetch} < ie + RAD) request(i + RAD + 1 + {cfg.prefetch});")
            return B

        K.append("  for (int i = ib; i < ie; ++i) {")
        K += plane_body()
        K.append("  }")
        K.append("  ok = __syncthreads_and(ok);  // uniform even when the march ran no plane")
        K.append("  if (!ok) { if (tid == 0) atomicExch(p.err, STEN_ERR_TMA_TIMEOUT); return%s; }"
                 % (" false" if batch else ""))
        K += ["  " + k for k in _red_flush(spec, "cta")]
        if batch:
            if tma_fields or lsu_fields:
                # every requested plane was waited on: retire the barriers before the
                # next item re-initialises this shared memory
                K.append("  __syncthreads();")
                K.append("  if (tid == 0) { for (int s = 0; s < NSLOT; ++s) mbar_inval(&bars[s]); }")
            K.append("  return true;")
    K.append("}")

    if regions:
        # shell: voxels within RAD of a face, one per thread, evaluated from global memory
        if batch:
            K.append("__device__ __forceinline__ void run_shell(const PView& p, const Params& pg, int bx) {")
            K.append("  double* red_scratch = (double*)(sten_smem + 128);")
        else:
            K.append(f'extern "C" __global__ void __launch_bounds__({SHELL_THREADS}) '
                     f"sten_shell(const __grid_constant__ Params p) {{")
            K.append("  const Params& pg = p;")
            K.append("  const int bx = blockIdx.x;")
            K.append(f"  __shared__ double red_scratch[{RED_SCRATCH_DOUBLES}];")
        K.append("  const int tid = threadIdx.x;")
        K += ["  " + k for k in _red_decls(spec, "shell")]
        # 32-bit decode when every count fits an int (unsigned divisions are a few
        # instructions; 64-bit ones a long emulated sequence per thread)
        T, Z = ("int", "0") if spec.idx32 else ("long long", "0ll")
        dv = (lambda a, b: f"(int)((unsigned)({a}) / (unsigned)({b}))") if spec.idx32 else (lambda a, b: f"({a}) / ({b})")
        K.append(f"  const {T} n0 = p.n0g, n1 = p.n1, n2 = p.n2;")
        K.append(f"  const {T} g_lo = ({T})p.out_lo + p.i_base, g_hi = g_lo + p.n_out;")
        K.append(f"  const {T} a1 = max(n1 - 2 * RAD, {Z}), a2 = max(n2 - 2 * RAD, {Z});")
        K.append(f"  const {T} c_low = max({Z}, min(g_hi, ({T})RAD) - g_lo);")
        K.append(f"  const {T} hs = max(g_lo, max(n0 - RAD, ({T})RAD));")
        K.append(f"  const {T} c_high = max({Z}, g_hi - hs);")
        K.append(f"  const {T} ii0 = max(g_lo, ({T})RAD), n_int = max({Z}, min(g_hi, n0 - RAD) - ii0);")
        if regions == "A":
            K.append(f"  const {T} cA = (c_low + c_high) * n1 * n2, cB = 0, cC = 0;")
        else:
            K.append(f"  const {T} cA = (c_low + c_high) * n1 * n2, cB = n_int * (n1 - a1) * n2, cC = n_int * a1 * (n2 - a2);")
        if batch:
            # a work item is one block of shell voxels
            K.append(f"  const {T} t = ({T})bx * blockDim.x + tid;")
            K.append("  if (t < cA + cB + cC) {")
        else:
            # at most SHELL_MAX_CTAS blocks stride over the shell: fewer partial rows
            # for the finalize and one block reduction per resident block
            K.append(f"  for ({T} t = ({T})bx * blockDim.x + tid; t < cA + cB + cC; t += ({T})gridDim.x * blockDim.x) {{")
        K.append(f"    {T} i, j, k;")
        K.append("    if (t < cA) {            // planes within RAD of a dim-0 face")
        K.append(f"      const {T} q = {dv('t', 'n1 * n2')}, r = t - q * n1 * n2;")
        K.append("      i = q < c_low ? g_lo + q : hs + (q - c_low);")
        K.append(f"      j = {dv('r', 'n2')}; k = r - j * n2;")
        K.append("    } else if (t < cA + cB) { // interior planes, rows within RAD of a dim-1 face")
        K.append(f"      const {T} u = t - cA, w1 = n1 - a1;")
        K.append(f"      const {T} q = {dv('u', 'w1 * n2')}, r = u - q * w1 * n2;")
        K.append(f"      const {T} jr = {dv('r', 'n2')}, lo = min(({T})RAD, n1);")
        K.append("      i = ii0 + q; j = jr < lo ? jr : n1 - (w1 - jr); k = r - jr * n2;")
        K.append("    } else {                  // interior rows, columns within RAD of a dim-2 face")
        # row-major (both faces' columns of a row next to each other): measured faster
        # on B200 than one face column per warp, which walks rows n2 apart
        K.append(f"      const {T} u = t - cA - cB, w2 = n2 - a2;")
        K.append(f"      const {T} q = {dv('u', 'a1 * w2')}, r = u - q * a1 * w2;")
        K.append(f"      const {T} jr = {dv('r', 'w2')}, kr = r - jr * w2, lo = min(({T})RAD, n2);")
        K.append("      i = ii0 + q; j = RAD + jr; k = kr < lo ? kr : n2 - (w2 - kr);")
        K.append("    }")
        K.append("    const int gi = (int)i;")
        K.append("    const size_t vox = ((size_t)(sten_plane(p, gi)) * p.n1 + j) * p.n2 + k;")
        K.append("    const size_t out_base = (size_t)p.out_lo * p.n1 * p.n2;")
        K.append(f"    float rv[{nroot}];")
        K.append("    eval_slow(pg, gi, (int)j, (int)k, rv);")
        K += ["    " + k for k in _epilogue(spec, e, scan_ok=False, where="shell")]
        K.append("  }")
        K += ["  " + k for k in _red_flush(spec, "p.cta_off + bx", "shell")]
        K.append("}")
    hists = [r for r in reds if r.red == "hist"]
    if hists and not batch:
        K.append('extern "C" __global__ void __launch_bounds__(256) sten_hist_final(const __grid_constant__ Params p) {')
        K.append(f"  __shared__ double red_scratch[{RED_SCRATCH_DOUBLES}];")
        K.append("  const double nvox = (double)p.n0g * (double)p.n1 * (double)p.n2;")
        for r in hists:
            nc = e.g.nodes[r.node].nc
            K.append(f"  {{ const double s_ = sten_hist_qlogq(p.hist + {r.slot}, {r.bins}, nvox * {nc}, red_scratch);")
            K.append(f"    if (threadIdx.x == 0) {{ const double lo_ = __ldcg(p.scal + {r.lohi_index}), "
                     f"hi_ = __ldcg(p.scal + {r.lohi_index + 1});")
            K.append(f"      ((double*)p.scal)[{r.table_index}] = hi_ > lo_ ? -s_ : 0.0; }} }}")
        K.append("}")
    if batch:
        K.append("__device__ __noinline__ bool run_item(const Params& pg, int kind, int bx, int by, int gdx, int shell_cta0) {")
        K.append("  PView p = make_view(pg);")
        if regions:
            K.append("  if (kind == 1) { p.cta_off = shell_cta0; run_shell(p, pg, bx); return true; }")
        K.append("  return run_tile(p, pg, bx, by, gdx);")
        K.append("}")
        K.append(f"}}  // namespace {batch_ns}")
        K.append("#undef TJ\n#undef TK\n#undef NT\n#undef RAD\n#undef NSLOT\n#undef VPT\n#undef NSLOTS_RED"
                 "\n#undef KV\n#undef TKT\n#undef FV\n#undef FITER")
    return "\n".join(L) + "\n" + "\n".join(K) + "\n"


# ----------------------------------------------------------------------------- batch module
BATCH_STRUCTS = r"""
struct BPhase {            // one pass of one job (80 bytes)
  unsigned long long params, part, table, hist;  // its Params; partial rows; scalar table; histograms
  int prog, n_items, dep, gdx;                    // program; work items; phase to wait for (-1); tiles per plane row
  int shell_cta0, ncta, nslots, red0;             // first shell partial row; partial rows; slots per row; first BRed
  int nred, hist0, nhist, pad;                    // reductions; first BHist; histograms
};
struct BRed { int kind, slot, out_index, unbiased; double count, eps; };
struct BHist { int base, bins, lohi, out_index; double count; };
struct BatchArgs {
  const int4* items;        // (phase, kind 0 tile | 1 shell, bx, by), in queue order
  const BPhase* phases; const BRed* reds; const BHist* hists;
  unsigned int* ctl;        // [0] queue head, [1] CTAs done, then done items and ready flag per phase
  int* err;
  int n_items, n_phases;
};
// the host packs these records with fixed layouts
static_assert(sizeof(BPhase) == 80 && sizeof(BRed) == 32 && sizeof(BHist) == 24 && sizeof(BatchArgs) == 56,
              "batch record layout");
"""


def emit_batch_module(specs: List[PassSpec], threads: int, min_blocks: int = 1) -> str:
    """One module holding every program of a batch (``specs[i]`` in namespace
    ``p<i>``) and ``sten_batch``, a persistent kernel whose CTAs take work items
    from a queue in order. An item is one z-march tile or one block of shell voxels
    of one pass of one job. The CTA completing the last item of a pass combines its
    partial rows and histograms into the job's scalar table (same fixed-order
    reduction as the standalone finalize) and sets the pass's ready flag; items of a
    pass that reads those scalars wait for the flag (bounded). Items are queued so a
    pass's prerequisites come first, so every wait is on items already taken by
    running CTAs. The last CTA to finish resets the queue for the next launch."""
    with open(HEADER_PATH) as fh:
        header = fh.read()
    L = [header, "extern __shared__ __align__(128) unsigned char sten_smem[];"]
    for i, sp_ in enumerate(specs):
        L.append(emit_pass(sp_, batch_ns=f"p{i}", batch_threads=threads))
    L.append(BATCH_STRUCTS)
    L.append(r"""
__device__ __noinline__ void sten_batch_finalize(const BatchArgs& a, const BPhase& ph) {
  double* scratch = (double*)(sten_smem + 128);
  double* table = (double*)ph.table;
  for (int r = 0; r < ph.nred; ++r) {
    const BRed d = a.reds[ph.red0 + r];
    sten_reduce_rows(d.kind, (const double*)ph.part, ph.ncta, ph.nslots, d.slot, d.unbiased, d.count, d.eps,
                     table + d.out_index, scratch);
  }
  for (int h = 0; h < ph.nhist; ++h) {
    const BHist d = a.hists[ph.hist0 + h];
    const double s = sten_hist_qlogq((unsigned long long*)ph.hist + d.base, d.bins, d.count, scratch);
    if (threadIdx.x == 0) {
      const double lo = __ldcg(table + d.lohi), hi = __ldcg(table + d.lohi + 1);
      table[d.out_index] = hi > lo ? -s : 0.0;
    }
  }
}
""")
    K = [f'extern "C" __global__ void __launch_bounds__({threads}, {min_blocks}) '
         "sten_batch(const __grid_constant__ BatchArgs a) {",
         "  __shared__ int s_item, s_last;",
         "  const int tid = threadIdx.x;",
         "  unsigned int* done = a.ctl + 2;",
         "  unsigned int* ready = a.ctl + 2 + a.n_phases;",
         "  bool ok = true;",
         "  for (;;) {",
         "    // a CTA that hit an error stops the others at their next item",
         "    if (tid == 0) s_item = *(volatile int*)a.err ? 0x7fffffff : (int)atomicAdd(a.ctl, 1u);",
         "    __syncthreads();",
         "    const int it = s_item;",
         "    if (it >= a.n_items) break;",
         "    const int4 w = a.items[it];",
         "    if ((unsigned)w.x >= (unsigned)a.n_phases) { ok = false; break; }  // corrupt queue: stop",
         "    const BPhase& ph = a.phases[w.x];",
         "    if (ph.dep >= 0) {",
         "      bool got = true;",
         "      if (tid == 0) got = flag_wait_bounded(ready + ph.dep, STEN_WAIT_LIMIT_NS);",
         "      if (!__syncthreads_and(got)) { ok = false; break; }",
         "    }",
         "    const void* prm = (const void*)ph.params;",
         "    switch (ph.prog) {"]
    for i in range(len(specs)):
        K.append(f"      case {i}: ok = p{i}::run_item(*(const p{i}::Params*)prm, w.y, w.z, w.w, ph.gdx, "
                 "ph.shell_cta0); break;")
    K += ["      default: ok = false; break;",
          "    }",
          "    if (!ok) break;",
          "    __threadfence();  // this item's partials and histogram counts, before it is counted done",
          "    __syncthreads();",
          "    if (tid == 0) { __threadfence(); s_last = atomicAdd(done + w.x, 1u) == (unsigned)ph.n_items - 1u; }",
          "    __syncthreads();",
          "    if (s_last) {",
          "      __threadfence();",
          "      sten_batch_finalize(a, ph);",
          "      __syncthreads();",
          "      if (tid == 0) { __threadfence(); atomicExch(ready + w.x, 1u); }",
          "    }",
          "  }",
          "  if (!ok && tid == 0) atomicExch(a.err, STEN_ERR_TMA_TIMEOUT);",
          "  __syncthreads();",
          "  if (tid == 0) {",
          "    __threadfence();",
          "    if (atomicAdd(a.ctl + 1, 1u) == gridDim.x - 1) {",
          "      for (int i = 0; i < 2 + 2 * a.n_phases; ++i) a.ctl[i] = 0u;",
          "      __threadfence();",
          "    }",
          "  }",
          "}"]
    return "\n".join(L) + "\n" + "\n".join(K) + "\n"

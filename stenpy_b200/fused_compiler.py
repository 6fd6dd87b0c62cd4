"""Fused executor: plans a ``Graph`` into passes of generated CUDA kernels and runs them.

This takes the slot of the reference's ``fused_compiler.compile_and_execute``
(fused_compiler.py:632-753, called from stenpy_engine.py:966-981): given a graph
and the wanted node ids it returns ``{node_id: tensor}``. Unlike the reference
(whose planner lowers only pointwise ops plus one Laplacian, and whose import is
circular so it never runs), every hot-path operator is fused here:

1. **Phases.** A global reduction (sum, mean, norm_l2, variance, entropy,
   integrate, min_max) is a barrier: nodes that use its value run in a later
   pass. A ``cumulative_integral`` is materialised by the pass that computes it
   and read as a field afterwards. (User-registered operators are split off by
   ``Runtime`` before planning.)
2. **Passes.** Each phase with work becomes one launch of a z-marching stencil
   kernel (``codegen.emit_pass``) evaluating every root of that phase — outputs,
   reduction partials, scans — directly from the input fields, recomputing
   shared per-voxel subexpressions instead of writing intermediates to HBM.
3. **Finalize.** Reductions of a pass are combined on the device
   (``stenpy_finalize``) into an FP64 scalar table read by later passes; nothing
   returns to the host between passes.

Plans are cached by the graph's structure (ops, params, field shapes and dtypes),
so repeated runs only re-pack pointers.
"""
from __future__ import annotations

import hashlib
import struct
import threading
from dataclasses import dataclass, field as dc_field
from typing import Any, Dict, List, Optional, Sequence, Set, Tuple

import torch

from . import _native as N
from .codegen import (ESIZE, SHELL_MAX_CTAS, SHELL_THREADS, STENCIL_PRIMS, FieldSpec, PassConfig, PassSpec, PGraph, RootSpec,
                      analyse_ghosts, emit_pass, param_layout, pass_grid, shell_count, shell_ctas, shell_regions,
                      smem_layout, tmap_specs)
from .graph import Graph
from .lowering import LoweringError, OpLowerer, dx3
from .registry import KNOWN_OPS

# operators fused on 2-D fields besides the pointwise ones (the reference's 2-D-only
# surface_normals, and global reductions of the values)
OPS_2D = {"surface_normals", "sum", "mean", "norm_l2", "variance", "entropy", "min_max", "entropy_hist"}

MAX_RING_SLOTS = 16         # one 8-byte mbarrier per plane-ring slot in a 128-byte block
MAX_SMEM_BYTES = 227 * 1024  # dynamic shared memory one CTA may opt into on sm_100a

TORCH_DT = {torch.float32: "f32", torch.float64: "f64", torch.bfloat16: "bf16", torch.float16: "f16"}
DT_TORCH = {v: k for k, v in TORCH_DT.items()}
NVRTC_OPTS = ["--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "-lineinfo"]

REDUCTIONS = {"sum": "sum", "mean": "sum", "norm_l2": "sumsq", "variance": "var",
              "entropy": "entropy", "integrate": "integrate", "min_max": "minmax"}
RED_SLOTS = {"sum": 1, "sumsq": 1, "var": 3, "entropy": 2, "integrate": 1, "minmax": 2, "cov": 6}
RED_KIND = {"sum": N.RED_SUM, "mean": N.RED_MEAN, "norm_l2": N.RED_NORM_L2, "variance": N.RED_VARIANCE,
            "entropy": N.RED_ENTROPY, "integrate": N.RED_INTEGRATE, "min_max": N.RED_MIN_MAX}


class FusionError(ValueError):
    """The graph cannot be executed by the fused executor (bad shapes/params)."""


def is_field_value(v: Any) -> bool:
    """A per-voxel input: a 3-D grid (scalar, (*, 3) or (*, 3, 3)) or a 2-D scalar
    field, which runs as a grid of one plane."""
    return isinstance(v, torch.Tensor) and v.ndim >= 2


def is_scalar_value(v: Any) -> bool:
    return (isinstance(v, (int, float)) and not isinstance(v, bool)) or \
        (isinstance(v, torch.Tensor) and v.ndim == 0)


def field_nc(shape: Sequence[int]) -> int:
    shape = tuple(shape)
    if len(shape) in (2, 3):
        return 1
    if len(shape) == 4 and shape[3] == 3:
        return 3
    if len(shape) == 5 and shape[3:] == (3, 3):
        return 9
    raise FusionError(f"field of shape {shape}: expected (n0,n1,n2), (...,3) or (...,3,3)")


def comp_shape(nc: int) -> Tuple[int, ...]:
    return {1: (), 3: (3,), 9: (3, 3)}[nc]


# --------------------------------------------------------------------------- plan
@dataclass
class _Info:
    kind: str                # field | scalar | voxel | red | scan
    avail: int               # first pass that can read the value
    nc: int = 1
    compute_pass: int = -1   # red / scan: the pass that computes it


@dataclass
class RedPlan:
    node: str
    slot: int
    table_index: int
    kind: int
    count: float
    unbiased: int
    eps: float


@dataclass
class PassPlan:
    spec: PassSpec
    field_nodes: List[str]                 # graph node read by each Params::fld slot
    out_nodes: List[Tuple[str, str, int]]  # (graph node, "out" | "scan", components) per Params::out slot
    reductions: List[RedPlan]
    hists: List[RootSpec] = dc_field(default_factory=list)  # histogram-entropy roots
    module: Optional[int] = None
    shell_module: Optional[int] = None
    hist_module: Optional[int] = None
    smem: int = 0
    source: str = ""
    key: str = ""


@dataclass
class FusedPlan:
    key: str
    shape: Tuple[int, int, int]
    infos: Dict[str, _Info]
    passes: List[PassPlan]
    table_size: int
    const_index: Dict[str, int]
    red_index: Dict[str, int]
    scalar_sinks: Dict[str, int]
    scalar_source: Optional[str]
    wanted: List[str]
    out_dtype: torch.dtype
    live: List[str] = dc_field(default_factory=list)
    buffers: Dict[str, torch.Tensor] = dc_field(default_factory=dict)
    scalar_module: Optional[int] = None
    hist_size: int = 0
    dims2: bool = False    # 2-D fields: the grid is (1, n0, n1), per-voxel results are (n0, n1, ...)
    keepdim: Set[str] = dc_field(default_factory=set)   # results with a trailing axis of 1 (norm_last)

    def out_shape(self, nc: int, nid: Optional[str] = None) -> Tuple[int, ...]:
        """Shape of a per-voxel result with ``nc`` components (of node ``nid``)."""
        return ((self.shape[1:] if self.dims2 else self.shape) + comp_shape(nc)
                + ((1,) if nid in self.keepdim else ()))

    def kernel_sources(self) -> List[str]:
        return [emit_pass(p.spec) for p in self.passes]


class Planner:
    def __init__(self, graph: Graph, wanted: Sequence[str], out_dtype: torch.dtype = torch.float32,
                 config: Optional[PassConfig] = None, ghosts: bool = True):
        self.ghosts = ghosts
        self.g = graph
        self.nodes = graph._nodes
        self.wanted = list(dict.fromkeys(wanted))
        self.out_dtype = out_dtype
        self.cfg = config or PassConfig()
        self.live = graph.live_nodes(self.wanted)
        self.hist_mm: Dict[str, int] = {}   # entropy_hist node -> pass of its min/max phase
        self.hist_base = 0                   # histogram bins allocated so far

    def analyse(self) -> None:
        infos: Dict[str, _Info] = {}
        shape: Optional[Tuple[int, int, int]] = None
        ndims = set()
        for nid in self.live:
            node = self.nodes[nid]
            op = node.op_name
            if op == "_constant":
                v = node.params.get("value")
                if is_field_value(v):
                    ndims.add(2 if v.ndim == 2 else 3)
                    if len(ndims) > 1:
                        raise FusionError("2-D and 3-D fields in one graph")
                    s = (1,) + tuple(int(x) for x in v.shape) if v.ndim == 2 else tuple(int(x) for x in v.shape[:3])
                    if shape is None:
                        shape = s
                    elif s != shape:
                        raise FusionError(f"fields on different grids in one graph: {shape} vs {s}")
                    if v.dtype not in TORCH_DT:
                        raise FusionError(f"field dtype {v.dtype} is not supported")
                    infos[nid] = _Info("field", 0, field_nc(v.shape))
                elif is_scalar_value(v):
                    infos[nid] = _Info("scalar", 0, 1)
                else:
                    raise FusionError(f"_constant {nid}: unsupported value of shape "
                                      f"{tuple(getattr(v, 'shape', ()))} (fields are 3-D)")
                continue
            spec = KNOWN_OPS.get(op)
            if spec is None:
                raise FusionError(f"operator '{op}' is not known to the fused executor")
            if ndims == {2} and op not in OPS_2D and spec.kind != "pointwise":
                raise FusionError(f"{op} on 2-D fields is not fused")
            ins = [infos[i] for i in node.input_ids]
            if spec.kind == "reduction":
                if not ins or ins[0].kind in ("scalar", "red"):
                    raise FusionError(f"{op} needs a per-voxel input")
                p = max(i.avail for i in ins)
                if op == "entropy_hist":
                    # two phases: min/max of the value, then its histogram over [min, max]
                    self.hist_mm[nid] = p
                    infos[nid] = _Info("red", p + 2, 1, compute_pass=p + 1)
                    continue
                infos[nid] = _Info("red", p + 1, 2 if op == "min_max" else 1, compute_pass=p)
            elif spec.kind == "scan":
                if int(node.params.get("dim", 0)) != 0:
                    raise FusionError("cumulative_integral: only dim=0 is fused")
                if ins[0].kind in ("scalar", "red"):
                    raise FusionError("cumulative_integral needs a per-voxel input")
                infos[nid] = _Info("scan", ins[0].avail + 1, 0, compute_pass=ins[0].avail)
            elif spec.kind == "pointwise" and all(i.kind in ("scalar", "red") for i in ins):
                if any(i.kind == "red" and self.nodes[x].op_name == "min_max"
                       for i, x in zip(ins, node.input_ids)):
                    raise FusionError("min_max results cannot feed other operators")
                infos[nid] = _Info("scalar", max([i.avail for i in ins] + [0]), 1)
            else:
                infos[nid] = _Info("voxel", max([i.avail for i in ins] + [0]), 0)
        if shape is None:
            if any(i.kind in ("voxel", "red", "scan") for i in infos.values()):
                raise FusionError("graph has no 3-D field input")
            shape = (1, 1, 1)  # scalar-only graph: evaluated by the scalar kernel alone
        self.infos, self.shape = infos, shape
        self.dims2 = ndims == {2}

    def plan(self, key: str = "") -> FusedPlan:
        self.analyse()
        infos = self.infos
        t = 0
        self.const_index: Dict[str, int] = {}
        self.red_index: Dict[str, int] = {}
        scalar_sinks: Dict[str, int] = {}
        for nid in self.live:
            if self.nodes[nid].op_name == "_constant" and infos[nid].kind == "scalar":
                self.const_index[nid] = t
                t += 1
        for nid in self.live:
            if infos[nid].kind == "red":
                self.red_index[nid] = t
                # min_max: (min, max); entropy_hist: (entropy, min, max)
                t += {"min_max": 2, "entropy_hist": 3}.get(self.nodes[nid].op_name, 1)
        for nid in self.wanted:
            if infos[nid].kind == "scalar" and self.nodes[nid].op_name != "_constant":
                scalar_sinks[nid] = t
                t += 1
        self.table_size = max(t, 1)
        last = max([i.compute_pass for i in infos.values()] + [i.avail for i in infos.values()] + [0])
        passes: List[PassPlan] = []
        for p in range(last + 1):
            roots: List[Tuple[str, str]] = []
            for nid in self.live:
                inf = infos[nid]
                if inf.kind == "voxel" and inf.avail == p and nid in self.wanted:
                    roots.append(("out", nid))
                elif inf.kind in ("red", "scan") and inf.compute_pass == p:
                    roots.append((inf.kind, nid))
                if self.hist_mm.get(nid) == p:
                    roots.append(("hist_mm", nid))
            if roots:
                passes.append(self._build_pass(roots))
        scalar_source = self._scalar_source(scalar_sinks) if scalar_sinks else None
        return FusedPlan(key, self.shape, infos, passes, self.table_size, self.const_index, self.red_index,
                         scalar_sinks, scalar_source, self.wanted, self.out_dtype, list(self.live),
                         hist_size=self.hist_base, dims2=self.dims2,
                         keepdim={n for n in self.wanted if self.nodes[n].op_name == "norm_last"})

    def _build_pass(self, roots: List[Tuple[str, str]]) -> PassPlan:
        pg = PGraph()
        low = OpLowerer(pg, self.shape, dims2=self.dims2)
        slots: Dict[str, int] = {}
        field_nodes: List[str] = []
        fields: List[FieldSpec] = []
        memo: Dict[str, int] = {}

        def field_of(nid: str, dtype: str, nc: int) -> int:
            if nid not in slots:
                slots[nid] = len(fields)
                field_nodes.append(nid)
                fields.append(FieldSpec(len(fields), dtype, nc))
            return pg.add("field", (), nc, 0, field=slots[nid])

        def lower(nid: str) -> int:
            if nid in memo:
                return memo[nid]
            node = self.nodes[nid]
            inf = self.infos[nid]
            if inf.kind == "field":
                r = field_of(nid, TORCH_DT[node.params["value"].dtype], inf.nc)
            elif inf.kind == "scalar" and node.op_name == "_constant":
                r = pg.add("scalar", (), 1, 0, index=self.const_index[nid])
            elif inf.kind == "red":
                r = pg.add("scalar", (), 1, 0, index=self.red_index[nid])
            elif inf.kind == "scan":
                r = field_of(nid, "f32", self.scan_nc[nid])
            else:
                ins = [lower(i) for i in node.input_ids]
                try:
                    r = low.lower(node.op_name, ins, node.params, None)
                except LoweringError as exc:
                    raise FusionError(f"{node.op_name} ({nid}): {exc}") from exc
            memo[nid] = r
            return r

        if not hasattr(self, "scan_nc"):
            self.scan_nc: Dict[str, int] = {}
        rspecs: List[RootSpec] = []
        out_nodes: List[Tuple[str, str, int]] = []
        reductions: List[RedPlan] = []
        nslots = 0
        has_scan = False
        hists: List[RootSpec] = []
        n_vox = self.shape[0] * self.shape[1] * self.shape[2]
        for kind, nid in roots:
            node = self.nodes[nid]
            if kind == "out":
                pn = lower(nid)
                nc = pg.nodes[pn].nc
                rspecs.append(RootSpec("out", pn, out_slot=len(out_nodes), out_dtype=TORCH_DT[self.out_dtype]))
                out_nodes.append((nid, "out", nc))
            elif kind == "scan":
                has_scan = True
                pn = lower(node.input_ids[0])
                nc = pg.nodes[pn].nc
                self.scan_nc[nid] = nc
                h = float(node.params.get("dx", 1.0))
                rspecs.append(RootSpec("scan", pn, out_slot=len(out_nodes), out_dtype="f32", dx=(h, h, h)))
                out_nodes.append((nid, "scan", nc))
            elif kind == "hist_mm":
                pn = lower(node.input_ids[0])
                nc = pg.nodes[pn].nc
                rspecs.append(RootSpec("red", pn, red="minmax", slot=nslots))
                reductions.append(RedPlan(nid, nslots, self.red_index[nid] + 1, N.RED_MIN_MAX,
                                          float(n_vox * nc), 0, 0.0))
                nslots += RED_SLOTS["minmax"]
            elif node.op_name == "surface_integral":
                # Σ over voxels of (t · normals) · area_weights (stenpy_engine.py:2486-2494)
                if len(node.input_ids) != 3:
                    raise FusionError("surface_integral: (t, normals, area_weights)")
                t_, n_, w_ = (lower(i) for i in node.input_ids)
                if pg.nodes[t_].nc != 3 or pg.nodes[n_].nc != 3 or pg.nodes[w_].nc != 1:
                    raise FusionError("surface_integral: two (*, 3) fields and a scalar weight field")

                def comp_(x, c):
                    y = low.component(x, c)
                    return y if y is not None else pg.add("select", (x,), 1, pg.nodes[x].radius, index=c)
                dots = [low.binop("mul", comp_(t_, c), comp_(n_, c)) for c in range(3)]
                pn = low.binop("mul", low.binop("add", low.binop("add", dots[0], dots[1]), dots[2]), w_)
                rspecs.append(RootSpec("red", pn, red="sum", slot=nslots))
                reductions.append(RedPlan(nid, nslots, self.red_index[nid], N.RED_SUM, float(n_vox), 0, 0.0))
                nslots += RED_SLOTS["sum"]
            elif node.op_name in ("covariance", "correlation"):
                # co-moments of the value pairs (stenpy_engine.py:2575-2613, CPU branch: the
                # centred dot product over n - 1, or over the product of centred norms)
                extra = set(node.params) - {"alloc", "mm"}
                if len(node.input_ids) != 2 or extra:
                    raise FusionError(f"{node.op_name}: two fields and no parameters")
                a_, b_ = (lower(i) for i in node.input_ids)
                nc = pg.nodes[a_].nc
                if pg.nodes[b_].nc != nc:
                    raise FusionError(f"{node.op_name}: shape mismatch ({nc} vs {pg.nodes[b_].nc} components)")
                pn = low.stack([a_, b_])
                rspecs.append(RootSpec("red", pn, red="cov", slot=nslots))
                kind = N.RED_COVARIANCE if node.op_name == "covariance" else N.RED_CORRELATION
                reductions.append(RedPlan(nid, nslots, self.red_index[nid], kind, float(n_vox * nc), 0, 1e-15))
                nslots += RED_SLOTS["cov"]
            elif node.op_name == "entropy_hist":
                extra = set(node.params) - {"bins", "alloc", "mm"}
                if extra:
                    raise FusionError(f"entropy_hist: unexpected parameters {sorted(extra)}")
                bins = int(node.params.get("bins", 256))
                if not 1 <= bins <= 4096:
                    raise FusionError(f"entropy_hist: bins={bins} outside [1, 4096]")
                pn = lower(node.input_ids[0])
                r = RootSpec("red", pn, red="hist", slot=self.hist_base, bins=bins,
                             lohi_index=self.red_index[nid] + 1, table_index=self.red_index[nid])
                self.hist_base += bins
                rspecs.append(r)
                hists.append(r)
            else:
                op = node.op_name
                extra = set(node.params) - {"dim", "keepdim", "unbiased", "eps", "dx", "dims", "method",
                                            "alloc", "mm"}
                if extra:
                    raise FusionError(f"{op}: unexpected parameters {sorted(extra)}")
                if node.params.get("dim") is not None:
                    raise FusionError(f"{op}: only dim=None is fused")
                pn = lower(node.input_ids[0])
                nc = pg.nodes[pn].nc
                red = REDUCTIONS[op]
                r = RootSpec("red", pn, red=red, slot=nslots)
                if op == "integrate":
                    if node.params.get("dims") is not None:
                        raise FusionError("integrate: only dims=None is fused")
                    if nc != 1:
                        raise FusionError("integrate: scalar fields only")
                    r.dx = dx3(node.params.get("dx", 1.0))
                    r.method = str(node.params.get("method", "simpson"))
                reductions.append(RedPlan(nid, nslots, self.red_index[nid], RED_KIND[op], float(n_vox * nc),
                                          1 if bool(node.params.get("unbiased", True)) else 0,
                                          float(node.params.get("eps", 1e-15))))
                nslots += RED_SLOTS[red]
                rspecs.append(r)
        radius = max([pg.nodes[r.node].radius for r in rspecs] + [0])
        staged: Set[int] = set()

        def mark(x: int) -> None:
            if x not in staged:
                staged.add(x)
                for y in pg.nodes[x].ins:
                    mark(y)

        for n in pg.nodes:
            if n.op in STENCIL_PRIMS:
                mark(n.ins[0])
        offset_read = {pg.nodes[x].a("field") for x in staged if pg.nodes[x].op == "field"}
        cfg = PassConfig(**vars(self.cfg))
        if has_scan:
            cfg.seg_len = self.shape[0]
        cfg.prefetch = max(cfg.prefetch, 1)
        spec = PassSpec(pg, fields, rspecs, self.table_size, max(nslots, 1), radius, cfg, has_scan)
        spec.nested_ok = self.shape[1] >= 4 and self.shape[2] >= 4
        # arrays hold at most n0 planes plus halo planes on both sides (a chunk of
        # the planes holds fewer): element offsets of all of them, and the shell
        # kernel's voxel index plus one grid stride, stay below 2^31
        max_nc = max([f.nc for f in fields] + [pg.nodes[r.node].nc for r in rspecs] + [1])
        spec.idx32 = ((self.shape[0] + 2 * radius + 2) * self.shape[1] * self.shape[2] * max_nc
                      + SHELL_MAX_CTAS * SHELL_THREADS < 1 << 31)
        n2 = self.shape[2]
        for f in fields:
            # every field goes through a TMA-filled plane ring when the layout allows;
            # fields read at offsets carry a halo of the pass radius
            f.halo = radius if f.slot in offset_read else 0
            es = ESIZE[f.dtype]
            f.tma = (n2 * f.nc * es) % 16 == 0        # the box (and its k-halo) as TMA stages it
            w, h = spec.box(f)
            f.tma = f.tma and (w * es) % 16 == 0 and w <= 256 and h <= 256
            f.staged = f.tma or f.slot in offset_read
            if f.staged and not f.tma and self.shape[1] * n2 * f.nc * es + 4 * w * es >= 1 << 31:
                # row staging addresses a unit by its 32-bit offset from the plane start
                raise FusionError(f"a plane of {self.shape[1]} x {n2} rows too large to row-stage "
                                  f"({n2 * f.nc * es} B rows are not 16-byte multiples)")
            if radius == 0 and not has_scan:
                f.tma = f.staged = False     # flat pass: vector loads straight from HBM
        if self.ghosts:
            analyse_ghosts(spec)
        if 2 * radius + 1 + cfg.prefetch > MAX_RING_SLOTS:
            raise FusionError(f"stencil reach {radius} needs more than {MAX_RING_SLOTS} plane-ring slots")
        if smem_layout(spec)[0] > MAX_SMEM_BYTES:
            raise FusionError(f"stencil reach {radius}: the plane rings exceed {MAX_SMEM_BYTES} B of shared memory")
        return PassPlan(spec, field_nodes, out_nodes, reductions, hists)

    def _scalar_source(self, sinks: Dict[str, int]) -> str:
        """One-thread FP64 kernel for sinks that are expressions of scalars only."""
        lines = ['extern "C" __global__ void sten_scalars(double* t) {', "  if (threadIdx.x != 0) return;"]
        memo: Dict[str, str] = {}

        def ev(nid: str) -> str:
            if nid in memo:
                return memo[nid]
            node = self.nodes[nid]
            if node.op_name == "_constant":
                r = f"t[{self.const_index[nid]}]"
            elif self.infos[nid].kind == "red":
                r = f"t[{self.red_index[nid]}]"
            else:
                a = [ev(i) for i in node.input_ids]
                op = node.op_name
                eps = float(node.params.get("eps", 1e-15))
                if op == "add":
                    e = f"({a[0]} + {a[1]})"
                elif op == "sub":
                    e = f"({a[0]} - {a[1]})"
                elif op == "mul":
                    e = f"({a[0]} * {a[1]})" if len(a) == 2 else f"({a[0]} * {float(node.params['scalar'])!r})"
                elif op == "div":
                    e = f"({a[0]} / (fabs({a[1]}) < {eps!r} ? ({a[1]} < 0 ? -{eps!r} : {eps!r}) : {a[1]}))"
                elif op == "neg":
                    e = f"(-{a[0]})"
                elif op in ("exp", "sin", "cos", "tanh"):
                    e = f"{op}({a[0]})"
                elif op == "abs":
                    e = f"fabs({a[0]})"
                elif op == "log":
                    e = f"log(fmax({a[0]}, {eps!r}))"
                elif op == "sqrt":
                    e = f"sqrt(fmax({a[0]}, {float(node.params.get('eps', 0.0))!r}))"
                elif op == "clamp":
                    lo = a[1] if len(a) > 1 else repr(float(node.params.get("lo", 0.0)))
                    hi = a[2] if len(a) > 2 else repr(float(node.params.get("hi", 1.0)))
                    e = f"fmin(fmax({a[0]}, {lo}), {hi})"
                else:
                    raise FusionError(f"{op} on scalars is not supported")
                r = f"s{len(memo)}"
                lines.append(f"  const double {r} = {e};")
            memo[nid] = r
            return r

        for nid, idx in sinks.items():
            lines.append(f"  t[{idx}] = {ev(nid)};")
        lines.append("}")
        return "\n".join(lines) + "\n"


def structure_key(graph: Graph, wanted: Sequence[str], out_dtype, cfg: Optional[PassConfig]) -> str:
    live = graph.live_nodes(wanted)
    index = {nid: i for i, nid in enumerate(live)}
    parts = [str(out_dtype), repr(vars(cfg)) if cfg else "-", ",".join(str(index[w]) for w in wanted)]
    for nid in live:
        node = graph._nodes[nid]
        if node.op_name == "_constant":
            v = node.params.get("value")
            parts.append(f"F{tuple(v.shape)}{v.dtype}" if is_field_value(v) else "S")
            continue
        params = sorted((k, repr(v)) for k, v in node.params.items() if k not in ("alloc", "mm"))
        parts.append(f"{node.op_name}:{[index[i] for i in node.input_ids]}:{params}")
    return hashlib.sha256("|".join(parts).encode()).hexdigest()[:40]


_plan_cache: Dict[str, FusedPlan] = {}
_plan_lock = threading.Lock()


def get_plan(graph: Graph, wanted: Sequence[str], out_dtype=torch.float32,
             config: Optional[PassConfig] = None) -> FusedPlan:
    key = structure_key(graph, wanted, out_dtype, config)
    with _plan_lock:
        plan = _plan_cache.get(key)
    if plan is None:
        plan = Planner(graph, wanted, out_dtype, config).plan(key)
        with _plan_lock:
            _plan_cache[key] = plan
    return plan


# --------------------------------------------------------------------------- execution
def compile_pass(pp: PassPlan, device: int) -> None:
    if pp.module is not None:
        return
    src = emit_pass(pp.spec)
    smem, _, _ = smem_layout(pp.spec)
    key, cubin = N.compile_cached(src, NVRTC_OPTS)
    pp.module = N.load_module(key, cubin, "sten_kernel", smem, device)
    if has_shell(pp.spec):
        pp.shell_module = N.load_module(key + ":shell", cubin, "sten_shell", 0, device)
    if pp.hists:
        pp.hist_module = N.load_module(key + ":hist", cubin, "sten_hist_final", 0, device)
    pp.smem, pp.source, pp.key = smem, src, key


def has_shell(spec: PassSpec) -> bool:
    return shell_regions(spec) != ""


def encode_tmaps(spec: PassSpec, ptrs: Sequence[int], nl: int, n1: int, n2: int) -> List[bytes]:
    """TMA descriptors of a pass, in the order the kernel's Params expects: each
    TMA field's plane box and, for periodic ghosts, its wrap-strip boxes. ``ptrs``
    are the field base addresses by slot, ``nl`` the planes of the arrays."""
    out = []
    for slot, kind, (bw, bh) in tmap_specs(spec):
        f = spec.fields[slot]
        es = ESIZE[f.dtype]
        if ptrs[slot] % 16:
            raise FusionError("TMA field base address must be 16-byte aligned")
        out.append(N.encode_tmap_3d(es, ptrs[slot], n2 * f.nc, n1, nl, n2 * f.nc * es,
                                    n1 * n2 * f.nc * es, (bw, bh, 1)))
    return out


def pack_params(spec: PassSpec, values: Dict[str, Any], tmaps: List[bytes]) -> bytes:
    layout = param_layout(spec)
    buf = bytearray(layout.size)
    o = layout.offsets
    for i, tm in enumerate(tmaps):
        buf[o["tmap"] + 128 * i: o["tmap"] + 128 * (i + 1)] = tm
    for i, ptr in enumerate(values["fld"]):
        struct.pack_into("<Q", buf, o["fld"] + 8 * i, ptr)
    for i, ptr in enumerate(values["out"]):
        struct.pack_into("<Q", buf, o["out"] + 8 * i, ptr)
    for name in ("scal", "part", "hist", "err"):
        struct.pack_into("<Q", buf, o[name], int(values.get(name, 0)))
    for name in ("n0g", "n1", "n2", "nl", "i_base", "out_lo", "n_out", "seg_len", "tiles_k", "cta_off"):
        struct.pack_into("<i", buf, o[name], int(values[name]))
    return bytes(buf)


class ErrorFlag:
    """Per-device status word that kernels set when a bounded wait gives up."""
    _flags: Dict[int, torch.Tensor] = {}

    @classmethod
    def get(cls, device: torch.device) -> torch.Tensor:
        idx = device.index if device.index is not None else torch.cuda.current_device()
        f = cls._flags.get(idx)
        if f is None:
            f = torch.zeros(1, dtype=torch.int32, device=torch.device("cuda", idx))
            cls._flags[idx] = f
        return f

    @classmethod
    def check(cls, device: torch.device) -> None:
        f = cls.get(device)
        v = int(f.item())
        if v:
            f.zero_()
            raise RuntimeError(f"stenpy_b200: a kernel reported device status {v} "
                               "(bounded wait on a TMA copy expired)")


@dataclass
class Launch:
    module: int
    grid: Tuple[int, int, int]
    block: Tuple[int, int, int]
    smem: int
    params: bytes


@dataclass
class Finalize:
    part: torch.Tensor
    ncta: int
    nslots: int
    descs: List[Any]
    table: torch.Tensor


@dataclass
class Program:
    """Everything one execution enqueues, fully resolved (pointers packed)."""
    ops: List[Any]
    results: Dict[str, Any]
    const_host: Optional[torch.Tensor]
    table: torch.Tensor

    @property
    def n_kernels(self) -> int:
        return sum(1 for op in self.ops if isinstance(op, (Launch, Finalize)))


def build_program(plan: FusedPlan, values: Dict[str, Any], device: torch.device,
                  outputs: Optional[Dict[str, torch.Tensor]] = None) -> Program:
    """Resolve a plan against concrete leaf tensors: compile kernels (cached),
    allocate outputs and scratch, encode TMA descriptors, pack parameters."""
    n0, n1, n2 = plan.shape
    dev_idx = device.index if device.index is not None else torch.cuda.current_device()
    table = plan.buffers.get("table")
    if table is None:
        table = torch.zeros(plan.table_size, dtype=torch.float64, device=device)
        plan.buffers["table"] = table
    err = ErrorFlag.get(device)
    const_host = None
    if plan.const_index:
        ch = torch.zeros(plan.table_size, dtype=torch.float64)
        for nid, idx in plan.const_index.items():
            v = values[nid]
            ch[idx] = float(v.item() if isinstance(v, torch.Tensor) else v)
        const_host = ch.pin_memory()
    ops: List[Any] = []
    results: Dict[str, Any] = {}
    produced: Dict[str, torch.Tensor] = {}
    hist_ptr = 0
    if plan.hist_size:
        hist = plan.buffers.get("hist")
        if hist is None:
            # zeroed once; the entropy kernel clears the counts after reading them
            hist = torch.zeros(plan.hist_size, dtype=torch.int64, device=device)
            plan.buffers["hist"] = hist
        hist_ptr = hist.data_ptr()
    for pi, pp in enumerate(plan.passes):
        compile_pass(pp, dev_idx)
        spec = pp.spec
        cfg = spec.cfg
        tiles_k = -(-n2 // cfg.tk)
        gx, gy = pass_grid(spec, n1, n2, n0)
        grid = (gx, gy, 1)
        ncta = grid[0] * grid[1]
        fptrs: List[int] = []
        for f, nid in zip(spec.fields, pp.field_nodes):
            t = produced[nid] if nid in produced else values[nid]
            if not isinstance(t, torch.Tensor) or t.device != device:
                raise FusionError(f"field {nid} must be a tensor on {device} (there is no CPU path)")
            if not t.is_contiguous():
                raise FusionError(f"field {nid} must be contiguous")
            if DT_TORCH[f.dtype] != t.dtype:
                raise FusionError(f"field {nid}: planned {f.dtype}, got {t.dtype}")
            fptrs.append(t.data_ptr())
        tmaps = encode_tmaps(spec, fptrs, n0, n1, n2)
        outs: List[torch.Tensor] = []
        for (nid, okind, nc), r in zip(pp.out_nodes, [r for r in spec.roots if r.kind in ("out", "scan")]):
            o = outputs.get(nid) if (outputs and okind == "out") else None
            if o is None:
                o = torch.empty(plan.out_shape(nc, nid), dtype=DT_TORCH[r.out_dtype], device=device)
            outs.append(o)
            produced[nid] = o
            if nid in plan.wanted:
                results[nid] = o
        n_shell = shell_count(plan.shape, spec.radius, regions=shell_regions(spec))
        n_sh_cta = shell_ctas(n_shell)
        total_cta = ncta + n_sh_cta
        part = plan.buffers.get(f"part{pi}")
        need = total_cta * spec.nslots
        if part is None or part.numel() < need:
            part = torch.zeros(max(need, 1), dtype=torch.float64, device=device)
            plan.buffers[f"part{pi}"] = part
        params = pack_params(spec, dict(fld=fptrs, out=[o.data_ptr() for o in outs], scal=table.data_ptr(),
                                        part=part.data_ptr(), hist=hist_ptr, err=err.data_ptr(), n0g=n0, n1=n1,
                                        n2=n2, nl=n0, i_base=0, out_lo=0, n_out=n0, seg_len=cfg.seg_len,
                                        tiles_k=tiles_k, cta_off=0), tmaps)
        ops.append(Launch(pp.module, grid, (cfg.threads, 1, 1), pp.smem, params))
        if n_sh_cta:
            shell_params = pack_params(spec, dict(fld=fptrs, out=[o.data_ptr() for o in outs],
                                                  scal=table.data_ptr(), part=part.data_ptr(), hist=hist_ptr,
                                                  err=err.data_ptr(), n0g=n0, n1=n1, n2=n2, nl=n0, i_base=0,
                                                  out_lo=0, n_out=n0, seg_len=cfg.seg_len, tiles_k=tiles_k,
                                                  cta_off=ncta), tmaps)
            ops.append(Launch(pp.shell_module, (n_sh_cta, 1, 1), (SHELL_THREADS, 1, 1), 0, shell_params))
        if pp.reductions:
            descs = [N.ReduceDesc(r.kind, r.slot, r.table_index, r.unbiased, r.count, r.eps)
                     for r in pp.reductions]
            ops.append(Finalize(part, total_cta, spec.nslots, descs, table))
        if pp.hists:
            ops.append(Launch(pp.hist_module, (1, 1, 1), (256, 1, 1), 0, params))
    if plan.scalar_source:
        if plan.scalar_module is None:
            key, cubin = N.compile_cached(plan.scalar_source, NVRTC_OPTS)
            plan.scalar_module = N.load_module(key, cubin, "sten_scalars", 0, dev_idx)
        ops.append(Launch(plan.scalar_module, (1, 1, 1), (32, 1, 1), 0, struct.pack("<Q", table.data_ptr())))
    for nid, idx in plan.red_index.items():
        if nid in plan.wanted:
            results[nid] = (nid, idx, 2 if plan.infos[nid].nc == 2 else 1)
    for nid, idx in plan.scalar_sinks.items():
        results[nid] = (nid, idx, 1)
    for nid in plan.wanted:
        if nid not in results:
            results[nid] = values[nid]
    return Program(ops, results, const_host, table)


def enqueue(prog: Program, stream: torch.cuda.Stream) -> int:
    """Enqueue a resolved program on ``stream``; returns the number of kernels launched."""
    s = stream.cuda_stream
    n = 0
    if prog.const_host is not None:
        with torch.cuda.stream(stream):
            prog.table.copy_(prog.const_host, non_blocking=True)
    for op in prog.ops:
        if isinstance(op, Launch):
            N.launch(op.module, op.grid, op.block, op.smem, s, op.params)
        else:
            N.finalize(op.part.data_ptr(), op.ncta, op.nslots, op.descs, op.table.data_ptr(), s)
        n += 1
    return n


def collect(prog: Program, stream: torch.cuda.Stream) -> Dict[str, Any]:
    """Results of an enqueued program: per-voxel outputs as produced, scalar results
    as fresh 0-d (or length-2) FP64 device tensors copied out of the scalar table."""
    out: Dict[str, Any] = {}
    with torch.cuda.stream(stream):
        for nid, v in prog.results.items():
            if isinstance(v, tuple):
                _, idx, n = v
                out[nid] = prog.table[idx:idx + n].clone() if n == 2 else prog.table[idx].clone()
            else:
                out[nid] = v
    return out


def bind(plan: FusedPlan, graph: Graph, wanted: Sequence[str]) -> Tuple[Dict[str, Any], Dict[str, str]]:
    """Leaf values of ``graph`` keyed by the plan's node ids, and the map from the
    plan's ids back to ``graph``'s (plans are shared by structurally equal graphs,
    whose live nodes correspond position by position)."""
    live = graph.live_nodes(list(dict.fromkeys(wanted)))
    if len(live) != len(plan.live):
        raise FusionError("internal: plan does not match graph structure")
    to_plan = dict(zip(live, plan.live))
    back = {v: k for k, v in to_plan.items()}
    values = {to_plan[nid]: graph._nodes[nid].params["value"] for nid in live
              if graph._nodes[nid].op_name == "_constant"}
    return values, back


def execute(graph: Graph, wanted: Sequence[str], device: torch.device, out_dtype=torch.float32,
            config: Optional[PassConfig] = None,
            outputs: Optional[Dict[str, torch.Tensor]] = None) -> Dict[str, Any]:
    plan = get_plan(graph, wanted, out_dtype, config)
    values, back = bind(plan, graph, wanted)
    to_plan = {v: k for k, v in back.items()}
    prog = build_program(plan, values, device,
                         {to_plan[k]: v for k, v in outputs.items()} if outputs else None)
    stream = torch.cuda.current_stream(device)
    enqueue(prog, stream)
    return {back[k]: v for k, v in collect(prog, stream).items()}

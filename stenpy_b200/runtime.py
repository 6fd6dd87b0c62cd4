"""``Runtime``: the executor slot of the reference (stenpy_engine.py:509-1146).

``Runtime(mm, device).run(graph, seed=None) -> Dict[node_id, value]`` keeps the
reference's contract. On a CUDA device the graph goes through the fused executor
(``fused_compiler``); with ``fusion_enabled=False`` each node runs as its own
one-node kernel with every intermediate materialised (the eager mode, the
structure of ``_run_original``). There is no CPU execution path: a CPU device is
rejected, and the CPU reference result lives only in the test oracle.

User-registered operators (``register_operator`` with a name the code generator
does not know) are opaque: their inputs are evaluated by the fused executor, the
operator is called on the GPU tensors with ``alloc=``/``mm=`` injected by
signature (stenpy_engine.py:1074-1080), and its output replaces the node as a leaf
(``Graph.clone_with_replacement``) for the rest of the graph.
"""
from __future__ import annotations

import inspect
import os
import warnings
from typing import Any, Dict, Iterable, List, Optional, Sequence

import torch

from . import fused_compiler as FC
from .codegen import PassConfig
from .graph import Graph
from .memory_manager import MemoryManager
from .registry import KNOWN_OPS, OP_REGISTRY

FUSION_ENABLED = os.environ.get("OPS_FUSION_ENABLED", "1").lower() in ("1", "true", "yes")


def _resolve_device(device: Any) -> torch.device:
    dev = torch.device(device)
    if dev.type != "cuda":
        raise NotImplementedError(
            f"stenpy_b200 executes on CUDA devices only (got {dev}); there is no CPU path")
    if not torch.cuda.is_available():
        raise RuntimeError("device='cuda' requested but no GPU is visible to this process")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def default_wanted(graph: Graph) -> List[str]:
    """Sinks of the graph, minus nodes the front end left orphaned by a rewrite."""
    dead = getattr(graph, "_orphans", set())
    return [s for s in graph.sinks() if s not in dead]


class Runtime:
    def __init__(self, mm: Optional[MemoryManager] = None, device: Any = "cuda", skip_pool: bool = False,
                 fusion_enabled: Optional[bool] = None, out_dtype: torch.dtype = torch.float32,
                 config: Optional[PassConfig] = None, check_errors: bool = True) -> None:
        self.mm = mm if mm is not None else MemoryManager()
        self.device = _resolve_device(device)
        self.skip_pool = skip_pool
        self.fusion_enabled = FUSION_ENABLED if fusion_enabled is None else bool(fusion_enabled)
        self.out_dtype = out_dtype
        self.config = config
        self.check_errors = check_errors

    # -- helpers
    def _to_device(self, v: Any) -> Any:
        if isinstance(v, torch.Tensor) and v.device != self.device:
            return v.to(self.device)
        return v

    def _with_seed(self, graph: Graph, seed: Optional[Dict[str, Any]]) -> Graph:
        g = graph
        for nid, val in (seed or {}).items():
            if nid in g._nodes:
                g = g.clone_with_replacement(nid, val)
        # leaf tensors are read in place: move them to the device once, contiguous
        for nid in list(g._order):
            v = g._nodes[nid].params.get("value") if g._nodes[nid].op_name == "_constant" else None
            if isinstance(v, torch.Tensor) and v.ndim >= 1 and (v.device != self.device or not v.is_contiguous()):
                g = g.clone_with_replacement(nid, v.to(self.device).contiguous())
        return g

    def _call_opaque(self, g: Graph, nid: str, values: Dict[str, Any]) -> Any:
        node = g._nodes[nid]
        fn = OP_REGISTRY[node.op_name]
        kwargs = dict(node.params)
        try:
            params = inspect.signature(fn).parameters
        except (TypeError, ValueError):
            params = {}
        if "alloc" in params:
            kwargs["alloc"] = self.mm.allocate
        if "mm" in params:
            kwargs["mm"] = self.mm
        args = [values[i] for i in node.input_ids]
        out = fn(*args, **kwargs)
        return self._to_device(out)

    def _execute(self, g: Graph, wanted: Sequence[str]) -> Dict[str, Any]:
        need = [w for w in wanted if g._nodes[w].op_name != "_constant"]
        res: Dict[str, Any] = {}
        if need:
            res = FC.execute(g, need, self.device, self.out_dtype, self.config)
        for w in wanted:
            if w not in res:
                res[w] = g._nodes[w].params["value"]
        return res

    # -- the contract
    def run(self, graph: Graph, seed: Optional[Dict[str, Any]] = None,
            wanted: Optional[Iterable[str]] = None) -> Dict[str, Any]:
        wanted = list(wanted) if wanted is not None else default_wanted(graph)
        g = self._with_seed(graph, seed)
        with torch.no_grad():
            if not self.fusion_enabled:
                results = self._run_eager(g, wanted)
            else:
                results = self._run_fused(g, wanted)
        if self.check_errors:
            torch.cuda.current_stream(self.device).synchronize()
            FC.ErrorFlag.check(self.device)
        out: Dict[str, Any] = dict(seed or {})
        for nid in g._order:
            if g._nodes[nid].op_name == "_constant" and nid in graph._nodes and \
                    graph._nodes[nid].op_name == "_constant":
                out[nid] = graph._nodes[nid].params.get("value")
        out.update(results)
        return out

    def _run_fused(self, g: Graph, wanted: List[str]) -> Dict[str, Any]:
        try:
            return self._run_fused_or_raise(g, wanted)
        except FC.FusionError as exc:
            # as the reference does when fusion fails (stenpy_engine.py:949-954): warn and
            # run the graph node by node, still on the GPU
            warnings.warn(f"Fusion failed, falling back to node-by-node execution: {exc}", RuntimeWarning)
            return self._run_eager(g, wanted)

    def _run_fused_or_raise(self, g: Graph, wanted: List[str]) -> Dict[str, Any]:
        while True:
            order = [n.id for n in g.topological_sort()]
            live = set(g.live_nodes(wanted))
            opaque = [n for n in order if n in live and g._nodes[n].op_name not in KNOWN_OPS
                      and g._nodes[n].op_name != "_constant"]
            if not opaque:
                break
            nid = opaque[0]
            ins = list(dict.fromkeys(g._nodes[nid].input_ids))
            vals = self._execute(g, ins) if ins else {}
            g = g.clone_with_replacement(nid, self._call_opaque(g, nid, vals))
        return self._execute(g, wanted)

    def _run_eager(self, g: Graph, wanted: List[str]) -> Dict[str, Any]:
        """One kernel per node, every intermediate materialised (reference structure)."""
        live = set(g.live_nodes(wanted))
        values: Dict[str, Any] = {}
        for node in g.topological_sort():
            if node.id not in live:
                continue
            if node.op_name == "_constant":
                values[node.id] = node.params["value"]
                continue
            if node.op_name not in KNOWN_OPS:
                values[node.id] = self._call_opaque(g, node.id, values)
                continue
            values[node.id] = run_single_op(node.op_name, [values[i] for i in node.input_ids],
                                            node.params, device=self.device, out_dtype=self.out_dtype)
        return {w: values[w] for w in wanted}


def run_single_op(name: str, inputs: Sequence[Any], params: Dict[str, Any],
                  device: Optional[torch.device] = None, out_dtype: Optional[torch.dtype] = None) -> Any:
    """Run one built-in operator through the fused executor (the registry's callables)."""
    params = {k: v for k, v in params.items() if k not in ("alloc", "mm")}
    if device is None:
        dev = next((t.device for t in inputs if isinstance(t, torch.Tensor) and t.ndim >= 1), None)
        if dev is None or dev.type != "cuda":
            raise NotImplementedError(f"{name}: stenpy_b200 operators run on CUDA tensors only")
        device = dev
    g = Graph()
    ids = [g.add("_constant", (), {"value": v}) for v in inputs]
    nid = g.add(name, ids, params)
    if out_dtype is None:
        out_dtype = torch.float32
    res = FC.execute(g, [nid], device, out_dtype)
    return res[nid]

"""Expression DAG: ``GraphNode`` and ``Graph``.

Mirrors the reference IR (stenpy_engine.py:351-444): a node is a frozen record
``(id, op_name, input_ids, params)``; a graph keeps insertion order in ``_order``
and nodes in ``_nodes`` (both read directly by callers, as in the reference's
stenpy.py:888 and fused_compiler.py:237), plus per-node shape/dtype hints filled
by the executor.

Added on top of the reference contract: ``live_nodes`` (dead-node elimination
from a set of sinks; the reference executes orphaned nodes such as the
``gradient`` left behind by the div∘grad → laplacian rewrite) and ``sinks``.
"""
from __future__ import annotations

import collections
import itertools
from dataclasses import dataclass, field as dc_field
from typing import Any, Dict, Iterable, List, Optional, Tuple

import torch

_call_counter = itertools.count()


def _uid(prefix: str = "t") -> str:
    """Unique node id ``<prefix>_<n>`` (stenpy_engine.py:89-90)."""
    return f"{prefix}_{next(_call_counter)}"


@dataclass(frozen=True)
class GraphNode:
    id: str
    op_name: str
    input_ids: Tuple[str, ...] = dc_field(default_factory=tuple)
    params: Dict[str, Any] = dc_field(default_factory=dict)


class Graph:
    """Insertion-ordered DAG of ``GraphNode`` (stenpy_engine.py:359-444)."""

    def __init__(self) -> None:
        self._nodes: Dict[str, GraphNode] = {}
        self._order: List[str] = []
        self._dtypes: Dict[str, torch.dtype] = {}
        self._shapes: Dict[str, Tuple[int, ...]] = {}

    def add(self, op_name: str, input_ids: Iterable[str] = (),
            params: Optional[Dict[str, Any]] = None,
            node_id: Optional[str] = None) -> str:
        nid = node_id or _uid(op_name)
        self._nodes[nid] = GraphNode(nid, op_name, tuple(input_ids), dict(params or {}))
        if nid not in self._order:
            self._order.append(nid)
        return nid

    def topological_sort(self) -> List[GraphNode]:
        """Kahn order; ties broken by insertion order (stenpy_engine.py:387-410)."""
        indeg = {nid: 0 for nid in self._nodes}
        children: Dict[str, List[str]] = {nid: [] for nid in self._nodes}
        for nid in self._order:
            for dep in self._nodes[nid].input_ids:
                if dep not in self._nodes:
                    raise ValueError(f"Node '{nid}' references unknown input '{dep}'")
                indeg[nid] += 1
                children[dep].append(nid)
        queue = collections.deque(nid for nid in self._order if indeg[nid] == 0)
        out: List[GraphNode] = []
        while queue:
            nid = queue.popleft()
            out.append(self._nodes[nid])
            for c in children[nid]:
                indeg[c] -= 1
                if indeg[c] == 0:
                    queue.append(c)
        if len(out) != len(self._nodes):
            raise ValueError("Graph contains a cycle")
        return out

    def clone_with_replacement(self, source_id: str, tensor: Any) -> "Graph":
        """Copy with node ``source_id`` replaced by a ``_constant`` holding ``tensor``
        (stenpy_engine.py:412-421)."""
        g = Graph()
        for nid in self._order:
            node = self._nodes[nid]
            if nid == source_id:
                g.add("_constant", (), {"value": tensor}, node_id=nid)
            else:
                g.add(node.op_name, node.input_ids, node.params, node_id=nid)
        return g

    def __len__(self) -> int:
        return len(self._nodes)

    def __repr__(self) -> str:
        return f"Graph({len(self._nodes)} nodes)"

    def set_node_shape(self, node_id: str, shape: Tuple[int, ...],
                       dtype: torch.dtype = torch.float64) -> None:
        self._shapes[node_id] = tuple(shape)
        self._dtypes[node_id] = dtype

    def get_node_shape(self, node_id: str) -> Optional[Tuple[int, ...]]:
        return self._shapes.get(node_id)

    def get_node_dtype(self, node_id: str) -> torch.dtype:
        return self._dtypes.get(node_id, torch.float64)

    def build_consumer_map(self) -> Dict[str, List[str]]:
        consumers: Dict[str, List[str]] = {nid: [] for nid in self._nodes}
        for nid in self._order:
            for dep in self._nodes[nid].input_ids:
                consumers[dep].append(nid)
        return consumers

    # -- additions -----------------------------------------------------------
    def sinks(self) -> List[str]:
        """Nodes nobody consumes, in insertion order (stenpy_engine.py:447-451)."""
        consumed = set()
        for node in self._nodes.values():
            consumed.update(node.input_ids)
        return [nid for nid in self._order if nid not in consumed]

    def live_nodes(self, wanted: Iterable[str]) -> List[str]:
        """Ids reachable backwards from ``wanted``, in insertion order."""
        keep = set()
        stack = list(wanted)
        while stack:
            nid = stack.pop()
            if nid in keep:
                continue
            keep.add(nid)
            stack.extend(self._nodes[nid].input_ids)
        return [nid for nid in self._order if nid in keep]

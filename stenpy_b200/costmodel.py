"""Learned schedule ranking: a small MLP over pass + schedule features.

The autotuner times every candidate schedule of a pass (24 of them); the cost
model predicts the (log) time of each candidate from features of the pass (op
mix, stencil reach, fields, dtypes, grid) and of the schedule (tile, threads,
rows per thread, z-segment, boundary strategy, shared memory) so that only the
top few need timing. It changes which schedule is picked, never any result.

* Network: in -> 64 -> ReLU -> 64 -> ReLU -> 1, trained with mean-squared error on
  log nanoseconds per voxel centred per pass (only the order of a pass's
  candidates matters, not the pass's absolute cost), Adam with weight decay; an
  ensemble of a few seeds is averaged. Forward, backward and the optimizer step
  are the library's own CUDA kernels (``stenpy_mlp_forward`` /
  ``stenpy_mlp_loss_grad`` / ``stenpy_adam_step``); PyTorch only holds the device
  buffers.
* Data: the autotuner's JSON-lines log (``autotune.LOG_PATH``).
* ``random_dag`` generates the cost-model workload: random expression DAGs of
  3-20 ops over the operator list, stencil reach 1-2, FP32 or BF16 fields, grids
  with every dimension a multiple of 32 in [64, 512].
* ``evaluate`` reports top-k selection regret against exhaustive tuning, and the
  same for the methods without the model (the default schedule, a random pick).
"""
from __future__ import annotations

import json
import math
import os
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _native as N

HIDDEN = 64
GRAPH_KEYS = ["radius", "n_fields", "in_bytes", "out_bytes", "n_d1", "n_lap", "n_trans", "n_arith", "n_eig",
              "n_out", "n_red", "n_slots", "narrow", "max_nc"]
SCHED_KEYS = ["tj", "tk", "threads", "vpt", "seg_len", "prefetch", "smem", "ghost", "shell", "kv"]
_LOG_KEYS = {"tj", "tk", "threads", "vpt", "seg_len", "kv"}


def vectorize(feat: Dict[str, float], sched: Dict[str, float]) -> List[float]:
    """Feature vector of (pass, schedule): raw counts, log2 sizes and derived
    occupancy / halo-overhead terms."""
    x = [float(feat.get(k, 0.0)) for k in GRAPH_KEYS]
    n0, n1, n2 = float(feat["n0"]), float(feat["n1"]), float(feat["n2"])
    x += [math.log2(n0), math.log2(n1), math.log2(n2), math.log2(max(feat["voxels"], 1.0))]
    for k in SCHED_KEYS:
        v = float(sched.get(k, 1.0 if k == "kv" else 0.0))
        x.append(math.log2(v) if k in _LOG_KEYS and v > 0 else (v / 1e5 if k == "smem" else v))
    tj, tk, seg = float(sched["tj"]), float(sched["tk"]), float(sched["seg_len"])
    ctas = math.ceil(n1 / tj) * math.ceil(n2 / tk) * math.ceil(n0 / seg)
    r = float(feat.get("radius", 0))
    x += [math.log2(ctas), ctas / 148.0 / 8.0, (tj + 2 * r) * (tk + 8 * (r > 0)) / (tj * tk),
          (seg + 2 * r) / seg]
    return x


def target(ms: float, feat: Dict[str, float]) -> float:
    """log of nanoseconds per voxel (comparable across grids)."""
    return math.log(ms * 1e6 / max(feat["voxels"], 1.0))


class CostModel:
    """MLP parameters + Adam state on the device; every numeric step runs in the
    library's kernels."""

    def __init__(self, in_dim: int, device: Any = "cuda", hidden: int = HIDDEN, seed: int = 0):
        self.in_dim, self.hidden = in_dim, hidden
        self.device = torch.device(device)
        n = N.mlp_param_count(in_dim, hidden)
        g = torch.Generator().manual_seed(seed)
        p = torch.zeros(n, dtype=torch.float32)
        o = 0
        for fan_in, fan_out in ((in_dim, hidden), (hidden, hidden), (hidden, 1)):
            lim = math.sqrt(6.0 / fan_in)      # He-uniform weights, zero biases
            p[o:o + fan_in * fan_out] = (torch.rand(fan_in * fan_out, generator=g) * 2 - 1) * lim
            o += fan_in * fan_out + fan_out
        self.params = p.to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.step_count = 0
        self.mu = torch.zeros(in_dim)
        self.sd = torch.ones(in_dim)
        self.y_mu = 0.0
        self._ws: Optional[torch.Tensor] = None

    def _workspace(self, n: int) -> torch.Tensor:
        need = N.mlp_workspace_floats(n, self.hidden)
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.float32, device=self.device)
        return self._ws

    def _norm(self, X: torch.Tensor) -> torch.Tensor:
        return ((X - self.mu) / self.sd).to(self.device, torch.float32).contiguous()

    def predict(self, X: torch.Tensor) -> torch.Tensor:
        """Predicted target for each row of raw (unnormalised) features X [n, in_dim]."""
        Xd = self._norm(X)
        n = Xd.shape[0]
        out = torch.empty(n, dtype=torch.float32, device=self.device)
        s = torch.cuda.current_stream(self.device).cuda_stream
        N.mlp_forward(self.params.data_ptr(), self.in_dim, self.hidden, Xd.data_ptr(), n, out.data_ptr(),
                      self._workspace(n).data_ptr(), s)
        return out.cpu().double() + self.y_mu

    def loss_grad(self, Xd: torch.Tensor, y: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        """Mean-squared loss and its gradient for normalised device inputs."""
        n = Xd.shape[0]
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        s = torch.cuda.current_stream(self.device).cuda_stream
        N.mlp_loss_grad(self.params.data_ptr(), self.in_dim, self.hidden, Xd.data_ptr(), y.data_ptr(), n,
                        self.grad.data_ptr(), loss.data_ptr(), self._workspace(n).data_ptr(), s)
        return loss, self.grad

    def fit(self, X: torch.Tensor, y: torch.Tensor, steps: int = 3000, batch: int = 256, lr: float = 2e-3,
            weight_decay: float = 1e-3, seed: int = 0) -> List[float]:
        self.mu = X.mean(0)
        self.sd = X.std(0).clamp(min=1e-6)
        self.y_mu = float(y.mean())
        Xd = self._norm(X)
        yd = (y - self.y_mu).to(self.device, torch.float32).contiguous()
        n = Xd.shape[0]
        gen = torch.Generator(device=self.device).manual_seed(seed)
        s = torch.cuda.current_stream(self.device).cuda_stream
        hist = []
        for it in range(steps):
            idx = torch.randint(0, n, (min(batch, n),), generator=gen, device=self.device)
            xb, yb = Xd[idx].contiguous(), yd[idx].contiguous()
            loss, grad = self.loss_grad(xb, yb)
            self.step_count += 1
            N.adam_step(self.params.data_ptr(), grad.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                        self.params.numel(), lr * (0.1 if it > 0.8 * steps else 1.0), 0.9, 0.999, 1e-8,
                        self.step_count, weight_decay, s)
            if it % 100 == 0 or it == steps - 1:
                hist.append(float(loss))
        return hist

    def save(self, path: str) -> None:
        np.savez(path, in_dim=self.in_dim, hidden=self.hidden, params=self.params.cpu().numpy(),
                 mu=self.mu.numpy(), sd=self.sd.numpy(), y_mu=self.y_mu)

    @classmethod
    def load(cls, path: str, device: Any = "cuda") -> "CostModel":
        z = np.load(path)
        m = cls(int(z["in_dim"]), device, int(z["hidden"]))
        m.params = torch.from_numpy(z["params"]).to(m.device)
        m.mu, m.sd, m.y_mu = torch.from_numpy(z["mu"]), torch.from_numpy(z["sd"]), float(z["y_mu"])
        return m


class Ensemble:
    """Average of several independently seeded models (lower-variance ranking)."""

    def __init__(self, models: Sequence[CostModel]):
        self.models = list(models)

    def predict(self, X: torch.Tensor) -> torch.Tensor:
        return sum(m.predict(X) for m in self.models) / len(self.models)

    @classmethod
    def train(cls, X: torch.Tensor, y: torch.Tensor, device: Any = "cuda", n: int = 5, seed: int = 0,
              **fit_kw) -> Tuple["Ensemble", List[List[float]]]:
        models, hists = [], []
        for i in range(n):
            m = CostModel(X.shape[1], device, seed=seed * 1000 + i)
            hists.append(m.fit(X, y, seed=seed * 1000 + i, **fit_kw))
            models.append(m)
        return cls(models), hists

    def save(self, path: str) -> None:
        np.savez(path, n=len(self.models), **{f"m{i}_{k}": v for i, m in enumerate(self.models)
                                              for k, v in (("in_dim", m.in_dim), ("hidden", m.hidden),
                                                           ("params", m.params.cpu().numpy()),
                                                           ("mu", m.mu.numpy()), ("sd", m.sd.numpy()),
                                                           ("y_mu", m.y_mu))})

    @classmethod
    def load(cls, path: str, device: Any = "cuda") -> "Ensemble":
        z = np.load(path)
        models = []
        for i in range(int(z["n"])):
            m = CostModel(int(z[f"m{i}_in_dim"]), device, int(z[f"m{i}_hidden"]))
            m.params = torch.from_numpy(z[f"m{i}_params"]).to(m.device)
            m.mu, m.sd = torch.from_numpy(z[f"m{i}_mu"]), torch.from_numpy(z[f"m{i}_sd"])
            m.y_mu = float(z[f"m{i}_y_mu"])
            models.append(m)
        return cls(models)


def centred_targets(recs: Sequence[Dict[str, Any]]) -> torch.Tensor:
    """log ns/voxel minus its mean over the timed candidates of the same pass."""
    _, y = records_to_xy(recs)
    groups: Dict[str, List[int]] = {}
    for i, r in enumerate(recs):
        groups.setdefault(r["tag"] + ":" + r["key"], []).append(i)
    for idx in groups.values():
        y[idx] -= y[idx].mean()
    return y


def analytic_cost(feat: Dict[str, float], sched: Dict[str, float]) -> float:
    """A roofline-style estimate without learning: bytes moved (staged halo and
    z-segment overlap included) times the wave-quantisation loss of the grid."""
    n0, n1, n2 = float(feat["n0"]), float(feat["n1"]), float(feat["n2"])
    tj, tk, seg, nt = float(sched["tj"]), float(sched["tk"]), float(sched["seg_len"]), float(sched["threads"])
    r = float(feat.get("radius", 0))
    halo = (tj + 2 * r) * (tk + (8 if r > 0 else 0)) / (tj * tk)
    zf = (min(seg, n0) + 2 * r) / min(seg, n0)
    ctas = math.ceil(n1 / tj) * math.ceil(n2 / tk) * math.ceil(n0 / seg)
    per_sm = max(1, min(2048 // int(nt), 32, int(227e3 // max(float(sched.get("smem", 1.0)), 1.0))))
    waves = ctas / (148.0 * per_sm)
    tail = math.ceil(waves) / waves if waves > 0 else 1.0
    cover = (math.ceil(n1 / tj) * tj * math.ceil(n2 / tk) * tk) / (n1 * n2)
    return (feat["in_bytes"] * halo * zf + feat["out_bytes"]) * cover * tail


def load_records(path: str, tags: Optional[Sequence[str]] = None) -> List[Dict[str, Any]]:
    out = []
    with open(path) as fh:
        for line in fh:
            r = json.loads(line)
            if tags is None or any(str(r.get("tag", "")).startswith(t) for t in tags):
                out.append(r)
    return out


def records_to_xy(recs: Sequence[Dict[str, Any]]) -> Tuple[torch.Tensor, torch.Tensor]:
    X = torch.tensor([vectorize(r["features"], r["schedule"]) for r in recs], dtype=torch.float32)
    y = torch.tensor([target(r["ms"], r["features"]) for r in recs], dtype=torch.float32)
    return X, y


def group_by_pass(recs: Sequence[Dict[str, Any]]) -> Dict[str, List[Dict[str, Any]]]:
    g: Dict[str, List[Dict[str, Any]]] = {}
    for r in recs:
        g.setdefault(r["tag"] + ":" + r["key"], []).append(r)
    return g


def _stats(v) -> Optional[Dict[str, float]]:
    v = np.asarray(v, dtype=np.float64)
    if not len(v):
        return None
    return {"mean": float(v.mean()), "median": float(np.median(v)), "p90": float(np.quantile(v, 0.9)),
            "max": float(v.max()), "frac_within_5pct": float((v <= 0.05).mean()), "n": int(len(v))}


def evaluate(model: CostModel, heldout: Sequence[Dict[str, Any]], k: int = 3, seed: int = 0) -> Dict[str, Any]:
    """Top-k regret on passes whose every candidate was timed: take the k schedules
    the model ranks fastest, keep the measured best of those, compare with the
    measured best of all candidates. Baselines without the model: the default
    schedule alone, and k schedules picked at random."""
    rng = np.random.default_rng(seed)
    # the fixed schedule closest to the executor's default (64 x 8 tiles, 128 threads)
    default = {"tj": 8, "tk": 64, "threads": 128, "seg_len": 32}
    reg_model, reg_rand, reg_def, reg_top1, reg_an, n_cands = [], [], [], [], [], []
    for key, rs in group_by_pass(heldout).items():
        if len(rs) < 8:
            continue
        X, _ = records_to_xy(rs)
        pred = model.predict(X).numpy()
        ms = np.array([r["ms"] for r in rs])
        best = ms.min()
        order = np.argsort(pred)
        n_cands.append(len(rs))
        reg_model.append(ms[order[:k]].min() / best - 1.0)
        reg_top1.append(ms[order[0]] / best - 1.0)
        reg_rand.append(ms[rng.choice(len(rs), size=min(k, len(rs)), replace=False)].min() / best - 1.0)
        an = np.array([analytic_cost(r["features"], r["schedule"]) for r in rs])
        reg_an.append(ms[np.argsort(an, kind="stable")[:k]].min() / best - 1.0)
        d = [r["ms"] for r in rs if all(r["cfg"].get(a) == default[a] for a in default)
             and r["cfg"].get("ghost", True) and r["cfg"].get("kv", 1) == 1]
        if d:
            reg_def.append(d[0] / best - 1.0)
    mean_c = float(np.mean(n_cands)) if n_cands else 0.0
    return {"top_k": k, "passes": len(reg_model), "candidates_per_pass": mean_c,
            "model_topk": _stats(reg_model), "model_top1": _stats(reg_top1),
            "random_topk": _stats(reg_rand), "analytic_topk": _stats(reg_an),
            "default_schedule": _stats(reg_def),
            "timing_runs_saved_frac": (1.0 - k / mean_c) if mean_c else None}


DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "costmodel_b200.npz")


def load_default(device: Any = "cuda") -> "Ensemble":
    """The ensemble trained on B200 autotuner timings of random DAGs (shipped with
    the package): ``autotune.tune_plan(plan, values, dev, chooser=chooser(load_default()))``
    then times only its top candidates."""
    return Ensemble.load(DEFAULT_MODEL, device)


def chooser(model: CostModel, k: int = 3):
    """``autotune.tune_plan(chooser=...)`` hook: keep the model's top-k candidates."""
    from . import autotune as AT

    def pick(pp, cands, shape):
        feats = AT.features(pp.spec, shape)
        X = torch.tensor([vectorize(feats, AT.schedule_features(pp.spec, c)) for c in cands], dtype=torch.float32)
        order = np.argsort(model.predict(X).numpy())
        return [cands[i] for i in order[:k]]
    return pick


# ------------------------------------------------------------------ random DAG workload
_UNARY = ["exp", "log", "sqrt", "sin", "cos", "tanh", "abs", "neg"]
_BINARY = ["add", "sub", "mul", "div"]


def random_dag(rng: np.random.Generator):
    """A random expression DAG of 3-20 ops; returns ``(graph, wanted, shape, dtype)``.
    Field leaves hold placeholders ``("field", shape, dtype, components)``; see
    ``materialize`` / ``placeholder_graph``."""
    from .graph import Graph
    shape = tuple(int(rng.integers(2, 17)) * 32 for _ in range(3))
    dtype = torch.float32 if rng.random() < 0.5 else torch.bfloat16
    boundary = "periodic" if rng.random() < 0.5 else "neumann"
    g = Graph()
    fields = {"f": g.add("_constant", (), {"value": ("field", shape, dtype, 1)})}
    if rng.random() < 0.5:
        fields["g"] = g.add("_constant", (), {"value": ("field", shape, dtype, 1)})
    if rng.random() < 0.35:
        fields["u"] = g.add("_constant", (), {"value": ("field", shape, dtype, 3)})
    scal = [(nid, 0) for k, nid in fields.items() if k != "u"]     # (node, stencil reach)
    vec = [(fields["u"], 0)] if "u" in fields else []
    st = {"dx": 1.0, "boundary": boundary}
    for _ in range(int(rng.integers(3, 21))):
        r = rng.random()
        a, ra = scal[int(rng.integers(len(scal)))]
        if r < 0.3:
            scal.append((g.add(_UNARY[int(rng.integers(len(_UNARY)))], (a,), {}), ra))
        elif r < 0.55:
            b, rb = scal[int(rng.integers(len(scal)))]
            scal.append((g.add(_BINARY[int(rng.integers(len(_BINARY)))], (a, b), {}), max(ra, rb)))
        elif r < 0.68 and ra <= 1:
            scal.append((g.add("laplacian", (a,), dict(st)), ra + 1))
        elif r < 0.76 and ra <= 1:
            scal.append((g.add("grad_mag", (a,), dict(st)), ra + 1))
        elif r < 0.82 and ra <= 1:
            vec.append((g.add("gradient", (a,), dict(st)), ra + 1))
        elif r < 0.86 and ra == 0:
            h = g.add("hessian", (a,), dict(st))
            if rng.random() < 0.5:
                scal.append((g.add("trace", (h,), {}), 2))
            else:
                ev = g.add("eigenvalues", (h,), {})
                scal.append((g.add("select_component", (ev,), {"index": int(rng.integers(3))}), 2))
        elif r < 0.9 and ra == 0:
            scal.append((g.add("mean_curvature", (a,), dict(st)), 2))
        elif vec:
            v, rv = vec[int(rng.integers(len(vec)))]
            if rng.random() < 0.5 and rv <= 1:
                scal.append((g.add("divergence", (v,), dict(st)), rv + 1))
            elif rv <= 1:
                vec.append((g.add("curl", (v,), dict(st)), rv + 1))
            else:
                scal.append((g.add("select_component", (v,), {"index": int(rng.integers(3))}), rv))
        else:
            scal.append((g.add("sin", (a,), {}), ra))
    out = scal[-1][0]
    for extra, _ in scal[-3:-1]:
        out = g.add("add", (out, extra), {})
    wanted = [out]
    if rng.random() < 0.3:
        wanted.append(g.add(["sum", "mean", "variance"][int(rng.integers(3))], (out,), {}))
    return g, wanted, shape, dtype


def materialize(g, device, seed: int = 0):
    """Replace placeholder leaves by seeded fields on ``device``."""
    from .synth import sinusoid_field, smoothed_vector
    for nid in list(g._order):
        v = g._nodes[nid].params.get("value")
        if isinstance(v, tuple) and v and v[0] == "field":
            _, shape, dtype, nc = v
            seed += 1
            t = (sinusoid_field(shape, seed=seed, device=device) if nc == 1
                 else smoothed_vector(shape, seed=seed, device=device)).to(dtype)
            g = g.clone_with_replacement(nid, t)
    return g


def placeholder_graph(g):
    """The graph with storage-free CPU tensors of the right shape and dtype in place
    of the placeholders (enough to plan and compile without device memory)."""
    for nid in list(g._order):
        v = g._nodes[nid].params.get("value")
        if isinstance(v, tuple) and v and v[0] == "field":
            _, shape, dtype, nc = v
            full = tuple(shape) + ((3,) if nc == 3 else ())
            g = g.clone_with_replacement(nid, torch.zeros(1, dtype=dtype).expand(*full))
    return g


def _compile_worker(src: str) -> int:
    from . import fused_compiler as FC
    N.compile_cached(src, FC.NVRTC_OPTS)
    return 1

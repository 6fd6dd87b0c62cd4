"""Kernel sources the GPU tests compile, enumerated on the CPU (no device needed),
so that a build step can fill the kernel cache before the tests run.

Each entry mirrors a graph a GPU test runs; planning uses stride-0 placeholders of
the test's shapes and dtypes. ``python tests/kernel_sources.py`` compiles them."""
import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def _ph(t_or_shape, dtype=torch.float32):
    shape = tuple(t_or_shape.shape) if isinstance(t_or_shape, torch.Tensor) else tuple(t_or_shape)
    dtype = t_or_shape.dtype if isinstance(t_or_shape, torch.Tensor) else dtype
    return torch.zeros(1, dtype=dtype).expand(*shape)


def eager_sources(g, S, O):
    """Sources of a node-by-node run: each node as a one-node graph on inputs of the
    shapes its producers give (values from the oracle)."""
    from stenpy_b200.prewarm import plan_sources
    src, vals = [], {}
    for node in g.topological_sort():
        if node.op_name == "_constant":
            vals[node.id] = node.params["value"]
            continue
        g1 = S.Graph()
        ids = [g1.add("_constant", (), {"value": vals[i] if (not isinstance(vals[i], torch.Tensor) or vals[i].ndim == 0)
                                        else _ph(vals[i].shape, torch.float32)})
               for i in node.input_ids]
        nid = g1.add(node.op_name, ids, node.params)
        src += plan_sources(g1, [nid])
        vals[node.id] = O.evaluate(g1, [nid])[nid]
    return src


def all_sources():
    import stenpy_b200 as S
    from stenpy_b200 import batch as B
    from stenpy_b200.codegen import PassConfig, emit_batch_module
    from stenpy_b200.prewarm import plan_sources
    from stenpy_b200.synth import BATCH_EXPRESSIONS, batch_specs
    from golden_cases import load_cases
    from oracle import stenpy_oracle as O

    src = []
    cases = load_cases()
    from stenpy_b200.registry import KNOWN_OPS
    for c in cases:       # fused parity against the goldens (graphs with FFT nodes compile at run time)
        g, sink, *_ = S.compile_expression(c["expr"], dx=c["dx"], boundary=c["boundary"],
                                           field_map={k: _ph(v) for k, v in c["inputs"].items()})
        if all(n.op_name in KNOWN_OPS for n in g.topological_sort()):
            src += plan_sources(g, [sink])
    for c in cases[:6]:   # eager mode: one kernel per node on the node's own inputs
        g, sink, *_ = S.compile_expression(c["expr"], dx=c["dx"], boundary=c["boundary"], field_map=c["inputs"])
        src += eager_sources(g, S, O)
    for shape in [(5, 7, 33), (3, 3, 3), (17, 9, 130), (2, 40, 64)]:   # ragged shapes
        for b in ["periodic", "neumann", "dirichlet"]:
            exprs = ["laplacian(f) + tanh(g)*exp(f)", "gradient(f)"]
            if min(shape) >= 3:
                exprs += ["_hessian(f)", "mean_curvature(g*g + 1)", "trace(_hessian(f)) + tanh(g)"]
            for e in exprs:
                g, sink, *_ = S.compile_expression(e, boundary=b, field_map={"f": _ph(shape), "g": _ph(shape)})
                src += plan_sources(g, [sink])
    g, sink, *_ = S.compile_expression("f**2 + tanh(f)*exp(f) + laplacian(g)", boundary="periodic",
                                       field_map={"f": _ph((128,) * 3), "g": _ph((128,) * 3)})
    src += plan_sources(g, [sink])
    g, sink, *_ = S.compile_expression("f**2 + tanh(f)*exp(f) + laplacian(g)", boundary="periodic",
                                       field_map={"f": _ph((24, 20, 64)), "g": _ph((24, 20, 64))})
    src += plan_sources(g, [sink, g.add("variance", (sink,), {})])     # smoke()
    g, sink, *_ = S.compile_expression("divergence(gradient(f)) + l2norm(curl(u))", boundary="periodic",
                                       field_map={"f": _ph((40, 48, 64)), "u": _ph((40, 48, 64, 3))})
    src += plan_sources(g, [sink] + [g.add(r, (sink,), {}) for r in ("sum", "mean", "variance")])  # no-alloc
    from stenpy_b200.synth import sinusoid_field   # node-by-node fallback (two grids)
    g, sinks, *_ = S.compile_expressions({"a": "laplacian(f)", "b": "laplacian(g) * 2"}, boundary="periodic",
                                         field_map={"f": sinusoid_field((8, 9, 16), seed=1).double(),
                                                    "g": sinusoid_field((10, 12, 16), seed=2).double()})
    src += eager_sources(g, S, O)
    g, sink, *_ = S.compile_expression("laplacian(f) * tanh(f)", boundary="periodic",   # cost-model chooser
                                       field_map={"f": _ph((64, 96, 128))})
    src += plan_sources(g, [sink])
    for shape in [(10, 17, 65), (9, 33, 97), (12, 18, 66)]:     # second-derivative ghosts
        for tk, tj in ((32, 16), (64, 8)):
            g, sink, *_ = S.compile_expression("trace(_hessian(f))", boundary="neumann", field_map={"f": _ph(shape)})
            src += plan_sources(g, [sink], torch.float32, PassConfig(tj=tj, tk=tk, threads=128, seg_len=8))
    expr = "divergence(gradient(f)) + l2norm(curl(u)) + laplacian(f)*tanh(f)"
    for dt in (torch.float32, torch.float16, torch.bfloat16):   # KV chunk parity
        for bnd in ("periodic", "neumann"):
            for shape in [(20, 33, 130), (9, 16, 64), (7, 5, 45)]:
                for kv, tk, tj in ((1, 64, 8), (2, 64, 16), (4, 64, 32), (2, 32, 8), (8, 64, 16), (8, 128, 8)):
                    g, sink, *_ = S.compile_expression(expr, boundary=bnd, field_map={
                        "f": _ph(shape, dt), "u": _ph(shape + (3,), dt)})
                    w = [sink, g.add("variance", (sink,), {})]
                    src += plan_sources(g, w, dt, PassConfig(tj=tj, tk=tk, threads=128, seg_len=8, kv=kv))
    for bnd in ("periodic", "neumann"):   # lazy mode
        g, sinks, *_ = S.compile_expressions({"eig": "eigenvalues(hessian(f))", "mc": "mean_curvature(f)",
                                              "lap": "laplacian(f)*2 + exp(f)"}, boundary=bnd,
                                             field_map={"f": _ph((37, 24, 64))})
        m = g.add("mean", (sinks["mc"],), {})
        src += plan_sources(g, list(sinks.values()) + [m])
    g, sinks, *_ = S.compile_expressions({"eig": "eigenvalues(hessian(f))", "mc": "mean_curvature(f)"},
                                         boundary="periodic", field_map={"f": _ph((96, 64, 64))})
    m = g.add("mean", (sinks["mc"],), {})
    src += plan_sources(g, list(sinks.values()) + [m], torch.bfloat16)
    for dt in (torch.float32, torch.bfloat16):   # entropy histograms
        exprs = {"e": "entropy_hist(f)", "e64": "entropy_hist(f, bins=64)", "el": "entropy_hist(laplacian(f))"}
        g, sinks, *_ = S.compile_expressions(exprs, boundary="neumann", field_map={"f": _ph((33, 20, 45), dt)})
        src += plan_sources(g, list(sinks.values()))
        g, sink, *_ = S.compile_expression("entropy_hist(f)", field_map={"f": _ph((8, 9, 16), dt)})
        src += plan_sources(g, [sink])
    for dt in (torch.float16, torch.bfloat16):   # 16-bit fields, one-sided edges, FP32 results
        for shape in [(12, 20, 64), (9, 17, 37)]:
            for e in ("curl(u)", "gradient(f) * 2", "_hessian(f)", "divergence(u) + laplacian(f)"):
                for ghost in (True, False):
                    g, sink, *_ = S.compile_expression(e, boundary="neumann", field_map={
                        "f": _ph(shape, dt), "u": _ph(shape + (3,), dt)})
                    src += plan_sources(g, [sink], torch.float32, PassConfig(ghost=ghost))
    # smoothing / advection stencils
    S4 = [(5, 7, 33), (17, 9, 130), (9, 33, 97), (3, 3, 3)]
    for shape in S4:
        for w in (3, 5):
            for b in ("neumann", "periodic", "dirichlet", "reflect"):
                g, sink, *_ = S.compile_expression(f"moving_average(f, window={w}, boundary='{b}')",
                                                   boundary="periodic", field_map={"f": _ph(shape)})
                src += plan_sources(g, [sink])
        for dt in (torch.float32, torch.bfloat16):
            g, sink, *_ = S.compile_expression("conv3d_spectral(f)", boundary="periodic",
                                               field_map={"f": _ph(shape, dt)})
            src += plan_sources(g, [sink]) + plan_sources(g, [sink], torch.bfloat16)
    for shape in S4 + [(2, 40, 64)]:
        for b in ("neumann", "periodic"):
            for e in ("material_derivative(f, u)", "material_derivative(f*f, curl(u)) + f")[:1 + (min(shape) >= 3)]:
                g, sink, *_ = S.compile_expression(e, boundary=b, field_map={"f": _ph(shape),
                                                                             "u": _ph(shape + (3,))})
                src += plan_sources(g, [sink])
    for shape in [(20, 33, 130), (7, 12, 45)]:
        for e in ("moving_average(laplacian(f)) + conv3d_spectral(g)*2",
                  "laplacian(moving_average(f, window=3, boundary='periodic'))",
                  "conv3d_spectral(tanh(f)) - moving_average(g, window=5, boundary='reflect')"):
            for kv, tk, tj in ((1, 64, 8), (2, 64, 16), (4, 64, 32), (2, 32, 8)):
                g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": _ph(shape), "g": _ph(shape)})
                src += plan_sources(g, [sink], torch.float32, PassConfig(tj=tj, tk=tk, threads=128, seg_len=8, kv=kv))
    g, sinks, *_ = S.compile_expressions({"a": "sum(f + 2)", "b": "sum(conv3d_spectral(f + 2))",
                                          "c": "sum(moving_average(f + 2, window=3, boundary='periodic'))"},
                                         boundary="periodic", field_map={"f": _ph((256,) * 3)})
    src += plan_sources(g, list(sinks.values()))
    for e in ("conv3d_spectral(f)", "moving_average(f, window=5)", "moving_average(f, boundary='periodic')"):
        for shape in ((33, 21, 45), (40, 24, 80), (37, 24, 64)):
            g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": _ph(shape)})
            src += plan_sources(g, [sink])
    for dt in (torch.float32, torch.bfloat16):   # 2-D surface normals
        for shape in [(3, 3), (5, 33), (40, 130), (64, 64), (37, 128)]:
            for e, bnd in (("surface_normals(f)", "neumann"), ("surface_normals(f*f) * 2 + mean(f)", "periodic"),
                           ("variance(tanh(f))", "periodic")):
                g, sink, *_ = S.compile_expression(e, boundary=bnd, field_map={"f": _ph(shape, dt)})
                src += plan_sources(g, [sink])
    for dt in (torch.float32, torch.bfloat16):   # entropy bins at edges / with offsets, and their batch
        ejobs = []
        for expr in ("entropy_hist(f)", "entropy_hist(f, bins=64)", "entropy_hist(f*f)"):
            g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": _ph((17, 24, 40), dt)})
            src += plan_sources(g, [sink])
            ejobs.append(B.BatchJob(g, [sink]))
        cfg = B.batch_candidates(128)[0]
        ps, seen = [], set()
        for j in ejobs * 3:
            for pp in B.plan_job(j, cfg).passes:
                k = B.program_key(pp.spec)
                if k not in seen:
                    seen.add(k)
                    ps.append(pp.spec)
        src.append(emit_batch_module(ps, 128, B.batch_min_blocks(128)))
    for dt in (torch.float32, torch.bfloat16):     # covariance / correlation
        for shape in [(17, 9, 130), (40, 33, 64), (3, 3, 3)]:
            exprs = {"c": "covariance(f, g)", "r": "correlation(f, g)", "rr": "correlation(f, f)",
                     "cl": "covariance(laplacian(g), f)"}
            g, sinks, *_ = S.compile_expressions(exprs, boundary="periodic",
                                                 field_map={"f": _ph(shape, dt), "g": _ph(shape, dt)})
            src += plan_sources(g, list(sinks.values()))
    from stenpy_b200.geometry import edt_source   # distance transform (per dtype and longest line)
    for dt in (torch.float32, torch.float64, torch.bfloat16, torch.float16):
        src += [edt_source(dt, nmax) for nmax in (16, 32, 64)]
    src.append(edt_source(torch.float32, 256))
    # batched executor: per-job runtime plans and the batch modules of the tests
    import test_gpu_batch as TB
    smooth = [(e, torch.float32, [(33, 21, 45), (40, 24, 80)][i % 2], 0) for i, e in
              enumerate(["conv3d_spectral(f)", "moving_average(f, window=5)",
                         "moving_average(f, boundary='periodic')"] * 2)]
    mixed2d = [("surface_normals(f)", torch.float32, (40, 130), 0), ("conv3d_spectral(f)", torch.float32, (20, 24, 80), 0),
               ("surface_normals(f)", torch.float32, (64, 64), 0), ("laplacian(f)", torch.float32, (19, 37, 50), 0)]
    for specs, threads in ((TB._mixed_specs(), 128), (TB._mixed_specs(), 256),
                           (batch_specs(48, seed=7, lo=32, hi=72), 128), (smooth, 128), (mixed2d, 128)):
        jobs = []
        for e, dt, shape, _ in specs:
            full = tuple(shape) + ((3,) if e.startswith("curl") else ())
            g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": _ph(full, dt)})
            jobs.append(B.BatchJob(g, [sink]))
            src += plan_sources(g, [sink], dt)
        cfg = B.batch_candidates(threads)[0]
        ps, seen = [], set()
        for j in jobs:
            for pp in B.plan_job(j, cfg).passes:
                k = B.program_key(pp.spec)
                if k not in seen:
                    seen.add(k)
                    ps.append(pp.spec)
        src.append(emit_batch_module(ps, threads, B.batch_min_blocks(threads)))
    return list(dict.fromkeys(src))


if __name__ == "__main__":
    from stenpy_b200.prewarm import compile_all
    s = all_sources()
    print(len(s), "sources;", compile_all(s), "compiled")

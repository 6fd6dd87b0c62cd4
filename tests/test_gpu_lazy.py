"""Lazy (out-of-core) mode: chunked runs from pinned host memory must reproduce the
whole-field run voxel for voxel (same arithmetic at every voxel: seam test), and
match the CPU FP64 oracle."""
import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
@pytest.mark.parametrize("chunk", [5, 7, 16])
def test_chunked_equals_whole_field(boundary, chunk):
    import stenpy_b200 as S
    from stenpy_b200.lazy import LazyPipeline
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    shape = (37, 24, 64)
    f = sinusoid_field(shape, seed=5)
    exprs = {"eig": "eigenvalues(hessian(f))", "mc": "mean_curvature(f)", "lap": "laplacian(f)*2 + exp(f)"}
    g, sinks, *_ = S.compile_expressions(exprs, boundary=boundary, field_map={"f": f.to(dev)})
    mean_id = g.add("mean", (sinks["mc"],), {})
    wanted = list(sinks.values()) + [mean_id]
    whole = S.Runtime(device=dev).run(g, wanted=wanted)
    gh, sinks_h, *_ = S.compile_expressions(exprs, boundary=boundary, field_map={"f": f.pin_memory()})
    mean_h = gh.add("mean", (sinks_h["mc"],), {})
    lp = LazyPipeline(gh, list(sinks_h.values()) + [mean_h], dev, chunk=chunk)
    res = lp.run()
    assert len(lp.passes[0]["chunks"]) == -(-shape[0] // max(chunk, 2 * lp.passes[0]["H"] + 1))
    for k in exprs:
        a = whole[sinks[k]].cpu()
        b = res[sinks_h[k]]
        assert torch.equal(a, b), (k, (a - b).abs().max().item())
    assert abs(float(whole[mean_id]) - float(res[mean_h])) <= 1e-12 * max(1.0, abs(float(whole[mean_id])))


def test_lazy_config2_shape_against_oracle():
    """Config-2 graph (eigenvalues of the hessian and mean curvature, BF16 outputs,
    FP32 compute, FP64 reductions) on a reduced grid with a budget forcing chunks."""
    import stenpy_b200 as S
    from stenpy_b200.lazy import LazyPipeline
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    shape = (96, 64, 64)
    f = sinusoid_field(shape, seed=0)
    exprs = {"eig": "eigenvalues(hessian(f))", "mc": "mean_curvature(f)"}
    g, sinks, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f.pin_memory()})
    mn = g.add("mean", (sinks["mc"],), {})
    budget = 12 * 64 * 64 * 4 * 6
    lp = LazyPipeline(g, list(sinks.values()) + [mn], dev, budget_bytes=budget + (256 << 20),
                      out_dtype=torch.bfloat16)
    res = lp.run()
    assert len(lp.passes[0]["chunks"]) > 1
    g2, sinks2, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f.double()})
    mn2 = g2.add("mean", (sinks2["mc"],), {})
    ref = O.evaluate(g2, list(sinks2.values()) + [mn2])
    # BF16 storage of the outputs: unit roundoff 2^-8 = 3.9e-3
    assert rel_err(res[sinks["eig"]], ref[sinks2["eig"]]) <= 4e-3
    assert rel_err(res[sinks["mc"]], ref[sinks2["mc"]]) <= 4e-3
    # the FP64 mean is formed from the FP32 values before BF16 rounding
    assert abs(float(res[mn]) - float(ref[mn2])) <= 1e-4 * max(1.0, abs(float(ref[mn2])))
    # FP32 results: the FP32 bound (eigenvalues of nearly equal pairs take the FP64 path)
    lp32 = LazyPipeline(g, list(sinks.values()) + [mn], dev, budget_bytes=budget + (256 << 20))
    r32 = lp32.run()
    assert rel_err(r32[sinks["eig"]], ref[sinks2["eig"]]) <= 1e-5
    assert rel_err(r32[sinks["mc"]], ref[sinks2["mc"]]) <= 1e-5


def test_captured_chunk_schedule_replays_bit_identically():
    """LazyPipeline.capture(): the whole chunk schedule (H2D copies, kernels, D2H
    copies, finalizes) as one CUDA graph. Replays give exactly the results of an
    eager enqueue, also after the pinned host input changes in place."""
    import stenpy_b200 as S
    from stenpy_b200.lazy import LazyPipeline
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    shape = (45, 32, 64)
    f = sinusoid_field(shape, seed=9).pin_memory()
    exprs = {"eig": "eigenvalues(hessian(f))", "mc": "mean_curvature(f)"}
    g, sinks, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f})
    mn = g.add("mean", (sinks["mc"],), {})
    wanted = list(sinks.values()) + [mn]
    lp = LazyPipeline(g, wanted, dev, chunk=8)
    eager = {k: (v.clone() if isinstance(v, torch.Tensor) else v) for k, v in lp.run().items()}
    assert len(lp.passes[0]["chunks"]) > 2
    graph = lp.capture()
    for k in sinks.values():                 # clear the host outputs before the replay
        lp.host_out[k].zero_()
    graph.replay()
    replayed = lp.results()
    for k in sinks.values():
        assert torch.equal(replayed[k], eager[k]), k
    assert float(replayed[mn]) == float(eager[mn])
    # new input values in the same pinned buffer: the replay reads them
    f.mul_(0.5).add_(0.25)
    graph.replay()
    again = {k: (v.clone() if isinstance(v, torch.Tensor) else v) for k, v in lp.results().items()}
    g2, sinks2, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f.to(dev)})
    mn2 = g2.add("mean", (sinks2["mc"],), {})
    ref = S.Runtime(device=dev).run(g2, wanted=list(sinks2.values()) + [mn2])
    for k in exprs:
        assert torch.equal(again[sinks[k]], ref[sinks2[k]].cpu()), k
    assert abs(float(again[mn]) - float(ref[mn2])) <= 1e-12 * max(1.0, abs(float(ref[mn2])))
    del graph


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_streamed_config1_step_equals_whole_field(dtype):
    """The end-to-end benchmark's streamed step: the two-phase config-1 graph (curl
    norm, then Laplacian + that scalar with sum/mean/variance) run chunk by chunk from
    pinned host fields gives the whole-field results: the same voxels up to one
    rounding of the output dtype (the scalar added is the same FP64 sum up to the
    order of its partial rows) and the same statistics to FP32 rounding of the plane
    sums (a thread's variance pivot is its first voxel, which a chunk moves)."""
    import stenpy_b200 as S
    from stenpy_b200.lazy import LazyPipeline
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    shape = (40, 24, 64)
    f = sinusoid_field(shape, seed=31).to(dtype)
    u = smoothed_vector(shape, seed=32).to(dtype)
    expr = "divergence(gradient(f)) + l2norm(curl(u))"
    g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev), "u": u.to(dev)})
    w = [sink] + [g.add(r, (sink,), {}) for r in ("sum", "mean", "variance")]
    whole = S.Runtime(device=dev, out_dtype=dtype).run(g, wanted=w)
    gh, sinkh, *_ = S.compile_expression(expr, boundary="periodic",
                                         field_map={"f": f.pin_memory(), "u": u.pin_memory()})
    wh = [sinkh] + [gh.add(r, (sinkh,), {}) for r in ("sum", "mean", "variance")]
    lp = LazyPipeline(gh, wh, dev, out_dtype=dtype, chunk=8)
    res = lp.run()
    assert len(lp.passes[0]["chunks"]) == 5
    a, b = whole[sink].cpu().float(), res[sinkh].float()
    tol = 1e-6 if dtype == torch.float32 else 1e-3
    assert (a - b).abs().max().item() <= tol * a.abs().max().item()
    for x, y in zip(w[1:], wh[1:]):
        assert abs(float(whole[x]) - float(res[y])) <= 1e-6 * max(1e-6, abs(float(whole[x]))), (x, y)

"""Batched persistent executor: one launch over many graphs of uneven shapes and
mixed storage dtypes must give, per job, exactly what ``Runtime.run`` gives for
that graph alone (bit-identical per-voxel outputs: same generated arithmetic;
reductions to FP64 rounding), match the CPU FP64 oracle, and leave its work queue
reset so a replay (also from a CUDA graph) reproduces the results."""
import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu

# per-expression bound of the norm-wise relative error of FP32-stored results vs
# the FP64 oracle; BF16-stored outputs add the BF16 unit roundoff 2^-9
TOL32 = {}
TOL_BF16_OUT = 8e-3


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _jobs(specs, dev):
    import stenpy_b200 as S
    from stenpy_b200.batch import BatchJob
    from stenpy_b200.synth import batch_field
    jobs, host = [], []
    for expr, dt, shape, seed in specs:
        f = batch_field(expr, dt, shape, seed)
        g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev)})
        jobs.append(BatchJob(g, [sink]))
        host.append((expr, f, sink))
    return jobs, host


def _mixed_specs():
    """All eight expressions x {FP32, BF16} x {rows TMA-aligned, ragged}."""
    from stenpy_b200.synth import BATCH_EXPRESSIONS
    specs = []
    shapes = {torch.float32: [(36, 40, 64), (33, 21, 45)], torch.bfloat16: [(40, 24, 80), (19, 37, 50)]}
    seed = 0
    for e in BATCH_EXPRESSIONS:
        for dt, shs in shapes.items():
            for sh in shs:
                specs.append((e, dt, sh, seed))
                seed += 1
    return specs


@pytest.mark.parametrize("threads", [128, 256])
def test_batch_equals_runtime_per_job(threads):
    import stenpy_b200 as S
    from stenpy_b200 import batch as B
    dev = _dev()
    jobs, host = _jobs(_mixed_specs(), dev)
    prog = B.build(jobs, dev, threads=threads)
    stream = torch.cuda.current_stream(dev)
    prog.enqueue(stream)
    stream.synchronize()
    prog.check()
    got = prog.collect()
    assert prog.n_ctas <= prog.mod.sm_count * prog.mod.blocks_per_sm
    for job, res in zip(jobs, got):
        ref = S.Runtime(device=dev, out_dtype=job.out_dtype).run(job.graph, wanted=job.wanted)
        for nid in job.wanted:
            a, b = res[nid], ref[nid]
            if a.ndim == 0:
                assert abs(float(a) - float(b)) <= 1e-12 * max(1.0, abs(float(b))), (nid, float(a), float(b))
            else:
                assert a.dtype == b.dtype and torch.equal(a, b), (job.graph._nodes[nid].op_name,
                                                                  (a.float() - b.float()).abs().max().item())


def test_batch_matches_oracle_and_replays():
    from stenpy_b200 import batch as B
    dev = _dev()
    jobs, host = _jobs(_mixed_specs(), dev)
    prog = B.build(jobs, dev)
    stream = torch.cuda.current_stream(dev)
    prog.enqueue(stream)
    stream.synchronize()
    prog.check()
    first = [{k: v.clone() for k, v in r.items()} for r in prog.collect()]
    for (expr, f, sink), res in zip(host, first):
        import stenpy_b200 as S
        g2, s2, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.double()})
        ref = O.evaluate(g2, [s2])[s2]
        got = res[sink]
        if got.ndim == 0:
            # entropy: the bins are formed in FP64 from the stored values, as the oracle does
            assert abs(float(got) - float(ref)) <= 1e-10 * max(1.0, abs(float(ref))), (expr, float(got), float(ref))
        else:
            tol = TOL_BF16_OUT if got.dtype == torch.bfloat16 else TOL32.get(expr, 1e-5)
            assert rel_err(got, ref) <= tol, (expr, f.dtype, tuple(f.shape), rel_err(got, ref))
    # a second launch and a CUDA-graph replay reproduce the first run exactly
    prog.enqueue(stream)
    stream.synchronize()
    prog.check()
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        graph.capture_begin()
        prog.enqueue(side)
        graph.capture_end()
    stream.wait_stream(side)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize(dev)
    prog.check()
    for a, b in zip(first, prog.collect()):
        for k in a:
            assert torch.equal(a[k], b[k]), k


def test_batch_config3_shape_small():
    """The batched workload's mix at reduced size: 48 fields, dims in [32, 72]."""
    from stenpy_b200 import batch as B
    from stenpy_b200.synth import batch_specs
    dev = _dev()
    specs = batch_specs(48, seed=7, lo=32, hi=72)
    jobs, host = _jobs(specs, dev)
    got = B.run_batch(jobs, dev)
    import stenpy_b200 as S
    for (expr, f, sink), res in zip(host, got):
        g2, s2, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.double()})
        ref = O.evaluate(g2, [s2])[s2]
        r = res[sink]
        if r.ndim == 0:
            assert abs(float(r) - float(ref)) <= 1e-10 * max(1.0, abs(float(ref))), expr
        else:
            tol = TOL_BF16_OUT if r.dtype == torch.bfloat16 else TOL32.get(expr, 1e-5)
            assert rel_err(r, ref) <= tol, (expr, tuple(f.shape), rel_err(r, ref))


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_entropy_hist_runtime_against_oracle(dtype):
    """Standalone Runtime path of entropy_hist: min/max pass, histogram pass, entropy."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    f = sinusoid_field((33, 20, 45), seed=3).to(dtype)
    exprs = {"e": "entropy_hist(f)", "e64": "entropy_hist(f, bins=64)", "el": "entropy_hist(laplacian(f))"}
    g, sinks, *_ = S.compile_expressions(exprs, boundary="neumann", field_map={"f": f.to(dev)})
    res = S.Runtime(device=dev).run(g, wanted=list(sinks.values()))
    g2, sinks2, *_ = S.compile_expressions(exprs, boundary="neumann", field_map={"f": f.double()})
    ref = O.evaluate(g2, list(sinks2.values()))
    for k in exprs:
        a, b = float(res[sinks[k]]), float(ref[sinks2[k]])
        # exact bins for a stored field; FP32 laplacian values may cross a bin edge
        tol = 1e-10 if k != "el" else 1e-3
        assert abs(a - b) <= tol * max(1.0, abs(b)), (k, a, b)
    # constant field: entropy 0 (empty range)
    c = torch.full((8, 9, 16), 2.5, device=dev, dtype=dtype)
    gc, sc, *_ = S.compile_expression("entropy_hist(f)", field_map={"f": c})
    assert float(S.Runtime(device=dev).run(gc)[sc]) == 0.0


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_entropy_hist_bins_at_edges_and_with_offsets(dtype):
    """Binning must equal the oracle's FP64 floor exactly: values on bin edges
    (i/256 patterns, where the FP32 shortcut must defer to FP64), values with a large
    offset relative to their range (the shortcut is disabled), and both in one batch."""
    import stenpy_b200 as S
    from stenpy_b200 import batch as B
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    shape = (17, 24, 40)
    i = torch.arange(shape[0] * shape[1] * shape[2], dtype=torch.float64).reshape(shape)
    fields = {"edges": ((i % 257) / 256.0).to(dtype),
              "offset": (sinusoid_field(shape, seed=8).double() * 0.01 + 1000.0).to(dtype),
              "smooth": sinusoid_field(shape, seed=9).to(dtype)}
    jobs, host = [], []
    for name, f in fields.items():
        for expr in ("entropy_hist(f)", "entropy_hist(f, bins=64)", "entropy_hist(f*f)"):
            g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev)})
            got = float(S.Runtime(device=dev).run(g)[sink])
            # the kernel bins the FP32 product: the oracle bins the same rounded values
            fo = (f.double() * f.double()).float().double() if "f*f" in expr else f.double()
            g2, s2, *_ = S.compile_expression(expr.replace("f*f", "f"), boundary="periodic", field_map={"f": fo})
            ref = float(O.evaluate(g2, [s2])[s2])
            assert abs(got - ref) <= 1e-10 * max(1.0, abs(ref)), (name, expr, got, ref)
            jobs.append(B.BatchJob(g, [sink]))
            host.append((name, expr, sink, ref))
    for (name, expr, sink, ref), res in zip(host, B.run_batch(jobs, dev)):
        assert abs(float(res[sink]) - ref) <= 1e-10 * max(1.0, abs(ref)), (name, expr, float(res[sink]), ref)

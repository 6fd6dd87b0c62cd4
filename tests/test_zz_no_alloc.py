"""The allocation-free pass entry point (stenpy_pass_noalloc) against the regular one.

Callers that cannot allocate device memory (a host that owns a fixed arena and
forbids further cudaMalloc, or a latency-critical loop where cudaMalloc would
synchronise the device) run a fused reduction pass through stenpy_pass_noalloc,
which keeps the FP64 partials in a static device array inside the library. This
test runs the config-1 graph (laplacian + ||curl u|| with sum / mean / variance)
through the regular path (caller-allocated partials: stenpy_launch +
stenpy_finalize), then twice in a row through the C ABI's no-alloc entry point,
and compares the reduction results and the output field (tolerance 1e-12
relative; the same kernels fold the same partials in the same order).
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_noalloc_pass_matches_regular_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import stenpy_b200 as S
    from stenpy_b200 import _native as N
    from stenpy_b200 import fused_compiler as FC
    from stenpy_b200.codegen import param_layout
    from stenpy_b200.synth import sinusoid_field, smoothed_vector

    dev = torch.device("cuda", 0)
    shape = (40, 48, 64)
    f = sinusoid_field(shape, seed=3).to(dev)
    u = smoothed_vector(shape, seed=4).to(dev)
    g, sink, *_ = S.compile_expression("divergence(gradient(f)) + l2norm(curl(u))", boundary="periodic",
                                       field_map={"f": f, "u": u})
    wanted = [sink] + [g.add(r, (sink,), {}) for r in ("sum", "mean", "variance")]
    plan = FC.get_plan(g, wanted)
    values, back = FC.bind(plan, g, wanted)
    prog = FC.build_program(plan, values, dev)
    stream = torch.cuda.current_stream(dev)

    # regular entry points: caller-allocated partials
    FC.enqueue(prog, stream)
    torch.cuda.synchronize()
    table_regular = prog.table.clone()
    out_node = [k for k, v in prog.results.items() if isinstance(v, torch.Tensor) and v.ndim == 3][0]
    field_regular = prog.results[out_node].clone()

    # the same passes through stenpy_pass_noalloc (scalars written to the same table)
    ops = prog.ops
    calls = []
    i = 0
    for pi, pp in enumerate(plan.passes):
        launches = []
        while i < len(ops) and isinstance(ops[i], FC.Launch):
            launches.append(ops[i])
            i += 1
        fin = ops[i]
        i += 1
        assert isinstance(fin, FC.Finalize)
        off = param_layout(pp.spec).offsets["part"]
        calls.append(([(L.module, L.grid, L.block, L.smem, L.params, off) for L in launches],
                      fin.ncta, fin.nslots, fin.descs))
    for attempt in range(2):
        prog.table.zero_()
        prog.results[out_node].zero_()
        if prog.const_host is not None:
            prog.table.copy_(prog.const_host)
        for launches, ncta, nslots, descs in calls:
            assert ncta * nslots <= N.NOALLOC_MAX_PARTIALS
            N.pass_noalloc(launches, ncta, nslots, descs, prog.table.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        FC.ErrorFlag.check(dev)
        for nid, (_, idx, n) in ((k, v) for k, v in prog.results.items() if isinstance(v, tuple)):
            a = table_regular[idx:idx + n].double()
            b = prog.table[idx:idx + n].double()
            assert torch.allclose(b, a, rtol=1e-12, atol=0.0), (attempt, nid, a.tolist(), b.tolist())
        assert torch.equal(prog.results[out_node], field_regular), attempt


def test_noalloc_rejects_oversized_request():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from stenpy_b200 import _native as N
    table = torch.zeros(4, dtype=torch.float64, device="cuda")
    d = N.ReduceDesc(N.RED_SUM, 0, 0, 0, 1.0, 0.0)
    with pytest.raises(N.NativeError, match="static scratch"):
        N.pass_noalloc([(0, (1, 1, 1), (32, 1, 1), 0, bytes(64), 0)], N.NOALLOC_MAX_PARTIALS + 1, 1, [d],
                       table.data_ptr(), torch.cuda.current_stream().cuda_stream)

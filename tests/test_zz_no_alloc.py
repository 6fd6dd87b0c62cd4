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


def _split_by_pass(plan, prog):
    """The program's ops grouped per pass: (main + shell launches, finalize or None,
    trailing launches such as the histogram-entropy kernel), then the launches
    after the last pass (the scalar kernel)."""
    from stenpy_b200 import fused_compiler as FC
    ops, i, groups = prog.ops, 0, []
    for pp in plan.passes:
        launches = [ops[i]]
        i += 1
        if pp.shell_module is not None and i < len(ops) and isinstance(ops[i], FC.Launch) \
                and ops[i].module == pp.shell_module:
            launches.append(ops[i])
            i += 1
        fin = None
        if pp.reductions:
            fin = ops[i]
            assert isinstance(fin, FC.Finalize)
            i += 1
        after = []
        if pp.hists:
            assert ops[i].module == pp.hist_module
            after.append(ops[i])
            i += 1
        groups.append((pp, launches, fin, after))
    return groups, ops[i:]


def _run_noalloc_twice(expr, reds, shape, seeds):
    import stenpy_b200 as S
    from stenpy_b200 import _native as N
    from stenpy_b200 import fused_compiler as FC
    from stenpy_b200.codegen import param_layout
    from stenpy_b200.synth import sinusoid_field, smoothed_vector

    dev = torch.device("cuda", 0)
    f = sinusoid_field(shape, seed=seeds[0]).to(dev)
    u = smoothed_vector(shape, seed=seeds[1]).to(dev)
    g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f, "u": u})
    wanted = [sink] + [g.add(r, (sink,), {}) for r in reds]
    plan = FC.get_plan(g, wanted)
    values, back = FC.bind(plan, g, wanted)
    prog = FC.build_program(plan, values, dev)
    stream = torch.cuda.current_stream(dev)

    # regular entry points: caller-allocated partials
    FC.enqueue(prog, stream)
    torch.cuda.synchronize()
    table_regular = prog.table.clone()
    out_nodes = [k for k, v in prog.results.items() if isinstance(v, torch.Tensor) and v.ndim == 3]
    fields_regular = {k: prog.results[k].clone() for k in out_nodes}

    groups, tail = _split_by_pass(plan, prog)
    s = stream.cuda_stream
    for attempt in range(2):
        prog.table.zero_()
        for k in out_nodes:
            prog.results[k].zero_()
        if prog.const_host is not None:
            prog.table.copy_(prog.const_host)
        for pp, launches, fin, after in groups:
            lay = param_layout(pp.spec).offsets
            if fin is None:
                for L in launches:
                    N.launch(L.module, L.grid, L.block, L.smem, s, L.params)
            else:
                assert fin.ncta * fin.nslots <= N.NOALLOC_MAX_PARTIALS
                N.pass_noalloc([(L.module, L.grid, L.block, L.smem, L.params, lay["part"], lay["cta_off"])
                                for L in launches], fin.ncta, fin.nslots, fin.descs, prog.table.data_ptr(), s)
            for L in after:
                N.launch(L.module, L.grid, L.block, L.smem, s, L.params)
        for L in tail:
            N.launch(L.module, L.grid, L.block, L.smem, s, L.params)
        torch.cuda.synchronize()
        FC.ErrorFlag.check(dev)
        for nid, (_, idx, n) in ((k, v) for k, v in prog.results.items() if isinstance(v, tuple)):
            a = table_regular[idx:idx + n].double()
            b = prog.table[idx:idx + n].double()
            assert torch.allclose(b, a, rtol=1e-12, atol=0.0), (attempt, nid, a.tolist(), b.tolist())
        for k in out_nodes:
            assert torch.equal(prog.results[k], fields_regular[k]), (attempt, k)


def test_noalloc_pass_matches_regular_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _run_noalloc_twice("divergence(gradient(f)) + l2norm(curl(u))", ("sum", "mean", "variance"),
                       (40, 48, 64), (3, 4))


def test_noalloc_pass_with_histogram_entropy_and_scalar_sink():
    """A graph whose passes end in the histogram-entropy kernel and whose last
    launch is the scalar kernel (a scalar result computed from two reductions)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _run_noalloc_twice("laplacian(f) + f*f", ("entropy_hist", "norm_l2"), (24, 40, 33), (5, 6))
    _run_noalloc_twice("sum(f) * mean(laplacian(f))", (), (20, 24, 36), (7, 8))
    _run_noalloc_twice("sum(f) * mean(laplacian(f)) + f", ("variance",), (20, 24, 36), (9, 10))


def test_noalloc_rejects_oversized_request():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from stenpy_b200 import _native as N
    table = torch.zeros(4, dtype=torch.float64, device="cuda")
    d = N.ReduceDesc(N.RED_SUM, 0, 0, 0, 1.0, 0.0)
    with pytest.raises(N.NativeError, match="static scratch"):
        N.pass_noalloc([(0, (1, 1, 1), (32, 1, 1), 0, bytes(64), 0, 8)], N.NOALLOC_MAX_PARTIALS + 1, 1, [d],
                       table.data_ptr(), torch.cuda.current_stream().cuda_stream)

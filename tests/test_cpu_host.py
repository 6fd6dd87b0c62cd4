"""CPU-only checks: the C ABI library loads and exports every declared symbol,
the front end keeps the reference's graph semantics, the planner/code generator
produces kernels NVRTC accepts for sm_100a, and the boundary-shell index decode
covers exactly the voxels within R of a face. No GPU calls."""
import ctypes
import itertools
import os
import re

import pytest
import torch

import stenpy_b200 as S
from stenpy_b200 import _native as N
from stenpy_b200 import fused_compiler as FC
from stenpy_b200.codegen import shell_count

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(REPO, "include", "stenpy_b200.h")).read()
    return sorted(set(re.findall(r"\b(stenpy_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(N.ABI_SYMBOLS) <= set(declared)
    assert lib.stenpy_abi_version() == 2


def test_abi_rejects_bad_arguments_without_gpu():
    L = N.lib()
    buf = ctypes.create_string_buffer(128)
    # misaligned base / bad strides are refused before any driver call
    assert L.stenpy_encode_tmap_3d(buf, 4, ctypes.c_void_p(8), 64, 8, 8, 256, 2048, 72, 10, 1) == -1
    assert b"aligned" in L.stenpy_last_error()
    assert L.stenpy_encode_tmap_3d(buf, 4, ctypes.c_void_p(256), 64, 8, 8, 100, 2048, 72, 10, 1) == -1
    assert L.stenpy_encode_tmap_3d(buf, 4, ctypes.c_void_p(256), 64, 8, 8, 256, 2048, 300, 10, 1) == -1
    assert L.stenpy_finalize(None, 1, 1, None, 1, None, None) == -1


def test_finalize_rejects_reductions_wider_than_the_row():
    """A variance reads 3 slots, entropy/min_max 2, covariance 6: a descriptor whose
    slots run past the row is refused before anything is launched."""
    L = N.lib()
    fake = ctypes.c_void_p(4096)
    for kind, width in ((N.RED_VARIANCE, 3), (N.RED_ENTROPY, 2), (N.RED_MIN_MAX, 2), (N.RED_COVARIANCE, 6),
                        (N.RED_SUM, 1)):
        d = (N.ReduceDesc * 1)(N.ReduceDesc(kind, 8 - width + 1, 0, 0, 1.0, 0.0))
        assert L.stenpy_finalize(fake, 4, 8, d, 1, fake, None) == -1, kind
        assert b"outside rows" in L.stenpy_last_error()
    d = (N.ReduceDesc * 1)(N.ReduceDesc(99, 0, 0, 0, 1.0, 0.0))
    assert L.stenpy_finalize(fake, 4, 8, d, 1, fake, None) == -1


def _noalloc_desc(grid, cta_off, nbytes=64, part_offset=0, cta_off_offset=8):
    params = bytearray(nbytes)
    params[cta_off_offset:cta_off_offset + 4] = int(cta_off).to_bytes(4, "little", signed=True)
    buf = ctypes.create_string_buffer(bytes(params), nbytes)
    d = N.LaunchDesc()
    d.module = None
    d.grid[:] = list(grid)
    d.block[:] = [128, 1, 1]
    d.dyn_smem = 0
    d.part_offset = part_offset
    d.cta_off_offset = cta_off_offset
    d.params = ctypes.cast(buf, ctypes.c_void_p)
    d.params_bytes = nbytes
    return d, buf


@pytest.mark.parametrize("grid,cta_off,ncta,nslots,msg", [
    ((4, 2, 1), 0, 7, 4, b"exceed ncta_total"),           # 8 rows written, 7 declared
    ((4, 1, 1), 5, 8, 4, b"exceed ncta_total"),           # rows 5..8 of 8
    ((4, 1, 1), -1, 8, 4, b"exceed ncta_total"),          # negative first row
    ((1, 1, 1), 0, N.NOALLOC_MAX_PARTIALS // 4 + 1, 4, b"static scratch"),
])
def test_noalloc_rejects_rows_outside_the_static_array(grid, cta_off, ncta, nslots, msg):
    """stenpy_pass_noalloc checks the rows each launch writes (its cta_off, read
    from the packed parameters, plus its grid size) against the declared partials
    before it touches the GPU."""
    L = N.lib()
    d, keep = _noalloc_desc(grid, cta_off)
    rd = (N.ReduceDesc * 1)(N.ReduceDesc(N.RED_SUM, 0, 0, 0, 1.0, 0.0))
    arr = (N.LaunchDesc * 1)(d)
    rc = L.stenpy_pass_noalloc(arr, 1, ncta, nslots, rd, 1, ctypes.c_void_p(4096), None)
    assert rc == -1
    assert msg in L.stenpy_last_error()
    # a misplaced cta_off field (past the parameter block) is refused too
    d2, keep2 = _noalloc_desc((1, 1, 1), 0, cta_off_offset=8)
    d2.cta_off_offset = 62
    arr2 = (N.LaunchDesc * 1)(d2)
    assert L.stenpy_pass_noalloc(arr2, 1, 4, 4, rd, 1, ctypes.c_void_p(4096), None) == -1
    assert b"bad parameter block" in L.stenpy_last_error()


def test_front_end_graph_semantics():
    f = torch.zeros(4, 4, 4, dtype=torch.float64)
    g, sink, warns, ids, _ = S.compile_expression("divergence(gradient(f)) + norm_l2(curl(u))",
                                                  field_map={"f": f, "u": torch.zeros(4, 4, 4, 3)})
    ops = [g._nodes[n].op_name for n in g._order]
    assert ops.count("laplacian") == 1 and ops.count("gradient") == 1  # orphan kept, as in the reference
    assert any("Simplified" in w for w in warns)
    orphan = [n for n in g._order if g._nodes[n].op_name == "gradient"][0]
    assert orphan in g._orphans and orphan in g.sinks()
    from stenpy_b200.runtime import default_wanted
    assert default_wanted(g) == [sink]
    # CSE: repeated subexpressions map to one node
    g2, s2, *_ = S.compile_expression("tanh(f)*exp(f) + tanh(f)", field_map={"f": f})
    assert sum(1 for n in g2._order if g2._nodes[n].op_name == "tanh") == 1
    # hessian spelled both ways, l2norm alias, abs, kwargs
    for e in ("hessian(f)", "_hessian(f)"):
        g3, s3, *_ = S.compile_expression(e, field_map={"f": f})
        assert g3._nodes[s3].op_name == "hessian"
    g4, s4, *_ = S.compile_expression("l2norm(abs(f))", field_map={"f": f})
    assert g4._nodes[s4].op_name == "norm_l2"
    g5, s5, *_ = S.compile_expression("gradient(f, dx=0.25, boundary=periodic)", field_map={"f": f})
    assert g5._nodes[s5].params == {"dx": 0.25, "boundary": "periodic"}
    with pytest.raises(ValueError):
        S.compile_expression("nosuchop(f)", field_map={"f": f})


def test_plan_structure_config1():
    f = torch.zeros(64, 64, 64)
    u = torch.zeros(64, 64, 64, 3)
    g, sink, *_ = S.compile_expression("divergence(gradient(f)) + norm_l2(curl(u))", boundary="periodic",
                                       field_map={"f": f, "u": u})
    wanted = [sink] + [g.add(r, (sink,), {}) for r in ("sum", "mean", "variance")]
    plan = FC.Planner(g, wanted).plan()
    # pass 0: ||curl u||^2 partials; pass 1: lap f + c, with sum/mean/var partials
    assert len(plan.passes) == 2
    assert [r.kind for r in plan.passes[0].spec.roots] == ["red"]
    assert sorted(r.kind for r in plan.passes[1].spec.roots) == ["out", "red", "red", "red"]
    assert plan.passes[0].spec.fields[0].nc == 3 and plan.passes[0].spec.radius == 1


@pytest.mark.parametrize("expr,boundary", [
    ("f**2 + tanh(f)*exp(f) + laplacian(g)", "periodic"),
    ("eigenvalues(hessian(f)) + 0*mean_curvature(f)", "neumann"),
    ("curl(u) * 2", "dirichlet"),
    ("cumulative_integral(exp(f)) + integrate(g) + entropy(f) + variance(g)", "periodic"),
    ("material_derivative(f, u) + conv3d_spectral(g) + moving_average(f, window=5, boundary='dirichlet')",
     "neumann"),
])
def test_generated_kernels_compile_for_sm100a(expr, boundary):
    fm = {"f": torch.zeros(20, 24, 32), "g": torch.zeros(20, 24, 32, dtype=torch.bfloat16),
          "u": torch.zeros(20, 24, 32, 3)}
    g, sink, *_ = S.compile_expression(expr, boundary=boundary, field_map=fm)
    plan = FC.Planner(g, [sink]).plan()
    for pp in plan.passes:
        key, cubin = N.compile_cached(FC.emit_pass(pp.spec), FC.NVRTC_OPTS)
        assert len(cubin) > 1000


def _shell_decode(t, shape, R, g_lo, g_hi):
    """Host model of ``sten_shell``'s voxel decode (regions A, B, C), formula for formula."""
    n0, n1, n2 = shape
    a1, a2 = max(n1 - 2 * R, 0), max(n2 - 2 * R, 0)
    c_low = max(0, min(g_hi, R) - g_lo)
    hs = max(g_lo, max(n0 - R, R))
    c_high = max(0, g_hi - hs)
    ii0 = max(g_lo, R)
    n_int = max(0, min(g_hi, n0 - R) - ii0)
    cA, cB = (c_low + c_high) * n1 * n2, n_int * (n1 - a1) * n2
    if t < cA:
        q, r = divmod(t, n1 * n2)
        return (g_lo + q if q < c_low else hs + (q - c_low), r // n2, r % n2)
    if t < cA + cB:
        u, w1 = t - cA, n1 - a1
        q, r = divmod(u, w1 * n2)
        jr, lo = r // n2, min(R, n1)
        return ii0 + q, (jr if jr < lo else n1 - (w1 - jr)), r - jr * n2
    u, w2 = t - cA - cB, n2 - a2
    q, r = divmod(u, a1 * w2)
    jr, kr = divmod(r, w2)
    lo = min(R, n2)
    return ii0 + q, R + jr, (kr if kr < lo else n2 - (w2 - kr))


def test_shell_decode_matches_boundary_shell():
    """Every global plane range of small grids: the count formula is the true shell
    size, and the kernel's decode (host model) maps thread indices one to one onto the
    shell voxels."""
    for shape in [(5, 7, 33), (3, 3, 3), (1, 4, 5), (9, 10, 11), (6, 2, 7), (12, 11, 9)]:
        for R in (1, 2, 3):
            n0, n1, n2 = shape
            for g_lo, g_hi in [(0, n0), (1, n0), (0, max(1, n0 - 1))]:
                truth = {(i, j, k) for i in range(g_lo, g_hi) for j in range(n1) for k in range(n2)
                         if not (R <= i < n0 - R and R <= j < n1 - R and R <= k < n2 - R)}
                cnt = shell_count(shape, R, g_lo, g_hi)
                assert cnt == len(truth)
                got = [_shell_decode(t, shape, R, g_lo, g_hi) for t in range(cnt)]
                assert set(got) == truth and len(set(got)) == cnt, (shape, R, g_lo, g_hi)


def test_shell_blocks_stride_over_every_voxel_once():
    """The shell launch has at most SHELL_MAX_CTAS blocks; their grid-stride loop
    (t = block * 256 + thread, step blocks * 256) visits every shell voxel index once,
    and the partial rows the finalize folds are the blocks launched."""
    from stenpy_b200.codegen import SHELL_MAX_CTAS, SHELL_THREADS, shell_ctas
    for n in (1, 255, 256, 257, SHELL_MAX_CTAS * SHELL_THREADS - 1, SHELL_MAX_CTAS * SHELL_THREADS + 1,
              3 * SHELL_MAX_CTAS * SHELL_THREADS + 17):
        b = shell_ctas(n)
        assert 1 <= b <= SHELL_MAX_CTAS and b == min(-(-n // SHELL_THREADS), SHELL_MAX_CTAS)
        seen = torch.zeros(n, dtype=torch.int32)
        stride = b * SHELL_THREADS
        for first in range(stride):
            seen[first:n:stride] += 1
        assert bool((seen == 1).all()), n


def test_32bit_shell_indexing_only_when_offsets_fit_an_int():
    """The planner enables 32-bit boundary indexing from the field shapes: every
    element offset of n0 (+ halo planes) x n1 x n2 x components must stay below 2^31."""
    def plan(n):
        u = torch.zeros(1).expand(n, n, n, 3)
        g, sink, *_ = S.compile_expression("l2norm(curl(u))", boundary="neumann", field_map={"u": u})
        return FC.Planner(g, [sink]).plan()
    assert plan(512).passes[0].spec.idx32
    assert not plan(1024).passes[0].spec.idx32      # 1026 * 1024 * 1024 * 3 > 2^31
    src = FC.emit_pass(plan(1024).passes[0].spec)
    assert "const long long n0 = p.n0g" in src and "const int n0 = p.n0g" not in src


@pytest.mark.parametrize("dx,expect", [(1.0, 0.25), (0.25, 4.0), (0.5, None), (0.3, None)])
def test_deferred_scale_of_curl_norm_only_for_power_of_two_spacing(dx, expect):
    """The z-march sums unscaled squares of the curl's differences and scales its
    block partial by (1/2h)^2 only when 1/2h is a power of two other than 1 (exact);
    the shell keeps scaled values and an unscaled flush."""
    from stenpy_b200.codegen import deferred_scale
    u = torch.zeros(20, 24, 32, 3)
    g, sink, *_ = S.compile_expression("l2norm(curl(u))", dx=dx, boundary="neumann", field_map={"u": u})
    spec = FC.Planner(g, [sink]).plan().passes[0].spec
    root = [r for r in spec.roots if r.kind == "red"][0]
    assert deferred_scale(spec, root) == expect
    src = FC.emit_pass(spec)
    main, shell = src.split("sten_shell(")[0], src.split("sten_shell(")[1]
    if expect is None:
        assert "block_sum(rv0_a * " not in main
    else:
        assert f"block_sum(rv0_a * {expect!r}, red_scratch)" in main
    assert "block_sum(rv0_a, red_scratch)" in shell
    # a plain sum of the same vector keeps per-voxel scaling
    g2, s2, *_ = S.compile_expression("sum(curl(u))", dx=dx, boundary="neumann", field_map={"u": u})
    spec2 = FC.Planner(g2, [s2]).plan().passes[0].spec
    assert all(deferred_scale(spec2, r) is None for r in spec2.roots)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
def test_mixed_precision_operands_only_for_16bit_staged_fields(dtype):
    """Central differences and Laplacian pairs of 16-bit staged fields take one value
    as stored (LDS / LDA accessors: sub/add.f32.f16 or .bf16); FP32 fields keep plain
    FP32 arithmetic. The kernels compile for sm_100a either way."""
    u = torch.zeros(20, 24, 32, 3, dtype=dtype)
    f = torch.zeros(20, 24, 32, dtype=dtype)
    g, sink, *_ = S.compile_expression("divergence(gradient(f)) + l2norm(curl(u))", boundary="periodic",
                                       field_map={"f": f, "u": u})
    plan = FC.Planner(g, [sink]).plan()
    a, b = (FC.emit_pass(pp.spec) for pp in plan.passes)
    sixteen = dtype != torch.float32
    assert ("LDS0<" in a) == sixteen and ("LDA0<" in b) == sixteen
    for src in (a, b):
        _, cubin = N.compile_cached(src, FC.NVRTC_OPTS)
        assert len(cubin) > 1000


def test_cpu_device_is_rejected():
    with pytest.raises(NotImplementedError):
        S.Runtime(device="cpu")


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16, torch.float16])
@pytest.mark.parametrize("expr,boundary", [
    ("divergence(gradient(f)) + l2norm(curl(u))", "periodic"),
    ("laplacian(f) + gradient(f)*0 + curl(u)", "neumann"),
    ("laplacian(f)", "periodic"),
    ("eigenvalues(hessian(f))", "periodic"),
    ("conv3d_spectral(f) + moving_average(f, window=5)", "neumann"),
    ("laplacian(f) + moving_average(f, window=9, boundary='reflect')", "periodic"),
])
def test_every_tma_x_coordinate_is_16_byte_aligned(dtype, expr, boundary):
    """The x coordinate of each tiled TMA load must be a multiple of 16 bytes (an
    unaligned one faults the GPU). Enumerate the coordinates the generated kernels
    issue — plane boxes for every tile and the periodic wrap strips — for every
    candidate schedule, and check them on the host."""
    from stenpy_b200 import autotune as AT
    from stenpy_b200.codegen import ESIZE, strip_boxes, tmap_specs, with_config
    import dataclasses
    shape = (24, 40, 96)
    fm = {"f": torch.zeros(shape, dtype=dtype), "u": torch.zeros(shape + (3,), dtype=dtype)}
    try:
        g, sink, *_ = S.compile_expression(expr, boundary=boundary, field_map=fm)
        plan = FC.Planner(g, [sink]).plan()
    except FC.FusionError:
        pytest.skip("graph not fusable")
    n2 = shape[2]
    for pp in plan.passes:
        for cfg in [pp.spec.cfg] + AT.candidates(pp.spec):
            spec = with_config(pp.spec, cfg)
            for slot, kind, (bw, bh) in tmap_specs(spec):
                f = spec.fields[slot]
                es = ESIZE[f.dtype]
                hk = spec.hk(f)
                assert (bw * es) % 16 == 0 and bw <= 256 and bh <= 256
                assert (n2 * f.nc * es) % 16 == 0
                xs = []
                if kind in ("box", "jstrip"):
                    xs = [(tk0 - hk) * f.nc for tk0 in range(0, n2, cfg.tk)]
                else:
                    xs = [(n2 - hk) * f.nc, 0]
                for x in xs:
                    assert (x * es) % 16 == 0, (kind, x, es, cfg)


def test_entropy_hist_plans_minmax_then_histogram():
    f = torch.zeros(10, 12, 16)
    g, sink, *_ = S.compile_expression("entropy_hist(f, bins=64)", field_map={"f": f})
    plan = FC.Planner(g, [sink]).plan()
    assert len(plan.passes) == 2 and plan.hist_size == 64
    assert [r.red for r in plan.passes[0].spec.roots] == ["minmax"] and not plan.passes[0].hists
    h = plan.passes[1].hists
    assert len(h) == 1 and h[0].bins == 64 and h[0].table_index == plan.red_index[sink]
    assert h[0].lohi_index == plan.red_index[sink] + 1
    assert plan.passes[0].reductions[0].table_index == h[0].lohi_index


def _batch_jobs_cpu():
    from stenpy_b200 import batch as B
    from stenpy_b200.synth import BATCH_EXPRESSIONS
    jobs = []
    for e in BATCH_EXPRESSIONS:
        for dt, shape in ((torch.float32, (20, 24, 64)), (torch.bfloat16, (17, 20, 51))):
            f = torch.zeros(shape + ((3,) if e.startswith("curl") else ()), dtype=dt)
            g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f})
            jobs.append(B.BatchJob(g, [sink]))
    return jobs


@pytest.mark.parametrize("threads", [128, 256])
def test_batch_module_compiles_for_sm100a(threads):
    from stenpy_b200 import batch as B
    from stenpy_b200.codegen import emit_batch_module
    jobs = _batch_jobs_cpu()
    cfg = B.batch_candidates(threads)[0]
    specs, seen = [], set()
    for j in jobs:
        for pp in B.plan_job(j, cfg).passes:
            k = B.program_key(pp.spec)
            if k not in seen:
                seen.add(k)
                specs.append(pp.spec)
    assert len(specs) >= 16          # 8 expressions x 2 dtypes (+ the entropy min/max passes)
    key, cubin = N.compile_cached(emit_batch_module(specs, threads, B.batch_min_blocks(threads)), FC.NVRTC_OPTS)
    assert len(cubin) > 10000
    # job outputs follow the storage dtype of the job's field
    assert {j.out_dtype for j in jobs} == {torch.float32, torch.bfloat16}


def test_batch_queue_orders_prerequisites_first():
    from stenpy_b200.batch import _Phase, build_queue
    # job 0: one pass; job 1: min/max pass then a dependent histogram pass; job 2 larger
    ph = [_Phase(0, 0, 0, 4, 2, 1, 9, 1, -1, 100.0),
          _Phase(1, 0, 1, 2, 1, 0, 2, 2, -1, 50.0),
          _Phase(1, 1, 2, 2, 1, 0, 2, 1, 1, 50.0),
          _Phase(2, 0, 0, 3, 3, 2, 11, 1, -1, 900.0)]
    items = build_queue(ph)
    quads = [tuple(items[i:i + 4]) for i in range(0, len(items), 4)]
    assert len(quads) == sum(p.ncta for p in ph)
    order = [q[0] for q in quads]
    # the pass with a dependent comes first, the dependent pass last, larger jobs before smaller
    assert order[0] == 1 and order[-1] == 2
    assert order.index(3) < order.index(0)
    assert max(i for i, p in enumerate(order) if p == 1) < min(i for i, p in enumerate(order) if p == 2)
    # every tile of every pass appears exactly once, shell blocks after the pass's tiles
    for pi, p in enumerate(ph):
        tiles = [(q[2], q[3]) for q in quads if q[0] == pi and q[1] == 0]
        assert sorted(tiles) == sorted((bx, by) for by in range(p.nseg) for bx in range(p.gdx))
        assert sum(1 for q in quads if q[0] == pi and q[1] == 1) == p.shell_items
    with pytest.raises(ValueError):
        build_queue([_Phase(0, 0, 0, 1, 1, 0, 1, 1, 0, 1.0)])


def test_batch_queue_check_rejects_bad_items():
    from stenpy_b200.batch import _Phase, build_queue, check_queue
    ph = [_Phase(0, 0, 0, 3, 2, 1, 7, 1, -1, 10.0), _Phase(1, 0, 1, 2, 1, 0, 2, 1, 0, 5.0)]
    items = torch.tensor(build_queue(ph), dtype=torch.int32).reshape(-1, 4)
    check_queue(items, ph)
    assert items.shape[0] == sum(p.ncta for p in ph)
    for bad in (items[:-1], torch.cat([items, items[:1]]),
                torch.cat([items[:-1], torch.tensor([[2, 0, 0, 0]], dtype=torch.int32)]),
                torch.cat([items[:-1], torch.tensor([[0, 0, 3, 0]], dtype=torch.int32)]),
                torch.cat([items[:-1], torch.tensor([[0, 1, 0, 1]], dtype=torch.int32)])):
        with pytest.raises(ValueError):
            check_queue(bad, ph)


def test_cost_model_fixture_and_baselines_without_gpu():
    """The timing fixture is well formed and the model-free baselines evaluate on it
    (the learned model itself trains with GPU kernels, see the GPU tests)."""
    import gzip
    import json
    from stenpy_b200 import costmodel as CM
    path = os.path.join(REPO, "tests", "golden", "autotune_timings.jsonl.gz")
    with gzip.open(path, "rt") as fh:
        recs = [json.loads(line) for line in fh]
    hold = [r for r in recs if r["tag"].startswith("cm-hold")]
    assert hold and any(r["tag"].startswith("cm-train") for r in recs)
    X, y = CM.records_to_xy(recs[:50])
    assert X.shape[0] == 50 and torch.isfinite(X).all() and torch.isfinite(y).all()
    yc = CM.centred_targets(hold)
    assert abs(float(yc.sum())) < 1e-3 * len(hold)   # centred per pass

    class Zero:
        def predict(self, X):
            return torch.zeros(X.shape[0], dtype=torch.float64)

    ev = CM.evaluate(Zero(), hold, k=3)
    assert ev["passes"] > 10 and 0.0 <= ev["analytic_topk"]["mean"] < ev["random_topk"]["mean"] + 0.1


def test_shipped_cost_model_matches_feature_layout():
    """The ensemble shipped with the package takes the current feature vector."""
    import numpy as np
    from stenpy_b200 import costmodel as CM
    z = np.load(CM.DEFAULT_MODEL)
    feat = {"radius": 1, "n0": 64, "n1": 64, "n2": 64, "voxels": 64.0 ** 3, "in_bytes": 4, "out_bytes": 4}
    sched = {"tj": 8, "tk": 64, "threads": 128, "vpt": 4, "seg_len": 32, "prefetch": 2, "smem": 1e4,
             "ghost": 1, "shell": 0, "kv": 1}
    d = len(CM.vectorize(feat, sched))
    assert int(z["n"]) >= 1
    for i in range(int(z["n"])):
        h = int(z[f"m{i}_hidden"])
        assert int(z[f"m{i}_in_dim"]) == d
        assert z[f"m{i}_params"].size == d * h + h + h * h + h + h + 1
        assert np.isfinite(z[f"m{i}_params"]).all()


def test_smoothing_plans_and_limits():
    """Weighted-tap stencils: reach = window // 2, no ghost cells (every face goes to
    the shell kernel), the widest window and the ring-slot bound raise FusionError,
    and chunked runs wrap dim 0 exactly when a pass reads across it periodically."""
    from stenpy_b200.lazy import wraps_dim0
    f = torch.zeros(16, 20, 32)
    u = torch.zeros(16, 20, 32, 3)

    def plan(expr, boundary="neumann"):
        g, sink, *_ = S.compile_expression(expr, boundary=boundary, field_map={"f": f, "u": u})
        return FC.Planner(g, [sink]).plan()

    p = plan("moving_average(f, window=5)")
    spec = p.passes[0].spec
    assert spec.radius == 2 and spec.ghosts is None
    assert [n.a("pad") for n in spec.graph.nodes if n.op == "taps"] == ["replicate"]
    assert not wraps_dim0(spec)
    assert wraps_dim0(plan("conv3d_spectral(f)").passes[0].spec)
    assert wraps_dim0(plan("laplacian(f)", "periodic").passes[0].spec)
    assert not wraps_dim0(plan("curl(u)", "periodic").passes[0].spec)
    taps = [n for n in plan("conv3d_spectral(f)").passes[0].spec.graph.nodes if n.op == "taps"][0]
    assert len(taps.a("taps")) == 27 and sum(t[3] for t in taps.a("taps")) * taps.a("scale") == 1.0
    assert plan("moving_average(f, window=9)").passes[0].spec.radius == 4
    for bad in ("moving_average(f, window=11)", "moving_average(f, window=4)"):
        with pytest.raises(FC.FusionError):
            plan(bad)
    # reach 8 needs 19 ring slots (nested keyword arguments do not parse, as in the
    # reference: the graph is built directly)
    g, sink, *_ = S.compile_expression("moving_average(f, window=9)", field_map={"f": f})
    outer = g.add("moving_average", (sink,), {"window": 9})
    with pytest.raises(FC.FusionError, match="ring"):
        FC.Planner(g, [outer]).plan()
    with pytest.raises(FC.FusionError):     # reflect padding wider than an axis
        g, sink, *_ = S.compile_expression("moving_average(f, window=7, boundary='reflect')",
                                           field_map={"f": torch.zeros(3, 20, 32)})
        FC.Planner(g, [sink]).plan()


def test_2d_fields_plan_as_one_plane_grids():
    """surface_normals needs 2-D fields (3-D raises, as in the reference); 2-D graphs
    plan on a (1, n0, n1) grid with (n0, n1, ...) results; stencils other than the
    surface normals, and 2-D next to 3-D fields, are not fused."""
    f2 = torch.zeros(12, 20)
    g, sink, *_ = S.compile_expression("surface_normals(f) * 2", field_map={"f": f2})
    plan = FC.Planner(g, [sink]).plan()
    assert plan.dims2 and plan.shape == (1, 12, 20) and plan.out_shape(3) == (12, 20, 3)
    spec = plan.passes[0].spec
    assert spec.radius == 1 and spec.ghosts is not None and spec.i_periodic
    g, sink, *_ = S.compile_expression("surface_normals(f)", field_map={"f": torch.zeros(4, 5, 6)})
    with pytest.raises(FC.FusionError, match="2-D"):
        FC.Planner(g, [sink]).plan()
    for expr in ("laplacian(f)", "integrate(f)"):
        g, sink, *_ = S.compile_expression(expr, field_map={"f": f2})
        with pytest.raises(FC.FusionError, match="2-D"):
            FC.Planner(g, [sink]).plan()
    g, sinks, *_ = S.compile_expressions({"a": "f*2", "b": "g*2"}, field_map={"f": f2, "g": torch.zeros(3, 12, 20)})
    with pytest.raises(FC.FusionError, match="2-D and 3-D"):
        FC.Planner(g, list(sinks.values())).plan()


def _emulate_row_staging(spec, f, tk0, tj0, n1, n2, rj, rk, nt, fb=0):
    """Host model of the row staging of one plane (the generated copies and in-place
    shift, formula for formula, on a one-plane field starting at byte ``fb``): returns
    {box element: global element, None for zero, or "free" for a column outside the
    grid that no rule asks for}, checking that every copy unit is 16-byte aligned,
    lies in the ring slot and reads only 16-byte units that overlap the field; that a
    warp reads all its chunks before it writes any, with every read inside
    its row; and that no other element takes a byte that was not copied from the
    field."""
    from stenpy_b200.codegen import ESIZE, rs_geometry
    es, nc = ESIZE[f.dtype], f.nc
    hk = spec.hk(f)
    w, h, _, rb, c, sr, rpw, ni = rs_geometry(spec, f, spec.cfg)
    nw = nt // 32
    assert rpw * nw >= h and ni * 32 >= rpw * c
    epc = 16 // es
    fe = fb + n1 * n2 * nc * es
    rbg = n2 * nc * es

    def remap(x, n, rule):
        if rule == "periodic":
            return x + n if x < 0 else (x - n if x >= n else x)
        if rule == "replicate":
            return min(max(x, 0), n - 1)
        if rule == "reflect" and n > 1:
            x = -x if x < 0 else x
            x = 2 * (n - 1) - x if x > n - 1 else x
            return min(max(x, 0), n - 1)
        return x

    slot = [None] * (h * sr)               # ring slot byte -> global byte ("outside": not the field)
    lo, hi = fb - fb % 16, (fe + 15) // 16 * 16
    for q in range(h * (c + 1)):            # request: unit q of the slot, one 16-byte copy
        r, u = divmod(q, c + 1)
        jg = remap(tj0 - f.halo + r, n1, rj)
        if not 0 <= jg < n1:
            continue
        a0 = fb + ((jg * n2 + (tk0 - hk)) * nc) * es
        g = a0 - a0 % 16 + 16 * u
        assert g % 16 == 0 and 16 * q + 16 <= h * sr
        if lo <= g < hi:                    # a unit that overlaps the field (first/last plane check)
            assert g < fe and g + 16 > fb
            for t in range(16):
                slot[16 * q + t] = g + t if fb <= g + t < fe else "outside"
        else:
            for t in range(16):
                slot[16 * q + t] = "zero-filled"

    gather = rk in ("periodic", "replicate", "reflect") and f.halo > 0
    ns = -(-(16 - es + f.halo * nc * es) // 16)
    strip = {}

    def window(side):
        ws = {("periodic", 0): n2 - f.halo, ("periodic", 1): 0, ("replicate", 0): 0,
              ("replicate", 1): n2 - f.halo, ("reflect", 0): 1, ("reflect", 1): n2 - 1 - f.halo}[(rk, side)]
        return min(max(ws, 0), max(n2 - f.halo, 0))

    if gather:                              # strips of tiles at a dim-2 face
        for r in range(h):
            jg = remap(tj0 - f.halo + r, n1, rj)
            if not 0 <= jg < n1:
                continue
            for sd in (0, 1):
                if (sd == 0 and tk0 != 0) or (sd == 1 and tk0 + spec.cfg.tk + hk <= n2):
                    continue
                g0 = fb + (jg * n2 + window(sd)) * nc * es
                al = g0 - g0 % 16
                for u in range(ns):
                    if g0 - al + f.halo * nc * es > 16 * u:
                        assert lo <= al + 16 * u < hi
                        for t in range(16):
                            g = al + 16 * u + t
                            strip[((2 * r + sd) * ns + u) * 16 + t] = g if fb <= g < fe else "outside"

    sz = fb + (tk0 - hk) * nc * es            # plane 0
    fixes = []
    for v in range(nw):                      # warps touch disjoint rows: one at a time
        lanes = []
        for i in range(ni):
            for lane in range(32):
                ix = i * 32 + lane
                m, cc = divmod(ix, c)
                r = v + nw * m
                if m >= rpw or r >= h:
                    continue
                jg = remap(tj0 - f.halo + r, n1, rj)
                off = r * sr + cc * 16
                if 0 <= jg < n1:
                    sh = (sz + (jg * rbg) % 16) % 16
                    assert sh == (fb + ((jg * n2 + (tk0 - hk)) * nc) * es) % 16
                    assert r * sr <= off and off + 32 <= (r + 1) * sr, "shifted read inside the row"
                    val = slot[off + sh:off + sh + 16]          # every lane reads ...
                    xl = cc * epc - hk * nc
                    if tk0 + xl // nc < 0 or tk0 + (xl + epc - 1) // nc >= n2:
                        fixes.append((r, cc, jg))
                else:
                    val = [None] * 16
                lanes.append((off, val))
        for off, val in lanes:                                 # ... before any lane writes
            slot[off:off + 16] = val
    zero = object()
    for r in range(h):                       # rows outside the grid were written as zeros
        if not 0 <= remap(tj0 - f.halo + r, n1, rj) < n1:
            slot[r * sr:r * sr + rb] = [zero] * rb
    fixed = {}
    for r, cc, jg in fixes:                  # the dim-2 fix-up after the shift
        rowb = fb + jg * rbg
        for e in range(epc):
            xr = cc * epc + e - hk * nc
            kg = tk0 + xr // nc
            if 0 <= kg < n2:
                continue
            if rk == "zero":
                fixed[r * w + cc * epc + e] = None
                continue
            if not gather or not -f.halo <= kg < n2 + f.halo:
                fixed[r * w + cc * epc + e] = "free"      # as copied: feeds no kept voxel
                continue
            ccomp = xr - (kg - tk0) * nc
            sd = 0 if kg < 0 else 1
            kr = remap(kg, n2, rk)
            ws = window(sd)
            if ws <= kr < ws + f.halo:                    # from the strip
                b0 = (rowb + ws * nc * es) % 16 + ((kr - ws) * nc + ccomp) * es
                by = [strip[(2 * r + sd) * ns * 16 + b0 + t] for t in range(es)]
                assert all(isinstance(x, int) for x in by) and all(by[t] == by[0] + t for t in range(es))
                assert by[0] == rowb + (kr * nc + ccomp) * es
                fixed[r * w + cc * epc + e] = (by[0] - fb) // es
            else:
                okk = 0 <= kr < n2
                fixed[r * w + cc * epc + e] = (rowb + (kr * nc + ccomp) * es - fb) // es if okk else None
    out = {}
    for r in range(h):
        for x in range(w):
            dst = r * w + x
            if dst in fixed:
                out[dst] = fixed[dst]
                continue
            bytes_ = slot[r * sr + x * es:r * sr + (x + 1) * es]
            if all(b_ is zero for b_ in bytes_):
                out[dst] = None
                continue
            assert all(isinstance(b_, int) for b_ in bytes_), ("byte not copied from the field", r, x, bytes_)
            assert all(bytes_[t] == bytes_[0] + t for t in range(es)) and (bytes_[0] - fb) % es == 0
            out[dst] = (bytes_[0] - fb) // es
    return out


@pytest.mark.parametrize("es,nc", [(4, 1), (4, 3), (2, 1), (2, 3), (8, 1)])
@pytest.mark.parametrize("rule", [None, "periodic", "replicate", "reflect", "zero"])
def test_row_staging_covers_every_box_element_once(es, nc, rule):
    """Row staging (fields whose rows TMA cannot describe): every element of a staged
    box is written exactly once — with the element its axis rules map it to, or zero
    outside the grid — from aligned 16-byte copies that read only the field, for
    interior, face and corner tiles of ragged grids, with 16-byte-aligned and merely
    element-aligned field bases."""
    from stenpy_b200.codegen import PassConfig, PassSpec, FieldSpec, PGraph

    def rm(x_, n_):
        if rule == "periodic":
            return x_ + n_ if x_ < 0 else (x_ - n_ if x_ >= n_ else x_)
        if rule == "replicate":
            return min(max(x_, 0), n_ - 1)
        if rule == "reflect" and n_ > 1:
            y = -x_ if x_ < 0 else x_
            y = 2 * (n_ - 1) - y if y > n_ - 1 else y
            return min(max(y, 0), n_ - 1)
        return x_

    dt = {4: "f32", 2: "bf16", 8: "f64"}[es]
    for tk, tj, nt in ((64, 8, 128), (32, 16, 128), (64, 16, 256)):
        cfg = PassConfig(tj=tj, tk=tk, threads=nt)
        for n1, n2 in ((37, 45), (9, 33), (40, 130), (5, 7), (12, 34), (11, 509), (6, 22)):
            f = FieldSpec(0, dt, nc, staged=True, halo=2)
            spec = PassSpec(PGraph(), [f], [], 1, 1, 2, cfg)
            hk = spec.hk(f)
            w, h = spec.box(f)
            for tj0 in range(0, n1, tj):
                for tk0 in range(0, n2, tk):
                    for fb in (0, es, 16 * 1000 + es * 3):
                        got = _emulate_row_staging(spec, f, tk0, tj0, n1, n2, rule, rule, nt, fb)
                        assert len(got) == w * h
                        for dst, g in got.items():
                            if g == "free":
                                continue
                            r, x = divmod(dst, w)
                            xr = x - hk * nc
                            kg, c = tk0 + xr // nc, xr % nc
                            jg, kg = rm(tj0 - f.halo + r, n1), rm(kg, n2)
                            want = (jg * n2 + kg) * nc + c if (0 <= jg < n1 and 0 <= kg < n2) else None
                            assert g == want, (dst, g, want, tj0, tk0, n1, n2, fb)


def test_spectral_operators_are_registered_and_gpu_only():
    """FFT operators run outside the fused passes (opaque graph nodes) and, like every
    operator here, refuse host tensors."""
    from stenpy_b200.registry import KNOWN_OPS
    for name in ("fft", "ifft", "fft_complex", "ifft_complex", "spectral_gradient", "spectral_laplacian"):
        assert name in S.OP_REGISTRY and name not in KNOWN_OPS
        assert S.OP_METADATA[name]["cost"] == "high"
        with pytest.raises(ValueError, match="CUDA"):
            S.OP_REGISTRY[name](torch.zeros(4, 5, 6))
    g, sink, *_ = S.compile_expression("spectral_gradient(f, dim=2, dx=0.5) + laplacian(f)",
                                       field_map={"f": torch.zeros(4, 5, 6)})
    ops = {n.op_name: n.params for n in g.topological_sort()}
    assert ops["spectral_gradient"] == {"dim": 2, "dx": 0.5}


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.float16, torch.bfloat16])
def test_distance_transform_kernels_compile_for_sm100a(dtype):
    """The distance transform's row, envelope and finalize kernels build for sm_100a
    for every storage dtype (no GPU needed: NVRTC only)."""
    from stenpy_b200.geometry import _OPTS, edt_source
    key, cubin = N.compile_cached(edt_source(dtype, 64), _OPTS)
    assert len(cubin) > 1000

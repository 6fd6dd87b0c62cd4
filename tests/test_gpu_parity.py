"""GPU parity: the fused CUDA executor against (a) the golden vectors produced by
the reference itself and (b) the CPU FP64 oracle on the same stored inputs.

Tolerance: norm-wise relative error max|y - y_ref| / max|y_ref| <= 1e-5 for FP32
storage and compute (the target the executor is built to), unless a case lists
its own bound in TOL below with the reason. Mean curvature meets it too: its
first differences are formed from stored (exact) values, so ∇f carries a relative
error of a few FP32 units even where |∇f| is small, and so does ∇f/|∇f|.
"""
import pytest
import torch

from golden_cases import load_cases, rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu

CASES = load_cases()
TOL: dict = {}


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_fused_matches_reference_golden(case):
    import stenpy_b200 as S
    dev = _dev()
    fmap = {k: v.to(dev) for k, v in case["inputs"].items()}
    g, sink, _, _, _ = S.compile_expression(case["expr"], dx=case["dx"], boundary=case["boundary"],
                                            field_map=fmap)
    got = S.Runtime(device=dev).run(g)[sink]
    assert tuple(got.shape) == tuple(case["expected"].shape)
    err = rel_err(got, case["expected"])
    assert err <= TOL.get(case["name"], 1e-5), f"{case['name']}: rel err {err:.3e}"


@pytest.mark.parametrize("case", CASES[:6], ids=[c["name"] for c in CASES[:6]])
def test_eager_mode_matches_golden(case):
    """fusion_enabled=False: one kernel per node, intermediates materialised."""
    import stenpy_b200 as S
    dev = _dev()
    fmap = {k: v.to(dev) for k, v in case["inputs"].items()}
    g, sink, _, _, _ = S.compile_expression(case["expr"], dx=case["dx"], boundary=case["boundary"],
                                            field_map=fmap)
    got = S.Runtime(device=dev, fusion_enabled=False).run(g)[sink]
    assert rel_err(got, case["expected"]) <= TOL.get(case["name"], 1e-5)


@pytest.mark.parametrize("shape", [(5, 7, 33), (3, 3, 3), (17, 9, 130), (2, 40, 64)])
@pytest.mark.parametrize("boundary", ["periodic", "neumann", "dirichlet"])
def test_ragged_shapes_against_oracle(shape, boundary):
    """Tiles that do not divide the grid, tiny grids, one-sided edges on every face."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, uniform_field
    dev = _dev()
    f = sinusoid_field(shape, seed=11)
    gg = uniform_field(shape, seed=12)
    exprs = ["laplacian(f) + tanh(g)*exp(f)", "gradient(f)"]
    if min(shape) >= 3:
        exprs += ["_hessian(f)", "mean_curvature(g*g + 1)", "trace(_hessian(f)) + tanh(g)"]
    for expr in exprs:
        g, sink, *_ = S.compile_expression(expr, boundary=boundary, field_map={"f": f.to(dev), "g": gg.to(dev)})
        got = S.Runtime(device=dev).run(g)[sink]
        g2, sink2, *_ = S.compile_expression(expr, boundary=boundary, field_map={"f": f.double(), "g": gg.double()})
        ref = O.evaluate(g2, [sink2])[sink2]
        assert rel_err(got, ref) <= 1e-4, (expr, shape, boundary)


def test_config0_shape_against_oracle():
    """Config 0 workload: f**2 + tanh(f)*exp(f) + laplacian(g) on 128^3, periodic."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, uniform_field
    dev = _dev()
    f = sinusoid_field((128, 128, 128), seed=0)
    gg = uniform_field((128, 128, 128), seed=1)
    expr = "f**2 + tanh(f)*exp(f) + laplacian(g)"
    g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev), "g": gg.to(dev)})
    got = S.Runtime(device=dev).run(g)[sink]
    g2, sink2, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.double(), "g": gg.double()})
    ref = O.evaluate(g2, [sink2])[sink2]
    assert rel_err(got, ref) <= 1e-5


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("boundary", ["periodic", "neumann"])
def test_kv_chunks_match_one_voxel_per_thread(dtype, boundary):
    """Several k-adjacent voxels per thread (vector shared-memory chunks, paired
    stores) compute every voxel exactly as one voxel per thread does; reductions of
    computed values agree to FP32 plane-sum rounding."""
    import stenpy_b200 as S
    from stenpy_b200.codegen import PassConfig
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    for shape in [(20, 33, 130), (9, 16, 64), (7, 5, 45)]:
        f = sinusoid_field(shape, seed=4).to(dtype).to(dev)
        u = smoothed_vector(shape, seed=5).to(dtype).to(dev)
        expr = "divergence(gradient(f)) + l2norm(curl(u)) + laplacian(f)*tanh(f)"
        outs = {}
        for kv, tk, tj in ((1, 64, 8), (2, 64, 16), (4, 64, 32), (2, 32, 8), (8, 64, 16), (8, 128, 8)):
            cfg = PassConfig(tj=tj, tk=tk, threads=128, seg_len=8, kv=kv)
            g, sink, *_ = S.compile_expression(expr, boundary=boundary, field_map={"f": f, "u": u})
            w = [sink, g.add("variance", (sink,), {})]
            res = S.Runtime(device=dev, out_dtype=dtype, config=cfg).run(g, wanted=w)
            outs[kv, tk, tj] = (res[w[0]], float(res[w[1]]))
        ref, vref = outs[1, 64, 8]
        for key, (o, v) in outs.items():
            assert torch.equal(o, ref), (key, shape, (o.float() - ref.float()).abs().max().item())
            # the variance of a computed value is summed per plane in FP32 over each
            # thread's voxels, which schedules group differently
            assert abs(v - vref) <= 1e-6 * abs(vref), (key, v, vref)


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_16bit_fields_with_one_sided_edges_keep_fp32_accuracy(dtype):
    """16-bit stored fields with FP32 results: one-sided edges must be formed from the
    stored values in FP32 (an extrapolated ghost written into the 16-bit ring would be
    rounded to 16 bits and show up as a ~1e-3 error at the faces)."""
    import stenpy_b200 as S
    from stenpy_b200.codegen import PassConfig
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    for shape in [(12, 20, 64), (9, 17, 37)]:
        f = sinusoid_field(shape, seed=70).to(dtype)
        u = smoothed_vector(shape, seed=71).to(dtype)
        for expr in ("curl(u)", "gradient(f) * 2", "_hessian(f)", "divergence(u) + laplacian(f)"):
            for ghost in (True, False):
                g, sink, *_ = S.compile_expression(expr, boundary="neumann", field_map={"f": f.to(dev), "u": u.to(dev)})
                got = S.Runtime(device=dev, config=PassConfig(ghost=ghost)).run(g)[sink]
                g2, s2, *_ = S.compile_expression(expr, boundary="neumann", field_map={"f": f.double(), "u": u.double()})
                ref = O.evaluate(g2, [s2])[s2]
                assert rel_err(got, ref) <= 1e-5, (expr, shape, ghost, rel_err(got, ref))


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_16bit_central_differences_equal_fp32_of_the_stored_values(dtype):
    """Interior central differences (and the Laplacian's neighbour pairs) of 16-bit
    fields take one stored value in a mixed-precision subtraction (addition): bit
    for bit the FP32 result of the converted values, so FP32 results equal those of
    the same values stored in FP32 at every voxel off the faces (whose one-sided
    rules run in another order)."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    for shape in [(12, 20, 64), (9, 17, 37)]:
        u = smoothed_vector(shape, seed=21).to(dtype)
        f = sinusoid_field(shape, seed=22).to(dtype)
        for expr in ("curl(u)", "divergence(u)", "gradient(f)", "laplacian(f)", "l2norm(curl(u))"):
            outs = []
            for cast in (lambda t: t, lambda t: t.float()):
                fm = {"u": cast(u).to(dev)} if "(u)" in expr else {"f": cast(f).to(dev)}
                g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map=fm)
                outs.append(S.Runtime(device=dev, out_dtype=torch.float32).run(g)[sink])
            if outs[0].dim() == 0:
                # the norm's faces come from the shell (16-bit) or ghost cells (FP32)
                assert abs(float(outs[0]) - float(outs[1])) <= 1e-6 * abs(float(outs[1])), (expr, shape)
                continue
            a, b = (o[1:-1, 1:-1, 1:-1] for o in outs)
            assert torch.equal(a, b), (expr, shape, (a - b).abs().max().item())


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_norm_of_curl_scales_exactly_with_power_of_two_spacing(dtype):
    """The z-march sums the squares of unscaled central differences and applies
    (1/2h)^2 once to each CTA's partial (the faces' kernel keeps scaled values in
    rows of its own). With power-of-two spacings that is bit for bit the sum of the
    scaled squares, so halving dx exactly doubles the norm; other spacings scale per
    voxel and meet the oracle as before."""
    import stenpy_b200 as S
    from stenpy_b200.synth import smoothed_vector
    dev = _dev()
    for shape in [(20, 33, 130), (9, 16, 64)]:
        u = smoothed_vector(shape, seed=11).to(dtype)
        vals = {}
        for dx in (1.0, 0.5, 0.25, 0.3):
            g, sink, *_ = S.compile_expression("l2norm(curl(u))", dx=dx, boundary="neumann", field_map={"u": u.to(dev)})
            vals[dx] = float(S.Runtime(device=dev).run(g)[sink])
            g2, s2, *_ = S.compile_expression("l2norm(curl(u))", dx=dx, boundary="neumann", field_map={"u": u.double()})
            ref = float(O.evaluate(g2, [s2])[s2])
            assert abs(vals[dx] - ref) <= 1e-6 * abs(ref), (shape, dx, vals[dx], ref)
        assert vals[1.0] * 2 == vals[0.5] and vals[0.5] * 2 == vals[0.25], (shape, vals)


@pytest.mark.parametrize("kv", [1, 2])
@pytest.mark.parametrize("tk,tj", [(32, 16), (64, 8)])
@pytest.mark.parametrize("shape", [(10, 17, 65), (9, 33, 97), (12, 18, 66)])
def test_second_derivative_ghosts_where_tile_halos_cross_faces(shape, tk, tj, kv):
    """Two-layer ghost cells of d1(d1(f)) (reach 2): tiles whose own voxels stop one
    short of a face still read past it and must get the extrapolated values; a last
    tile holding one column reads the four before it (row-staged grids: the k-halo
    depends on the voxels per thread)."""
    import stenpy_b200 as S
    from stenpy_b200.codegen import PassConfig
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    f = sinusoid_field(shape, seed=9)
    cfg = PassConfig(tj=tj, tk=tk, threads=128, seg_len=8, kv=kv)
    g, sink, *_ = S.compile_expression("trace(_hessian(f))", boundary="neumann", field_map={"f": f.to(dev)})
    got = S.Runtime(device=dev, config=cfg).run(g)[sink]
    g2, sink2, *_ = S.compile_expression("trace(_hessian(f))", boundary="neumann", field_map={"f": f.double()})
    ref = O.evaluate(g2, [sink2])[sink2]
    assert rel_err(got, ref) <= 1e-5, (shape, tk, tj, rel_err(got, ref))


def test_unfusable_graph_warns_and_runs_node_by_node():
    """Fields on two different grids cannot share fused passes: like the reference,
    the runtime warns and runs the graph node by node (on the GPU)."""
    import warnings as W
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    f = sinusoid_field((8, 9, 16), seed=1)
    g = sinusoid_field((10, 12, 16), seed=2)
    gr, sinks, *_ = S.compile_expressions({"a": "laplacian(f)", "b": "laplacian(g) * 2"}, boundary="periodic",
                                          field_map={"f": f.to(dev), "g": g.to(dev)})
    with W.catch_warnings(record=True) as rec:
        W.simplefilter("always")
        res = S.Runtime(device=dev).run(gr, wanted=list(sinks.values()))
    assert any("Fusion failed" in str(w.message) for w in rec)
    g2, sinks2, *_ = S.compile_expressions({"a": "laplacian(f)", "b": "laplacian(g) * 2"}, boundary="periodic",
                                           field_map={"f": f.double(), "g": g.double()})
    ref = O.evaluate(g2, list(sinks2.values()))
    for k in ("a", "b"):
        assert rel_err(res[sinks[k]], ref[sinks2[k]]) <= 1e-5, k


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_covariance_and_correlation(dtype):
    """Co-moment reductions (pivot-shifted per thread, Chan-merged per block and across
    CTAs in FP64) on stored values: FP64 agreement with the oracle's centred dot
    products, on ragged grids, offset data (where Σab − n·μa·μb would cancel) and fused
    with stencils."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, uniform_field
    dev = _dev()
    for shape in [(17, 9, 130), (40, 33, 64), (3, 3, 3)]:
        f = (sinusoid_field(shape, seed=41).double() * 0.01 + 100.0).to(dtype)
        g = uniform_field(shape, seed=42).to(dtype)
        exprs = {"c": "covariance(f, g)", "r": "correlation(f, g)", "rr": "correlation(f, f)",
                 "cl": "covariance(laplacian(g), f)"}
        gr, sinks, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f.to(dev), "g": g.to(dev)})
        res = S.Runtime(device=dev).run(gr, wanted=list(sinks.values()))
        g2, s2, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f.double(), "g": g.double()})
        ref = O.evaluate(g2, list(s2.values()))
        for k in exprs:
            a, b = float(res[sinks[k]]), float(ref[s2[k]])
            tol = 1e-5 if k == "cl" else 1e-9   # cl: an FP32 Laplacian
            assert abs(a - b) <= tol * max(abs(b), 1e-6), (k, shape, a, b)

"""Smoothing, advection and surface stencils on the fused executor —
``moving_average`` (box mean, every padding rule), ``conv3d_spectral`` (27-point
Gaussian, circular), ``material_derivative`` and ``surface_normals`` (2-D fields) —
against the CPU FP64 oracle on the same stored values.

Tolerance: norm-wise relative error <= 1e-5 for FP32-stored results (FP32 compute of
at most 125 taps); BF16-stored results add the BF16 unit roundoff."""
import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(5, 7, 33), (17, 9, 130), (9, 33, 97), (3, 3, 3)]
TOL_BF16_OUT = 8e-3


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _check(expr, fields, boundary="periodic", tol=1e-5, out_dtype=torch.float32, cfg=None):
    import stenpy_b200 as S
    dev = _dev()
    g, sink, *_ = S.compile_expression(expr, boundary=boundary, field_map={k: v.to(dev) for k, v in fields.items()})
    got = S.Runtime(device=dev, out_dtype=out_dtype, config=cfg).run(g)[sink]
    g2, s2, *_ = S.compile_expression(expr, boundary=boundary, field_map={k: v.double() for k, v in fields.items()})
    ref = O.evaluate(g2, [s2])[s2]
    assert tuple(got.shape) == tuple(ref.shape), (expr, tuple(got.shape))
    err = rel_err(got, ref)
    assert err <= tol, (expr, tuple(next(iter(fields.values())).shape), err)
    return got


@pytest.mark.parametrize("boundary", ["neumann", "periodic", "dirichlet", "reflect"])
@pytest.mark.parametrize("window", [3, 5])
def test_moving_average_against_oracle(window, boundary):
    from stenpy_b200.synth import sinusoid_field
    for shape in SHAPES:
        f = sinusoid_field(shape, seed=21)
        _check(f"moving_average(f, window={window}, boundary='{boundary}')", {"f": f})


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_gauss27_against_oracle(dtype):
    from stenpy_b200.synth import sinusoid_field
    for shape in SHAPES:
        f = sinusoid_field(shape, seed=22).to(dtype)
        _check("conv3d_spectral(f)", {"f": f})
        _check("conv3d_spectral(f)", {"f": f}, out_dtype=torch.bfloat16, tol=TOL_BF16_OUT)


@pytest.mark.parametrize("boundary", ["neumann", "periodic"])
def test_material_derivative_against_oracle(boundary):
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    for shape in SHAPES + [(2, 40, 64)]:
        f = sinusoid_field(shape, seed=23)
        u = smoothed_vector(shape, seed=24)
        _check("material_derivative(f, u)", {"f": f, "u": u}, boundary=boundary)
        if min(shape) >= 3:   # curl needs edge order 2 on every axis
            _check("material_derivative(f*f, curl(u)) + f", {"f": f, "u": u}, boundary=boundary)


def test_smoothing_fused_with_other_stencils_under_every_schedule():
    """Taps nested under and over other stencils, several taps nodes in one pass, and
    the same voxels under thread mappings with 1, 2 and 4 voxels per thread. Nested
    stencils are inlined per offset, so the compiler may contract a different set of
    multiply-adds per schedule: schedules agree to FP32 rounding, not bit for bit."""
    from stenpy_b200.codegen import PassConfig
    from stenpy_b200.synth import sinusoid_field, uniform_field
    exprs = ["moving_average(laplacian(f)) + conv3d_spectral(g)*2",
             "laplacian(moving_average(f, window=3, boundary='periodic'))",
             "conv3d_spectral(tanh(f)) - moving_average(g, window=5, boundary='reflect')"]
    for shape in [(20, 33, 130), (7, 12, 45)]:
        f = sinusoid_field(shape, seed=25)
        g = uniform_field(shape, seed=26)
        for expr in exprs:
            outs = [_check(expr, {"f": f, "g": g}, cfg=PassConfig(tj=tj, tk=tk, threads=128, seg_len=8, kv=kv))
                    for kv, tk, tj in ((1, 64, 8), (2, 64, 16), (4, 64, 32), (2, 32, 8))]
            for o in outs[1:]:
                assert rel_err(o, outs[0]) <= 2e-6, (expr, shape, rel_err(o, outs[0]))


def test_smoothing_preserves_the_sum_at_256():
    """On a periodic grid a normalised filter moves mass around without changing the
    total: Σ conv3d_spectral(f) = Σ moving_average(f) = Σ f (a size-independent check
    at a size the oracle does not run)."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    f = sinusoid_field((256, 256, 256), seed=27).to(dev)
    exprs = {"a": "sum(f + 2)", "b": "sum(conv3d_spectral(f + 2))",
             "c": "sum(moving_average(f + 2, window=3, boundary='periodic'))"}
    g, sinks, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f})
    res = S.Runtime(device=dev).run(g, wanted=list(sinks.values()))
    a = float(res[sinks["a"]])
    for k in ("b", "c"):
        assert abs(float(res[sinks[k]]) - a) <= 1e-6 * abs(a), (k, float(res[sinks[k]]), a)


def test_smoothing_in_batch_and_lazy_modes():
    """The same kernels behind the batched executor and the chunked (lazy) runner."""
    import stenpy_b200 as S
    from stenpy_b200 import batch as B
    from stenpy_b200.lazy import LazyPipeline
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    exprs = ["conv3d_spectral(f)", "moving_average(f, window=5)", "moving_average(f, boundary='periodic')"]
    jobs, host = [], []
    for i, e in enumerate(exprs * 2):
        shape = [(33, 21, 45), (40, 24, 80)][i % 2]
        f = sinusoid_field(shape, seed=30 + i)
        g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f.to(dev)})
        jobs.append(B.BatchJob(g, [sink]))
        host.append((e, f, sink))
    for (e, f, sink), res in zip(host, B.run_batch(jobs, dev)):
        g2, s2, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f.double()})
        assert rel_err(res[sink], O.evaluate(g2, [s2])[s2]) <= 1e-5, (e, tuple(f.shape))
    f = sinusoid_field((37, 24, 64), seed=40)
    for e in exprs:
        g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f.to(dev)})
        whole = S.Runtime(device=dev).run(g)[sink].cpu()
        gh, sh, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f.pin_memory()})
        got = LazyPipeline(gh, [sh], dev, chunk=7).run()[sh]
        assert torch.equal(whole, got), (e, (whole - got).abs().max().item())


def test_window_limits_raise():
    """Even windows change the grid in the reference (it fails); so does this."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    f = sinusoid_field((8, 9, 16), seed=1).to(dev)
    g, sink, *_ = S.compile_expression("moving_average(f, window=4)", field_map={"f": f})
    with pytest.raises(Exception, match="window"):
        S.Runtime(device=dev).run(g)


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_surface_normals_on_2d_fields(dtype):
    """2-D height fields run as one-plane grids; the normals come back (n0, n1, 3).
    Shapes cover TMA rows (64 FP32 / 128 BF16 columns) and ragged ones."""
    from stenpy_b200.synth import sinusoid_field
    for shape in [(3, 3), (5, 33), (40, 130), (64, 64), (37, 128)]:
        f = sinusoid_field((1,) + shape, seed=50)[0].contiguous().to(dtype)
        got = _check("surface_normals(f)", {"f": f}, boundary="neumann")
        assert tuple(got.shape) == shape + (3,)
        _check("surface_normals(f*f) * 2 + mean(f)", {"f": f})
        _check("variance(tanh(f))", {"f": f})


def test_surface_normals_in_a_batch():
    """2-D jobs next to 3-D ones in one persistent launch."""
    import stenpy_b200 as S
    from stenpy_b200 import batch as B
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    items = [("surface_normals(f)", (1, 40, 130)), ("conv3d_spectral(f)", (20, 24, 80)),
             ("surface_normals(f)", (1, 64, 64)), ("laplacian(f)", (19, 37, 50))]
    jobs, host = [], []
    for i, (e, shape) in enumerate(items):
        f = sinusoid_field(shape, seed=60 + i)
        if shape[0] == 1:
            f = f[0].contiguous()
        g, sink, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f.to(dev)})
        jobs.append(B.BatchJob(g, [sink]))
        host.append((e, f, sink))
    for (e, f, sink), res in zip(host, B.run_batch(jobs, dev)):
        g2, s2, *_ = S.compile_expression(e, boundary="periodic", field_map={"f": f.double()})
        ref = O.evaluate(g2, [s2])[s2]
        assert tuple(res[sink].shape) == tuple(ref.shape)
        assert rel_err(res[sink], ref) <= 1e-5, (e, tuple(f.shape))

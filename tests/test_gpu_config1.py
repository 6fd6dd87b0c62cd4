"""The headline workload at full size, and global reductions of stored values.

1. Config 1 at 512^3: ``divergence(gradient(f)) + l2norm(curl(u))`` with the
   sum / mean / variance of the result, periodic, unit spacing, f and u generated
   as the benchmark generates them. Every storage form runs on the whole field
   on the GPU; the CPU FP64 oracle evaluates the same graph on the same stored
   (rounded) inputs over the whole field, slab by slab (curl and the Laplacian
   of a slab need one plane of halo; the global L2 norm is the FP64 sum of the
   slabs' squares), so every voxel of the GPU result is compared.
   Bounds, norm-wise (max |y - y64| / max |y64|): FP32 storage 1e-5; FP16
   storage 1e-3 (the target for 16-bit storage; FP16's unit roundoff is
   2^-11 = 4.9e-4); BF16 inputs with an FP32 result 1e-5; BF16 storage 4e-3
   (BF16 keeps 8 significant bits: its unit roundoff 2^-8 = 3.9e-3 alone exceeds
   1e-3). Scalars (formed in FP64 from the FP32 per-voxel values, before output
   rounding): 1e-6 relative.
2. sum / mean / norm_l2 / integrate of raw stored fields (FP32, FP16, BF16,
   vector fields included) against the FP64 oracle at 1e-12 relative: the values
   are exact, so only FP64 accumulation order separates the two.
"""
import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu

N = 512
EXPR = "divergence(gradient(f)) + l2norm(curl(u))"
REDS = ("sum", "mean", "variance")
FORMS = {  # name: (input storage, result storage, norm-wise bound)
    "fp32": (torch.float32, torch.float32, 1e-5),
    "fp16": (torch.float16, torch.float16, 1e-3),
    "bf16in": (torch.bfloat16, torch.float32, 1e-5),
    "bf16": (torch.bfloat16, torch.bfloat16, 4e-3),
}


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def fields():
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    f = sinusoid_field((N,) * 3, seed=0, device=dev)
    u = smoothed_vector((N,) * 3, seed=2, device=dev)
    return f, u


def _oracle_whole_field(f64: torch.Tensor, u64: torch.Tensor, slab: int = 32):
    """FP64 oracle of the config-1 graph over the whole field, slab by slab:
    returns the per-voxel result and its sum / mean / unbiased variance."""
    n0 = f64.shape[0]
    torch.set_num_threads(max(1, torch.get_num_threads()))
    sq = torch.zeros((), dtype=torch.float64)
    for a in range(0, n0, slab):            # ||curl u||^2, curl ignores periodic (torch.gradient)
        b = min(a + slab, n0)
        lo, hi = max(a - 1, 0), min(b + 1, n0)
        c = O.OPS["curl"](u64[lo:hi], dx=1.0, boundary="periodic")[a - lo:a - lo + (b - a)]
        sq += (c * c).sum()
    cnorm = torch.sqrt(sq)
    out = torch.empty_like(f64)
    for a in range(0, n0, slab):            # periodic Laplacian: wrap one plane each side
        b = min(a + slab, n0)
        idx = torch.arange(a - 1, b + 1) % n0
        lap = O.OPS["laplacian"](f64[idx], dx=1.0, boundary="periodic")[1:-1]
        out[a:b] = lap + cnorm
    return out, {"sum": out.sum().item(), "mean": out.mean().item(), "variance": out.var().item()}


@pytest.mark.parametrize("form", list(FORMS))
def test_config1_full_size_every_voxel_against_oracle(fields, form):
    import stenpy_b200 as S
    dev = _dev()
    f, u = fields
    din, dout, bound = FORMS[form]
    fs, us = f.to(din), u.to(din)
    g, sink, *_ = S.compile_expression(EXPR, dx=1.0, boundary="periodic", field_map={"f": fs, "u": us})
    wanted = [sink] + [g.add(r, (sink,), {}) for r in REDS]
    res = S.Runtime(device=dev, out_dtype=dout).run(g, wanted=wanted)
    y = res[sink]
    assert y.dtype == dout and tuple(y.shape) == (N,) * 3
    y64 = y.double().cpu()
    ref, scal = _oracle_whole_field(fs.double().cpu(), us.double().cpu())
    err = (y64 - ref).abs().max().item() / ref.abs().max().item()
    assert err <= bound, (form, err)
    for r, w in zip(REDS, wanted[1:]):
        got = float(res[w])
        assert abs(got - scal[r]) <= 1e-6 * abs(scal[r]), (form, r, got, scal[r])


RAW = [
    ("sum(f)", "f", (70, 33, 129)),
    ("mean(f)", "f", (64, 64, 64)),
    ("norm_l2(f)", "f", (41, 50, 77)),
    ("integrate(f)", "f", (31, 40, 66)),
    ("integrate(f)", "f", (30, 41, 65)),
    ("norm_l2(u)", "u", (33, 36, 40)),
    ("sum(u)", "u", (21, 30, 44)),
]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("expr,name,shape", RAW, ids=[f"{e}-{s[0]}" for e, _, s in RAW])
def test_reductions_of_stored_values_at_1e12(expr, name, shape, dtype):
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    x = sinusoid_field(shape, seed=51) if name == "f" else smoothed_vector(shape, seed=52)
    x = (x + 3.0).to(dtype)          # an offset keeps the sums away from cancellation
    g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={name: x.to(dev)})
    got = float(S.Runtime(device=dev).run(g)[sink])
    g2, s2, *_ = S.compile_expression(expr, boundary="periodic", field_map={name: x.double()})
    ref = float(O.evaluate(g2, [s2])[s2])
    assert abs(got - ref) <= 1e-12 * abs(ref), (expr, dtype, got, ref, abs(got - ref) / abs(ref))

"""Exact distance transform (``distance_transform``) against the reference's CPU
definition (SciPy's exact EDT of ``t == 0``, through the oracle): random masks, every
storage dtype, anisotropic spacing, 1-D to 3-D fields, and inside graphs."""
import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.bfloat16, torch.float16])
def test_distance_transform_matches_scipy(dtype):
    from stenpy_b200.geometry import distance_transform
    dev = _dev()
    gen = torch.Generator().manual_seed(5)
    for shape, density, dx in (((17, 23, 31), 0.05, 1.0), ((9, 40, 13), 0.01, (0.5, 1.0, 2.0)),
                               ((64, 3, 70), 0.2, 0.7), ((1, 1, 50), 0.1, 1.0), ((5, 6, 7), 0.9, 1.0)):
        mask = torch.rand(shape, generator=gen) < density
        mask.view(-1)[0] = True                  # at least one voxel with t != 0
        t = torch.where(mask, torch.rand(shape, generator=gen) + 0.5, torch.zeros(shape)).to(dtype)
        t[0, 0, -1] = -0.0                       # a negative zero is a zero
        got = distance_transform(t.to(dev), dx=dx)
        ref = O.distance_transform(t.double(), dx=dx)
        assert got.dtype == torch.float64 and tuple(got.shape) == shape
        assert rel_err(got, ref) <= 1e-12, (shape, dx, rel_err(got, ref))
    t1 = torch.tensor([0.0, 0.0, 3.0, 0.0, 0.0, 0.0], dtype=dtype)
    assert torch.equal(distance_transform(t1.to(dev)).cpu(), O.distance_transform(t1.double()))
    t2 = torch.zeros(6, 9, dtype=dtype)
    t2[2, 3] = 1
    assert rel_err(distance_transform(t2.to(dev), dx=(1.0, 0.5)), O.distance_transform(t2.double(), dx=(1.0, 0.5))) <= 1e-12


def test_distance_transform_in_graphs_and_at_256():
    """As a graph node between fused passes, and at 256^3 (sizes the oracle also runs:
    SciPy is exact there too)."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field
    dev = _dev()
    f = sinusoid_field((256, 256, 256), seed=3)
    expr = "distance_transform(clamp(f - 1.5)) * 0.5 + tanh(f)"
    g, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev)})
    got = S.Runtime(device=dev).run(g)[sink]
    g2, s2, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.double()})
    ref = O.evaluate(g2, [s2])[s2]
    assert rel_err(got, ref) <= 1e-6, rel_err(got, ref)

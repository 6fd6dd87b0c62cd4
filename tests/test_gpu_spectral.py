"""FFT operators (cuFFT through torch.fft, outside the fused passes) inside graphs run
by the fused runtime: against the CPU FP64 oracle on ragged grids, and against exact
Fourier identities at a size the oracle does not run."""
import math

import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.mark.parametrize("shape", [(8, 9, 16), (5, 7, 33), (12, 20, 64)])
def test_spectral_graphs_against_oracle(shape):
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, uniform_field
    dev = _dev()
    f = sinusoid_field(shape, seed=31)
    g = uniform_field(shape, seed=32)
    for expr in ("spectral_laplacian(f)", "spectral_gradient(f, dim=0) * g", "ifft(fft(f)) - f",
                 "spectral_laplacian(tanh(f)) - laplacian(tanh(f)) + mean(spectral_gradient(g, dim=2))"):
        gr, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev), "g": g.to(dev)})
        got = S.Runtime(device=dev).run(gr)[sink]
        g2, s2, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.double(), "g": g.double()})
        ref = O.evaluate(g2, [s2])[s2]
        assert tuple(got.shape) == tuple(ref.shape)
        assert rel_err(got, ref) <= 1e-5, (expr, shape, rel_err(got, ref))
        eager = S.Runtime(device=dev, fusion_enabled=False).run(gr)[sink]
        assert rel_err(eager, ref) <= 1e-5, (expr, shape, "eager")


def test_spectral_derivatives_of_fourier_modes_at_256():
    """sin(k·x) on a periodic 256³ grid: the spectral derivative is exact (to FP64
    rounding; the wavenumbers m/256, rounded to FP32 as the reference forms them, are
    exact): ∂₂ = k₂ cos(k·x), ∇² = −|k|² sin(k·x)."""
    import stenpy_b200 as S
    dev = _dev()
    n = 256
    ax = torch.arange(n, device=dev, dtype=torch.float64)
    i, j, k = torch.meshgrid(ax, ax, ax, indexing="ij")
    kv = [2 * math.pi * m / n for m in (3, 5, 7)]
    ph = kv[0] * i + kv[1] * j + kv[2] * k
    f = torch.sin(ph)
    exprs = {"d2": "spectral_gradient(f, dim=2)", "lap": "spectral_laplacian(f)"}
    g, sinks, *_ = S.compile_expressions(exprs, boundary="periodic", field_map={"f": f})
    res = S.Runtime(device=dev).run(g, wanted=list(sinks.values()))
    assert rel_err(res[sinks["d2"]], kv[2] * torch.cos(ph)) <= 1e-10
    assert rel_err(res[sinks["lap"]], -sum(v * v for v in kv) * f) <= 1e-10

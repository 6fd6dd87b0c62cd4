"""The drop-in boundary on the GPU: a user operator registered with
``register_operator`` (the reference's plugin contract, stenpy_engine.py:1188-1212,
with ``alloc=``/``mm=`` injected by signature, :1074-1080) running between fused
stencil passes; the attribute-configured ``Pipeline`` (stenpy.py:621-951); and the
``stenpy`` command line (README.md:21). Results are compared with the CPU FP64
oracle on the same stored inputs (norm-wise relative error <= 1e-5, the FP32
executor's bound).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from golden_cases import rel_err
from oracle import stenpy_oracle as O

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


CALLS = []


def soft_threshold(x, t=0.25, dx=1.0, boundary="periodic", alloc=None, mm=None):
    """A user operator written against the reference's contract: it asks for an
    output buffer through ``alloc`` (FP64, like the reference's memory manager)
    and records what the runtime injected."""
    CALLS.append({"alloc": alloc is not None, "mm": mm is not None, "device": x.device.type})
    out = alloc(tuple(x.shape), x.device, key=None)
    torch.mul(torch.sign(x), torch.clamp(x.abs() - t, min=0.0), out=out)
    return out


def _soft_threshold_cpu(x, t=0.25, **_):
    return torch.sign(x) * torch.clamp(x.abs() - t, min=0.0)


@pytest.fixture
def user_op(monkeypatch):
    import stenpy_b200 as S
    from stenpy_b200.registry import OP_METADATA, OP_REGISTRY
    S.register_operator("soft_threshold", soft_threshold, radius=0, cost="low")
    monkeypatch.setitem(O.OPS, "soft_threshold", _soft_threshold_cpu)
    CALLS.clear()
    yield
    OP_REGISTRY.pop("soft_threshold", None)
    OP_METADATA.pop("soft_threshold", None)


@pytest.mark.parametrize("fusion", [True, False])
def test_registered_operator_between_fused_stencils(user_op, fusion):
    import stenpy_b200 as S
    from stenpy_b200.registry import OP_METADATA
    from stenpy_b200.synth import sinusoid_field, uniform_field
    dev = _dev()
    assert OP_METADATA["soft_threshold"]["stencil_radius"] == 0
    shape = (20, 33, 70)
    f = sinusoid_field(shape, seed=21)
    g = uniform_field(shape, seed=22)
    expr = "laplacian(soft_threshold(laplacian(f) + g)) + sum(soft_threshold(f*g)) * g"
    gr, sink, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.to(dev), "g": g.to(dev)})
    mm = S.MemoryManager()
    got = S.Runtime(mm, device=dev, fusion_enabled=fusion).run(gr)[sink]
    g2, sink2, *_ = S.compile_expression(expr, boundary="periodic", field_map={"f": f.double(), "g": g.double()})
    ref = O.evaluate(g2, [sink2])[sink2]
    assert rel_err(got, ref) <= 1e-5
    assert len(CALLS) == 2 and all(c["alloc"] and c["mm"] and c["device"] == "cuda" for c in CALLS)


def test_registered_operator_is_called_directly(user_op):
    """OP_REGISTRY[name] is the user's callable, as in the reference."""
    from stenpy_b200.registry import OP_REGISTRY
    import stenpy_b200 as S
    dev = _dev()
    x = torch.linspace(-1, 1, 64, dtype=torch.float64, device=dev).reshape(4, 4, 4)
    out = OP_REGISTRY["soft_threshold"](x, t=0.5, alloc=S.MemoryManager().allocate)
    assert torch.equal(out.cpu(), _soft_threshold_cpu(x.cpu(), t=0.5))


def test_pipeline_attribute_run(tmp_path):
    """Pipeline configured by attribute assignment: field paths, a constant, the
    boundary, and ``.output`` triggering the run and writing field + spacing + origin."""
    import stenpy_b200 as S
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    _dev()
    shape = (18, 24, 40)
    f = sinusoid_field(shape, seed=31)
    u = smoothed_vector(shape, seed=32)
    np.savez(tmp_path / "f.npz", field=f.numpy(), spacing=np.array([0.5, 0.5, 0.5]), origin=np.zeros(3))
    np.savez(tmp_path / "u.npz", field=u.numpy(), spacing=np.array([0.5, 0.5, 0.5]), origin=np.ones(3))
    p = S.Pipeline("cfg1", "divergence(gradient(f)) + l2norm(curl(u)) * c")
    p.f = str(tmp_path / "f.npz")
    p.u = str(tmp_path / "u.npz")
    p.c = 0.5
    p.boundary = "neumann"
    p.dx = 0.5
    p.output = str(tmp_path / "out.npz")          # runs the pipeline
    z = np.load(tmp_path / "out.npz")
    got = torch.from_numpy(z["field"])
    g2, sink2, *_ = S.compile_expression("divergence(gradient(f)) + norm_l2(curl(u)) * c", dx=0.5,
                                         boundary="neumann",
                                         field_map={"f": f.double(), "u": u.double(),
                                                    "c": torch.tensor(0.5, dtype=torch.float64)})
    ref = O.evaluate(g2, [sink2])[sink2]
    assert rel_err(got, ref) <= 1e-5
    # as in the reference, the file keeps the spacing/origin of the last field loaded
    assert list(z["spacing"]) == [0.5, 0.5, 0.5] and list(z["origin"]) == [1.0, 1.0, 1.0]
    assert rel_err(p.value, ref) <= 1e-5                 # cached result, no second run
    # module-level dispatch: stenpy_b200.<op>(expr, **settings) is a Pipeline
    q = S.laplacian("laplacian(f)", f=f.to("cuda"), boundary="periodic")
    g3, s3, *_ = S.compile_expression("laplacian(f)", boundary="periodic", field_map={"f": f.double()})
    assert rel_err(q.value, O.evaluate(g3, [s3])[s3]) <= 1e-5


def test_console_entry_point_is_declared():
    import tomllib
    with open(os.path.join(REPO, "pyproject.toml"), "rb") as fh:
        proj = tomllib.load(fh)
    target = proj["project"]["scripts"]["stenpy"]
    mod, fn = target.split(":")
    import importlib
    assert callable(getattr(importlib.import_module(mod), fn))


def test_stenpy_command_line_curl(tmp_path):
    """``stenpy --field u=… --expr "curl(u)" --device cuda --output …`` (the
    reference's advertised command) in a fresh process, against the oracle."""
    from stenpy_b200.synth import smoothed_vector
    import stenpy_b200 as S
    _dev()
    u = smoothed_vector((16, 20, 36), seed=41)
    np.save(tmp_path / "u.npy", u.numpy())
    out = tmp_path / "curl.npy"
    code = "import sys; from stenpy_b200.cli import main; sys.exit(main())"
    r = subprocess.run([sys.executable, "-c", code, "--field", f"u={tmp_path / 'u.npy'}", "--expr", "curl(u)",
                        "--device", "cuda", "--output", str(out)],
                       cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    summary = json.loads(r.stdout.strip().splitlines()[-1])
    got = torch.from_numpy(np.load(out))
    assert summary["shape"] == [16, 20, 36, 3]
    g2, s2, *_ = S.compile_expression("curl(u)", boundary="periodic", field_map={"u": u.double()})
    assert rel_err(got, O.evaluate(g2, [s2])[s2]) <= 1e-5
    # --device cpu is refused: there is no CPU path
    r = subprocess.run([sys.executable, "-c", code, "--field", f"u={tmp_path / 'u.npy'}", "--expr", "curl(u)",
                        "--device", "cpu"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 2 and "CUDA devices only" in r.stderr

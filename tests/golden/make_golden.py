"""Generate golden vectors by running the REFERENCE implementation itself.

Run in the development container, where the reference sources are mounted:

    python tests/golden/make_golden.py [/path/to/reference]

It imports the reference's ``stenpy_engine`` in-process and evaluates each case
below with the reference's own CPU eager path::

    compile_expression(expr, dx, boundary, field_map)
    Runtime(MemoryManager(), device="cpu").run(graph)[sink]

The reference imports ``h5py`` and ``zict`` unconditionally; neither is installed
here and neither is on this path, so two minimal stand-ins are registered first
(``h5py.File`` raises; ``zict`` mappings are plain dicts). Inputs are stored as
float32 (the storage dtype the GPU executor reads), outputs as float64, in
``golden.npz``; case metadata and library versions go to ``cases.json``.
The fixtures are read by the tests; the reference is not needed to run them.
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from stenpy_b200.synth import sinusoid_field, smoothed_vector, uniform_field  # noqa: E402


def _install_stand_ins() -> None:
    h5 = types.ModuleType("h5py")

    class _NoFile:
        def __init__(self, *a, **k):
            raise OSError("h5py stand-in: HDF5 is not available in this harness")

    h5.File = _NoFile
    h5.Dataset = type("Dataset", (), {})
    sys.modules["h5py"] = h5

    zict = types.ModuleType("zict")

    class _Map(dict):
        def __init__(self, *a, **k):
            super().__init__()

    zict.File = _Map
    zict.Func = _Map
    zict.Buffer = _Map
    sys.modules["zict"] = zict


S_EVEN = (12, 14, 16)
S_ODD = (5, 7, 9)
S_MIX = (9, 10, 11)


def _fields(shape, seed, names):
    if len(shape) == 2:     # 2-D fields: the first plane of a one-plane 3-D field
        return {k: v[0].contiguous() for k, v in _fields((1,) + tuple(shape), seed, names).items()}
    out = {}
    for n in names:
        if n == "f":
            out[n] = sinusoid_field(shape, seed=seed)
        elif n == "g":
            out[n] = uniform_field(shape, seed=seed + 1)
        elif n == "u":
            out[n] = smoothed_vector(shape, seed=seed + 2)
        else:
            raise KeyError(n)
    return out


# name, expression, fields, boundary, dx, shape
CASES = [
    ("cfg0_periodic", "f**2 + tanh(f)*exp(f) + laplacian(g)", "fg", "periodic", 1.0, S_EVEN),
    ("cfg0_neumann", "f**2 + tanh(f)*exp(f) + laplacian(g)", "fg", "neumann", 1.0, S_MIX),
    ("lap_dirichlet", "laplacian(f)", "f", "dirichlet", 1.0, S_ODD),
    ("lap_reflect", "laplacian(f)", "f", "reflect", 1.0, S_ODD),
    ("lap_dx", "laplacian(f)*2", "f", "periodic", 0.5, S_MIX),
    ("grad_periodic", "gradient(f)", "f", "periodic", 1.0, S_EVEN),
    ("grad_neumann", "gradient(f)", "f", "neumann", 1.0, S_MIX),
    ("grad_dx", "gradient(f)", "f", "neumann", 0.5, S_ODD),
    ("div_periodic", "divergence(u)", "u", "periodic", 1.0, S_EVEN),
    ("div_neumann", "divergence(u)", "u", "neumann", 1.0, S_MIX),
    ("curl_periodic", "curl(u)", "u", "periodic", 1.0, S_EVEN),
    ("curl_neumann", "curl(u)", "u", "neumann", 0.5, S_MIX),
    ("hess_neumann", "_hessian(f)", "f", "neumann", 1.0, S_MIX),
    ("hess_periodic", "_hessian(f)", "f", "periodic", 0.5, S_EVEN),
    ("eig_hess", "eigenvalues(_hessian(f))", "f", "neumann", 1.0, S_MIX),
    ("trace_hess", "trace(_hessian(f))", "f", "periodic", 1.0, S_EVEN),
    ("mc_periodic", "mean_curvature(f)", "f", "periodic", 1.0, S_EVEN),
    ("mc_neumann", "mean_curvature(f)", "f", "neumann", 1.0, S_MIX),
    ("cfg1_expr", "divergence(gradient(f)) + norm_l2(curl(u))", "fu", "periodic", 1.0, S_EVEN),
    ("cfg1_sum", "sum(divergence(gradient(f)) + norm_l2(curl(u)))", "fu", "periodic", 1.0, S_EVEN),
    ("cfg1_mean", "mean(divergence(gradient(f)) + norm_l2(curl(u)))", "fu", "periodic", 1.0, S_EVEN),
    ("cfg1_var", "variance(divergence(gradient(f)) + norm_l2(curl(u)))", "fu", "periodic", 1.0, S_EVEN),
    ("norm_l2", "norm_l2(f*g)", "fg", "periodic", 1.0, S_MIX),
    ("entropy", "entropy(f)", "f", "periodic", 1.0, S_MIX),
    ("integrate_even", "integrate(f)", "f", "periodic", 1.0, S_EVEN),
    ("integrate_odd", "integrate(f + g)", "fg", "periodic", 1.0, S_ODD),
    ("integrate_mix", "integrate(exp(f))", "f", "periodic", 1.0, S_MIX),
    ("cumint", "cumulative_integral(f*g)", "fg", "periodic", 1.0, S_MIX),
    ("elementwise_a", "sqrt(f) + log(g) - sin(f)/(g*g + 1)", "fg", "periodic", 1.0, S_MIX),
    ("elementwise_b", "clamp(log(f*f + 1), 0, 2)", "f", "periodic", 1.0, S_MIX),
    ("elementwise_c", "f**-2 + f**1.5 + tanh(g)**3", "fg", "periodic", 1.0, S_MIX),
    ("elementwise_d", "exp(f)*2 + 3 - clamp(g)", "fg", "periodic", 1.0, S_ODD),
    ("div_eps_guard", "f/clamp(g, 0, 0) + g/(f*f)", "fg", "periodic", 1.0, S_ODD),
    ("elementwise_e", "-f + sqrt(g) * 0.25", "fg", "periodic", 1.0, S_ODD),
    ("lap_of_pointwise", "laplacian(tanh(f)*exp(g)) + 0.5*laplacian(g)", "fg", "neumann", 1.0, S_MIX),
    ("lap_lap", "laplacian(laplacian(f))", "f", "periodic", 1.0, S_EVEN),
    ("grad_scalar_mix", "sum(f) * laplacian(f) - mean(g)", "fg", "periodic", 1.0, S_MIX),
    ("jacobian_neumann", "jacobian(u)", "u", "neumann", 1.0, S_MIX),
    ("jacobian_dx", "jacobian(u)", "u", "periodic", 0.5, S_EVEN),
    ("matderiv_neumann", "material_derivative(f, u)", "fu", "neumann", 1.0, S_MIX),
    ("matderiv_dx", "material_derivative(f, u) + f", "fu", "periodic", 0.5, S_ODD),
    ("movavg_default", "moving_average(f)", "f", "periodic", 1.0, S_MIX),
    ("movavg_w5", "moving_average(f, window=5)", "f", "periodic", 1.0, S_EVEN),
    ("movavg_periodic", "moving_average(f, window=3, boundary='periodic')", "f", "neumann", 1.0, S_MIX),
    ("movavg_dirichlet", "moving_average(f, window=5, boundary='dirichlet')", "f", "neumann", 1.0, S_ODD),
    ("movavg_reflect", "moving_average(g, window=3, boundary='reflect')", "g", "neumann", 1.0, S_ODD),
    ("movavg_w1", "moving_average(g, window=1)", "g", "neumann", 1.0, S_ODD),
    ("movavg_of_expr", "moving_average(tanh(f)*g) + laplacian(f)", "fg", "periodic", 1.0, S_MIX),
    ("gauss27", "conv3d_spectral(f)", "f", "periodic", 1.0, S_MIX),
    ("gauss27_odd", "conv3d_spectral(g)", "g", "neumann", 1.0, S_ODD),
    ("gauss27_of_expr", "conv3d_spectral(f*g + 1)", "fg", "periodic", 1.0, S_EVEN),
    ("surfnorm_a", "surface_normals(f)", "f", "periodic", 1.0, (10, 11)),
    ("surfnorm_dx", "surface_normals(f)", "f", "neumann", 0.5, (12, 16)),
    ("surfnorm_small", "surface_normals(f*g)", "fg", "neumann", 1.0, (3, 5)),
    ("field2d_reduce", "sum(f*f) + mean(g)", "fg", "periodic", 1.0, (9, 13)),
    ("field2d_pointwise", "tanh(f)*exp(g) + f**2", "fg", "periodic", 1.0, (9, 13)),
    ("spec_lap", "spectral_laplacian(f)", "f", "periodic", 1.0, S_EVEN),
    ("spec_grad", "spectral_gradient(f, dim=1)", "f", "periodic", 1.0, S_MIX),
    ("spec_grad_dx", "spectral_gradient(f, dim=2, dx=0.5)", "f", "periodic", 1.0, S_ODD),
    ("fft_roundtrip", "ifft(fft(f*g))", "fg", "periodic", 1.0, S_MIX),
    ("spec_vs_fd", "spectral_laplacian(f) - laplacian(f) + sum(spectral_laplacian(g))", "fg", "periodic", 1.0, S_EVEN),
    ("edt_clamp", "distance_transform(clamp(f))", "f", "periodic", 1.0, S_MIX),
    ("edt_even", "distance_transform(clamp(f*g))", "fg", "periodic", 1.0, S_EVEN),
    ("edt_plus", "distance_transform(clamp(f - 1)) + f", "f", "neumann", 1.0, S_ODD),
    ("det_hess", "determinant(_hessian(f))", "f", "neumann", 1.0, S_MIX),
    ("dev_hess", "deviatoric(_hessian(f)) * 2", "f", "periodic", 1.0, S_EVEN),
    ("inv_spd", "inverse(_hessian(f) + scale_eye(f*f + 4, D=3))", "f", "neumann", 1.0, S_MIX),
    ("gnd", "gradient_nd(f)", "f", "periodic", 0.5, S_ODD),
    ("stack3", "stack_components(f, g, f*g)", "fg", "periodic", 1.0, S_MIX),
    ("normlast", "norm_last(gradient(f))", "f", "neumann", 1.0, S_MIX),
    ("divlast", "div_last(gradient(f), norm_last(gradient(f)))", "f", "periodic", 1.0, S_EVEN),
    ("divlast_scalar", "div_last(curl(u), f*f + 1)", "fu", "neumann", 1.0, S_MIX),
    ("negstack", "neg_stack3(f, g)", "fg", "periodic", 1.0, S_ODD),
    ("vdotg", "velocity_dot_grad(f, g) + 1", "fg", "periodic", 1.0, S_ODD),
    ("surfint", "surface_integral(gradient(f), curl(u), f*f)", "fu", "neumann", 1.0, S_MIX),
    ("aat_hess", "matmul_batched_custom(_hessian(f))", "f", "neumann", 1.0, S_MIX),
    ("cov_fg", "covariance(f, g)", "fg", "periodic", 1.0, S_MIX),
    ("corr_fg", "correlation(f*g, laplacian(f))", "fg", "periodic", 1.0, S_EVEN),
    ("cov_vec", "covariance(curl(u), gradient(f)) + correlation(f, f)", "fu", "neumann", 1.0, S_MIX),
]

# The reference's expression path hands conv3d_spectral and matmul_batched_custom a
# ``dx`` they do not accept (a TypeError at run time), so these cases build the
# reference graph directly: the inner expression, then the operator node on top
# (stenpy_engine.py:2735-2748, 2800-2860).
GRAPH_BUILT = {"gauss27": ("f", "conv3d_spectral"), "gauss27_odd": ("g", "conv3d_spectral"),
               "gauss27_of_expr": ("f*g + 1", "conv3d_spectral"), "aat_hess": ("_hessian(f)", "matmul_batched_custom")}


def main(ref_dir: str) -> None:
    _install_stand_ins()
    sys.dont_write_bytecode = True
    sys.path.insert(0, ref_dir)
    import sympy
    import stenpy_engine as E  # the reference

    arrays = {}
    meta = []
    for name, expr, fnames, bnd, dx, shape in CASES:
        fields32 = _fields(shape, seed=len(meta) * 7 + 3, names=fnames)
        fmap = {k: v.to(torch.float64) for k, v in fields32.items()}
        if name in GRAPH_BUILT:
            inner, op = GRAPH_BUILT[name]
            g, sink, warns, _, _ = E.compile_expression(inner, dx=dx, boundary=bnd, field_map=fmap)
            sink = g.add(op, (sink,), {})
        else:
            g, sink, warns, _, _ = E.compile_expression(expr, dx=dx, boundary=bnd, field_map=fmap)
        rt = E.Runtime(E.MemoryManager(), device="cpu", fusion_enabled=False)
        with torch.no_grad():
            out = rt.run(g)[sink]
        out = out.detach().to(torch.float64).numpy()
        for k, v in fields32.items():
            arrays[f"{name}__in__{k}"] = v.numpy().astype(np.float32)
        arrays[f"{name}__out"] = np.asarray(out, dtype=np.float64)
        meta.append({"name": name, "expr": expr, "fields": list(fnames), "boundary": bnd,
                     "dx": dx, "shape": list(shape), "out_shape": list(np.shape(out)),
                     "warnings": list(warns), "graph_built": name in GRAPH_BUILT})
        print(f"{name:18s} {expr:55s} -> {np.shape(out)}")
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "cases.json"), "w") as fh:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "oracle_path": "reference stenpy_engine compile_expression + Runtime(device='cpu')",
                   "versions": {"torch": torch.__version__, "sympy": sympy.__version__,
                                "numpy": np.__version__},
                   "cases": meta}, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <directory holding the reference's stenpy_engine.py>")
    main(sys.argv[1])

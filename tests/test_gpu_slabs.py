"""Dim-0 slab decomposition on one GPU: 2 and 3 ranks emulated in one process
(``LocalRanks``: the halo planes travel by the same point-to-point pairing the
process-group driver uses, partial rows are stacked in rank order). Per-voxel
results reassembled from the ranks' owned planes equal the whole-field run bit
for bit (every voxel takes the same arithmetic), and the scalars agree with it to
1e-12 relative (FP64 partial rows folded in another grouping; variances to 1e-6,
their FP32 plane sums being pivoted at each thread's first voxel)."""
import pytest
import torch

pytestmark = pytest.mark.gpu

CASES = [
    ({"y": "divergence(gradient(f)) + l2norm(curl(u))"}, "periodic", ("sum", "mean", "variance")),
    ({"eig": "eigenvalues(hessian(f))", "mc": "mean_curvature(f)"}, "neumann", ("mean",)),
    ({"y": "laplacian(f)*tanh(f) + f", "c": "curl(u)"}, "dirichlet", ("norm_l2",)),
]


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _build(exprs, bnd, f, u, reds):
    import stenpy_b200 as S
    g, sinks, *_ = S.compile_expressions(exprs, boundary=bnd, field_map={"f": f, "u": u})
    first = next(iter(sinks.values()))
    red_ids = [g.add(r, (first,), {}) for r in reds]
    return g, sinks, red_ids


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", range(3))
def test_emulated_ranks_equal_whole_field(world, case):
    import stenpy_b200 as S
    from stenpy_b200.slabs import LocalRanks, owned_range
    from stenpy_b200.synth import sinusoid_field, smoothed_vector
    dev = _dev()
    exprs, bnd, reds = CASES[case]
    shape = (29, 24, 40)
    f = sinusoid_field(shape, seed=61).to(dev)
    u = smoothed_vector(shape, seed=62).to(dev)
    g, sinks, red_ids = _build(exprs, bnd, f, u, reds)
    whole = S.Runtime(device=dev).run(g, wanted=list(sinks.values()) + red_ids)
    graphs, wanted, ids = [], [], []
    for r in range(world):
        s, e = owned_range(shape[0], r, world)
        gr, sk, rd = _build(exprs, bnd, f[s:e].contiguous(), u[s:e].contiguous(), reds)
        graphs.append(gr)
        wanted.append(list(sk.values()) + rd)
        ids.append((sk, rd))
    res = LocalRanks(graphs, wanted, shape[0], dev).run()
    for k, nid in sinks.items():
        parts = [res[r][ids[r][0][k]] for r in range(world)]
        got = torch.cat(parts, 0)
        assert torch.equal(got, whole[nid]), (k, (got.float() - whole[nid].float()).abs().max().item())
    for i, nid in enumerate(red_ids):
        ref = float(whole[nid])
        for r in range(world):
            v = float(res[r][ids[r][1][i]])
            # a variance pivots each thread's FP32 plane sums at its first voxel, which
            # moves with the slab bounds (FP32 rounding of those sums); the sum and mean
            # of the same value come from the variance's accumulators
            tol = 1e-6 if "variance" in reds else 1e-12
            assert abs(v - ref) <= tol * max(abs(ref), 1e-300), (reds[i], r, v, ref)
        # every rank holds the same scalar, bit for bit
        assert len({float(res[r][ids[r][1][i]]) for r in range(world)}) == 1

"""Pin the CPU oracle (and this package's expression front end) against golden
vectors produced by running the reference implementation itself."""
import pytest
import torch

from golden_cases import load_cases, rel_err
from oracle import stenpy_oracle as O
from stenpy_b200.frontend import compile_expression

CASES = load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_golden(case):
    fmap = {k: v.to(torch.float64) for k, v in case["inputs"].items()}
    g, sink, _, _, _ = compile_expression(case["expr"], dx=case["dx"], boundary=case["boundary"],
                                          field_map=fmap)
    got = O.evaluate(g, [sink])[sink]
    assert tuple(got.shape) == tuple(case["expected"].shape)
    assert rel_err(got, case["expected"]) <= 1e-12

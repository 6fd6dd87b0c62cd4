"""Loader for the golden vectors produced by tests/golden/make_golden.py."""
import json
import os

import numpy as np
import torch

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_cases():
    with open(os.path.join(HERE, "cases.json")) as fh:
        meta = json.load(fh)
    data = np.load(os.path.join(HERE, "golden.npz"))
    cases = []
    for c in meta["cases"]:
        fields = {k: torch.from_numpy(data[f"{c['name']}__in__{k}"].copy()) for k in c["fields"]}
        out = torch.from_numpy(np.asarray(data[f"{c['name']}__out"]).copy())
        cases.append(dict(c, inputs=fields, expected=out))
    return cases


def rel_err(got, ref):
    got = got.to(torch.float64).cpu()
    ref = ref.to(torch.float64).cpu()
    scale = ref.abs().max().item() if ref.numel() else 1.0
    if scale == 0.0:
        scale = 1.0
    return (got - ref).abs().max().item() / scale

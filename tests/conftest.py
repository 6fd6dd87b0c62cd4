import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
for p in (REPO, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_collection_modifyitems(session, config, items):
    """Before any GPU test runs, compile the kernels the selected GPU tests need
    into the on-disk NVRTC cache with a spawn-started pool (no CUDA state exists
    yet at collection time). Sources already cached cost nothing."""
    if os.environ.get("STENPY_TEST_PREWARM", "1") == "0":
        return
    if not any(item.get_closest_marker("gpu") for item in items):
        return
    import torch
    if not torch.cuda.is_available():
        return
    import kernel_sources
    from stenpy_b200.prewarm import compile_all
    compile_all(kernel_sources.all_sources())

"""Loader for the unmodified reference implementation — TEST/BENCH INFRASTRUCTURE ONLY.

The reference (Stenpy) is pure Python. ``bench.py --impl reference`` times its own
CPU eager path — ``compile_expression`` + ``Runtime(MemoryManager(), device="cpu")``
(stenpy_engine.py:3762, 945, 983-1146) — on the host cores, and
``tests/golden/make_golden.py`` runs it to produce golden vectors. Only those two
and ``tests/`` import this module; the product package never does.

Where the reference comes from: a directory holding its modules
(``stenpy_engine.py`` and the modules it imports). ``bench.py`` uses the copy
installed into ``baseline/_ref`` (``pip install --target baseline/_ref`` from a copy
of the reference with a packaging file added; the sources are not changed), which
travels with the repository to the GPU machine.

The reference imports ``h5py`` (stenpy_engine.py:14) and ``zict``
(memory_manager.py:230-233) unconditionally; neither is installed and neither is
on the in-memory CPU path, so minimal stand-ins are registered first when the
real packages are absent: ``h5py.File`` raises, ``zict`` mappings are plain dicts.
"""
from __future__ import annotations

import os
import sys
import types
from typing import Optional

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INSTALLED = os.path.join(REPO, "baseline", "_ref")


def install_stand_ins() -> None:
    try:
        import h5py  # noqa: F401
    except ImportError:
        h5 = types.ModuleType("h5py")

        class _NoFile:
            def __init__(self, *a, **k):
                raise OSError("h5py stand-in: HDF5 is not available in this harness")

        h5.File = _NoFile
        h5.Dataset = type("Dataset", (), {})
        sys.modules["h5py"] = h5
    try:
        import zict  # noqa: F401
    except ImportError:
        zict = types.ModuleType("zict")

        class _Map(dict):
            def __init__(self, *a, **k):
                super().__init__()

        zict.File = _Map
        zict.Func = _Map
        zict.Buffer = _Map
        sys.modules["zict"] = zict


def load_engine(ref_dir: Optional[str] = None):
    """The reference's ``stenpy_engine`` module, imported from ``ref_dir`` (default:
    the ``baseline/_ref`` install). Raises ImportError when it is not there."""
    d = ref_dir or INSTALLED
    if not os.path.isfile(os.path.join(d, "stenpy_engine.py")):
        raise ImportError(f"reference not installed at {d}")
    install_stand_ins()
    sys.dont_write_bytecode = True
    if d not in sys.path:
        sys.path.insert(0, d)
    import stenpy_engine  # the reference
    return stenpy_engine

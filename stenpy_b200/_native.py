"""ctypes binding of libstenpy_b200.so (the C ABI in include/stenpy_b200.h).

There is no CPU fallback: if the library is missing, every entry point raises
``NativeUnavailable`` with the build command. Kernel CUBINs produced by NVRTC are
cached on disk, keyed by a hash of the generated source, the compile options and
the NVRTC version (``STENPY_JIT_CACHE``, default ``<package>/_jit_cache``), and
loaded modules are cached per device in memory.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import threading
from typing import Dict, Optional, Sequence, Tuple

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libstenpy_b200.so")
CACHE_DIR = os.environ.get("STENPY_JIT_CACHE", os.path.join(_PKG, "_jit_cache"))

ABI_SYMBOLS = (
    "stenpy_abi_version", "stenpy_last_error", "stenpy_nvrtc_version", "stenpy_device_props",
    "stenpy_nvrtc_compile", "stenpy_free", "stenpy_module_load", "stenpy_module_free",
    "stenpy_launch", "stenpy_encode_tmap_3d", "stenpy_finalize", "stenpy_pass_noalloc",
    "stenpy_mlp_param_count", "stenpy_mlp_workspace_floats", "stenpy_mlp_forward", "stenpy_mlp_loss_grad",
    "stenpy_adam_step", "stenpy_module_info",
)


class NativeUnavailable(RuntimeError):
    pass


class NativeError(RuntimeError):
    pass


class ReduceDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("slot", ctypes.c_int32), ("out_index", ctypes.c_int32),
                ("unbiased", ctypes.c_int32), ("count", ctypes.c_double), ("eps", ctypes.c_double)]


class LaunchDesc(ctypes.Structure):
    _fields_ = [("module", ctypes.c_void_p), ("grid", ctypes.c_uint32 * 3), ("block", ctypes.c_uint32 * 3),
                ("dyn_smem", ctypes.c_uint32), ("part_offset", ctypes.c_uint32),
                ("cta_off_offset", ctypes.c_uint32), ("params", ctypes.c_void_p), ("params_bytes", ctypes.c_size_t)]


NOALLOC_MAX_PARTIALS = 1 << 19

RED_SUM, RED_MEAN, RED_NORM_L2, RED_VARIANCE, RED_ENTROPY, RED_INTEGRATE, RED_MIN_MAX, RED_COVARIANCE, \
    RED_CORRELATION = range(9)
MAX_REDUCTIONS = 32

_lib: Optional[ctypes.CDLL] = None
_lock = threading.Lock()
_modules: Dict[Tuple[str, int], int] = {}


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise NativeUnavailable(
                f"{LIB_PATH} is missing: build it with `python -m stenpy_b200.csrc.build` "
                "(the executor has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        c = ctypes
        L.stenpy_abi_version.restype = c.c_int
        L.stenpy_last_error.restype = c.c_char_p
        L.stenpy_nvrtc_version.restype = c.c_int
        L.stenpy_device_props.argtypes = [c.c_int] + [c.POINTER(c.c_int)] * 4
        L.stenpy_nvrtc_compile.argtypes = [c.c_char_p, c.c_char_p, c.POINTER(c.c_void_p),
                                           c.POINTER(c.c_size_t), c.POINTER(c.c_void_p)]
        L.stenpy_free.argtypes = [c.c_void_p]
        L.stenpy_free.restype = None
        L.stenpy_module_load.argtypes = [c.c_void_p, c.c_size_t, c.c_char_p, c.c_int, c.POINTER(c.c_void_p)]
        L.stenpy_module_free.argtypes = [c.c_void_p]
        L.stenpy_module_info.argtypes = [c.c_void_p, c.c_int, c.c_int] + [c.POINTER(c.c_int)] * 3
        L.stenpy_module_free.restype = None
        L.stenpy_launch.argtypes = [c.c_void_p] + [c.c_uint] * 7 + [c.c_void_p, c.c_void_p, c.c_size_t]
        L.stenpy_encode_tmap_3d.argtypes = [c.c_void_p, c.c_int, c.c_void_p, c.c_uint64, c.c_uint64,
                                            c.c_uint64, c.c_uint64, c.c_uint64, c.c_uint32, c.c_uint32,
                                            c.c_uint32]
        L.stenpy_finalize.argtypes = [c.c_void_p, c.c_int, c.c_int, c.POINTER(ReduceDesc), c.c_int,
                                      c.c_void_p, c.c_void_p]
        L.stenpy_pass_noalloc.argtypes = [c.POINTER(LaunchDesc), c.c_int, c.c_int, c.c_int,
                                          c.POINTER(ReduceDesc), c.c_int, c.c_void_p, c.c_void_p]
        L.stenpy_mlp_param_count.argtypes = [c.c_int, c.c_int]
        L.stenpy_mlp_workspace_floats.argtypes = [c.c_int, c.c_int]
        L.stenpy_mlp_forward.argtypes = [c.c_void_p, c.c_int, c.c_int, c.c_void_p, c.c_int, c.c_void_p,
                                         c.c_void_p, c.c_void_p]
        L.stenpy_mlp_loss_grad.argtypes = [c.c_void_p, c.c_int, c.c_int, c.c_void_p, c.c_void_p, c.c_int,
                                           c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
        L.stenpy_adam_step.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p, c.c_int, c.c_float,
                                       c.c_float, c.c_float, c.c_float, c.c_int, c.c_float, c.c_void_p]
        for name in ABI_SYMBOLS:
            if not hasattr(L, name):
                raise NativeUnavailable(f"{LIB_PATH} lacks {name}; rebuild it")
        if L.stenpy_abi_version() != 2:
            raise NativeUnavailable("libstenpy_b200.so ABI version mismatch; rebuild it")
        _lib = L
        return L


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().stenpy_last_error().decode(errors="replace")
        raise NativeError(f"{what}: {msg} (code {rc})")


def device_props(device: int) -> Tuple[int, int, int, int]:
    v = [ctypes.c_int() for _ in range(4)]
    _check(lib().stenpy_device_props(device, *[ctypes.byref(x) for x in v]), "device_props")
    return tuple(x.value for x in v)  # sm_count, major, minor, smem_optin


def nvrtc_compile(source: str, options: Sequence[str]) -> bytes:
    L = lib()
    out = ctypes.c_void_p()
    size = ctypes.c_size_t()
    log = ctypes.c_void_p()
    rc = L.stenpy_nvrtc_compile(source.encode(), "\n".join(options).encode(), ctypes.byref(out),
                                ctypes.byref(size), ctypes.byref(log))
    if log.value:
        L.stenpy_free(log)
    _check(rc, "nvrtc_compile")
    try:
        return ctypes.string_at(out.value, size.value)
    finally:
        L.stenpy_free(out)


def compile_cached(source: str, options: Sequence[str]) -> Tuple[str, bytes]:
    """CUBIN for ``source``; compiled once per (source, options, NVRTC version)."""
    ver = lib().stenpy_nvrtc_version()
    key = hashlib.sha256(("\0".join([source, *options, str(ver)])).encode()).hexdigest()[:32]
    path = os.path.join(CACHE_DIR, key + ".cubin")
    if os.path.exists(path):
        with open(path, "rb") as fh:
            return key, fh.read()
    cubin = nvrtc_compile(source, options)
    try:
        os.makedirs(CACHE_DIR, exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "wb") as fh:
            fh.write(cubin)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only cache only costs a recompile
    return key, cubin


def load_module(key: str, cubin: bytes, kernel_name: str, dyn_smem_max: int, device: int) -> int:
    with _lock:
        h = _modules.get((key, device))
        if h is not None:
            return h
    out = ctypes.c_void_p()
    _check(lib().stenpy_module_load(cubin, len(cubin), kernel_name.encode(), int(dyn_smem_max),
                                    ctypes.byref(out)), "module_load")
    with _lock:
        _modules[(key, device)] = out.value
    return out.value


def unload_module(key: str, device: int) -> None:
    """Release a loaded module (the caller guarantees no launch of it is pending)."""
    with _lock:
        h = _modules.pop((key, device), None)
    if h is not None:
        lib().stenpy_module_free(h)


def module_info(module: int, block_threads: int, dyn_smem: int) -> Tuple[int, int, int]:
    """(resident blocks per SM, registers per thread, local bytes per thread)."""
    b, r, loc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().stenpy_module_info(module, int(block_threads), int(dyn_smem), ctypes.byref(b), ctypes.byref(r),
                                    ctypes.byref(loc)), "module_info")
    return b.value, r.value, loc.value


def launch(module: int, grid: Tuple[int, int, int], block: Tuple[int, int, int], dyn_smem: int,
           stream: int, params: bytes) -> None:
    buf = ctypes.create_string_buffer(params, len(params))
    _check(lib().stenpy_launch(module, grid[0], grid[1], grid[2], block[0], block[1], block[2],
                               int(dyn_smem), ctypes.c_void_p(stream), buf, len(params)), "launch")


def encode_tmap_3d(elem_bytes: int, base: int, x: int, y: int, z: int, row_bytes: int,
                   plane_bytes: int, box: Tuple[int, int, int]) -> bytes:
    out = ctypes.create_string_buffer(128)
    _check(lib().stenpy_encode_tmap_3d(out, elem_bytes, ctypes.c_void_p(base), x, y, z, row_bytes,
                                       plane_bytes, box[0], box[1], box[2]), "encode_tmap_3d")
    return out.raw


def finalize(partials_ptr: int, ncta: int, nslots: int, descs: Sequence[ReduceDesc], scalars_ptr: int,
             stream: int) -> None:
    arr = (ReduceDesc * len(descs))(*descs)
    _check(lib().stenpy_finalize(ctypes.c_void_p(partials_ptr), ncta, nslots, arr, len(descs),
                                 ctypes.c_void_p(scalars_ptr), ctypes.c_void_p(stream)), "finalize")


def pass_noalloc(launches, ncta_total: int, nslots: int, descs: Sequence[ReduceDesc], scalars_ptr: int,
                 stream: int) -> None:
    """Run one fused reduction pass with the library's static partials array (no
    device allocation). ``launches``: (module, grid, block, dyn_smem, params bytes,
    byte offset of the partials pointer in params, byte offset of the int32
    ``cta_off`` (first partial row) in params)."""
    keep = []
    arr = (LaunchDesc * len(launches))()
    for d, (module, grid, block, smem, params, part_offset, cta_off_offset) in zip(arr, launches):
        buf = ctypes.create_string_buffer(params, len(params))
        keep.append(buf)
        d.module = module
        d.grid[:] = list(grid)
        d.block[:] = list(block)
        d.dyn_smem = smem
        d.part_offset = part_offset
        d.cta_off_offset = cta_off_offset
        d.params = ctypes.cast(buf, ctypes.c_void_p)
        d.params_bytes = len(params)
    rd = (ReduceDesc * len(descs))(*descs)
    _check(lib().stenpy_pass_noalloc(arr, len(launches), ncta_total, nslots, rd, len(descs),
                                     ctypes.c_void_p(scalars_ptr), ctypes.c_void_p(stream)), "pass_noalloc")


def mlp_param_count(in_dim: int, hidden: int) -> int:
    return int(lib().stenpy_mlp_param_count(in_dim, hidden))


def mlp_workspace_floats(n: int, hidden: int) -> int:
    return int(lib().stenpy_mlp_workspace_floats(n, hidden))


def mlp_forward(params: int, in_dim: int, hidden: int, X: int, n: int, out: int, ws: int, stream: int) -> None:
    v = ctypes.c_void_p
    _check(lib().stenpy_mlp_forward(v(params), in_dim, hidden, v(X), n, v(out), v(ws), v(stream)), "mlp_forward")


def mlp_loss_grad(params: int, in_dim: int, hidden: int, X: int, target: int, n: int, grad: int, loss: int,
                  ws: int, stream: int) -> None:
    v = ctypes.c_void_p
    _check(lib().stenpy_mlp_loss_grad(v(params), in_dim, hidden, v(X), v(target), n, v(grad), v(loss), v(ws),
                                      v(stream)), "mlp_loss_grad")


def adam_step(params: int, grad: int, m: int, vv: int, n: int, lr: float, b1: float, b2: float, eps: float,
              step: int, wd: float, stream: int) -> None:
    v = ctypes.c_void_p
    _check(lib().stenpy_adam_step(v(params), v(grad), v(m), v(vv), n, lr, b1, b2, eps, step, wd, v(stream)),
           "adam_step")

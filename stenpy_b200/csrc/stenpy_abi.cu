// stenpy_abi.cu — libstenpy_b200.so: the C ABI declared in include/stenpy_b200.h.
//
// * NVRTC compilation of generated kernels to sm_100a CUBINs,
// * module loading / launching through the CUDA driver API, resolved lazily with
//   dlopen so the library also loads on hosts without a driver (symbol checks),
// * 3-D TMA descriptor encoding (cuTensorMapEncodeTiled),
// * the deterministic FP64 reduction-finalize kernel (compiled ahead of time).
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/stenpy_b200.h"

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

static int fail(int code, const char* fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

// ------------------------------------------------------------------ lazy driver API
namespace {
struct Driver {
  bool loaded = false;
  std::string why;
  CUresult (*Init)(unsigned) = nullptr;
  CUresult (*CtxGetCurrent)(CUcontext*) = nullptr;
  CUresult (*CtxSetCurrent)(CUcontext) = nullptr;
  CUresult (*DeviceGet)(CUdevice*, int) = nullptr;
  CUresult (*DevicePrimaryCtxRetain)(CUcontext*, CUdevice) = nullptr;
  CUresult (*DeviceGetAttribute)(int*, CUdevice_attribute, CUdevice) = nullptr;
  CUresult (*ModuleLoadData)(CUmodule*, const void*) = nullptr;
  CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*ModuleUnload)(CUmodule) = nullptr;
  CUresult (*FuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*FuncGetAttribute)(int*, CUfunction_attribute, CUfunction) = nullptr;
  CUresult (*OccupancyMaxActiveBlocksPerMultiprocessor)(int*, CUfunction, int, size_t) = nullptr;
  CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned,
                           unsigned, unsigned, CUstream, void**, void**) = nullptr;
  CUresult (*TensorMapEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill) = nullptr;
  CUresult (*GetErrorString)(CUresult, const char**) = nullptr;
};

Driver g_drv;
std::once_flag g_drv_once;

template <typename F>
bool bind(void* h, const char* name, F& fn) {
  fn = reinterpret_cast<F>(dlsym(h, name));
  return fn != nullptr;
}

void load_driver() {
  void* h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libcuda.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) { g_drv.why = "libcuda.so.1 not found (no NVIDIA driver on this host)"; return; }
  bool ok = bind(h, "cuInit", g_drv.Init) && bind(h, "cuCtxGetCurrent", g_drv.CtxGetCurrent) &&
            bind(h, "cuCtxSetCurrent", g_drv.CtxSetCurrent) && bind(h, "cuDeviceGet", g_drv.DeviceGet) &&
            bind(h, "cuDevicePrimaryCtxRetain", g_drv.DevicePrimaryCtxRetain) &&
            bind(h, "cuDeviceGetAttribute", g_drv.DeviceGetAttribute) &&
            bind(h, "cuModuleLoadData", g_drv.ModuleLoadData) &&
            bind(h, "cuModuleGetFunction", g_drv.ModuleGetFunction) &&
            bind(h, "cuModuleUnload", g_drv.ModuleUnload) &&
            bind(h, "cuFuncSetAttribute", g_drv.FuncSetAttribute) &&
            bind(h, "cuFuncGetAttribute", g_drv.FuncGetAttribute) &&
            bind(h, "cuOccupancyMaxActiveBlocksPerMultiprocessor", g_drv.OccupancyMaxActiveBlocksPerMultiprocessor) &&
            bind(h, "cuLaunchKernel", g_drv.LaunchKernel) &&
            bind(h, "cuTensorMapEncodeTiled", g_drv.TensorMapEncodeTiled) &&
            bind(h, "cuGetErrorString", g_drv.GetErrorString);
  if (!ok) { g_drv.why = "libcuda.so.1 lacks a required entry point"; return; }
  if (g_drv.Init(0) != CUDA_SUCCESS) { g_drv.why = "cuInit failed"; return; }
  g_drv.loaded = true;
}

int need_driver() {
  std::call_once(g_drv_once, load_driver);
  if (!g_drv.loaded) return fail(STENPY_E_DRIVER, "CUDA driver unavailable: %s", g_drv.why.c_str());
  return STENPY_OK;
}

int drv_fail(CUresult r, const char* what) {
  const char* s = "?";
  if (g_drv.GetErrorString) g_drv.GetErrorString(r, &s);
  return fail(STENPY_E_DRIVER, "%s failed: %s (%d)", what, s ? s : "?", (int)r);
}

// Make sure a context is current on this thread: the caller's (PyTorch's) if any,
// else the primary context of the runtime's current device.
int ensure_context() {
  int rc = need_driver();
  if (rc) return rc;
  CUcontext ctx = nullptr;
  CUresult r = g_drv.CtxGetCurrent(&ctx);
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuCtxGetCurrent");
  if (ctx) return STENPY_OK;
  int dev_ord = 0;
  cudaGetDevice(&dev_ord);
  CUdevice dev;
  if ((r = g_drv.DeviceGet(&dev, dev_ord)) != CUDA_SUCCESS) return drv_fail(r, "cuDeviceGet");
  if ((r = g_drv.DevicePrimaryCtxRetain(&ctx, dev)) != CUDA_SUCCESS) return drv_fail(r, "cuDevicePrimaryCtxRetain");
  if ((r = g_drv.CtxSetCurrent(ctx)) != CUDA_SUCCESS) return drv_fail(r, "cuCtxSetCurrent");
  return STENPY_OK;
}
}  // namespace

struct StenModule {
  CUmodule mod = nullptr;
  CUfunction fn = nullptr;
};

extern "C" {

// Lets other translation units of the library report errors through stenpy_last_error.
void sten_internal_set_error(const char* msg) { g_last_error = msg ? msg : ""; }

// The context launches go to (the caller's current one, else the primary context of
// the runtime's current device, made current), for per-context caches elsewhere.
int sten_internal_current_context(void** out) {
  int rc = ensure_context();
  if (rc) return rc;
  CUcontext c = nullptr;
  CUresult r = g_drv.CtxGetCurrent(&c);
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuCtxGetCurrent");
  *out = (void*)c;
  return STENPY_OK;
}

int stenpy_abi_version(void) { return STENPY_ABI_VERSION; }

const char* stenpy_last_error(void) { return g_last_error.c_str(); }

int stenpy_nvrtc_version(void) {
  int major = 0, minor = 0;
  if (nvrtcVersion(&major, &minor) != NVRTC_SUCCESS) return 0;
  return major * 1000 + minor * 10;
}

int stenpy_device_props(int device, int* sm_count, int* cc_major, int* cc_minor, int* smem_optin) {
  int rc = need_driver();
  if (rc) return rc;
  CUdevice dev;
  CUresult r = g_drv.DeviceGet(&dev, device);
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuDeviceGet");
  if (sm_count) g_drv.DeviceGetAttribute(sm_count, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev);
  if (cc_major) g_drv.DeviceGetAttribute(cc_major, CU_DEVICE_ATTRIBUTE_COMPUTE_CAPABILITY_MAJOR, dev);
  if (cc_minor) g_drv.DeviceGetAttribute(cc_minor, CU_DEVICE_ATTRIBUTE_COMPUTE_CAPABILITY_MINOR, dev);
  if (smem_optin) g_drv.DeviceGetAttribute(smem_optin, CU_DEVICE_ATTRIBUTE_MAX_SHARED_MEMORY_PER_BLOCK_OPTIN, dev);
  return STENPY_OK;
}

int stenpy_nvrtc_compile(const char* source, const char* options, void** cubin, size_t* cubin_size,
                         char** log) {
  if (!source || !cubin || !cubin_size) return fail(STENPY_E_INVALID, "nvrtc_compile: null argument");
  *cubin = nullptr;
  *cubin_size = 0;
  if (log) *log = nullptr;
  std::vector<std::string> opts;
  if (options) {
    std::string all(options), cur;
    for (char c : all) {
      if (c == '\n') { if (!cur.empty()) opts.push_back(cur); cur.clear(); }
      else cur.push_back(c);
    }
    if (!cur.empty()) opts.push_back(cur);
  }
  std::vector<const char*> argv;
  for (auto& o : opts) argv.push_back(o.c_str());

  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, source, "sten_kernel.cu", 0, nullptr, nullptr);
  if (r != NVRTC_SUCCESS) return fail(STENPY_E_NVRTC, "nvrtcCreateProgram: %s", nvrtcGetErrorString(r));
  r = nvrtcCompileProgram(prog, (int)argv.size(), argv.data());
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  std::string text(log_size > 1 ? log_size : 1, '\0');
  if (log_size > 1) nvrtcGetProgramLog(prog, &text[0]);
  if (log && log_size > 1) {
    *log = (char*)malloc(log_size);
    memcpy(*log, text.data(), log_size);
  }
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return fail(STENPY_E_NVRTC, "nvrtc compile failed: %s\n%.1500s", nvrtcGetErrorString(r), text.c_str());
  }
  size_t n = 0;
  r = nvrtcGetCUBINSize(prog, &n);
  if (r != NVRTC_SUCCESS || n == 0) {
    nvrtcDestroyProgram(&prog);
    return fail(STENPY_E_NVRTC, "nvrtcGetCUBINSize: %s (a real sm_ architecture must be requested)",
                nvrtcGetErrorString(r));
  }
  void* buf = malloc(n);
  r = nvrtcGetCUBIN(prog, (char*)buf);
  nvrtcDestroyProgram(&prog);
  if (r != NVRTC_SUCCESS) { free(buf); return fail(STENPY_E_NVRTC, "nvrtcGetCUBIN: %s", nvrtcGetErrorString(r)); }
  *cubin = buf;
  *cubin_size = n;
  return STENPY_OK;
}

void stenpy_free(void* p) { free(p); }

int stenpy_module_load(const void* cubin, size_t cubin_size, const char* kernel_name, int dyn_smem_max,
                       StenModule** out) {
  if (!cubin || !cubin_size || !kernel_name || !out) return fail(STENPY_E_INVALID, "module_load: null argument");
  int rc = ensure_context();
  if (rc) return rc;
  StenModule* m = new StenModule();
  CUresult r = g_drv.ModuleLoadData(&m->mod, cubin);
  if (r != CUDA_SUCCESS) { delete m; return drv_fail(r, "cuModuleLoadData"); }
  r = g_drv.ModuleGetFunction(&m->fn, m->mod, kernel_name);
  if (r != CUDA_SUCCESS) { g_drv.ModuleUnload(m->mod); delete m; return drv_fail(r, "cuModuleGetFunction"); }
  if (dyn_smem_max > 48 * 1024) {
    r = g_drv.FuncSetAttribute(m->fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, dyn_smem_max);
    if (r != CUDA_SUCCESS) { g_drv.ModuleUnload(m->mod); delete m; return drv_fail(r, "cuFuncSetAttribute"); }
  }
  *out = m;
  return STENPY_OK;
}

int stenpy_module_info(StenModule* m, int block_threads, int dyn_smem, int* blocks_per_sm, int* regs,
                       int* local_bytes) {
  if (!m || !m->fn || !blocks_per_sm || !regs || !local_bytes) return fail(STENPY_E_INVALID, "module_info: null argument");
  if (block_threads <= 0 || block_threads > 1024 || dyn_smem < 0) return fail(STENPY_E_INVALID, "module_info: bad block");
  int rc = ensure_context();
  if (rc) return rc;
  CUresult r = g_drv.OccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, m->fn, block_threads, (size_t)dyn_smem);
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
  if ((r = g_drv.FuncGetAttribute(regs, CU_FUNC_ATTRIBUTE_NUM_REGS, m->fn)) != CUDA_SUCCESS)
    return drv_fail(r, "cuFuncGetAttribute");
  if ((r = g_drv.FuncGetAttribute(local_bytes, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, m->fn)) != CUDA_SUCCESS)
    return drv_fail(r, "cuFuncGetAttribute");
  return STENPY_OK;
}

void stenpy_module_free(StenModule* m) {
  if (!m) return;
  if (g_drv.loaded && m->mod) g_drv.ModuleUnload(m->mod);
  delete m;
}

int stenpy_launch(StenModule* m, unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by,
                  unsigned bz, unsigned dyn_smem, void* stream, const void* params, size_t params_bytes) {
  if (!m || !m->fn) return fail(STENPY_E_INVALID, "launch: no module");
  if (!params || params_bytes == 0 || params_bytes > 32768) return fail(STENPY_E_INVALID, "launch: bad params");
  if (gx == 0 || gy == 0 || gz == 0 || bx == 0 || by == 0 || bz == 0) return fail(STENPY_E_INVALID, "launch: empty grid");
  int rc = ensure_context();
  if (rc) return rc;
  // One by-value struct parameter: kernelParams[0] points at its bytes.
  void* args[1] = {const_cast<void*>(params)};
  CUresult r = g_drv.LaunchKernel(m->fn, gx, gy, gz, bx, by, bz, dyn_smem, (CUstream)stream, args, nullptr);
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuLaunchKernel");
  return STENPY_OK;
}

int stenpy_encode_tmap_3d(void* out128, int elem_bytes, const void* base, uint64_t x, uint64_t y, uint64_t z,
                          uint64_t row_bytes, uint64_t plane_bytes, uint32_t box_x, uint32_t box_y,
                          uint32_t box_z) {
  if (!out128 || !base) return fail(STENPY_E_INVALID, "encode_tmap: null argument");
  CUtensorMapDataType dt;
  switch (elem_bytes) {
    case 1: dt = CU_TENSOR_MAP_DATA_TYPE_UINT8; break;
    case 2: dt = CU_TENSOR_MAP_DATA_TYPE_UINT16; break;
    case 4: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; break;
    case 8: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64; break;
    default: return fail(STENPY_E_INVALID, "encode_tmap: elem_bytes %d", elem_bytes);
  }
  if (((uintptr_t)base) % 16) return fail(STENPY_E_INVALID, "encode_tmap: base not 16-byte aligned");
  if (row_bytes % 16 || plane_bytes % 16) return fail(STENPY_E_INVALID, "encode_tmap: strides must be multiples of 16");
  if ((box_x * (uint64_t)elem_bytes) % 16) return fail(STENPY_E_INVALID, "encode_tmap: box inner bytes not a multiple of 16");
  if (box_x == 0 || box_y == 0 || box_z == 0 || box_x > 256 || box_y > 256 || box_z > 256)
    return fail(STENPY_E_INVALID, "encode_tmap: box dims must be in [1, 256]");
  int rc = need_driver();
  if (rc) return rc;
  cuuint64_t dims[3] = {x, y, z};
  cuuint64_t strides[2] = {row_bytes, plane_bytes};
  cuuint32_t box[3] = {box_x, box_y, box_z};
  cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMap map;
  CUresult r = g_drv.TensorMapEncodeTiled(&map, dt, 3, const_cast<void*>(base), dims, strides, box, estr,
                                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuTensorMapEncodeTiled");
  static_assert(sizeof(CUtensorMap) == 128, "CUtensorMap size");
  memcpy(out128, &map, 128);
  return STENPY_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ reduction finalize
struct FinalizeArgs {
  StenReduceDesc d[STENPY_MAX_REDUCTIONS];
};

__device__ static void co(double* x, const double* y) {
  // co-moments (n, mean a, mean b, C, M2 a, M2 b) of two groups merged
  double nt = x[0] + y[0];
  if (nt == 0.0) return;
  double da = y[1] - x[1], db = y[2] - x[2], w = y[0] / nt, f = x[0] * w;
  x[1] += da * w; x[2] += db * w;
  x[3] += y[3] + da * db * f; x[4] += y[4] + da * da * f; x[5] += y[5] + db * db * f;
  x[0] = nt;
}

__device__ static void chan(double& n, double& m, double& q, double nb, double mb, double qb) {
  double nt = n + nb;
  if (nt == 0.0) return;
  double dd = mb - m, w = nb / nt;
  m += dd * w;
  q += qb + dd * dd * n * w;
  n = nt;
}

// One block per reduction; each thread folds a strided subset of CTA rows in order,
// then a fixed shared-memory tree combines the 256 thread results: deterministic.
__global__ void __launch_bounds__(256) sten_finalize_kernel(const double* __restrict__ part, int ncta,
                                                            int nslots, FinalizeArgs a,
                                                            double* __restrict__ out) {
  __shared__ double s0[256], s1[256], s2[256];
  __shared__ double sc[6][256];
  const StenReduceDesc d = a.d[blockIdx.x];
  const int t = threadIdx.x;
  if (d.kind == STENPY_RED_COVARIANCE || d.kind == STENPY_RED_CORRELATION) {
    // rows folded in order as below, then a fixed tree
    double x[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int c = t; c < ncta; c += 256) {
      const double* row = part + (size_t)c * nslots + d.slot;
      double y[6];
      for (int i = 0; i < 6; ++i) y[i] = row[i];
      co(x, y);
    }
    for (int i = 0; i < 6; ++i) sc[i][t] = x[i];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (t < w) {
        double xa[6], yb[6];
        for (int i = 0; i < 6; ++i) { xa[i] = sc[i][t]; yb[i] = sc[i][t + w]; }
        co(xa, yb);
        for (int i = 0; i < 6; ++i) sc[i][t] = xa[i];
      }
      __syncthreads();
    }
    if (t == 0) {
      double* o = out + d.out_index;
      const double n = sc[0][0], c = sc[3][0];
      // covariance: C / max(n - 1, 1); correlation: C / (|a - mean a| |b - mean b| + eps)
      o[0] = d.kind == STENPY_RED_COVARIANCE ? c / (n - 1.0 > 1.0 ? n - 1.0 : 1.0)
                                             : c / (sqrt(sc[4][0]) * sqrt(sc[5][0]) + d.eps);
    }
    return;
  }
  double x0 = 0.0, x1 = 0.0, x2 = 0.0;
  if (d.kind == STENPY_RED_MIN_MAX) { x0 = INFINITY; x1 = -INFINITY; }
  // rows t, t + 256, ... folded in that order; the loads of up to FOLD_U rows are
  // issued before their folds so that their latencies overlap, the last group's
  // only for the rows that exist (the order, and so the result, is the same as one
  // row at a time)
  const int width = d.kind == STENPY_RED_VARIANCE ? 3 : (d.kind == STENPY_RED_ENTROPY || d.kind == STENPY_RED_MIN_MAX ? 2 : 1);
  constexpr int FOLD_U = 16;
  for (int c = t; c < ncta; c += FOLD_U * 256) {
    double v[FOLD_U][3];
#pragma unroll
    for (int u = 0; u < FOLD_U; ++u) {
      v[u][0] = v[u][1] = v[u][2] = 0.0;
      if (c + u * 256 < ncta) {
        const double* row = part + (size_t)(c + u * 256) * nslots + d.slot;
        v[u][0] = row[0];
        if (width > 1) v[u][1] = row[1];
        if (width > 2) v[u][2] = row[2];
      }
    }
#pragma unroll
    for (int u = 0; u < FOLD_U; ++u) {
      if (c + u * 256 >= ncta) break;
      switch (d.kind) {
        case STENPY_RED_VARIANCE: chan(x0, x1, x2, v[u][0], v[u][1], v[u][2]); break;
        case STENPY_RED_ENTROPY: x0 += v[u][0]; x1 += v[u][1]; break;
        case STENPY_RED_MIN_MAX: x0 = fmin(x0, v[u][0]); x1 = fmax(x1, v[u][1]); break;
        default: x0 += v[u][0]; break;
      }
    }
  }
  s0[t] = x0; s1[t] = x1; s2[t] = x2;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) {
      switch (d.kind) {
        case STENPY_RED_VARIANCE: chan(s0[t], s1[t], s2[t], s0[t + w], s1[t + w], s2[t + w]); break;
        case STENPY_RED_ENTROPY: s0[t] += s0[t + w]; s1[t] += s1[t + w]; break;
        case STENPY_RED_MIN_MAX: s0[t] = fmin(s0[t], s0[t + w]); s1[t] = fmax(s1[t], s1[t + w]); break;
        default: s0[t] += s0[t + w]; break;
      }
    }
    __syncthreads();
  }
  if (t != 0) return;
  double* o = out + d.out_index;
  switch (d.kind) {
    case STENPY_RED_SUM:
    case STENPY_RED_INTEGRATE: o[0] = s0[0]; break;
    case STENPY_RED_MEAN: o[0] = s0[0] / d.count; break;
    case STENPY_RED_NORM_L2: o[0] = sqrt(s0[0]); break;
    case STENPY_RED_VARIANCE: {
      double n = s0[0], den = d.unbiased ? (n - 1.0 > 1.0 ? n - 1.0 : 1.0) : (n > 1.0 ? n : 1.0);
      o[0] = s2[0] / den;
      break;
    }
    case STENPY_RED_ENTROPY: {
      // p = |x| / (S + eps); -sum p log p = (S log(S + eps) - sum |x| log|x|) / (S + eps)
      double S = s0[0], T = s1[0], Z = S + d.eps;
      o[0] = (S * log(Z) - T) / Z;
      break;
    }
    case STENPY_RED_MIN_MAX: o[0] = s0[0]; o[1] = s1[0]; break;
  }
}

extern "C" int stenpy_finalize(const double* partials, int ncta, int nslots, const StenReduceDesc* descs,
                               int nred, double* scalars, void* stream) {
  if (!partials || !descs || !scalars) return fail(STENPY_E_INVALID, "finalize: null argument");
  if (nred <= 0 || nred > STENPY_MAX_REDUCTIONS) return fail(STENPY_E_INVALID, "finalize: nred %d", nred);
  if (ncta <= 0 || nslots <= 0) return fail(STENPY_E_INVALID, "finalize: empty partials");
  FinalizeArgs a;
  memset(&a, 0, sizeof a);
  for (int i = 0; i < nred; ++i) {
    // every slot the kernel folds for this kind must lie inside the row
    const int k = descs[i].kind;
    if (k < STENPY_RED_SUM || k > STENPY_RED_CORRELATION) return fail(STENPY_E_INVALID, "finalize: kind %d", k);
    const int width = k == STENPY_RED_VARIANCE ? 3
                    : (k == STENPY_RED_ENTROPY || k == STENPY_RED_MIN_MAX) ? 2
                    : (k == STENPY_RED_COVARIANCE || k == STENPY_RED_CORRELATION) ? 6 : 1;
    if (descs[i].slot < 0 || descs[i].slot + width > nslots)
      return fail(STENPY_E_INVALID, "finalize: slots %d..%d of kind %d outside rows of %d", descs[i].slot,
                  descs[i].slot + width - 1, k, nslots);
    a.d[i] = descs[i];
  }
  sten_finalize_kernel<<<nred, 256, 0, (cudaStream_t)stream>>>(partials, ncta, nslots, a, scalars);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(STENPY_E_RUNTIME, "finalize launch: %s", cudaGetErrorString(e));
  return STENPY_OK;
}

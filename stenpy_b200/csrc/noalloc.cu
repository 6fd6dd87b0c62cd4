// noalloc.cu — the allocation-free variant of a fused reduction pass.
//
// A fused pass that computes global reductions writes one row of FP64 partials per
// CTA to scratch memory and then folds the rows into scalars (stenpy_launch +
// stenpy_finalize, with the partials buffer allocated by the caller). Some callers
// cannot allocate device memory at all: a host application that hands the library
// one pre-sized arena and forbids any further cudaMalloc, code that runs while
// another component owns the device allocator, or a latency-critical loop where
// cudaMalloc/cudaFree would synchronise the device. For them,
// stenpy_pass_noalloc runs the same launches with the partials placed in the
// file-scope array below, so the call itself allocates nothing.
//
// The array (STENPY_NOALLOC_MAX_PARTIALS doubles, 4 MiB) exists once per device
// that loads the library and stays allocated until the process exits. Its device
// address is looked up with cudaGetSymbolAddress the first time the entry point is
// called on a device, with that device current, and kept for that device's
// context: a call from another context on the device (after a device reset, or a
// context the caller created) looks it up again. Make the first call on each
// device before any stream capture. All calls share the array and it keeps the
// previous call's contents: every partial row is rewritten by its CTA on each
// call, so nothing has to be cleared, but two calls that overlap on the same GPU
// (for example issued on two streams without ordering between them) race on it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/stenpy_b200.h"

extern "C" void sten_internal_set_error(const char* msg);       // stenpy_abi.cu
extern "C" int sten_internal_current_context(void** ctx);      // stenpy_abi.cu

static __device__ __align__(256) double g_noalloc_partials[STENPY_NOALLOC_MAX_PARTIALS];

namespace {
constexpr int kMaxDevices = 64;
struct PartialsAddr {
  void* ctx = nullptr;     // context the address belongs to
  double* addr = nullptr;  // device address of g_noalloc_partials in it
};
std::mutex g_setup_mu;
PartialsAddr g_partials[kMaxDevices];

// Host code must not use g_noalloc_partials directly: its name is a host-side
// stand-in, not the device address. Resolve the address per device and context.
int partials_for_current_device(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices) return STENPY_E_RUNTIME;
  void* ctx = nullptr;
  if (sten_internal_current_context(&ctx) != STENPY_OK || !ctx) return STENPY_E_DRIVER;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  PartialsAddr& slot = g_partials[dev];
  if (!slot.addr || slot.ctx != ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) return STENPY_E_RUNTIME;
    slot.addr = static_cast<double*>(p);
    slot.ctx = ctx;
  }
  *out = slot.addr;
  return STENPY_OK;
}
}  // namespace

extern "C" int stenpy_pass_noalloc(const StenLaunchDesc* launches, int n_launch, int ncta_total, int nslots,
                                   const StenReduceDesc* descs, int nred, double* scalars, void* stream) {
  if (!launches || n_launch <= 0 || !descs || !scalars) {
    sten_internal_set_error("pass_noalloc: null argument");
    return STENPY_E_INVALID;
  }
  if (ncta_total <= 0 || nslots <= 0 ||
      (unsigned long long)ncta_total * (unsigned long long)nslots > STENPY_NOALLOC_MAX_PARTIALS) {
    sten_internal_set_error("pass_noalloc: partials exceed the static scratch (STENPY_NOALLOC_MAX_PARTIALS doubles); "
                     "use stenpy_launch + stenpy_finalize with caller-allocated partials");
    return STENPY_E_INVALID;
  }
  // Every launch writes rows cta_off .. cta_off + (its CTAs) - 1 of nslots doubles:
  // check those rows against ncta_total before anything runs.
  for (int i = 0; i < n_launch; ++i) {
    const StenLaunchDesc& L = launches[i];
    if (!L.params || L.params_bytes > 8192 || L.part_offset + sizeof(double*) > L.params_bytes ||
        L.cta_off_offset + sizeof(int32_t) > L.params_bytes || (L.part_offset % 8) || (L.cta_off_offset % 4)) {
      sten_internal_set_error("pass_noalloc: bad parameter block");
      return STENPY_E_INVALID;
    }
    int32_t cta_off = 0;
    std::memcpy(&cta_off, static_cast<const unsigned char*>(L.params) + L.cta_off_offset, sizeof cta_off);
    const unsigned long long ctas =
        (unsigned long long)L.grid[0] * (unsigned long long)L.grid[1] * (unsigned long long)L.grid[2];
    if (cta_off < 0 || ctas == 0 || (unsigned long long)cta_off + ctas > (unsigned long long)ncta_total) {
      sten_internal_set_error("pass_noalloc: a launch's partial rows (cta_off + grid size) exceed ncta_total");
      return STENPY_E_INVALID;
    }
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    sten_internal_set_error("pass_noalloc: cudaGetDevice failed");
    return STENPY_E_RUNTIME;
  }
  int stream_dev = -1;
  if (cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &stream_dev) != cudaSuccess || stream_dev != dev) {
    sten_internal_set_error("pass_noalloc: the stream does not belong to the current device");
    return STENPY_E_INVALID;
  }
  double* part = nullptr;
  if (partials_for_current_device(dev, &part) != STENPY_OK) {
    sten_internal_set_error("pass_noalloc: cudaGetSymbolAddress of the static partials failed");
    return STENPY_E_RUNTIME;
  }
  unsigned char buf[8192];
  for (int i = 0; i < n_launch; ++i) {
    const StenLaunchDesc& L = launches[i];
    std::memcpy(buf, L.params, L.params_bytes);
    std::memcpy(buf + L.part_offset, &part, sizeof(double*));
    int rc = stenpy_launch(L.module, L.grid[0], L.grid[1], L.grid[2], L.block[0], L.block[1], L.block[2],
                           L.dyn_smem, stream, buf, L.params_bytes);
    if (rc != STENPY_OK) return rc;
  }
  return stenpy_finalize(part, ncta_total, nslots, descs, nred, scalars, stream);
}

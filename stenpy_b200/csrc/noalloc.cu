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
// called on a device, with that device current; make that first call before any
// stream capture. All calls share the array and it keeps the previous call's
// contents: every partial row is rewritten by its CTA on each call, so nothing has
// to be cleared, but two calls that overlap on the same GPU (for example issued on
// two streams without ordering between them) race on it.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/stenpy_b200.h"

extern "C" void sten_internal_set_error(const char* msg);  // stenpy_abi.cu

static __device__ __align__(256) double g_noalloc_partials[STENPY_NOALLOC_MAX_PARTIALS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_partials_addr[kMaxDevices] = {nullptr};

// Host code must not use g_noalloc_partials directly: its name is a host-side
// stand-in, not the device address. Resolve the address once per device.
int partials_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return STENPY_E_RUNTIME;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_partials_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) return STENPY_E_RUNTIME;
    g_partials_addr[dev] = static_cast<double*>(p);
  }
  *out = g_partials_addr[dev];
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
  double* part = nullptr;
  if (partials_for_current_device(&part) != STENPY_OK) {
    sten_internal_set_error("pass_noalloc: cudaGetSymbolAddress of the static partials failed");
    return STENPY_E_RUNTIME;
  }
  unsigned char buf[8192];
  for (int i = 0; i < n_launch; ++i) {
    const StenLaunchDesc& L = launches[i];
    if (!L.params || L.params_bytes > sizeof buf || L.part_offset + sizeof(double*) > L.params_bytes) {
      sten_internal_set_error("pass_noalloc: bad parameter block");
      return STENPY_E_INVALID;
    }
    std::memcpy(buf, L.params, L.params_bytes);
    std::memcpy(buf + L.part_offset, &part, sizeof(double*));
    int rc = stenpy_launch(L.module, L.grid[0], L.grid[1], L.grid[2], L.block[0], L.block[1], L.block[2],
                           L.dyn_smem, stream, buf, L.params_bytes);
    if (rc != STENPY_OK) return rc;
  }
  return stenpy_finalize(part, ncta_total, nslots, descs, nred, scalars, stream);
}

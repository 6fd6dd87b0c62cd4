/* stenpy_b200.h — C ABI of libstenpy_b200.so, the native boundary of the fused
 * stencil-graph executor.
 *
 * The reference (Stenpy) is pure Python: its fused path writes Triton source per
 * fusion group, imports it and launches it (fused_compiler.py:560-575, 595-629,
 * 744-746), and its reductions call torch and `.item()` (stenpy_engine.py:2546-2667).
 * These entry points are what a host binding needs to replace that path with
 * CUDA C++ kernels for sm_100a: compile a generated kernel, load it, launch it on a
 * caller-owned stream with a packed parameter block, encode TMA descriptors for
 * caller-owned device buffers, and finalize FP64 reduction partials on the device.
 *
 * Conventions: every function returns 0 on success and a negative STENPY_E_* code
 * on failure, with a message from stenpy_last_error() (thread-local). All device
 * memory is allocated by the caller (PyTorch in the Python host); pointers are
 * device pointers in the caller's current CUDA context. Streams are cudaStream_t /
 * CUstream handles passed as void*. No torch types cross this boundary.
 */
#ifndef STENPY_B200_H
#define STENPY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STENPY_ABI_VERSION 2

#define STENPY_OK 0
#define STENPY_E_INVALID (-1)   /* bad argument */
#define STENPY_E_DRIVER (-2)    /* CUDA driver missing or a driver call failed */
#define STENPY_E_NVRTC (-3)     /* run-time compilation failed (log in last_error) */
#define STENPY_E_RUNTIME (-4)   /* CUDA runtime call / kernel launch failed */

typedef struct StenModule StenModule;

/* ABI version (STENPY_ABI_VERSION). */
int stenpy_abi_version(void);

/* Thread-local message describing the last failure on this thread. */
const char* stenpy_last_error(void);

/* NVRTC version as major*1000 + minor*10 (part of the kernel cache key). */
int stenpy_nvrtc_version(void);

/* Device properties used for launch sizing: SM count, compute capability and
 * the opt-in shared memory limit per block (bytes). */
int stenpy_device_props(int device, int* sm_count, int* cc_major, int* cc_minor,
                        int* smem_optin);

/* Compile CUDA C++ `source` with NVRTC to a CUBIN (`options` is a '\n'-separated
 * option list, e.g. "--gpu-architecture=sm_100a\n-std=c++17"). On success
 * *cubin / *cubin_size describe a malloc'd buffer released with stenpy_free().
 * On failure the compiler log is returned in *log (also malloc'd, may be NULL).
 * Replaces TritonCodegen.emit → _compile_kernel_from_source
 * (fused_compiler.py:404-529, 560-575). */
int stenpy_nvrtc_compile(const char* source, const char* options, void** cubin,
                         size_t* cubin_size, char** log);

/* Release a buffer returned by stenpy_nvrtc_compile. */
void stenpy_free(void* p);

/* Load a CUBIN into the current context (the device's primary context when none
 * is current) and resolve `kernel_name`; `dyn_smem_max` raises the kernel's
 * dynamic shared memory limit. Replaces the import of the generated module and
 * the KernelCache entry (fused_compiler.py:531-557, 612-621). */
int stenpy_module_load(const void* cubin, size_t cubin_size, const char* kernel_name,
                       int dyn_smem_max, StenModule** out);

/* Resident blocks per SM for `block_threads` threads and `dyn_smem` bytes of
 * dynamic shared memory, registers per thread and local (spill/stack) bytes per
 * thread of the module's kernel. Sizes the persistent batch grid. New entry
 * point: the reference launches Triton kernels with fixed grids
 * (stenpy_engine.py:1961-1981) and has no persistent kernel. */
int stenpy_module_info(StenModule* m, int block_threads, int dyn_smem, int* blocks_per_sm, int* regs,
                       int* local_bytes);

/* Unload a module. */
void stenpy_module_free(StenModule* m);

/* Launch the module's kernel. The kernel takes ONE by-value struct parameter;
 * `params` points to its packed bytes (`params_bytes` long, <= 32 KiB).
 * Replaces `task.kernel[grid](*args, BLOCK_SIZE=512)` (fused_compiler.py:743-746). */
int stenpy_launch(StenModule* m, unsigned gx, unsigned gy, unsigned gz,
                  unsigned bx, unsigned by, unsigned bz, unsigned dyn_smem,
                  void* stream, const void* params, size_t params_bytes);

/* Encode a 3-D tiled TMA descriptor (128 bytes written to `out128`) for a
 * row-major array of `z` planes × `y` rows × `x` elements of `elem_bytes` each
 * (1, 2, 4 or 8; x counts elements including interleaved components), with
 * byte strides `row_bytes` (y) and `plane_bytes` (z), both multiples of 16, and a
 * base address aligned to 16 bytes. The box is box_x × box_y × box_z elements
 * (box_x * elem_bytes a multiple of 16, each box dim <= 256). Out-of-range
 * elements of a box read as zero. No counterpart in the reference (it has no TMA). */
int stenpy_encode_tmap_3d(void* out128, int elem_bytes, const void* base,
                          uint64_t x, uint64_t y, uint64_t z,
                          uint64_t row_bytes, uint64_t plane_bytes,
                          uint32_t box_x, uint32_t box_y, uint32_t box_z);

/* Reduction kinds for stenpy_finalize (partial-slot layout in parentheses). */
#define STENPY_RED_SUM 0       /* (sum x)                       -> sum        */
#define STENPY_RED_MEAN 1      /* (sum x)                       -> sum/count  */
#define STENPY_RED_NORM_L2 2   /* (sum x^2)                     -> sqrt       */
#define STENPY_RED_VARIANCE 3  /* (n, mean, M2), Chan-merged    -> M2/(n-u)   */
#define STENPY_RED_ENTROPY 4   /* (sum|x|, sum|x|log|x|)        -> entropy    */
#define STENPY_RED_INTEGRATE 5 /* (sum w x)                     -> sum        */
#define STENPY_RED_MIN_MAX 6   /* (min, max)                    -> 2 values   */
#define STENPY_RED_COVARIANCE 7  /* (n, mean a, mean b, C, M2a, M2b) -> C/(n-1)   */
#define STENPY_RED_CORRELATION 8 /* same co-moments -> C/(sqrt(M2a M2b)+eps)       */

typedef struct StenReduceDesc {
  int32_t kind;      /* STENPY_RED_* */
  int32_t slot;      /* first partial slot of this reduction */
  int32_t out_index; /* index into the scalar table */
  int32_t unbiased;  /* variance: 1 -> divide by n-1 */
  double count;      /* number of values reduced (mean) */
  double eps;        /* entropy: eps of p = |x|/(sum|x| + eps) */
} StenReduceDesc;

#define STENPY_MAX_REDUCTIONS 32

/* Combine per-CTA FP64 partials `partials[cta * nslots + slot]` (device memory,
 * `ncta` rows) into final scalars written to the device FP64 table `scalars`,
 * in a fixed order (deterministic), on `stream`. `descs` is a HOST array of
 * `nred` <= STENPY_MAX_REDUCTIONS descriptors. Replaces the torch reductions and
 * the `.item()` host round trips of sum/mean/norm_l2/variance/entropy/integrate
 * (stenpy_engine.py:2340-2459, 2546-2572, 2638-2667). */
int stenpy_finalize(const double* partials, int ncta, int nslots,
                    const StenReduceDesc* descs, int nred, double* scalars,
                    void* stream);

/* ---- schedule cost model (MLP) -----------------------------------------------
 * No counterpart in the reference, whose only schedule model is an analytic
 * arithmetic-intensity / register estimate (fused_compiler.py:20-43). A 2-hidden-
 * layer ReLU perceptron (hidden = 64) predicts a pass's log run time under a
 * schedule; it is trained on the autotuner's timings with these kernels and only
 * ranks candidate schedules. Parameters: one FP32 device buffer laid out
 * W1[in][h], b1[h], W2[h][h], b2[h], w3[h], b3. All buffers are caller-owned
 * device memory; `workspace` holds stenpy_mlp_workspace_floats(n, hidden) floats. */
int stenpy_mlp_param_count(int in_dim, int hidden);
int stenpy_mlp_workspace_floats(int n, int hidden);
/* out[n] = MLP(X[n][in_dim]). */
int stenpy_mlp_forward(const float* params, int in_dim, int hidden, const float* X, int n,
                       float* out, float* workspace, void* stream);
/* Mean squared error against target[n]: *loss (device scalar) and grad (same
 * layout as params) of the mean loss, by explicit backpropagation. */
int stenpy_mlp_loss_grad(const float* params, int in_dim, int hidden, const float* X,
                         const float* target, int n, float* grad, float* loss,
                         float* workspace, void* stream);
/* One Adam update (bias-corrected, decoupled weight decay added to the gradient). */
int stenpy_adam_step(float* params, const float* grad, float* m, float* v, int n_params,
                     float lr, float beta1, float beta2, float eps, int step,
                     float weight_decay, void* stream);

/* ---- allocation-free variant ------------------------------------------------
 * No counterpart in the reference. For hosts that cannot allocate device memory
 * (an application that owns a fixed arena and forbids further cudaMalloc, code
 * running while another component owns the allocator, latency-critical loops
 * where cudaMalloc/cudaFree would synchronise the device): runs a fused
 * reduction pass — its kernel launches, then the finalize — with the FP64
 * partials in a static device array of STENPY_NOALLOC_MAX_PARTIALS doubles
 * (4 MiB, held by every device that loads the library until exit) instead of a
 * caller-allocated buffer. Each launch's packed parameters are copied and the
 * partials pointer at byte offset `part_offset` is replaced by the static
 * array's device address. That address is looked up on the first call on a
 * device (so make that call before any stream capture) and kept per device and
 * context: a call from a different context on the device, for example after a
 * device reset, looks it up again.
 *
 * Sizes: a launch writes partial rows cta_off .. cta_off + gx*gy*gz - 1, where
 * cta_off is the int32 at byte offset `cta_off_offset` of its params, each row
 * `nslots` doubles wide. `nslots` must equal the row width the kernels were
 * generated with (the pass's NSLOTS_RED); every launch's rows must lie below
 * `ncta_total`, and ncta_total * nslots must not exceed the maximum: otherwise
 * the call fails with STENPY_E_INVALID before launching anything. The stream
 * must belong to the current device (STENPY_E_INVALID otherwise). Calls share
 * the array: every partial row is rewritten each call, but calls that overlap
 * on one GPU race. */
#define STENPY_NOALLOC_MAX_PARTIALS (1u << 19)

typedef struct StenLaunchDesc {
  StenModule* module;
  uint32_t grid[3];
  uint32_t block[3];
  uint32_t dyn_smem;
  uint32_t part_offset;    /* byte offset of the partials pointer in params (8-aligned) */
  uint32_t cta_off_offset; /* byte offset of the int32 first partial row in params */
  const void* params;      /* packed kernel parameters (<= 8 KiB) */
  size_t params_bytes;
} StenLaunchDesc;

int stenpy_pass_noalloc(const StenLaunchDesc* launches, int n_launch, int ncta_total, int nslots,
                        const StenReduceDesc* descs, int nred, double* scalars, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* STENPY_B200_H */

// sten_device.cuh — device-side building blocks for the per-graph stencil kernels.
//
// The code generator (stenpy_b200/codegen.py) prepends this header to every kernel it
// emits; kernels are compiled at run time with NVRTC for sm_100a. The header is
// self-contained (no CUDA headers), so NVRTC needs no include path.
//
// Contents
//   * storage-dtype loads/stores (fp32, bf16, fp16, fp64) — compute is always fp32
//   * mbarrier + TMA (cp.async.bulk.tensor, no multicast) plane loads with bounded waits
//   * boundary index helpers for periodic / replicate / zero / reflect padding
//   * fp64 block reductions: sum, Chan-merged (n, mean, M2), min/max
//   * closed-form symmetric 3x3 eigenvalues (trigonometric method of O. K. Smith,
//     "Eigenvalues of a symmetric 3x3 matrix", CACM 4(4):168, 1961) in fp32 with an
//     fp64 re-evaluation when the spread of the spectrum is small against its centre.
#pragma once

typedef unsigned long long u64;
typedef long long i64;
typedef unsigned int u32;
typedef unsigned short u16;

#define STEN_DEV __device__ __forceinline__

// ------------------------------------------------------------------ dtype I/O
struct bf16_t { u16 bits; };
struct f16_t { u16 bits; };

STEN_DEV float ld_as_f32(const float* p) { return *p; }
STEN_DEV float ld_as_f32(const double* p) { return (float)(*p); }
STEN_DEV float ld_as_f32(const bf16_t* p) { return __int_as_float(((u32)p->bits) << 16); }
STEN_DEV float ld_as_f32(const f16_t* p) {
  float f; asm("cvt.f32.f16 %0, %1;" : "=f"(f) : "h"(p->bits)); return f;
}
STEN_DEV float ldg_as_f32(const float* p) { return __ldg(p); }
STEN_DEV float ldg_as_f32(const double* p) { return (float)__ldg(p); }
STEN_DEV float ldg_as_f32(const bf16_t* p) {
  return __int_as_float(((u32)__ldg((const u16*)p)) << 16);
}
STEN_DEV float ldg_as_f32(const f16_t* p) {
  u16 b = __ldg((const u16*)p); float f; asm("cvt.f32.f16 %0, %1;" : "=f"(f) : "h"(b)); return f;
}
// raw element loads through the read-only path (no conversion)
STEN_DEV float ldg_raw(const float* p) { return __ldg(p); }
STEN_DEV double ldg_raw(const double* p) { return __ldg(p); }
STEN_DEV bf16_t ldg_raw(const bf16_t* p) { bf16_t v; v.bits = __ldg((const u16*)p); return v; }
STEN_DEV f16_t ldg_raw(const f16_t* p) { f16_t v; v.bits = __ldg((const u16*)p); return v; }
STEN_DEV void st_from_f32(float* p, float v) { *p = v; }
STEN_DEV void st_from_f32(double* p, float v) { *p = (double)v; }
STEN_DEV void st_from_f32(bf16_t* p, float v) {
  u16 b; asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(b) : "f"(v)); p->bits = b;
}
STEN_DEV void st_from_f32(f16_t* p, float v) {
  u16 b; asm("cvt.rn.f16.f32 %0, %1;" : "=h"(b) : "f"(v)); p->bits = b;
}
STEN_DEV void st_from_f64(double* p, double v) { *p = v; }
STEN_DEV void st_from_f64(float* p, double v) { *p = (float)v; }
STEN_DEV void st_from_f64(bf16_t* p, double v) { st_from_f32(p, (float)v); }
STEN_DEV void st_from_f64(f16_t* p, double v) { st_from_f32(p, (float)v); }

// ------------------------------------------------------------------ math helpers
// ------------------------------------------------------------------ k-vector chunks
// A thread's KV k-adjacent voxels of one row are one contiguous chunk of CW bytes in
// shared memory, aligned to 16 (CW % 16 == 0), 8 (CW % 8 == 0) or 4 bytes. Element
// loads at byte B of the chunk become one wide load per 16/8/4 bytes (identical
// loads from different taps are merged by the compiler) and a register extract.
template <typename T> struct is_bf16_t { static constexpr bool value = false; };
template <> struct is_bf16_t<bf16_t> { static constexpr bool value = true; };
STEN_DEV float f16_bits_to_f32(u16 b) { float f; asm("cvt.f32.f16 %0, %1;" : "=f"(f) : "h"(b)); return f; }
// The low / high FP16 half of a 32-bit word as FP32: the halves are named as the
// word's register pair (no shift or mask), so the conversion reads the half directly.
STEN_DEV float f16_lo_to_f32(u32 w) {
  float f; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; cvt.f32.f16 %0, l_; }" : "=f"(f) : "r"(w)); return f;
}
STEN_DEV float f16_hi_to_f32(u32 w) {
  float f; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; cvt.f32.f16 %0, h_; }" : "=f"(f) : "r"(w)); return f;
}
// a - c for a 16-bit element a (the low / high half of a 32-bit word) and an FP32 c
// in one mixed-precision subtraction (sm_100 sub.f32.f16 / sub.f32.bf16): a is
// widened exactly and the difference rounded once to FP32, the value of the FP32
// subtraction of the converted element, without the conversion instruction.
STEN_DEV float f16_lo_sub_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; sub.rn.f32.f16 %0, l_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float f16_hi_sub_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; sub.rn.f32.f16 %0, h_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float bf16_lo_sub_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; sub.rn.f32.bf16 %0, l_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float bf16_hi_sub_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; sub.rn.f32.bf16 %0, h_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
// a + c likewise (add.f32.f16 / add.f32.bf16)
STEN_DEV float f16_lo_add_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; add.rn.f32.f16 %0, l_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float f16_hi_add_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; add.rn.f32.f16 %0, h_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float bf16_lo_add_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; add.rn.f32.bf16 %0, l_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float bf16_hi_add_f32(u32 w, float c) {
  float d; asm("{ .reg .b16 l_, h_; mov.b32 {l_, h_}, %1; add.rn.f32.bf16 %0, h_, %2; }" : "=f"(d) : "r"(w), "f"(c)); return d;
}
STEN_DEV float add_as_f32(const f16_t* p, float c) {
  float d; asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(p->bits), "f"(c)); return d;
}
STEN_DEV float add_as_f32(const bf16_t* p, float c) {
  float d; asm("add.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(p->bits), "f"(c)); return d;
}
STEN_DEV float sub_as_f32(const f16_t* p, float c) {
  float d; asm("sub.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(p->bits), "f"(c)); return d;
}
STEN_DEV float sub_as_f32(const bf16_t* p, float c) {
  float d; asm("sub.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(p->bits), "f"(c)); return d;
}
// element at byte B of the chunk minus c (ADD false) or plus c (ADD true), 16-bit T
template <typename T, int CW, int B, bool ADD = false>
STEN_DEV float chunk_sub(const unsigned char* row, float c) {
  u32 w;
  if constexpr (CW % 16 == 0) {
    const uint4 v = *(const uint4*)(row + (B / 16) * 16);
    constexpr int q = (B % 16) / 4;
    w = q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
  } else if constexpr (CW % 8 == 0) {
    const uint2 v = *(const uint2*)(row + (B / 8) * 8);
    w = ((B % 8) / 4) == 0 ? v.x : v.y;
  } else {
    w = *(const u32*)(row + (B / 4) * 4);
  }
  if constexpr (is_bf16_t<T>::value && ADD) {
    return (B % 4) ? bf16_hi_add_f32(w, c) : bf16_lo_add_f32(w, c);
  } else if constexpr (is_bf16_t<T>::value) {
    return (B % 4) ? bf16_hi_sub_f32(w, c) : bf16_lo_sub_f32(w, c);
  } else if constexpr (ADD) {
    return (B % 4) ? f16_hi_add_f32(w, c) : f16_lo_add_f32(w, c);
  } else {
    return (B % 4) ? f16_hi_sub_f32(w, c) : f16_lo_sub_f32(w, c);
  }
}
template <typename T, int CW, int B>
STEN_DEV float chunk_elem(const unsigned char* row) {
  u32 w;
  if constexpr (CW % 16 == 0) {
    const uint4 v = *(const uint4*)(row + (B / 16) * 16);
    constexpr int q = (B % 16) / 4;
    w = q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
  } else if constexpr (CW % 8 == 0) {
    const uint2 v = *(const uint2*)(row + (B / 8) * 8);
    w = ((B % 8) / 4) == 0 ? v.x : v.y;
  } else {
    w = *(const u32*)(row + (B / 4) * 4);
  }
  if constexpr (sizeof(T) == 4) {
    return __uint_as_float(w);
  } else if constexpr (is_bf16_t<T>::value) {
    return __uint_as_float((B % 4) ? (w & 0xffff0000u) : (w << 16));
  } else {
    return (B % 4) ? f16_hi_to_f32(w) : f16_lo_to_f32(w);
  }
}
// N consecutive elements from global memory (read-only path) as floats: one 16/8/4-byte
// load per 16/8/4 bytes when the address is aligned to that width (ld_vec_f32), or
// element by element with the first n valid (ld_part_f32; the rest are zero).
STEN_DEV void unpack_f32(u32 w, const float*, float* o) { o[0] = __uint_as_float(w); }
STEN_DEV void unpack_f32(u32 w, const bf16_t*, float* o) {
  o[0] = __uint_as_float(w << 16); o[1] = __uint_as_float(w & 0xffff0000u);
}
STEN_DEV void unpack_f32(u32 w, const f16_t*, float* o) {
  o[0] = f16_lo_to_f32(w); o[1] = f16_hi_to_f32(w);
}
template <typename T, int N>
STEN_DEV void ld_vec_f32(const T* p, float* out) {
  constexpr int B = N * (int)sizeof(T), PW = 4 / (int)sizeof(T);   // elements per 32-bit word
  if constexpr (B % 16 == 0) {
    #pragma unroll
    for (int q = 0; q < B / 16; ++q) {
      const uint4 v = __ldg((const uint4*)p + q);
      unpack_f32(v.x, p, out + (4 * q + 0) * PW); unpack_f32(v.y, p, out + (4 * q + 1) * PW);
      unpack_f32(v.z, p, out + (4 * q + 2) * PW); unpack_f32(v.w, p, out + (4 * q + 3) * PW);
    }
  } else if constexpr (B % 8 == 0) {
    #pragma unroll
    for (int q = 0; q < B / 8; ++q) {
      const uint2 v = __ldg((const uint2*)p + q);
      unpack_f32(v.x, p, out + (2 * q + 0) * PW); unpack_f32(v.y, p, out + (2 * q + 1) * PW);
    }
  } else {
    #pragma unroll
    for (int q = 0; q < B / 4; ++q) unpack_f32(__ldg((const u32*)p + q), p, out + q * PW);
  }
}
template <typename T, int N>
STEN_DEV void ld_part_f32(const T* p, int n, float* out) {
  #pragma unroll
  for (int q = 0; q < N; ++q) out[q] = q < n ? ldg_as_f32(p + q) : 0.0f;
}
// KV consecutive values to a (KV x element size)-aligned global address.
STEN_DEV u32 pack2(const f16_t*, float lo, float hi) {
  u32 w; asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(w) : "f"(hi), "f"(lo)); return w;
}
STEN_DEV u32 pack2(const bf16_t*, float lo, float hi) {
  u32 w; asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(w) : "f"(hi), "f"(lo)); return w;
}
template <int KV> STEN_DEV void st_vec(float* p, const float* v) {
  if constexpr (KV == 2) *(float2*)p = make_float2(v[0], v[1]);
  else if constexpr (KV == 4) *(float4*)p = make_float4(v[0], v[1], v[2], v[3]);
  else if constexpr (KV == 8) {
    *(float4*)p = make_float4(v[0], v[1], v[2], v[3]);
    *(float4*)(p + 4) = make_float4(v[4], v[5], v[6], v[7]);
  } else { for (int q = 0; q < KV; ++q) p[q] = v[q]; }
}
template <int KV, typename T> STEN_DEV void st_vec(T* p, const float* v) {
  if constexpr (KV == 2) *(u32*)p = pack2(p, v[0], v[1]);
  else if constexpr (KV == 4) *(uint2*)p = make_uint2(pack2(p, v[0], v[1]), pack2(p, v[2], v[3]));
  else if constexpr (KV == 8)
    *(uint4*)p = make_uint4(pack2(p, v[0], v[1]), pack2(p, v[2], v[3]), pack2(p, v[4], v[5]), pack2(p, v[6], v[7]));
  else { for (int q = 0; q < KV; ++q) st_from_f32(p + q, v[q]); }
}

STEN_DEV float sten_clamp(float a, float lo, float hi) {
  // torch.clamp: min(max(a, lo), hi), NaN propagates
  return (a != a) ? a : fminf(fmaxf(a, lo), hi);
}
STEN_DEV float sten_div(float a, float b, float eps) {
  // divisor with |b| < eps replaced by +-eps
  float bs = (fabsf(b) < eps) ? (b < 0.0f ? -eps : eps) : b;
  return a / bs;
}
STEN_DEV float sten_log(float a, float eps) { return logf((a != a) ? a : fmaxf(a, eps)); }
STEN_DEV float sten_sqrt(float a, float eps) { return sqrtf((a != a) ? a : fmaxf(a, eps)); }

// ------------------------------------------------------------------ boundary indices
// x is within one period of [0, n): every stencil tap moves one cell per level
STEN_DEV int wrap_idx(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }
STEN_DEV int clamp_idx(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
// mirror without repeating the edge, radius 1: -1 -> 1, n -> n-2
STEN_DEV int reflect_idx(int x, int n) {
  if (x < 0) x = -x;
  if (x > n - 1) x = 2 * (n - 1) - x;
  return x < 0 ? 0 : (x > n - 1 ? n - 1 : x);
}

// ------------------------------------------------------------------ mbarrier + TMA
struct __align__(64) TmaDesc { u64 opaque[16]; };

STEN_DEV u32 smem_u32(const void* p) {
  return (u32)__cvta_generic_to_shared(p);
}
STEN_DEV void mbar_init(u64* bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
STEN_DEV void mbar_inval(u64* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
STEN_DEV void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
STEN_DEV void st_shared_u32(u32 saddr, u32 v) { asm volatile("st.shared.u32 [%0], %1;" :: "r"(saddr), "r"(v) : "memory"); }
STEN_DEV void st_shared_u64(u32 saddr, u64 v) { asm volatile("st.shared.u64 [%0], %1;" :: "r"(saddr), "l"(v) : "memory"); }
STEN_DEV void st_shared_u128(u32 saddr, u32 a, u32 b, u32 c, u32 d) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" :: "r"(saddr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}
// The 16 bytes of v with bytes outside [lo, hi) zeroed.
STEN_DEV uint4 keep_bytes16(uint4 v, u32 lo, u32 hi) {
  u32 w[4] = {v.x, v.y, v.z, v.w};
  #pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int l = min(max((int)lo - 4 * i, 0), 4), h = min(max((int)hi - 4 * i, 0), 4);
    const u32 below_h = h >= 4 ? 0xffffffffu : ((1u << (8 * h)) - 1u);
    const u32 below_l = l >= 4 ? 0xffffffffu : ((1u << (8 * l)) - 1u);
    w[i] &= below_h & ~below_l;
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}
// 16-byte asynchronous global->shared copy (L2 only) of which the first src_bytes
// (16 or 0) come from gsrc, the rest zero; completion tracked by cp_async_mbar_arrive.
STEN_DEV void cp_async16_cg(u32 sdst, const void* gsrc, u32 src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(sdst), "l"(gsrc), "r"(src_bytes) : "memory");
}
// One arrival on `bar` once every cp.async this thread issued so far has completed
// (the barrier's expected count includes it).
STEN_DEV void cp_async_mbar_arrive(u64* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
// 16-byte shared-memory load / store at a 32-bit shared address.
STEN_DEV uint4 ld_shared_v4(u32 saddr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(saddr) : "memory");
  return v;
}
STEN_DEV void st_shared_v4(u32 saddr, uint4 v) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" :: "r"(saddr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}
STEN_DEV uint2 ld_shared_v2(u32 saddr) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(saddr) : "memory");
  return v;
}
// The 16 bytes that start `sh` (0..15, a multiple of ES) bytes into the 32 bytes at the
// 16-byte aligned 32-bit shared address src. 2- and 8-byte elements: the 8-byte half of
// the offset taken by the load address (8-byte loads), the rest by one select step and
// funnel shifts; 4-byte elements: two 16-byte loads and two select steps (measured
// faster for them at 509^3).
template <int ES> STEN_DEV uint4 shifted16s(u32 src, u32 sh) {
  if constexpr (ES == 4) {
    const uint4 a = ld_shared_v4(src), b = ld_shared_v4(src + 16u);
    const u32 w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    const bool s8 = (sh & 8u) != 0u, s4 = (sh & 4u) != 0u;
    u32 x[5];
    #pragma unroll
    for (int j = 0; j < 5; ++j) x[j] = s8 ? w[j + 2] : w[j];
    return s4 ? make_uint4(x[1], x[2], x[3], x[4]) : make_uint4(x[0], x[1], x[2], x[3]);
  } else {
    const u32 base = src + (sh & 8u);
    const uint2 a = ld_shared_v2(base), b = ld_shared_v2(base + 8u);
    if constexpr (ES >= 8) {
      return make_uint4(a.x, a.y, b.x, b.y);
    } else {
      const uint2 c = ld_shared_v2(base + 16u);
      const u32 v[6] = {a.x, a.y, b.x, b.y, c.x, c.y};
      const bool s4 = (sh & 4u) != 0u;
      u32 y[5];
      #pragma unroll
      for (int j = 0; j < 5; ++j) y[j] = s4 ? v[j + 1] : v[j];
      const u32 bs = (sh & 3u) * 8u;
      return make_uint4(__funnelshift_r(y[0], y[1], bs), __funnelshift_r(y[1], y[2], bs),
                        __funnelshift_r(y[2], y[3], bs), __funnelshift_r(y[3], y[4], bs));
    }
  }
}
STEN_DEV void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
STEN_DEV void mbar_arrive_expect_tx(u64* bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
STEN_DEV bool mbar_try_wait(u64* bar, u32 parity) {
  u32 ok;
  asm volatile("{\n .reg .pred p;\n"
               " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
STEN_DEV u64 global_ns() {
  u64 t; asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t)); return t;
}
// Bounded wait: gives up after `limit_ns` of wall time and returns false.
STEN_DEV bool mbar_wait_bounded(u64* bar, u32 parity, u64 limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  u64 t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}
// Bounded wait for a flag that another CTA of this launch sets to non-zero (after a
// __threadfence); acquire loads with a short back-off. False after limit_ns.
STEN_DEV bool flag_wait_bounded(const unsigned int* f, u64 limit_ns) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
  if (v) return true;
  const u64 t0 = global_ns();
  for (;;) {
    __nanosleep(200);
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
    if (v) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}
// 3-D tiled TMA load of one box into shared memory; completion counted on `bar`.
// Coordinates: x innermost (elements), y, z. x * elem_size must be a multiple of 16.
STEN_DEV void tma_load_3d(void* smem_dst, const TmaDesc* map, u64* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];"
      :: "r"(smem_u32(smem_dst)), "l"((u64)map), "r"(smem_u32(bar)),
         "r"(x), "r"(y), "r"(z) : "memory");
}
STEN_DEV void tma_prefetch_desc(const TmaDesc* map) {
  asm volatile("prefetch.tensormap [%0];" :: "l"((u64)map) : "memory");
}

// ------------------------------------------------------------------ fp64 reductions
STEN_DEV double warp_sum(double v) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
STEN_DEV double warp_min(double v) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
STEN_DEV double warp_max(double v) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Chan et al. pairwise merge of (n, mean, M2) moments.
STEN_DEV void chan_merge(double& n, double& mean, double& m2, double nb, double meanb, double m2b) {
  double nt = n + nb;
  if (nt == 0.0) return;
  double d = meanb - mean;
  double w = nb / nt;
  mean += d * w;
  m2 += m2b + d * d * n * w;
  n = nt;
}
STEN_DEV void warp_chan(double& n, double& mean, double& m2) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double nb = __shfl_xor_sync(0xffffffffu, n, o);
    double mb = __shfl_xor_sync(0xffffffffu, mean, o);
    double qb = __shfl_xor_sync(0xffffffffu, m2, o);
    // fixed operand order per lane pair keeps the result identical on both lanes
    if ((threadIdx.x & o) == 0) { chan_merge(n, mean, m2, nb, mb, qb); }
    else { double n2 = nb, m2_ = mb, q2 = qb; chan_merge(n2, m2_, q2, n, mean, m2); n = n2; mean = m2_; m2 = q2; }
  }
}

// co-moments of two variables: (n, mean a, mean b, C = sum da db, M2 a, M2 b), merged as
// Chan et al. merge (n, mean, M2) pairs, with C's cross term da db n nb / (n + nb)
STEN_DEV void co_merge(double* x, const double* y) {
  const double nt = x[0] + y[0];
  if (nt == 0.0) return;
  const double da = y[1] - x[1], db = y[2] - x[2], w = y[0] / nt, f = x[0] * w;
  x[1] += da * w; x[2] += db * w;
  x[3] += y[3] + da * db * f;
  x[4] += y[4] + da * da * f;
  x[5] += y[5] + db * db * f;
  x[0] = nt;
}
STEN_DEV void warp_co(double* x) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double y[6];
    #pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = __shfl_xor_sync(0xffffffffu, x[i], o);
    // fixed operand order per lane pair keeps the result identical on both lanes
    if ((threadIdx.x & o) == 0) co_merge(x, y);
    else { co_merge(y, x); for (int i = 0; i < 6; ++i) x[i] = y[i]; }
  }
}

// Block-level reductions through a small shared scratch (one value per warp).
// All threads of the block must call these; `scratch` holds >= 6*32 doubles.
STEN_DEV double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < nw ? scratch[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;  // valid in thread 0
}
STEN_DEV double block_min(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_min(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = __longlong_as_double(0x7ff0000000000000ll);
  if (warp == 0) { r = lane < nw ? scratch[lane] : r; r = warp_min(r); }
  return r;
}
STEN_DEV double block_max(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = __longlong_as_double(0xfff0000000000000ll);
  if (warp == 0) { r = lane < nw ? scratch[lane] : r; r = warp_max(r); }
  return r;
}
STEN_DEV void block_chan(double& n, double& mean, double& m2, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  warp_chan(n, mean, m2);
  __syncthreads();
  if (lane == 0) { scratch[warp] = n; scratch[32 + warp] = mean; scratch[64 + warp] = m2; }
  __syncthreads();
  if (warp == 0) {
    double a = 0.0, b = 0.0, c = 0.0;
    if (lane < nw) { a = scratch[lane]; b = scratch[32 + lane]; c = scratch[64 + lane]; }
    warp_chan(a, b, c);
    n = a; mean = b; m2 = c;
  }
}

STEN_DEV void block_co(double* x, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  warp_co(x);
  __syncthreads();
  if (lane == 0) for (int i = 0; i < 6; ++i) scratch[32 * i + warp] = x[i];
  __syncthreads();
  if (warp == 0) {
    double y[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (lane < nw) for (int i = 0; i < 6; ++i) y[i] = scratch[32 * i + lane];
    warp_co(y);
    for (int i = 0; i < 6; ++i) x[i] = y[i];
  }
}

// ------------------------------------------------------------------ histograms
// sum over non-empty bins of q log q, q = count / n (the entropy is its negation),
// clearing the counts for the next run. Fixed bins per thread and a fixed
// reduction tree: deterministic. Whole block; the result is valid in thread 0.
STEN_DEV double sten_hist_qlogq(unsigned long long* h, int bins, double n, double* scratch) {
  double acc = 0.0;
  for (int b = threadIdx.x; b < bins; b += blockDim.x) {
    const unsigned long long c = __ldcg(h + b);
    if (c) { const double q = (double)c / n; acc += q * log(q); }
    h[b] = 0ull;
  }
  return block_sum(acc, scratch);
}

// ------------------------------------------------------------------ in-kernel finalize
// Kinds of per-CTA partial rows (same numbering as the library's STENPY_RED_*).
#define STEN_RED_SUM 0
#define STEN_RED_MEAN 1
#define STEN_RED_NORM_L2 2
#define STEN_RED_VARIANCE 3
#define STEN_RED_ENTROPY 4
#define STEN_RED_INTEGRATE 5
#define STEN_RED_MIN_MAX 6
#define STEN_RED_COVARIANCE 7
#define STEN_RED_CORRELATION 8
// Combine rows part[c * nslots + slot], c < ncta, into the final value(s) at out[0]
// (out[1] for min/max). Each thread folds rows t, t + blockDim, ... in order and a
// fixed warp/block tree combines them: deterministic for a given block size.
// Whole block; partials are read through L2 (written by other CTAs of this launch).
STEN_DEV void sten_reduce_rows(int kind, const double* part, int ncta, int nslots, int slot, int unbiased,
                               double count, double eps, double* out, double* scratch) {
  const int t = threadIdx.x;
  if (kind == STEN_RED_COVARIANCE || kind == STEN_RED_CORRELATION) {
    double x[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int c = t; c < ncta; c += blockDim.x) {
      const double* row = part + (size_t)c * nslots + slot;
      double y[6];
      for (int i = 0; i < 6; ++i) y[i] = __ldcg(row + i);
      co_merge(x, y);
    }
    block_co(x, scratch);
    if (t == 0) out[0] = kind == STEN_RED_COVARIANCE ? x[3] / (x[0] - 1.0 > 1.0 ? x[0] - 1.0 : 1.0)
                                                    : x[3] / (sqrt(x[4]) * sqrt(x[5]) + eps);
    return;
  }
  double x0 = 0.0, x1 = 0.0, x2 = 0.0;
  if (kind == STEN_RED_MIN_MAX) { x0 = __longlong_as_double(0x7ff0000000000000ll); x1 = -x0; }
  for (int c = t; c < ncta; c += blockDim.x) {
    const double* row = part + (size_t)c * nslots + slot;
    if (kind == STEN_RED_VARIANCE) chan_merge(x0, x1, x2, __ldcg(row), __ldcg(row + 1), __ldcg(row + 2));
    else if (kind == STEN_RED_ENTROPY) { x0 += __ldcg(row); x1 += __ldcg(row + 1); }
    else if (kind == STEN_RED_MIN_MAX) { x0 = fmin(x0, __ldcg(row)); x1 = fmax(x1, __ldcg(row + 1)); }
    else x0 += __ldcg(row);
  }
  double r0, r1 = 0.0, r2 = 0.0;
  if (kind == STEN_RED_VARIANCE) { block_chan(x0, x1, x2, scratch); r0 = x0; r2 = x2; }
  else if (kind == STEN_RED_MIN_MAX) { r0 = block_min(x0, scratch); r1 = block_max(x1, scratch); }
  else if (kind == STEN_RED_ENTROPY) { r0 = block_sum(x0, scratch); r1 = block_sum(x1, scratch); }
  else r0 = block_sum(x0, scratch);
  if (t != 0) return;
  switch (kind) {
    case STEN_RED_MEAN: out[0] = r0 / count; break;
    case STEN_RED_NORM_L2: out[0] = sqrt(r0); break;
    case STEN_RED_VARIANCE: {
      const double den = unbiased ? (r0 - 1.0 > 1.0 ? r0 - 1.0 : 1.0) : (r0 > 1.0 ? r0 : 1.0);
      out[0] = r2 / den;
      break;
    }
    case STEN_RED_ENTROPY: { const double Z = r0 + eps; out[0] = (r0 * log(Z) - r1) / Z; break; }
    case STEN_RED_MIN_MAX: out[0] = r0; out[1] = r1; break;
    default: out[0] = r0; break;
  }
}

// ------------------------------------------------------------------ 3x3 symmetric eigenvalues
STEN_DEV float m_sqrt(float x) { return sqrtf(x); }
STEN_DEV double m_sqrt(double x) { return sqrt(x); }
STEN_DEV float m_acos(float x) { return acosf(x); }
STEN_DEV double m_acos(double x) { return acos(x); }
STEN_DEV float m_cos(float x) { return cosf(x); }
STEN_DEV double m_cos(double x) { return cos(x); }
// Ascending eigenvalues of the symmetric matrix whose lower triangle is
// (a00; a10 a11; a20 a21 a22), trigonometric closed form.
// Returns r = det((A - qI)/p)/2 = cos(3 phi), clamped to [-1, 1] (1 for a multiple of I).
template <typename T>
STEN_DEV T eig3_trig(T a00, T a10, T a11, T a20, T a21, T a22, T* w) {
  const T p1 = a10 * a10 + a20 * a20 + a21 * a21;
  const T q = (a00 + a11 + a22) / T(3);
  const T b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
  const T p2 = b00 * b00 + b11 * b11 + b22 * b22 + T(2) * p1;
  if (p2 <= T(0)) { w[0] = q; w[1] = q; w[2] = q; return T(1); }
  const T p = m_sqrt(p2 / T(6));
  const T ip = T(1) / p;
  const T c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip;
  const T c10 = a10 * ip, c20 = a20 * ip, c21 = a21 * ip;
  // det(B)/2
  T r = (c00 * (c11 * c22 - c21 * c21) - c10 * (c10 * c22 - c21 * c20) + c20 * (c10 * c21 - c11 * c20)) / T(2);
  r = r < T(-1) ? T(-1) : (r > T(1) ? T(1) : r);
  const T phi = m_acos(r) / T(3);
  const T two_pi_3 = T(2.0943951023931954923);
  const T e_hi = q + T(2) * p * m_cos(phi);
  const T e_lo = q + T(2) * p * m_cos(phi + two_pi_3);
  const T e_mid = T(3) * q - e_hi - e_lo;
  w[0] = e_lo; w[1] = e_mid; w[2] = e_hi;
  return r;
}
// fp32 evaluation, re-evaluated in fp64 in two cases: (a) the spectrum spread p is
// below 1e-3 of the matrix scale (the fp32 shift A - qI loses digits); (b) two
// eigenvalues nearly coincide, |r| > 0.999: acos amplifies the fp32 rounding of r
// (a few units of 2^-24) by 1/sqrt(1 - r^2), and at |r| = 0.999 the eigenvalue error
// stays near 1e-6 of the scale (checked against LAPACK on smooth fields, where a few
// percent of voxels take the fp64 path).
STEN_DEV void eig3_sym(const float* m, float* w) {
  const float a00 = m[0], a10 = m[3], a11 = m[4], a20 = m[6], a21 = m[7], a22 = m[8];
  const float scale = fmaxf(fmaxf(fabsf(a00), fabsf(a11)), fmaxf(fabsf(a22),
                      fmaxf(fmaxf(fabsf(a10), fabsf(a20)), fabsf(a21))));
  const float q = (a00 + a11 + a22) * (1.0f / 3.0f);
  const float p2 = (a00 - q) * (a00 - q) + (a11 - q) * (a11 - q) + (a22 - q) * (a22 - q)
                 + 2.0f * (a10 * a10 + a20 * a20 + a21 * a21);
  float r = 1.0f;
  if (p2 > 1e-6f * scale * scale) r = eig3_trig<float>(a00, a10, a11, a20, a21, a22, w);
  if (fabsf(r) > 0.999f) {
    double wd[3];
    eig3_trig<double>((double)a00, (double)a10, (double)a11, (double)a20, (double)a21, (double)a22, wd);
    w[0] = (float)wd[0]; w[1] = (float)wd[1]; w[2] = (float)wd[2];
  }
}

// ------------------------------------------------------------------ status word
// Device-side error codes written to Params::err (host raises on non-zero).
#define STEN_ERR_TMA_TIMEOUT 1
#define STEN_ERR_BAD_ALIGN 2
#define STEN_WAIT_LIMIT_NS 2000000000ull

// Shared device-side building blocks for the flagsparse_b200 CSR kernels.
//
// Value types, compensated accumulators and small warp/block primitives used by
// the SpMV, SpMM and SDDMM kernels.  Everything here is sm_100a-only code; the
// library is built with -gencode arch=compute_100a,code=sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/flagsparse_b200.h"

namespace fsb {

// ---------------------------------------------------------------------------
// Value-type traits.  `Store` is the element type in HBM, `Real` the scalar
// arithmetic type, `kComplex` selects interleaved (re, im) arithmetic.
// ---------------------------------------------------------------------------
template <int DT> struct VT;
template <> struct VT<FSB_F16> {
  using Store = __half; using Real = float; static constexpr bool kComplex = false;
  // a half*half product is exact in fp32 (11+11 significant bits <= 24).
  static constexpr bool kExactProduct = true;
};
template <> struct VT<FSB_BF16> {
  using Store = __nv_bfloat16; using Real = float; static constexpr bool kComplex = false;
  static constexpr bool kExactProduct = true;   // 8+8 significant bits <= 24
};
template <> struct VT<FSB_F32> {
  using Store = float; using Real = float; static constexpr bool kComplex = false;
  static constexpr bool kExactProduct = false;
};
template <> struct VT<FSB_F64> {
  using Store = double; using Real = double; static constexpr bool kComplex = false;
  static constexpr bool kExactProduct = false;
};
template <> struct VT<FSB_C64> {
  using Store = float2; using Real = float; static constexpr bool kComplex = true;
  static constexpr bool kExactProduct = false;
};
template <> struct VT<FSB_C128> {
  using Store = double2; using Real = double; static constexpr bool kComplex = true;
  static constexpr bool kExactProduct = false;
};

__device__ __forceinline__ float to_real(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_real(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_real(float v) { return v; }
__device__ __forceinline__ double to_real(double v) { return v; }

template <typename S> __device__ __forceinline__ S from_real(float v);
template <> __device__ __forceinline__ __half from_real<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_real<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ float from_real<float>(float v) { return v; }
template <typename S> __device__ __forceinline__ S from_real_d(double v);
template <> __device__ __forceinline__ double from_real_d<double>(double v) { return v; }

// ---------------------------------------------------------------------------
// Error-free transformations (Knuth TwoSum, FMA-based TwoProduct) and the
// compensated accumulator built on them.  The accumulator follows the Sum2 /
// Dot2 scheme of Ogita, Rump and Oishi, "Accurate sum and dot product",
// SIAM J. Sci. Comput. 26(6), 2005: the running sum `hi` is exact up to the
// rounding errors collected in `lo`, so the rounded result hi+lo is as
// accurate as a dot product evaluated in twice the working precision.
// ---------------------------------------------------------------------------
// Round-to-nearest add/sub/mul that the compiler may never contract into an
// FMA: the error-free transformations below rely on every step being rounded.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename R>
__device__ __forceinline__ void two_sum(R a, R b, R& s, R& e) {
  s = add_rn(a, b);
  R bb = sub_rn(s, a);
  e = add_rn(sub_rn(a, sub_rn(s, bb)), sub_rn(b, bb));
}

template <typename R>
struct Comp {            // compensated real accumulator: value == hi + lo
  R hi, lo;
  __device__ __forceinline__ void zero() { hi = R(0); lo = R(0); }
  __device__ __forceinline__ void add(R v) {
    R s, e; two_sum(hi, v, s, e); hi = s; lo = add_rn(lo, e);
  }
  // add the exact product a*b: p + pe == a*b exactly (FMA TwoProduct)
  __device__ __forceinline__ void add_prod(R a, R b) {
    R p = mul_rn(a, b);
    R pe = fma_rn(a, b, -p);
    R s, e; two_sum(hi, p, s, e); hi = s; lo = add_rn(lo, add_rn(e, pe));
  }
  __device__ __forceinline__ void add_comp(R ohi, R olo) {
    R s, e; two_sum(hi, ohi, s, e); hi = s; lo = add_rn(lo, add_rn(e, olo));
  }
  __device__ __forceinline__ R value() const { return add_rn(hi, lo); }
};

// Plain accumulator with the same interface (used where the error analysis
// shows compensation is not needed, e.g. short bf16 rows).
template <typename R>
struct Plain {
  R hi;
  __device__ __forceinline__ void zero() { hi = R(0); }
  __device__ __forceinline__ void add(R v) { hi += v; }
  __device__ __forceinline__ void add_prod(R a, R b) { hi = fma(a, b, hi); }
  __device__ __forceinline__ void add_comp(R ohi, R /*olo*/) { hi += ohi; }
  __device__ __forceinline__ R value() const { return hi; }
};

// ---------------------------------------------------------------------------
// Warp shuffles over teams of T lanes (T a power of two <= 32).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R shfl_xor(R v, int mask, int width = 32) {
  return __shfl_xor_sync(0xffffffffu, v, mask, width);
}

template <int T, typename R>
__device__ __forceinline__ void team_reduce(Comp<R>& a) {
#pragma unroll
  for (int m = T / 2; m > 0; m >>= 1) {
    R oh = shfl_xor(a.hi, m, T);
    R ol = shfl_xor(a.lo, m, T);
    a.add_comp(oh, ol);
  }
}
template <int T, typename R>
__device__ __forceinline__ void team_reduce(Plain<R>& a) {
#pragma unroll
  for (int m = T / 2; m > 0; m >>= 1) a.hi += shfl_xor(a.hi, m, T);
}

// Dynamic-width variant: width is a runtime power of two <= 32.
template <typename R>
__device__ __forceinline__ void team_reduce_dyn(Comp<R>& a, int T) {
  for (int m = T >> 1; m > 0; m >>= 1) {
    R oh = __shfl_xor_sync(0xffffffffu, a.hi, m, 32);
    R ol = __shfl_xor_sync(0xffffffffu, a.lo, m, 32);
    a.add_comp(oh, ol);
  }
}

// ---------------------------------------------------------------------------
// Misc helpers.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

template <typename P>
__device__ __forceinline__ int64_t ld_ptr(const P* p, int64_t i) { return static_cast<int64_t>(__ldg(p + i)); }

}  // namespace fsb

// Status plumbing shared by every C-ABI entry point: never throw, never abort.
// A grid launched as a programmatic dependent of the grid before it in the
// stream may start while that grid still runs.  Its last block waits for that
// grid before exiting, so the dependent grid completes only after both have:
// work later in the stream sees both grids' results.  Waiting after its own
// work keeps the overlap.
__device__ __forceinline__ void pdl_join_primary() {
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) asm volatile("griddepcontrol.wait;" ::: "memory");
}

#define FSB_LAUNCH_CHECK()                                   \
  do {                                                       \
    cudaError_t _e = cudaGetLastError();                     \
    if (_e != cudaSuccess) return FSB_ERR_LAUNCH;            \
  } while (0)

#define FSB_CUDA_CHECK(call)                                 \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return FSB_ERR_CUDA;              \
  } while (0)

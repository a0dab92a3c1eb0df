// CSR SpMM  C = A B  for sm_100a (A sparse M x K in CSR, B dense K x N row-major).
//
// The launch reuses the SpMV unit plan (plan.cu), built with the SpMM window
// cap (64) and chunk (256): every warp executes one (unit, column tile) pair.
// The lanes of a warp own consecutive column groups of V elements of the tile
// (16-byte loads when N and the leading dimensions allow it), so one nonzero
// costs the warp a single coalesced read of its B-row slice:
//
//  * row-block unit: a run of rows with < 128 nonzeros.  The warp stages the
//    nonzeros (value, column, local row) in its shared-memory slice, writes
//    zero rows for empty rows, then walks the nonzeros in order, loading the
//    B slices of 4 nonzeros ahead of the multiply-adds across row boundaries
//    and storing a C row slice whenever the row changes.
//  * long-row chunk: `chunk_nnz` nonzeros of a row with > cap nonzeros, staged
//    in 128-nonzero batches.  A one-chunk row is written directly; otherwise
//    the chunk's partial row slice goes to its scratch slot and the warp that
//    completes the row's ticket adds the partials in chunk order.
//
// Accumulation: fp32 for half / bfloat16 / fp32 values (half and bfloat16
// products are exact in fp32), fp64 for fp64, componentwise for complex.
// FSB_SPMM_COMPENSATED switches every sum to Dot2 compensated accumulation.
// Every sum runs in a fixed order, so results are bitwise reproducible.
//
// The same file holds the narrow-row team kernel (k_spmm_team, also fused
// with an SpMV for the batched step) and the one-launch backward of Y = A X
// (k_spmm_bwd: dX = A^T dY and the SDDMM dvals from one gather of dY).
//
// Replaces _triton_spmm_csr_impl / _spmm_csr_real_kernel / the complex kernel
// (sparse_operations/spmm_csr.py:3373-3466, 144-339) and the bucketed
// alg1 / alg2 / opt kernels (spmm_csr.py:1091-2449, spmm_csr_opt_alg2.py) of
// flagos-ai/FlagSparse.
#include <atomic>
#include <cstring>
#include <type_traits>

#include "fsb_common.cuh"

namespace fsb {
namespace {

constexpr int kSpmmWarps = 8;      // warps per block; one (unit, tile) per warp
constexpr int kSpmmBatch = 128;    // nonzeros staged per batch
constexpr int kSpmmMaxCap = 64;    // row blocks hold < 2*cap <= kSpmmBatch nonzeros
constexpr int kSpmmAhead = 4;      // B slices loaded ahead of the multiply-adds
// the same for a team's row in the narrow-row kernel: 8 for fp32 (measured
// 2-6 % faster), 4 where the slices, sums or the fused y terms need the registers
template <int DT>
struct TeamAhead { static constexpr int value = (DT == FSB_F32) ? 8 : 4; };
constexpr int kSpmmTileLanes = 32;

template <int BYTES> struct RawT;
template <> struct RawT<2> { using T = unsigned short; };
template <> struct RawT<4> { using T = unsigned int; };
template <> struct RawT<8> { using T = uint2; };
template <> struct RawT<16> { using T = uint4; };

// V consecutive elements starting at p; the first nv < V only when the slice
// crosses column N (the rest read as zero).  ONCE: a streaming (evict-first)
// load, for data read once that should not displace gathered rows in L2.
template <typename S, int V, bool ONCE = false>
__device__ __forceinline__ void load_slice(const S* p, int nv, S (&out)[V]) {
  if (nv == V) {
    using Raw = typename RawT<int(sizeof(S)) * V>::T;
    Raw r = ONCE ? __ldcs(reinterpret_cast<const Raw*>(p)) : __ldg(reinterpret_cast<const Raw*>(p));
    memcpy(out, &r, sizeof(Raw));
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if (j < nv) {
        out[j] = p[j];
      } else {
        memset(&out[j], 0, sizeof(S));
      }
    }
  }
}

// One whole 16-byte slice at B + row * ldb (row, ldb < 2^32: a single wide
// 32 x 32-bit multiply), no partial-slice test: the team kernels point lanes
// without columns at a valid slice and discard what they load.  (L2
// evict-last hints on these gathers, with evict-first on A and C, measured no
// better: fp32 N = 128 on a 1,000,000-row power-law matrix kept its 11 % L2
// hit rate.)
template <typename S, int V>
__device__ __forceinline__ void load_row16(const S* __restrict__ B, uint32_t row, uint32_t ldb, S (&out)[V]) {
  static_assert(int(sizeof(S)) * V == 16, "one 16-byte slice");
  const uint4 r = __ldg(reinterpret_cast<const uint4*>(B + static_cast<uint64_t>(row) * ldb));
  memcpy(out, &r, 16);
}

// Output slices are written once: STREAM makes them streaming (evict-first)
// stores, so the output does not displace gathered rows in L2.
template <typename S, int V, bool STREAM = false>
__device__ __forceinline__ void store_slice(S* p, int nv, const S (&v)[V]) {
  if (nv == V) {
    using Raw = typename RawT<int(sizeof(S)) * V>::T;
    Raw r;
    memcpy(&r, v, sizeof(Raw));
    if (STREAM) __stcs(reinterpret_cast<Raw*>(p), r);
    else *reinterpret_cast<Raw*>(p) = r;
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j)
      if (j < nv) p[j] = v[j];
  }
}

__device__ __forceinline__ __half spmm_store(float v, __half*) { return __float2half_rn(v); }
__device__ __forceinline__ __nv_bfloat16 spmm_store(float v, __nv_bfloat16*) { return __float2bfloat16_rn(v); }
__device__ __forceinline__ float spmm_store(float v, float*) { return v; }
__device__ __forceinline__ double spmm_store(double v, double*) { return v; }

// c0 += a * b0, c1 += a * b1 in one packed fp32x2 FMA (sm_100a); each half is
// rounded exactly as a scalar fma.rn, so results equal the scalar loop's.
__device__ __forceinline__ void ffma2(float& c0, float& c1, float a, float b0, float b1) {
  unsigned long long cc, aa, bb;
  asm("mov.b64 %0, {%1, %2};" : "=l"(cc) : "f"(c0), "f"(c1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(aa) : "f"(a), "f"(a));
  asm("mov.b64 %0, {%1, %2};" : "=l"(bb) : "f"(b0), "f"(b1));
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(cc) : "l"(aa), "l"(bb));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(c0), "=f"(c1) : "l"(cc));
}

// (c0, c1) += (a * lo(b), a * hi(b)) for a 16-bit a and two packed 16-bit
// values b: sm_100a's mixed-precision fma.rn.f32.{bf16,f16} multiplies the
// 16-bit inputs exactly (the product fits fp32) and rounds each sum once, so
// the results equal widening to fp32 and calling fmaf, with no widening
// instructions.
template <typename S>
__device__ __forceinline__ void fma_mixed2(float& c0, float& c1, S a, unsigned b) {
  unsigned short ab;
  memcpy(&ab, &a, 2);
  if constexpr (std::is_same<S, __nv_bfloat16>::value) {
    asm("{\n .reg .b16 bl, bh;\n mov.b32 {bl, bh}, %3;\n fma.rn.f32.bf16 %0, %2, bl, %0;\n"
        " fma.rn.f32.bf16 %1, %2, bh, %1;\n}"
        : "+f"(c0), "+f"(c1) : "h"(ab), "r"(b));
  } else {
    asm("{\n .reg .b16 bl, bh;\n mov.b32 {bl, bh}, %3;\n fma.rn.f32.f16 %0, %2, bl, %0;\n"
        " fma.rn.f32.f16 %1, %2, bh, %1;\n}"
        : "+f"(c0), "+f"(c1) : "h"(ab), "r"(b));
  }
}

// Per-lane accumulator of V output elements.
template <int DT, bool COMP, int V>
struct SpmmAcc {
  using Vt = VT<DT>;
  using S = typename Vt::Store;
  using R = typename Vt::Real;
  static constexpr bool kCplx = Vt::kComplex;
  static constexpr int kNC = kCplx ? 2 : 1;            // real components per element
  using Sum = typename std::conditional<COMP, Comp<R>, Plain<R>>::type;
  Sum s[kNC][V];

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int c = 0; c < kNC; ++c)
#pragma unroll
      for (int j = 0; j < V; ++j) s[c][j].zero();
  }

  __device__ __forceinline__ static void term(Sum& acc, R a, R b) {
    if constexpr (COMP && Vt::kExactProduct) acc.add(mul_rn(a, b));  // exact product
    else acc.add_prod(a, b);
  }

  __device__ __forceinline__ void add(S a, const S (&b)[V]) {
    if constexpr (kCplx) {
#pragma unroll
      for (int j = 0; j < V; ++j) {
        term(s[0][j], a.x, b[j].x);
        term(s[0][j], -a.y, b[j].y);
        term(s[1][j], a.x, b[j].y);
        term(s[1][j], a.y, b[j].x);
      }
    } else {
      const R ar = to_real(a);
      if constexpr (!COMP && sizeof(S) == 2 && V % 2 == 0) {
        unsigned bw[V / 2];
        memcpy(bw, b, sizeof(bw));
#pragma unroll
        for (int j = 0; j < V; j += 2) fma_mixed2(s[0][j].hi, s[0][j + 1].hi, a, bw[j / 2]);
      } else if constexpr (!COMP && std::is_same<R, float>::value && V % 2 == 0) {
#pragma unroll
        for (int j = 0; j < V; j += 2) ffma2(s[0][j].hi, s[0][j + 1].hi, ar, to_real(b[j]), to_real(b[j + 1]));
      } else {
#pragma unroll
        for (int j = 0; j < V; ++j) term(s[0][j], ar, to_real(b[j]));
      }
    }
  }

  __device__ __forceinline__ void result(S (&out)[V]) const {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if constexpr (kCplx) {
        out[j].x = s[0][j].value();
        out[j].y = s[1][j].value();
      } else {
        out[j] = spmm_store(s[0][j].value(), static_cast<S*>(nullptr));
      }
    }
  }

  // scratch layout per element: (hi, lo) per real component
  __device__ __forceinline__ void store_partial(R* p) const {
#pragma unroll
    for (int j = 0; j < V; ++j)
#pragma unroll
      for (int c = 0; c < kNC; ++c) {
        p[(j * kNC + c) * 2] = s[c][j].hi;
        if constexpr (COMP) p[(j * kNC + c) * 2 + 1] = s[c][j].lo;
        else p[(j * kNC + c) * 2 + 1] = R(0);
      }
  }

  __device__ __forceinline__ void add_partial(const R* p) {
#pragma unroll
    for (int j = 0; j < V; ++j)
#pragma unroll
      for (int c = 0; c < kNC; ++c)
        s[c][j].add_comp(__ldcg(p + (j * kNC + c) * 2), __ldcg(p + (j * kNC + c) * 2 + 1));
  }
};

// Per-warp shared-memory slice: staged values, columns, the unit's row
// offsets and each staged nonzero's local row; a multiple of 16 bytes.
template <typename S>
constexpr int spmm_warp_smem_bytes() {
  return (kSpmmBatch * int(sizeof(S)) + kSpmmBatch * 4 + (kSpmmMaxCap + 1) * 4 + kSpmmBatch + 15) & ~15;
}

template <int DT>
struct SpmmMinBlocks { static constexpr int value = (DT == FSB_C128) ? 2 : (DT == FSB_F64 || DT == FSB_C64) ? 3 : 4; };

// Gather of x for the fused y sums: L2-only.
template <typename T> __device__ __forceinline__ T ld_gather(const T* p) { return __ldcg(p); }
template <> __device__ __forceinline__ __half ld_gather<__half>(const __half* p) {
  return __ushort_as_half(__ldcg(reinterpret_cast<const unsigned short*>(p)));
}
template <> __device__ __forceinline__ __nv_bfloat16 ld_gather<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __ushort_as_bfloat16(__ldcg(reinterpret_cast<const unsigned short*>(p)));
}
__device__ __forceinline__ void put_y(__half& o, float v) { o = __float2half_rn(v); }
__device__ __forceinline__ void put_y(__nv_bfloat16& o, float v) { o = __float2bfloat16_rn(v); }
__device__ __forceinline__ void put_y(float& o, float v) { o = v; }
__device__ __forceinline__ void put_y(double& o, double v) { o = v; }

// y accumulator of the fused SpMM + SpMV.  For 2- and 4-byte values every
// product is exact in fp64, so an fp64 sum is at least as accurate as Dot2 in
// fp32 and costs one DFMA per term; fp64 values keep the Dot2 pair.  A
// long-row partial takes the two real slots of scratch column n.
template <typename R> struct YAcc;
template <> struct YAcc<float> {
  double s;
  __device__ __forceinline__ void zero() { s = 0.0; }
  __device__ __forceinline__ void add_prod(float a, float b) { s = __fma_rn(double(a), double(b), s); }
  __device__ __forceinline__ void shfl_join(int m) { s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, m)); }
  __device__ __forceinline__ void shfl_up(int d) { s = __shfl_up_sync(0xffffffffu, s, d); }
  __device__ __forceinline__ void combine(const YAcc& o) { s = __dadd_rn(s, o.s); }
  __device__ __forceinline__ void store(float* p) const { *reinterpret_cast<double*>(p) = s; }
  __device__ __forceinline__ void add_stored(const float* p) {
    s = __dadd_rn(s, __ldcg(reinterpret_cast<const double*>(p)));
  }
  __device__ __forceinline__ float value() const { return __double2float_rn(s); }
};
template <> struct YAcc<double> {
  Comp<double> c;
  __device__ __forceinline__ void zero() { c.zero(); }
  __device__ __forceinline__ void add_prod(double a, double b) { c.add_prod(a, b); }
  __device__ __forceinline__ void shfl_join(int m) {
    const double oh = __shfl_xor_sync(0xffffffffu, c.hi, m), ol = __shfl_xor_sync(0xffffffffu, c.lo, m);
    c.add_comp(oh, ol);
  }
  __device__ __forceinline__ void shfl_up(int d) {
    c.hi = __shfl_up_sync(0xffffffffu, c.hi, d);
    c.lo = __shfl_up_sync(0xffffffffu, c.lo, d);
  }
  __device__ __forceinline__ void combine(const YAcc& o) { c.add_comp(o.c.hi, o.c.lo); }
  __device__ __forceinline__ void store(double* p) const { p[0] = c.hi; p[1] = c.lo; }
  __device__ __forceinline__ void add_stored(const double* p) { c.add_comp(__ldcg(p), __ldcg(p + 1)); }
  __device__ __forceinline__ double value() const { return c.value(); }
};

template <typename T> __device__ __forceinline__ T ld_once(const T* p) { return __ldcs(p); }
template <> __device__ __forceinline__ __half ld_once<__half>(const __half* p) {
  return __ushort_as_half(__ldcs(reinterpret_cast<const unsigned short*>(p)));
}
template <> __device__ __forceinline__ __nv_bfloat16 ld_once<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short*>(p)));
}

// Asynchronous global -> shared copies of one 4-, 8- or 16-byte element
// (cp.async): every copy of a staging pass is in flight at once, with no
// registers held; cp_async_wait_all() then __syncwarp() before reading.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Stages values and columns [s0, s0 + cnt) (cnt <= MAXN) into the warp's
// shared slices by cp.async, every copy in flight at once; returns the
// offset of value s0 in sh_a (the values start at sh_a + the offset).  2-byte
// values move as 4-byte words from the even element at or below s0 (offset 1
// when s0 is odd; the slice holds MAXN + 2 values); a last value left alone
// in its word is copied by itself, so nothing past value s0 + cnt - 1 is
// read.  The caller's __syncwarp() makes the slices visible to all lanes.
template <typename S, int MAXN>
__device__ __forceinline__ int stage_nz(S* sh_a, int32_t* sh_c, const S* __restrict__ data,
                                        const int32_t* __restrict__ col, int64_t s0, int cnt, int lane) {
  int shift = 0;
  for (int k = lane; k < cnt; k += 32) cp_async<4>(sh_c + k, col + s0 + k);
  if constexpr (sizeof(S) >= 4) {
    for (int k = lane; k < cnt; k += 32) cp_async<int(sizeof(S))>(sh_a + k, data + s0 + k);
  } else {
    shift = static_cast<int>(s0 & 1);
    const S* base = data + (s0 - shift);  // 4-byte aligned (data is)
    const int words = (cnt + shift) >> 1;
    for (int w = lane; w < words; w += 32) cp_async<4>(sh_a + 2 * w, base + 2 * w);
    if (((cnt + shift) & 1) && lane == 0) sh_a[cnt + shift - 1] = ld_once(data + s0 + cnt - 1);
  }
  cp_async_wait_all();
  return shift;
}

// Run-local row offsets off[i] = ptr[r0 + i] - s0 for i <= nr (nr < MAXR),
// every load issued before the first store.
template <int MAXR>
__device__ __forceinline__ void stage_offsets(int32_t* sh_off, const int64_t* __restrict__ ptr, int64_t r0, int nr,
                                              int64_t s0, int lane) {
  constexpr int kQ = (MAXR + 32) / 32;
  int64_t v[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q) {
    const int i = lane + 32 * q;
    if (i <= nr) v[q] = __ldg(ptr + r0 + i);
  }
#pragma unroll
  for (int q = 0; q < kQ; ++q) {
    const int i = lane + 32 * q;
    if (i <= nr) sh_off[i] = static_cast<int32_t>(v[q] - s0);
  }
}

// Rows of more than this many nonzeros accumulate compensated in the types
// whose sums run in fp32 (f16, bf16, f32), whatever the plan's flags: their
// sums are the long ones.  Shorter rows keep the plan's accumulation.  The
// forward kernels use Dot2 (blocked in the team kernel), the backward fp64
// sums of the exact products.
constexpr int64_t kCompensateAbove = 1024;
template <int DT, bool COMP>
constexpr bool kCompLong = !COMP && (DT == FSB_F16 || DT == FSB_BF16 || DT == FSB_F32);

// grid: x = groups of kSpmmWarps units, y = column tiles of 32*V columns.
// pstride: scratch elements per slot; cps: tickets per slot.
template <int DT, int V, bool COMP>
__global__ void __launch_bounds__(kSpmmWarps * 32, SpmmMinBlocks<DT>::value)
k_spmm_csr(const typename VT<DT>::Store* __restrict__ data, const int32_t* __restrict__ col,
           const int64_t* __restrict__ ptr, const typename VT<DT>::Store* __restrict__ B, int64_t ldb, int64_t n,
           typename VT<DT>::Store* __restrict__ C, int64_t ldc, fsb_spmv_plan plan, int64_t pstride, int64_t cps) {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  using Acc = SpmmAcc<DT, COMP, V>;
  constexpr int kER = Acc::kNC * 2;  // scratch reals per element

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t unit = int64_t(blockIdx.x) * kSpmmWarps + warp;
  if (unit >= plan.n_units) return;  // whole warp leaves together
  const int tile = blockIdx.y;
  const int64_t c0 = int64_t(tile) * (kSpmmTileLanes * V) + int64_t(lane) * V;  // this lane's first column
  const int nv = static_cast<int>(n - c0 >= V ? int64_t(V) : (n > c0 ? n - c0 : int64_t(0)));

  unsigned char* wbase = smem_raw + warp * spmm_warp_smem_bytes<S>();
  S* sh_a = reinterpret_cast<S*>(wbase);
  int32_t* sh_c = reinterpret_cast<int32_t*>(wbase + kSpmmBatch * sizeof(S));
  int32_t* sh_off = sh_c + kSpmmBatch;
  uint8_t* sh_rid = reinterpret_cast<uint8_t*>(sh_off + kSpmmMaxCap + 1);

  const fsb_spmv_unit* ud = plan.units + unit;
  const int64_t s0 = __ldg(&ud->nnz_begin), s1 = __ldg(&ud->nnz_end);
  const int32_t row = __ldg(&ud->row), tag = __ldg(&ud->tag);

  auto flush = [&](const Acc& acc, int64_t r) {
    if (nv > 0) {
      S o[V];
      acc.result(o);
      store_slice(C + r * ldc + c0, nv, o);
    }
  };

  if (tag >= 0) {
    // ------------------------------------------------------------ row block
    const int nr = tag - row;
    const int cnt = static_cast<int>(s1 - s0);
    for (int i = lane; i <= nr; i += 32) sh_off[i] = static_cast<int32_t>(__ldg(ptr + row + i) - s0);
    for (int k = lane; k < cnt; k += 32) {
      sh_a[k] = ld_once(data + s0 + k);
      sh_c[k] = ld_once(col + s0 + k);
    }
    __syncwarp();
    for (int k = lane; k < cnt; k += 32) {  // local row of nonzero k: first i with off[i+1] > k
      int lo = 0, hi = nr - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sh_off[mid + 1] > k) hi = mid; else lo = mid + 1;
      }
      sh_rid[k] = static_cast<uint8_t>(lo);
    }
    for (int i0 = 0; i0 < nr; i0 += 32) {  // empty rows get zero slices
      const int i = i0 + lane;
      unsigned m = __ballot_sync(0xffffffffu, i < nr && sh_off[i] == sh_off[i + 1]);
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        Acc z;
        z.zero();
        flush(z, int64_t(row) + i0 + b);
      }
    }
    __syncwarp();
    if (cnt == 0) return;
    Acc acc;
    acc.zero();
    int cur = sh_rid[0];
    for (int k = 0; k < cnt; k += kSpmmAhead) {
      S bv[kSpmmAhead][V];
#pragma unroll
      for (int u = 0; u < kSpmmAhead; ++u) {
        const int kk = k + u < cnt ? k + u : k;
        load_slice<S, V>(B + int64_t(sh_c[kk]) * ldb + c0, k + u < cnt ? nv : 0, bv[u]);
      }
#pragma unroll
      for (int u = 0; u < kSpmmAhead; ++u) {
        if (k + u < cnt) {
          const int r = sh_rid[k + u];
          if (r != cur) {  // uniform across the warp
            flush(acc, int64_t(row) + cur);
            acc.zero();
            cur = r;
          }
          acc.add(sh_a[k + u], bv[u]);
        }
      }
    }
    flush(acc, int64_t(row) + cur);
    return;
  }

  // ------------------------------------------------------------ long-row chunk
  const int32_t nch = __ldg(&ud->n_chunks), slot = __ldg(&ud->slot);
  // A2: the accumulator of this row's chunks (Dot2 for long rows, see kCompLong)
  auto run_chunk = [&](auto proto) {
    using A2 = decltype(proto);
    A2 acc;
    acc.zero();
    for (int64_t b0 = s0; b0 < s1; b0 += kSpmmBatch) {
      const int cnt = static_cast<int>(s1 - b0 < kSpmmBatch ? s1 - b0 : int64_t(kSpmmBatch));
      __syncwarp();
      for (int k = lane; k < cnt; k += 32) {
        sh_a[k] = ld_once(data + b0 + k);
        sh_c[k] = ld_once(col + b0 + k);
      }
      __syncwarp();
      for (int k = 0; k < cnt; k += kSpmmAhead) {
        S bv[kSpmmAhead][V];
#pragma unroll
        for (int u = 0; u < kSpmmAhead; ++u) {
          const int kk = k + u < cnt ? k + u : k;
          load_slice<S, V>(B + int64_t(sh_c[kk]) * ldb + c0, k + u < cnt ? nv : 0, bv[u]);
        }
#pragma unroll
        for (int u = 0; u < kSpmmAhead; ++u)
          if (k + u < cnt) acc.add(sh_a[k + u], bv[u]);
      }
    }
    auto put = [&](const A2& a) {
      if (nv > 0) {
        S o[V];
        a.result(o);
        store_slice(C + int64_t(row) * ldc + c0, nv, o);
      }
    };
    if (nch == 1) {
      put(acc);
      return;
    }
    R* part = static_cast<R*>(plan.partials);
    const int64_t first = int64_t(slot) + (tag + 1);  // slot of the row's first chunk
    acc.store_partial(part + (int64_t(slot) * pstride + c0) * kER);
    __threadfence();
    __syncwarp();
    int ticket = 0;
    if (lane == 0) ticket = atomicAdd(plan.counters + first * cps + tile, 1);
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    if (ticket != nch - 1) return;
    __threadfence();
    A2 fin;
    fin.zero();
#pragma unroll 4
    for (int c = 0; c < nch; ++c) fin.add_partial(part + ((first + c) * pstride + c0) * kER);
    put(fin);
    if (lane == 0) plan.counters[first * cps + tile] = 0;  // ready for the next call
  };
  if (kCompLong<DT, COMP> && int64_t(nch) * plan.chunk_nnz > kCompensateAbove)
    run_chunk(SpmmAcc<DT, true, V>());
  else
    run_chunk(Acc());
}

// ---------------------------------------------------------------------------
// Dense rows made of whole aligned 16-byte slices: the team kernel.  Teams of
// T lanes (1 to 32) own the 16-byte slices of a column tile of T * 16 bytes,
// G = 32 / T teams per warp.  Rows wider than the tile run as several column
// tiles; the tile is the slowest work dimension, so while one tile is in
// flight only that tile's slice of B is being gathered, and a slice that fits
// in L2 is read from HBM about once.
//
// Persistent warps stride over the work items of every tile in tile order.
// An item is either
//  * a row group: up to kRowUnits consecutive row-block units, split into runs
//    of adjacent rows.  A run (<= 256 rows, < 512 nonzeros) is staged in the
//    warp's shared memory and cut by a merge path over its list of row ends
//    and nonzeros: every team walks the same number of positions whatever the
//    row lengths, summing nonzeros and writing a row at its end.  A row that
//    spans teams is finished by a segmented scan over the teams' partial sums
//    (keys: row indices) in team order;
//  * a long-row chunk: team g takes nonzeros g, g+G, ...; the team partials
//    are combined by xor-shuffles over the team index, then the chunk is
//    stored directly (one-chunk rows) or as a slot partial whose ticket's
//    last taker adds the partials in chunk order.
// FUSED: every lane also gathers x[col] beside B's row and sums y = A x for
// the team's rows (identical sums on the team's lanes; lane 0 writes y).
// ---------------------------------------------------------------------------
constexpr int kRowUnits = 4;                            // row-block units per row group
constexpr int kRowStage = kRowUnits * 2 * kSpmmMaxCap;  // staged nonzeros of a run (< 512)
constexpr int kRowRows = kRowUnits * kSpmmMaxCap;       // rows of a run (<= 256)
static_assert(kSpmmBatch <= kRowStage, "the long-row batch must fit the run staging");

// Per-warp slice: staged values, columns and run-local row offsets, then
// (16-byte aligned) one parked accumulator per lane.
template <typename S>
constexpr int spmm_team_vals_bytes() {
  return ((kRowStage + 2) * int(sizeof(S)) + 15) & ~15;  // 2-byte values may start one element early
}
template <typename S>
constexpr int spmm_team_park_offset() {
  return (spmm_team_vals_bytes<S>() + kRowStage * 4 + (kRowRows + 1) * 4 + 15) & ~15;
}
template <int DT, bool COMP>
constexpr int spmm_team_warp_smem_bytes() {
  using S = typename VT<DT>::Store;
  constexpr int V = 16 / int(sizeof(S));
  return spmm_team_park_offset<S>() + 32 * int(sizeof(SpmmAcc<DT, COMP, V>));
}

// Resident blocks the register budget is sized for: 4 (64 registers) for
// plain sums of 2- and 4-byte values, 3 (85) for 8-byte values and for
// compensated or fused sums, 2 for complex fp64.  More resident warps keep
// more B rows in flight: wide rows measured up to 15 % faster at 4 blocks with
// 4 slices ahead than at 3 blocks with 6 ahead.
template <int DT, bool COMP, bool FUSED, int KP>
struct SpmmTeamMinBlocks {
  static constexpr int value = (DT == FSB_C128) ? 2 : (!COMP && !FUSED && DT != FSB_F64 && DT != FSB_C64) ? 4 : 3;
};

// B-row slices a team loads ahead of its sums in the row walk (KP): 4 for
// teams narrower than the warp, 6 for 32-lane teams, whose warp walks its
// rows alone and needs more of them in flight.
template <int DT, bool COMP, int V>
__device__ __forceinline__ void acc_shfl_add(SpmmAcc<DT, COMP, V>& a, int m) {
#pragma unroll
  for (int c = 0; c < SpmmAcc<DT, COMP, V>::kNC; ++c)
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const auto hi = __shfl_xor_sync(0xffffffffu, a.s[c][j].hi, m);
      if constexpr (COMP) {
        const auto lo = __shfl_xor_sync(0xffffffffu, a.s[c][j].lo, m);
        a.s[c][j].add_comp(hi, lo);
      } else {
        a.s[c][j].add(hi);
      }
    }
}

// b = the accumulator of the lane `delta` below (the lane itself where there is none)
template <int DT, bool COMP, int V>
__device__ __forceinline__ void acc_shfl_up(const SpmmAcc<DT, COMP, V>& a, SpmmAcc<DT, COMP, V>& b, int delta) {
#pragma unroll
  for (int c = 0; c < SpmmAcc<DT, COMP, V>::kNC; ++c)
#pragma unroll
    for (int j = 0; j < V; ++j) {
      b.s[c][j].hi = __shfl_up_sync(0xffffffffu, a.s[c][j].hi, delta);
      if constexpr (COMP) b.s[c][j].lo = __shfl_up_sync(0xffffffffu, a.s[c][j].lo, delta);
    }
}

template <int DT, bool COMP, int V>
__device__ __forceinline__ void acc_combine(SpmmAcc<DT, COMP, V>& a, const SpmmAcc<DT, COMP, V>& b) {
#pragma unroll
  for (int c = 0; c < SpmmAcc<DT, COMP, V>::kNC; ++c)
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if constexpr (COMP) a.s[c][j].add_comp(b.s[c][j].hi, b.s[c][j].lo);
      else a.s[c][j].add(b.s[c][j].hi);
    }
}

// a += t elementwise, each add an error-free TwoSum into the compensated a
template <int DT, int V>
__device__ __forceinline__ void acc_fold(SpmmAcc<DT, true, V>& a, const SpmmAcc<DT, false, V>& t) {
#pragma unroll
  for (int c = 0; c < SpmmAcc<DT, true, V>::kNC; ++c)
#pragma unroll
    for (int j = 0; j < V; ++j) a.s[c][j].add(t.s[c][j].hi);
}

// fp64 accumulator for a long row of a real type accumulated in fp32 (bf16,
// f16, f32): each product is exact in fp64 and the fp64 sum of n of them is
// within n 2^-53 sum|a||b| of the exact sum -- inside the Dot2 bound of the
// compensated fp32 sum for rows under 2^26 nonzeros, at one DFMA per term and
// no temporaries.  Partials keep the (hi, lo) fp32 pairs of SpmmAcc<DT, true>.
template <int DT, int V>
struct WideAcc {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  static_assert(std::is_same<R, float>::value, "fp32-accumulated real types only");
  static constexpr int kNC = 1;  // real components per element
  double s[V];

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int j = 0; j < V; ++j) s[j] = 0.0;
  }
  __device__ __forceinline__ void add(S a, const S (&b)[V]) {
    const double ad = to_real(a);
#pragma unroll
    for (int j = 0; j < V; ++j) s[j] = fma(ad, double(to_real(b[j])), s[j]);
  }
  __device__ __forceinline__ void shfl_add(int m) {
#pragma unroll
    for (int j = 0; j < V; ++j) s[j] += __shfl_xor_sync(0xffffffffu, s[j], m);
  }
  __device__ __forceinline__ void result(S (&out)[V]) const {
#pragma unroll
    for (int j = 0; j < V; ++j) out[j] = spmm_store(__double2float_rn(s[j]), static_cast<S*>(nullptr));
  }
  __device__ __forceinline__ void store_partial(R* p) const {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const float hi = __double2float_rn(s[j]);
      p[j * 2] = hi;
      p[j * 2 + 1] = __double2float_rn(s[j] - double(hi));
    }
  }
  __device__ __forceinline__ void add_partial(const R* p) {
#pragma unroll
    for (int j = 0; j < V; ++j) s[j] += double(__ldcg(p + j * 2)) + double(__ldcg(p + j * 2 + 1));
  }
};

template <int DT, int V>
__device__ __forceinline__ void acc_shfl_add(WideAcc<DT, V>& a, int m) { a.shfl_add(m); }

// Accumulation of a long-row chunk: MODE 0 plain sums; 1 Dot2 on every term
// (plans with FSB_SPMM_COMPENSATED); 2 blocked compensation: each step's
// KA products of a team are summed plainly, then folded into a Dot2
// accumulator, so the error is at most gamma_(KA+1) * sum|a||b| plus
// the final rounding whatever the row length (the chunk and team partials
// are combined compensated as well); 3 fp64 sums of the exact products
// (WideAcc), far inside that bound.  Modes 2 and 3 serve the same rows of
// the fp32-accumulated types: 3 in the one-team kernel, where it measured
// faster (fp32, 128 columns: 2.21 against 2.25 ms), 2 elsewhere (fp64 sums
// cost 4-5 % on 256-byte rows).
template <int DT, int MODE, int V>
struct ChunkAcc;
template <int DT, int V>
struct ChunkAcc<DT, 0, V> { using T = SpmmAcc<DT, false, V>; };
template <int DT, int V>
struct ChunkAcc<DT, 1, V> { using T = SpmmAcc<DT, true, V>; };
template <int DT, int V>
struct ChunkAcc<DT, 2, V> { using T = SpmmAcc<DT, true, V>; };
template <int DT, int V>
struct ChunkAcc<DT, 3, V> { using T = WideAcc<DT, V>; };

// One long-row chunk of the team kernel: team g takes nonzeros g, g+G, ...,
// KA B-row slices in flight; the team partials are combined by xor-shuffles
// over the team index, then the chunk is stored directly (one-chunk rows) or
// as a slot partial whose ticket's last taker adds the partials in chunk order.
template <int DT, int MODE, bool FUSED, int KA>
__device__ __forceinline__ void team_chunk(const typename VT<DT>::Store* __restrict__ data,
                                           const int32_t* __restrict__ col,
                                           const typename VT<DT>::Store* __restrict__ B, uint32_t ldb, int64_t n,
                                           typename VT<DT>::Store* __restrict__ C, int64_t ldc,
                                           const fsb_spmv_plan& plan, const fsb_spmv_unit* ud, int T, int64_t tile,
                                           int64_t c0, int nv, int64_t pstride, int64_t cps,
                                           const typename VT<DT>::Store* __restrict__ x,
                                           typename VT<DT>::Store* __restrict__ y, typename VT<DT>::Store* sh_a,
                                           int32_t* sh_c) {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  constexpr int V = 16 / int(sizeof(S));
  using Acc = typename ChunkAcc<DT, MODE, V>::T;
  constexpr int kER = Acc::kNC * 2;
  const int lane = threadIdx.x & 31;
  const int G = 32 / T, team = lane / T;
  const int64_t s0 = __ldg(&ud->nnz_begin), s1 = __ldg(&ud->nnz_end);
  const int32_t row = __ldg(&ud->row), tag = __ldg(&ud->tag);
  const int32_t nch = __ldg(&ud->n_chunks), slot = __ldg(&ud->slot);
  const S* Bl = B + (nv > 0 ? c0 : 0);  // lanes without columns load column 0 and discard it
  Acc acc;
  acc.zero();
  YAcc<R> yacc;
  yacc.zero();
  for (int64_t b0 = s0; b0 < s1; b0 += kRowStage) {
    const int cnt = static_cast<int>(s1 - b0 < kRowStage ? s1 - b0 : int64_t(kRowStage));
    __syncwarp();
    const S* sv = sh_a + stage_nz<S, kRowStage>(sh_a, sh_c, data, col, b0, cnt, lane);
    __syncwarp();
    for (int k = 0; k < cnt; k += KA * G) {
      S bv[KA][V];
      S xv[KA];
#pragma unroll
      for (int q = 0; q < KA; ++q) {
        const int kk = k + q * G + team;
        load_row16<S, V>(Bl, static_cast<uint32_t>(sh_c[kk < cnt ? kk : cnt - 1]), ldb, bv[q]);
      }
      if constexpr (FUSED) {
        // the y terms of these KA * G items, one per lane in order
#pragma unroll
        for (int q = 0; q * 32 < KA * G; ++q) {
          const int kk = k + q * 32 + lane;
          if (q * 32 + lane < KA * G && kk < cnt) xv[q] = ld_gather(x + sh_c[kk]);
        }
      }
      if constexpr (MODE == 2) {
        SpmmAcc<DT, false, V> step;
        step.zero();
#pragma unroll
        for (int q = 0; q < KA; ++q) {
          const int kk = k + q * G + team;
          if (kk < cnt) step.add(sv[kk], bv[q]);
        }
        acc_fold(acc, step);
      } else {
#pragma unroll
        for (int q = 0; q < KA; ++q) {
          const int kk = k + q * G + team;
          if (kk < cnt) acc.add(sv[kk], bv[q]);
        }
      }
      if constexpr (FUSED) {
#pragma unroll
        for (int q = 0; q * 32 < KA * G; ++q) {
          const int kk = k + q * 32 + lane;
          if (q * 32 + lane < KA * G && kk < cnt) yacc.add_prod(to_real(sv[kk]), to_real(xv[q]));
        }
      }
    }
  }
  for (int m = T; m < 32; m <<= 1) acc_shfl_add(acc, m);  // every team now holds the chunk's sum
  if constexpr (FUSED) {
    // every lane's y terms, joined over the warp in a fixed order
    for (int m = 1; m < 32; m <<= 1) yacc.shfl_join(m);
  }
  if (nch == 1) {
    if (team == 0 && nv > 0) {
      S o[V];
      acc.result(o);
      store_slice<S, V, true>(C + int64_t(row) * ldc + c0, nv, o);
    }
    if constexpr (FUSED)
      if (lane == 0 && tile == 0) put_y(y[row], yacc.value());
    return;
  }
  R* part = static_cast<R*>(plan.partials);
  const int64_t first = int64_t(slot) + (tag + 1);  // slot of the row's first chunk
  if (team == 0) acc.store_partial(part + (int64_t(slot) * pstride + c0) * kER);
  if constexpr (FUSED) {
    // y's partial sits in the slot's column n (n < pstride for the fused path)
    if (lane == 0 && tile == 0) yacc.store(part + (int64_t(slot) * pstride + n) * kER);
  }
  __threadfence();
  __syncwarp();
  int ticket = 0;
  if (lane == 0) ticket = atomicAdd(plan.counters + first * cps + tile, 1);
  ticket = __shfl_sync(0xffffffffu, ticket, 0);
  if (ticket != nch - 1) return;
  __threadfence();
  if (team == 0) {
    Acc fin;
    fin.zero();
#pragma unroll 4
    for (int c = 0; c < nch; ++c) fin.add_partial(part + ((first + c) * pstride + c0) * kER);
    if (nv > 0) {
      S o[V];
      fin.result(o);
      store_slice<S, V, true>(C + int64_t(row) * ldc + c0, nv, o);
    }
    if constexpr (FUSED) {
      if (lane == 0 && tile == 0) {
        YAcc<R> fy;
        fy.zero();
        for (int c = 0; c < nch; ++c) fy.add_stored(part + ((first + c) * pstride + n) * kER);
        put_y(y[row], fy.value());
      }
    }
    if (lane == 0) plan.counters[first * cps + tile] = 0;  // ready for the next call
  }
}

template <int DT, bool COMP, bool FUSED, int KP>
__global__ void __launch_bounds__(kSpmmWarps * 32, SpmmTeamMinBlocks<DT, COMP, FUSED, KP>::value)
k_spmm_team(const typename VT<DT>::Store* __restrict__ data, const int32_t* __restrict__ col,
            const int64_t* __restrict__ ptr, const typename VT<DT>::Store* __restrict__ B, uint32_t ldb, int64_t n,
            typename VT<DT>::Store* __restrict__ C, int64_t ldc, fsb_spmv_plan plan, int T, int64_t tiles,
            int64_t pstride, int64_t cps, const typename VT<DT>::Store* __restrict__ x,
            typename VT<DT>::Store* __restrict__ y) {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  constexpr int V = 16 / int(sizeof(S));
  using Acc = SpmmAcc<DT, COMP, V>;
  constexpr int kP = KP;
  // the KP != 4 instantiation runs 32-lane teams only (one team per warp): a
  // run's rows all end inside the team, so it has no scan and parks nothing
  constexpr bool kOneTeam = KP != 4;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int G = 32 / T, team = lane / T, tl = lane % T;
  unsigned char* wbase = smem_raw + warp * spmm_team_warp_smem_bytes<DT, COMP>();
  S* sh_a = reinterpret_cast<S*>(wbase);
  int32_t* sh_c = reinterpret_cast<int32_t*>(wbase + spmm_team_vals_bytes<S>());
  int32_t* sh_off = sh_c + kRowStage;
  Acc* sh_park = reinterpret_cast<Acc*>(wbase + spmm_team_park_offset<S>()) + lane;

  const int64_t nb = plan.n_block_units;
  const uint32_t n_groups = static_cast<uint32_t>(ceil_div(nb, kRowUnits));
  const uint32_t n_items = n_groups + static_cast<uint32_t>(plan.n_units - nb);
  const uint32_t total = n_items * static_cast<uint32_t>(tiles);
  const uint32_t nwarps = gridDim.x * kSpmmWarps;

  for (uint32_t it = blockIdx.x * kSpmmWarps + warp; it < total; it += nwarps) {
    const uint32_t tile = it / n_items, item = it - tile * n_items;
    const int64_t c0 = int64_t(tile) * (int64_t(T) * V) + int64_t(tl) * V;  // this lane's first column
    const int nv = c0 + V <= n ? V : 0;                       // n is a multiple of V
    const S* Bl = B + (nv > 0 ? c0 : 0);  // lanes without columns load column 0 and discard it
    __syncwarp();  // the staging slice of the previous item is free

    if (item < n_groups) {
      // ---------------------------------------------------------- row group
      // lanes 0 .. kRowUnits-1 hold the group's unit descriptors
      const int64_t ua = int64_t(item) * kRowUnits;
      const int nu = static_cast<int>(nb - ua < kRowUnits ? nb - ua : int64_t(kRowUnits));
      int64_t d_s0 = 0, d_s1 = 0;
      int32_t d_row = 0, d_tag = 0;
      if (lane < nu) {
        const int4* p = reinterpret_cast<const int4*>(plan.units + ua + lane);
        const int4 a = __ldg(p), b = __ldg(p + 1);
        d_s0 = (int64_t)(uint32_t)a.x | ((int64_t)a.y << 32);
        d_s1 = (int64_t)(uint32_t)a.z | ((int64_t)a.w << 32);
        d_row = b.x;
        d_tag = b.y;
      }
      int u = 0;
      while (u < nu) {
        // the run: units u .. v-1 whose rows join up (a long row between two
        // units, listed among the chunks, breaks the run)
        const int32_t r0 = __shfl_sync(0xffffffffu, d_row, u);
        const int64_t s0 = __shfl_sync(0xffffffffu, d_s0, u);
        int32_t r1 = __shfl_sync(0xffffffffu, d_tag, u);
        int64_t s1 = __shfl_sync(0xffffffffu, d_s1, u);
        int v = u + 1;
        for (; v < nu; ++v) {
          if (__shfl_sync(0xffffffffu, d_row, v) != r1) break;
          r1 = __shfl_sync(0xffffffffu, d_tag, v);
          s1 = __shfl_sync(0xffffffffu, d_s1, v);
        }
        u = v;
        const int nr = r1 - r0;
        const int cnt = static_cast<int>(s1 - s0);
        __syncwarp();
        const S* sv = sh_a + stage_nz<S, kRowStage>(sh_a, sh_c, data, col, s0, cnt, lane);
        stage_offsets<kRowRows>(sh_off, ptr, r0, nr, s0, lane);
        __syncwarp();
        // empty rows get zero slices (one team each)
        for (int i0 = 0; i0 < nr; i0 += 32) {
          const int i = i0 + lane;
          const bool empty = i < nr && sh_off[i] == sh_off[i + 1];
          unsigned m = __ballot_sync(0xffffffffu, empty);
          for (int q = 0; m; ++q) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            if (q % G == team) {
              if (nv > 0) {
                Acc z;
                z.zero();
                S o[V];
                z.result(o);
                store_slice<S, V, true>(C + (int64_t(r0) + i0 + b) * ldc + c0, nv, o);
              }
              if constexpr (FUSED)
                if (tl == 0 && tile == 0) put_y(y[int64_t(r0) + i0 + b], 0.0f);
            }
          }
        }
        __syncwarp();

        // team g sums nonzeros [jb, je) of the run: an equal share whatever the
        // row lengths.  A row is written by the team holding its last nonzero;
        // the partials of a row spanning several teams are totalled by a
        // segmented scan over the teams (keys: run-local rows).
        const int per = (cnt + G - 1) / G;
        const int jb = min(team * per, cnt), je = min(jb + per, cnt);
        Acc acc;
        acc.zero();
        YAcc<R> yacc, ypark;
        yacc.zero();
        ypark.zero();
        int cur = 0;  // the row of nonzero jb: the last row whose offset is <= jb
        {
          int lo = 0, hi = nr - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sh_off[mid] <= jb) lo = mid; else hi = mid - 1;
          }
          cur = lo;
        }
        int next_end = jb < je ? sh_off[cur + 1] : 0;  // where row cur ends
        bool open_start = jb < je && sh_off[cur] < jb;  // row cur began in an earlier team
        int park_row = -1;
        auto put_row = [&](const Acc& a, const YAcc<R>& ya, int r) {
          if (nv > 0) {
            S o[V];
            a.result(o);
            store_slice<S, V, true>(C + (int64_t(r0) + r) * ldc + c0, nv, o);
          }
          if constexpr (FUSED)
            if (tl == 0 && tile == 0) put_y(y[int64_t(r0) + r], ya.value());
        };
        for (int j0 = jb; j0 < je; j0 += kP) {
          S bv[kP][V];
          S xv[kP];
#pragma unroll
          for (int q = 0; q < kP; ++q) {  // past je: the last nonzero again, loaded and not summed
            const int j = j0 + q < je ? j0 + q : je - 1;
            load_row16<S, V>(Bl, static_cast<uint32_t>(sh_c[j]), ldb, bv[q]);
            if constexpr (FUSED) xv[q] = ld_gather(x + sh_c[j]);
          }
#pragma unroll
          for (int q = 0; q < kP; ++q) {
            const int j = j0 + q;
            if (j < je) {
              if (j == next_end) {  // row cur ended before nonzero j
                if (!kOneTeam && open_start) {
                  *sh_park = acc;  // finished after the scan
                  ypark = yacc;
                  park_row = cur;
                  open_start = false;
                } else {
                  put_row(acc, yacc, cur);
                }
                acc.zero();
                yacc.zero();
                do {  // past the empty rows (already zeroed) to the row of nonzero j
                  ++cur;
                  next_end = sh_off[cur + 1];
                } while (next_end == j);
              }
              const S a = sv[j];
              acc.add(a, bv[q]);
              if constexpr (FUSED) yacc.add_prod(to_real(a), to_real(xv[q]));
            }
          }
        }
        if constexpr (kOneTeam) {  // one team walked the whole run: its last row ends here
          if (jb < je) put_row(acc, yacc, cur);
          __syncwarp();
          continue;
        }
        const bool open_end = jb < je && next_end > je;  // row cur goes on in later teams
        // inclusive segmented scan of the open-ended partials over the teams
        const int key = open_end ? cur : -1;
        Acc sc = acc;
        YAcc<R> ysc = yacc;
        if (!open_end) {
          sc.zero();
          ysc.zero();
        }
        for (int o = 1; o < G; o <<= 1) {
          Acc other;
          acc_shfl_up(sc, other, o * T);
          YAcc<R> oy = ysc;
          if constexpr (FUSED) oy.shfl_up(o * T);
          const int okey = __shfl_up_sync(0xffffffffu, key, o * T);
          if (team >= o && key >= 0 && okey == key) {
            acc_combine(sc, other);
            if constexpr (FUSED) ysc.combine(oy);
          }
        }
        Acc carry;
        acc_shfl_up(sc, carry, T);
        YAcc<R> ycarry = ysc;
        if constexpr (FUSED) ycarry.shfl_up(T);
        // the partials of earlier teams belong to the row this team began inside
        if (park_row >= 0) {
          Acc f = *sh_park;
          acc_combine(f, carry);
          if constexpr (FUSED) ypark.combine(ycarry);
          put_row(f, ypark, park_row);
        }
        if (jb < je && !open_end) {
          if (open_start) {  // this team holds the end of a row begun before it
            acc_combine(acc, carry);
            if constexpr (FUSED) yacc.combine(ycarry);
          }
          put_row(acc, yacc, cur);
        }
        __syncwarp();  // the staging slice is rewritten by the next run
      }
      continue;
    }

    // ------------------------------------------------------------ long-row chunk
    const fsb_spmv_unit* ud = plan.units + nb + (item - n_groups);
    const int32_t nch = __ldg(&ud->n_chunks);
    // rows of more than kCompensateAbove nonzeros sum compensated in the
    // fp32-accumulated types, partials and all (blocked Dot2, or fp64 sums
    // in the one-team kernel)
    if constexpr (COMP) {
      team_chunk<DT, 1, FUSED, KP>(data, col, B, ldb, n, C, ldc, plan, ud, T, tile, c0, nv, pstride, cps, x, y,
                                   sh_a, sh_c);
      continue;
    }
    if constexpr (kCompLong<DT, COMP>) {
      if (int64_t(nch) * plan.chunk_nnz > kCompensateAbove) {
        team_chunk<DT, (KP > kSpmmAhead ? 3 : 2), FUSED, KP>(data, col, B, ldb, n, C, ldc, plan, ud, T, tile, c0, nv,
                                                             pstride, cps, x, y, sh_a, sh_c);
        continue;
      }
    }
    team_chunk<DT, 0, FUSED, KP>(data, col, B, ldb, n, C, ldc, plan, ud, T, tile, c0, nv, pstride, cps, x, y, sh_a,
                                 sh_c);
  }
}

// ---------------------------------------------------------------------------
// Backward of Y = A X in one launch, over the unit plan of A^T (built with the
// SpMM window and chunk).  Nonzero q of A^T sits in row c (a column of A) and
// column r (a row of A) and is nonzero p = perm[q] of A:
//   dX[c]   += vals[p] * dY[r]      A^T dY, laid out as in k_spmm_team
//   dvals[p] = <dY[r], X[c]>        the SDDMM of dY and X on A's pattern
// The dY row slice of each nonzero is gathered once and serves both sums; A's
// values are read through perm (no transposed copy), and X[c] is loaded once
// per row of A^T.  Teams of T lanes (T * V >= n, T <= 32) own 16-byte column
// slices.  The dot products of each group of slices loaded ahead reduce across
// the team by a transpose butterfly (log2 of the group size halving steps, then
// plain xor steps) in a fixed order; the lanes left holding a finished product
// write it.  With DV false dvals is not formed (dX only).  X is read with
// streaming loads and dX written with streaming stores, which keep more of the
// gathered dY rows in L2 (measured 0.5 % faster).
// ---------------------------------------------------------------------------
// dY row slices loaded ahead of the sums: 8 for 4- and 8-byte values, 4 for
// half / bfloat16, whose 8-wide slices and widened products spill at 8
template <int DT>
struct BwdAhead { static constexpr int value = (DT == FSB_F16 || DT == FSB_BF16) ? 4 : 8; };

template <typename S>
constexpr int spmm_bwd_warp_smem_bytes() {
  return (kSpmmBatch * (int(sizeof(S)) + 8) + (kSpmmMaxCap + 1) * 4 + 15) & ~15;
}

// Reduces d[0..M) of every lane across the T lanes of its team.  On return the
// lane holds the team sums of items first .. first + held - 1 in d[0..held),
// and `writer` is set on exactly one lane of each group holding the same items.
template <typename R, int M>
__device__ __forceinline__ void team_transpose_sum(R (&d)[M], int T, int tl, int& first, int& held, bool& writer) {
  first = 0;
  held = M;
  int m = T >> 1;
#pragma unroll
  for (int h = M / 2; h >= 1; h >>= 1) {
    if (m == 0) break;  // teams narrower than M keep M / T items per lane
    const bool up = (tl & m) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const R keep = up ? d[i + h] : d[i];
      const R send = up ? d[i] : d[i + h];
      d[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
    }
    if (up) first += h;
    held = h;
    m >>= 1;
  }
  const int rest = m;  // lanes tl and tl ^ j (j < 2 * rest) now hold the same items
  for (; m > 0; m >>= 1) d[0] += __shfl_xor_sync(0xffffffffu, d[0], m);
  writer = (tl & (2 * rest - 1)) == 0 || rest == 0;
}

// (c0, c1) += (a0 * b0, a1 * b1) in one packed fp32x2 FMA, each half rounded
// as a scalar fma.rn.
__device__ __forceinline__ void ffma2x(float& c0, float& c1, float a0, float a1, float b0, float b1) {
  unsigned long long cc, aa, bb;
  asm("mov.b64 %0, {%1, %2};" : "=l"(cc) : "f"(c0), "f"(c1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(aa) : "f"(a0), "f"(a1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(bb) : "f"(b0), "f"(b1));
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(cc) : "l"(aa), "l"(bb));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(c0), "=f"(c1) : "l"(cc));
}

// Per-lane partial dot products of the kA dY slices with this lane's X slice
// (already widened to R); fp32 sums run as two packed halves added at the end.
// (c0, c1) += (lo(x) * lo(b), hi(x) * hi(b)) for packed 16-bit x and b, one
// rounding each (see fma_mixed2).
template <typename S>
__device__ __forceinline__ void fma_mixed2x(float& c0, float& c1, unsigned x, unsigned b) {
  if constexpr (std::is_same<S, __nv_bfloat16>::value) {
    asm("{\n .reg .b16 xl, xh, bl, bh;\n mov.b32 {xl, xh}, %2;\n mov.b32 {bl, bh}, %3;\n"
        " fma.rn.f32.bf16 %0, bl, xl, %0;\n fma.rn.f32.bf16 %1, bh, xh, %1;\n}"
        : "+f"(c0), "+f"(c1) : "r"(x), "r"(b));
  } else {
    asm("{\n .reg .b16 xl, xh, bl, bh;\n mov.b32 {xl, xh}, %2;\n mov.b32 {bl, bh}, %3;\n"
        " fma.rn.f32.f16 %0, bl, xl, %0;\n fma.rn.f32.f16 %1, bh, xh, %1;\n}"
        : "+f"(c0), "+f"(c1) : "r"(x), "r"(b));
  }
}

// xs: the same X slice as xf, unwidened (16-bit values multiply from it).
template <typename S, typename R, int KA, int V>
__device__ __forceinline__ void bwd_dots(const S (&bv)[KA][V], const R (&xf)[V], const S (&xs)[V], R (&d)[KA]) {
#pragma unroll
  for (int u = 0; u < KA; ++u) {
    if constexpr (sizeof(S) == 2 && V % 2 == 0) {
      unsigned xw[V / 2], bw[V / 2];
      memcpy(xw, xs, sizeof(xw));
      memcpy(bw, bv[u], sizeof(bw));
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int j = 0; j < V / 2; ++j) fma_mixed2x<S>(s0, s1, xw[j], bw[j]);
      d[u] = s0 + s1;
    } else if constexpr (std::is_same<R, float>::value && V % 2 == 0) {
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int j = 0; j < V; j += 2) ffma2x(s0, s1, to_real(bv[u][j]), to_real(bv[u][j + 1]), xf[j], xf[j + 1]);
      d[u] = s0 + s1;
    } else {
      R s = R(0);
#pragma unroll
      for (int j = 0; j < V; ++j) s = fma(to_real(bv[u][j]), xf[j], s);
      d[u] = s;
    }
  }
}

// Team sums of d, each written once to dvals[perm of its staged entry]; item u
// of the group is staged entry base + u * stride, present when below limit.
template <typename S, typename R, int KA>
__device__ __forceinline__ void bwd_put_dots(R (&d)[KA], int base, int stride, int limit, int T, int tl,
                                             const int32_t* sh_p, S* __restrict__ dvals) {
  int first, held;
  bool writer;
  team_transpose_sum<R, KA>(d, T, tl, first, held, writer);
  if (!writer) return;
#pragma unroll
  for (int i = 0; i < KA; ++i) {
    const int k = base + (first + i) * stride;
    if (i < held && k < limit) dvals[sh_p[k]] = spmm_store(d[i], static_cast<S*>(nullptr));
  }
}

template <int DT, bool DV>
__global__ void __launch_bounds__(kSpmmWarps * 32, SpmmMinBlocks<DT>::value)
k_spmm_bwd(const typename VT<DT>::Store* __restrict__ vals, const int32_t* __restrict__ perm,
           const int32_t* __restrict__ col, const int64_t* __restrict__ ptr,
           const typename VT<DT>::Store* __restrict__ dY, int64_t lddy, int64_t n,
           const typename VT<DT>::Store* __restrict__ X, int64_t ldx, typename VT<DT>::Store* __restrict__ dX,
           int64_t lddx, typename VT<DT>::Store* __restrict__ dvals, fsb_spmv_plan plan, int T, int64_t pstride,
           int64_t cps) {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  constexpr int V = 16 / int(sizeof(S));
  using Acc = SpmmAcc<DT, false, V>;
  constexpr int kER = Acc::kNC * 2;
  constexpr int kA = BwdAhead<DT>::value;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t unit = int64_t(blockIdx.x) * kSpmmWarps + warp;
  if (unit >= plan.n_units) return;  // whole warp leaves together
  const int G = 32 / T, team = lane / T, tl = lane % T;
  const int64_t c0 = int64_t(tl) * V;
  const int nv = c0 + V <= n ? V : 0;  // n is a multiple of V

  unsigned char* wbase = smem_raw + warp * spmm_bwd_warp_smem_bytes<S>();
  S* sh_a = reinterpret_cast<S*>(wbase);
  int32_t* sh_c = reinterpret_cast<int32_t*>(wbase + kSpmmBatch * sizeof(S));
  int32_t* sh_p = sh_c + kSpmmBatch;
  int32_t* sh_off = sh_p + kSpmmBatch;

  const fsb_spmv_unit* ud = plan.units + unit;
  const int64_t s0 = __ldg(&ud->nnz_begin), s1 = __ldg(&ud->nnz_end);
  const int32_t row = __ldg(&ud->row), tag = __ldg(&ud->tag);

  // stages a batch of <= kSpmmBatch nonzeros (a strided loop: unrolling the
  // loads ahead costs registers that the gathers below need)
  auto stage = [&](int64_t from, int cnt) {
    for (int k = lane; k < cnt; k += 32) {
      const int32_t p = ld_once(perm + from + k);
      sh_p[k] = p;
      sh_a[k] = vals[p];
      sh_c[k] = ld_once(col + from + k);
    }
  };
  if (tag >= 0) {
    // ------------------------------------------------------------ row block
    const int nr = tag - row;
    const int cnt = static_cast<int>(s1 - s0);
    stage_offsets<kSpmmMaxCap>(sh_off, ptr, row, nr, s0, lane);
    stage(s0, cnt);
    __syncwarp();
    for (int i0 = 0; i0 < nr; i0 += G) {
      const int i = i0 + team;
      const bool has = i < nr;
      const int b = has ? sh_off[i] : 0;
      const int len = has ? sh_off[i + 1] - b : 0;
      int maxlen = len;
      for (int m = T; m < 32; m <<= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, m));
      R xf[V];
      S xs[V];
      if constexpr (DV) {
        load_slice<S, V, true>(X + (int64_t(row) + (has ? i : 0)) * ldx + c0, len > 0 ? nv : 0, xs);
#pragma unroll
        for (int j = 0; j < V; ++j) xf[j] = to_real(xs[j]);
      }
      Acc acc;
      acc.zero();
      for (int k = 0; k < maxlen; k += kA) {
        S bv[kA][V];
#pragma unroll
        for (int u = 0; u < kA; ++u) {
          const bool ok = k + u < len;
          load_slice<S, V>(dY + int64_t(sh_c[ok ? b + k + u : 0]) * lddy + c0, ok ? nv : 0, bv[u]);
        }
#pragma unroll
        for (int u = 0; u < kA; ++u)
          if (k + u < len) acc.add(sh_a[b + k + u], bv[u]);
        if constexpr (DV) {
          R d[kA];
          bwd_dots<S, R, kA, V>(bv, xf, xs, d);
          bwd_put_dots<S, R, kA>(d, b + k, 1, b + len, T, tl, sh_p, dvals);
        }
      }
      if (has && nv > 0) {
        S o[V];
        acc.result(o);
        store_slice<S, V, true>(dX + (int64_t(row) + i) * lddx + c0, nv, o);
      }
    }
    return;
  }

  // ------------------------------------------------------------ long-row chunk
  const int32_t nch = __ldg(&ud->n_chunks), slot = __ldg(&ud->slot);
  R xf[V];
  S xs[V];
  if constexpr (DV) {
    load_slice<S, V, true>(X + int64_t(row) * ldx + c0, nv, xs);
#pragma unroll
    for (int j = 0; j < V; ++j) xf[j] = to_real(xs[j]);
  }
  // WIDE (rows over kCompensateAbove nonzeros, see kCompLong): fp64 sums of
  // the exact products (WideAcc) with kA / 2 dY slices in flight, which keeps
  // the kernel within the plain path's registers (measured on the 500,000-node
  // Chung-Lu graph, 128 columns: fp32 no slower than plain sums, bf16 3.5 %
  // slower; Dot2 sums cost 3.5 % / 8 %); else plain sums
  auto run_chunk = [&](auto wide) {
    constexpr bool kWide = decltype(wide)::value;
    using A2 = typename std::conditional<kWide, WideAcc<DT, V>, Acc>::type;
    constexpr int kAc = kWide ? kA / 2 : kA;
    A2 acc;
    acc.zero();
    for (int64_t b0 = s0; b0 < s1; b0 += kSpmmBatch) {
      const int cnt = static_cast<int>(s1 - b0 < kSpmmBatch ? s1 - b0 : int64_t(kSpmmBatch));
      __syncwarp();
      stage(b0, cnt);
      __syncwarp();
      for (int k = 0; k < cnt; k += kAc * G) {
        S bv[kAc][V];
#pragma unroll
        for (int u = 0; u < kAc; ++u) {
          const int kk = k + u * G + team;
          load_slice<S, V>(dY + int64_t(sh_c[kk < cnt ? kk : 0]) * lddy + c0, kk < cnt ? nv : 0, bv[u]);
        }
#pragma unroll
        for (int u = 0; u < kAc; ++u) {
          const int kk = k + u * G + team;
          if (kk < cnt) acc.add(sh_a[kk], bv[u]);
        }
        if constexpr (DV) {
          R d[kAc];
          bwd_dots<S, R, kAc, V>(bv, xf, xs, d);
          bwd_put_dots<S, R, kAc>(d, k + team, G, cnt, T, tl, sh_p, dvals);
        }
      }
    }
    for (int m = T; m < 32; m <<= 1) acc_shfl_add(acc, m);  // every team now holds the chunk's sum
    if (nch == 1) {
      if (team == 0 && nv > 0) {
        S o[V];
        acc.result(o);
        store_slice<S, V, true>(dX + int64_t(row) * lddx + c0, nv, o);
      }
      return;
    }
    R* part = static_cast<R*>(plan.partials);
    const int64_t first = int64_t(slot) + (tag + 1);
    if (team == 0) acc.store_partial(part + (int64_t(slot) * pstride + c0) * kER);
    __threadfence();
    __syncwarp();
    int ticket = 0;
    if (lane == 0) ticket = atomicAdd(plan.counters + first * cps, 1);
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    if (ticket != nch - 1) return;
    __threadfence();
    if (team != 0) return;
    A2 fin;
    fin.zero();
#pragma unroll 4
    for (int c = 0; c < nch; ++c) fin.add_partial(part + ((first + c) * pstride + c0) * kER);
    if (nv > 0) {
      S o[V];
      fin.result(o);
      store_slice<S, V, true>(dX + int64_t(row) * lddx + c0, nv, o);
    }
    if (lane == 0) plan.counters[first * cps] = 0;  // ready for the next call
  };
  if constexpr (kCompLong<DT, false>) {
    if (int64_t(nch) * plan.chunk_nnz > kCompensateAbove) {
      run_chunk(std::true_type());
      return;
    }
  }
  run_chunk(std::false_type());
}

}  // namespace
}  // namespace fsb

namespace fsb {
namespace {

inline int64_t spmm_real_bytes(int dtype) {
  switch (dtype) {
    case FSB_F16: case FSB_BF16: case FSB_F32: case FSB_C64: return 4;
    case FSB_F64: case FSB_C128: return 8;
    default: return -1;
  }
}

inline int64_t spmm_elem_bytes(int dtype) {
  switch (dtype) {
    case FSB_F16: case FSB_BF16: return 2;
    case FSB_F32: return 4;
    case FSB_F64: case FSB_C64: return 8;
    case FSB_C128: return 16;
    default: return -1;
  }
}

inline int64_t spmm_pstride(int64_t n) { return ceil_div(n, 256) * 256; }
// Tickets per slot: one per column tile.  The narrowest tile of any kernel is
// one 16-byte slice, so ceil(n * elem / 16) covers every tiling.
inline int64_t spmm_cps_bytes(int64_t n, int64_t elem) { return n > 0 ? ceil_div(n * elem, 16) : 1; }
template <int DT>
inline int64_t spmm_cps(int64_t n) { return spmm_cps_bytes(n, sizeof(typename VT<DT>::Store)); }

// Column tile of the team kernel, in bytes (a power of two, 16 .. 512).  The
// default is the whole row (rounded up to a power of two of 16-byte slices) up
// to 512 bytes.  A positive `hint` (fsb_spmv_plan.tile_bytes) asks for
// narrower tiles: then only a tile's slice of B (n_cols x tile bytes) is
// gathered at a time, which stays in L2 when it fits, at the cost of reading
// A once per tile.  On B200 the whole-row tile measured faster for every
// width up to 512 bytes on 1,000,000-row matrices (fp32 N = 128: 2.4 ms
// against 3.6 ms at 128-byte and 5.5 ms at 64-byte tiles), so narrow tiles
// are opt-in.
inline int spmm_team_tile_bytes(int64_t row_bytes, int32_t hint) {
  int w = 16;
  while (w < row_bytes && w < 512) w *= 2;
  if (hint > 0) {
    int h = 16;
    while (h < hint && h < 512) h *= 2;
    return h < w ? h : w;
  }
  return w;
}

template <int DT, int V, bool COMP>
int spmm_launch_v(const void* data, const int32_t* idx, const int64_t* ptr, const void* B, int64_t ldb, int64_t n,
                  void* C, int64_t ldc, const fsb_spmv_plan& plan, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  const int64_t tiles = ceil_div(n, kSpmmTileLanes * V);
  if (tiles > 65535) return FSB_ERR_UNSUPPORTED;
  const int64_t blocks = ceil_div(plan.n_units, kSpmmWarps);
  const size_t smem = size_t(spmm_warp_smem_bytes<S>()) * kSpmmWarps;
  dim3 grid((unsigned)blocks, (unsigned)tiles);
  k_spmm_csr<DT, V, COMP><<<grid, kSpmmWarps * 32, smem, st>>>(
      static_cast<const S*>(data), idx, ptr, static_cast<const S*>(B), ldb, n, static_cast<S*>(C), ldc, plan,
      spmm_pstride(n), spmm_cps<DT>(n));
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

// Widest per-lane vector (elements) that 32 lanes need for N columns and that
// the B / C base addresses and leading dimensions allow.
template <int DT>
int spmm_pick_v(const void* B, int64_t ldb, const void* C, int64_t ldc, int64_t n) {
  using S = typename VT<DT>::Store;
  constexpr int kVmax = 16 / int(sizeof(S));
  int v = 1;
  while (v < kVmax && int64_t(kSpmmTileLanes) * v < n) v *= 2;
  auto ok = [&](int w) {
    const uintptr_t a = uintptr_t(w) * sizeof(S);
    return reinterpret_cast<uintptr_t>(B) % a == 0 && reinterpret_cast<uintptr_t>(C) % a == 0 && ldb % w == 0 &&
           ldc % w == 0;
  };
  while (v > 1 && !ok(v)) v /= 2;
  return v;
}

// The team kernel: one work item per warp, the items of every tile in tile
// order (tile bytes = T * 16), so the blocks of one tile run together; with
// FSB_SPMM_PERSISTENT, the resident blocks, whose warps stride over the items
// in the same order.
template <int DT, bool COMP, bool FUSED = false>
int spmm_launch_team(const void* data, const int32_t* idx, const int64_t* ptr, const void* B, int64_t ldb, int64_t n,
                     void* C, int64_t ldc, const fsb_spmv_plan& plan, int T, int64_t tiles, cudaStream_t st,
                     const void* x = nullptr, void* y = nullptr) {
  using S = typename VT<DT>::Store;
  const size_t smem = size_t(spmm_team_warp_smem_bytes<DT, COMP>()) * kSpmmWarps;
  const int wide = (!FUSED && T == 32) ? 1 : 0;
  auto kern = wide ? k_spmm_team<DT, COMP, FUSED, 6> : k_spmm_team<DT, COMP, FUSED, 4>;
  if (smem > 48 * 1024) {  // opt in to the larger dynamic shared memory once per kernel and device
    static std::atomic<uint64_t> done[2];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
      (void)cudaGetLastError();
      return FSB_ERR_CUDA;
    }
    const uint64_t bit = uint64_t(1) << (dev & 63);
    if (!(done[wide].load(std::memory_order_acquire) & bit)) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return FSB_ERR_CUDA;
      }
      done[wide].fetch_or(bit, std::memory_order_release);
    }
  }
  const int64_t nb = plan.n_block_units;
  const int64_t items = (ceil_div(nb, kRowUnits) + (plan.n_units - nb)) * tiles;
  int64_t blocks = ceil_div(items, kSpmmWarps);  // one work item per warp, tiles in block order
  if (items >= (int64_t(1) << 32) || blocks > INT32_MAX || ldb > UINT32_MAX) return FSB_ERR_UNSUPPORTED;
  if (blocks < 1) return FSB_OK;
  if (plan.flags & FSB_SPMM_PERSISTENT) {  // the resident blocks; warps stride over the items
    static std::atomic<int64_t> resident[2][64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
      (void)cudaGetLastError();
      return FSB_ERR_CUDA;
    }
    int64_t r = resident[wide][dev].load(std::memory_order_acquire);
    if (r == 0) {
      int per_sm = 0, sms = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSpmmWarps * 32, smem) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || per_sm < 1 ||
          sms < 1) {
        (void)cudaGetLastError();
        return FSB_ERR_CUDA;
      }
      r = int64_t(per_sm) * sms;
      resident[wide][dev].store(r, std::memory_order_release);
    }
    if (blocks > r) blocks = r;
  }
  kern<<<(unsigned)blocks, kSpmmWarps * 32, smem, st>>>(
      static_cast<const S*>(data), idx, ptr, static_cast<const S*>(B), static_cast<uint32_t>(ldb), n,
      static_cast<S*>(C), ldc, plan, T, tiles, spmm_pstride(n), spmm_cps<DT>(n), static_cast<const S*>(x),
      static_cast<S*>(y));
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

// C = A B and y = A x in one launch: the team kernel with the fused y sums.
// Real types, narrow aligned rows (the team conditions) and n < the slot
// stride, so that y's long-row partial has a column of its own.
template <int DT>
int spmm_spmv_fused(const void* data, const int32_t* idx, const int64_t* ptr, const void* B, int64_t ldb, int64_t n,
                    void* C, int64_t ldc, const void* x, void* y, const fsb_spmv_plan& plan, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  constexpr int kVmax = 16 / int(sizeof(S));
  if constexpr (VT<DT>::kComplex) {
    return FSB_ERR_UNSUPPORTED;
  } else {
    if (!(n * int64_t(sizeof(S)) <= 256 && n % kVmax == 0 && ldb % kVmax == 0 && ldc % kVmax == 0 &&
          reinterpret_cast<uintptr_t>(B) % 16 == 0 && reinterpret_cast<uintptr_t>(C) % 16 == 0 &&
          n < spmm_pstride(n)))
      return FSB_ERR_UNSUPPORTED;
    int T = 1;
    while (int64_t(T) * kVmax < n) T *= 2;
    if (plan.flags & FSB_SPMM_COMPENSATED)
      return spmm_launch_team<DT, true, true>(data, idx, ptr, B, ldb, n, C, ldc, plan, T, 1, st, x, y);
    return spmm_launch_team<DT, false, true>(data, idx, ptr, B, ldb, n, C, ldc, plan, T, 1, st, x, y);
  }
}

// dX = A^T dY (and dvals = SDDMM(dY, X) on A's pattern when dvals is given) in
// one launch of k_spmm_bwd.  Real types, 16-byte aligned rows of at most 512
// bytes whose width n is a multiple of 16 / sizeof(value); plain sums, fp64
// sums on rows over kCompensateAbove nonzeros for the fp32-accumulated types.
template <int DT>
int spmm_backward(const void* vals, const int32_t* perm, const int32_t* idx, const int64_t* ptr, const void* dY,
                  int64_t lddy, const void* X, int64_t ldx, int64_t n, void* dX, int64_t lddx, void* dvals,
                  const fsb_spmv_plan& plan, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  constexpr int kVmax = 16 / int(sizeof(S));
  if constexpr (VT<DT>::kComplex) {
    return FSB_ERR_UNSUPPORTED;
  } else {
    auto a16 = [](const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; };
    if (!(n * int64_t(sizeof(S)) <= 512 && n % kVmax == 0 && lddy % kVmax == 0 && lddx % kVmax == 0 && a16(dY) &&
          a16(dX) && (!dvals || (ldx % kVmax == 0 && a16(X)))) ||
        (plan.flags & FSB_SPMM_COMPENSATED))
      return FSB_ERR_UNSUPPORTED;
    int T = 1;
    while (int64_t(T) * kVmax < n) T *= 2;
    const int64_t blocks = ceil_div(plan.n_units, kSpmmWarps);
    const size_t smem = size_t(spmm_bwd_warp_smem_bytes<S>()) * kSpmmWarps;
    const S* v = static_cast<const S*>(vals);
    if (dvals) {
      k_spmm_bwd<DT, true><<<(unsigned)blocks, kSpmmWarps * 32, smem, st>>>(
          v, perm, idx, ptr, static_cast<const S*>(dY), lddy, n, static_cast<const S*>(X), ldx,
          static_cast<S*>(dX), lddx, static_cast<S*>(dvals), plan, T, spmm_pstride(n), spmm_cps<DT>(n));
    } else {
      k_spmm_bwd<DT, false><<<(unsigned)blocks, kSpmmWarps * 32, smem, st>>>(
          v, perm, idx, ptr, static_cast<const S*>(dY), lddy, n, nullptr, 0, static_cast<S*>(dX), lddx, nullptr,
          plan, T, spmm_pstride(n), spmm_cps<DT>(n));
    }
    FSB_LAUNCH_CHECK();
    return FSB_OK;
  }
}

template <int DT, bool COMP>
int spmm_dispatch(const void* data, const int32_t* idx, const int64_t* ptr, const void* B, int64_t ldb, int64_t n,
                  int64_t n_cols, void* C, int64_t ldc, const fsb_spmv_plan& plan, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  constexpr int kVmax = 16 / int(sizeof(S));
  // rows of whole, aligned 16-byte slices: teams of T lanes over column tiles
  // of T * 16 bytes (spmm_team_tile_bytes)
  if (n % kVmax == 0 && ldb % kVmax == 0 && ldc % kVmax == 0 && reinterpret_cast<uintptr_t>(B) % 16 == 0 &&
      reinterpret_cast<uintptr_t>(C) % 16 == 0 && ldb <= UINT32_MAX && n_cols < (int64_t(1) << 32)) {
    const int w = spmm_team_tile_bytes(n * int64_t(sizeof(S)), plan.tile_bytes);
    const int T = w / 16;
    return spmm_launch_team<DT, COMP>(data, idx, ptr, B, ldb, n, C, ldc, plan, T, ceil_div(n, int64_t(T) * kVmax),
                                      st);
  }
  const int v = spmm_pick_v<DT>(B, ldb, C, ldc, n);
  if constexpr (kVmax >= 8)
    if (v == 8) return spmm_launch_v<DT, 8, COMP>(data, idx, ptr, B, ldb, n, C, ldc, plan, st);
  if constexpr (kVmax >= 4)
    if (v == 4) return spmm_launch_v<DT, 4, COMP>(data, idx, ptr, B, ldb, n, C, ldc, plan, st);
  if constexpr (kVmax >= 2)
    if (v == 2) return spmm_launch_v<DT, 2, COMP>(data, idx, ptr, B, ldb, n, C, ldc, plan, st);
  return spmm_launch_v<DT, 1, COMP>(data, idx, ptr, B, ldb, n, C, ldc, plan, st);
}

template <int DT>
int spmm_mode(const void* data, const int32_t* idx, const int64_t* ptr, const void* B, int64_t ldb, int64_t n,
              int64_t n_cols, void* C, int64_t ldc, const fsb_spmv_plan& plan, cudaStream_t st) {
  if (plan.flags & FSB_SPMM_COMPENSATED)
    return spmm_dispatch<DT, true>(data, idx, ptr, B, ldb, n, n_cols, C, ldc, plan, st);
  return spmm_dispatch<DT, false>(data, idx, ptr, B, ldb, n, n_cols, C, ldc, plan, st);
}

}  // namespace
}  // namespace fsb

using namespace fsb;

extern "C" {

int32_t fsb_spmm_default_cap(int dtype) { (void)dtype; return kSpmmMaxCap; }

int32_t fsb_spmm_default_chunk(int dtype) { (void)dtype; return 2 * kSpmmBatch; }

int fsb_spmm_scratch_layout(int dtype, int64_t n, int64_t* partial_bytes_per_slot, int64_t* tickets_per_slot) {
  const int64_t rb = spmm_real_bytes(dtype);
  if (rb < 0) return FSB_ERR_UNSUPPORTED;
  if (n < 0 || !partial_bytes_per_slot || !tickets_per_slot) return FSB_ERR_INVALID_ARG;
  const int64_t comps = (dtype == FSB_C64 || dtype == FSB_C128) ? 2 : 1;
  *partial_bytes_per_slot = spmm_pstride(n) * comps * 2 * rb;
  *tickets_per_slot = spmm_cps_bytes(n, spmm_elem_bytes(dtype));
  return FSB_OK;
}

int fsb_spmm_csr(int dtype, const void* data, const int32_t* indices, const int64_t* indptr, int64_t n_rows,
                 int64_t n_cols, const void* B, int64_t ldb, int64_t n, void* C, int64_t ldc,
                 const fsb_spmv_plan* plan, void* stream) {
  if (!plan || n_rows < 0 || n_cols < 0 || n < 0 || ldb < n || ldc < n) return FSB_ERR_INVALID_ARG;
  if (n_rows == 0 || n == 0) return FSB_OK;
  if (!indptr || !C || !plan->units || plan->n_units < 1 || plan->cap < 1 || plan->cap > kSpmmMaxCap ||
      plan->chunk_nnz < kSpmmBatch || plan->chunk_nnz % kSpmmBatch != 0 || plan->n_slots < 0 ||
      (plan->n_slots > 0 && (!plan->partials || !plan->counters)))
    return FSB_ERR_INVALID_ARG;
  if (n_cols > 0 && !B) return FSB_ERR_INVALID_ARG;
  if (plan->n_units >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16: return spmm_mode<FSB_F16>(data, indices, indptr, B, ldb, n, n_cols, C, ldc, *plan, st);
    case FSB_BF16: return spmm_mode<FSB_BF16>(data, indices, indptr, B, ldb, n, n_cols, C, ldc, *plan, st);
    case FSB_F32: return spmm_mode<FSB_F32>(data, indices, indptr, B, ldb, n, n_cols, C, ldc, *plan, st);
    case FSB_F64: return spmm_mode<FSB_F64>(data, indices, indptr, B, ldb, n, n_cols, C, ldc, *plan, st);
    case FSB_C64: return spmm_mode<FSB_C64>(data, indices, indptr, B, ldb, n, n_cols, C, ldc, *plan, st);
    case FSB_C128: return spmm_mode<FSB_C128>(data, indices, indptr, B, ldb, n, n_cols, C, ldc, *plan, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

int fsb_spmm_spmv_csr(int dtype, const void* data, const int32_t* indices, const int64_t* indptr, int64_t n_rows,
                      int64_t n_cols, const void* B, int64_t ldb, int64_t n, void* C, int64_t ldc, const void* x,
                      void* y, const fsb_spmv_plan* plan, void* stream) {
  if (!plan || n_rows < 0 || n_cols < 0 || n < 1 || ldb < n || ldc < n || !x || !y) return FSB_ERR_INVALID_ARG;
  if (n_rows == 0) return FSB_OK;
  if (!indptr || !C || !plan->units || plan->n_units < 1 || plan->cap < 1 || plan->cap > kSpmmMaxCap ||
      plan->chunk_nnz < kSpmmBatch || plan->chunk_nnz % kSpmmBatch != 0 || plan->n_slots < 0 ||
      (plan->n_slots > 0 && (!plan->partials || !plan->counters)))
    return FSB_ERR_INVALID_ARG;
  if (n_cols > 0 && !B) return FSB_ERR_INVALID_ARG;
  if (plan->n_units >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16: return spmm_spmv_fused<FSB_F16>(data, indices, indptr, B, ldb, n, C, ldc, x, y, *plan, st);
    case FSB_BF16: return spmm_spmv_fused<FSB_BF16>(data, indices, indptr, B, ldb, n, C, ldc, x, y, *plan, st);
    case FSB_F32: return spmm_spmv_fused<FSB_F32>(data, indices, indptr, B, ldb, n, C, ldc, x, y, *plan, st);
    case FSB_F64: return spmm_spmv_fused<FSB_F64>(data, indices, indptr, B, ldb, n, C, ldc, x, y, *plan, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

int fsb_spmm_csr_backward(int dtype, const void* vals, const int32_t* perm, const int32_t* t_indices,
                          const int64_t* t_indptr, int64_t n_rows, int64_t n_cols, const void* dY, int64_t lddy,
                          const void* X, int64_t ldx, int64_t n, void* dX, int64_t lddx, void* dvals,
                          const fsb_spmv_plan* t_plan, void* stream) {
  const fsb_spmv_plan* plan = t_plan;
  if (!plan || n_rows < 0 || n_cols < 0 || n < 0 || lddy < n || lddx < n || !dX || (dvals && (!X || ldx < n)))
    return FSB_ERR_INVALID_ARG;
  if (n == 0) return FSB_ERR_UNSUPPORTED;  // dvals would be all zero: left to the separate kernels
  if (n_cols == 0) return FSB_OK;
  if (!t_indptr || !plan->units || plan->n_units < 1 || plan->cap < 1 || plan->cap > kSpmmMaxCap ||
      plan->chunk_nnz < kSpmmBatch || plan->chunk_nnz % kSpmmBatch != 0 || plan->n_slots < 0 ||
      (plan->n_slots > 0 && (!plan->partials || !plan->counters)))
    return FSB_ERR_INVALID_ARG;
  if (n_rows > 0 && !dY) return FSB_ERR_INVALID_ARG;
  if (plan->n_units >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16:
      return spmm_backward<FSB_F16>(vals, perm, t_indices, t_indptr, dY, lddy, X, ldx, n, dX, lddx, dvals, *plan, st);
    case FSB_BF16:
      return spmm_backward<FSB_BF16>(vals, perm, t_indices, t_indptr, dY, lddy, X, ldx, n, dX, lddx, dvals, *plan,
                                     st);
    case FSB_F32:
      return spmm_backward<FSB_F32>(vals, perm, t_indices, t_indptr, dY, lddy, X, ldx, n, dX, lddx, dvals, *plan, st);
    case FSB_F64:
      return spmm_backward<FSB_F64>(vals, perm, t_indices, t_indptr, dY, lddy, X, ldx, n, dX, lddx, dvals, *plan, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

}  // extern "C"

// BSR SpMV y = A x for sm_100a, any block dimension.
//
// Blocks are stored row-major, blocks[k][r][c], so row r of block k is a
// contiguous run of bd values and the x slice a block multiplies,
// x[bcol * bd, bcol * bd + bd), is contiguous too.  One thread owns one
// (padded) row: it walks the blocks of its block row, two blocks per step so
// several loads are in flight, and reads its bd-value row slice and the x
// slice with 16-byte vector loads whenever bd * sizeof(value) is a multiple
// of 16 (the threads of a block row read the block's rows side by side; x is
// shared by all of them through L1).  Sums are compensated (Dot2) and run in
// block order, so results are deterministic; every padded row is written,
// empty block rows with 0.
//
// op = trans / conj runs the same kernel on A^T, prepared once by
// fsb_csr_transpose on the block pattern plus fsb_bsr_transpose_values.
//
// Replaces _spmv_bsr_non_real_kernel / _spmv_bsr_non_complex_kernel,
// _spmv_bsr_blockrow_reduce_*_kernel and _spmv_bsr_trans_*_kernel
// (sparse_operations/spmv_bsr.py:183-446) of flagos-ai/FlagSparse, which
// accumulate per BLOCK_NNZ segment with atomic adds.
#include <algorithm>

#include "fsb_common.cuh"

namespace fsb {

template <typename S>
struct alignas(16) Vec16 {
  static constexpr int N = 16 / int(sizeof(S));
  S v[N];
};

template <typename S>
__device__ __forceinline__ Vec16<S> ld_vec_stream(const S* p) {
  union { uint4 u; Vec16<S> s; } t;
  t.u = __ldcs(reinterpret_cast<const uint4*>(p));
  return t.s;
}
template <typename S>
__device__ __forceinline__ Vec16<S> ld_vec(const S* p) {
  union { uint4 u; Vec16<S> s; } t;
  t.u = __ldg(reinterpret_cast<const uint4*>(p));
  return t.s;
}

template <typename S> __device__ __forceinline__ S ld_one(const S* p) { return *p; }

// compensated accumulator for real and complex values
template <int DT, bool CPLX = VT<DT>::kComplex>
struct BsrAcc;

__device__ __forceinline__ void put_rn(float v, __half& o) { o = __float2half_rn(v); }
__device__ __forceinline__ void put_rn(float v, __nv_bfloat16& o) { o = __float2bfloat16_rn(v); }
__device__ __forceinline__ void put_rn(float v, float& o) { o = v; }
__device__ __forceinline__ void put_rn(double v, double& o) { o = v; }

template <int DT>
struct BsrAcc<DT, false> {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  Comp<R> c;
  __device__ __forceinline__ void zero() { c.zero(); }
  __device__ __forceinline__ void add(S a, S x) { c.add_prod(to_real(a), to_real(x)); }
  __device__ __forceinline__ void shfl_combine(int m) {
    const R oh = __shfl_xor_sync(0xffffffffu, c.hi, m), ol = __shfl_xor_sync(0xffffffffu, c.lo, m);
    c.add_comp(oh, ol);
  }
  __device__ __forceinline__ S result() const { S o; put_rn(c.value(), o); return o; }
};

template <int DT>
struct BsrAcc<DT, true> {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  Comp<R> re, im;
  __device__ __forceinline__ void zero() { re.zero(); im.zero(); }
  __device__ __forceinline__ void add(S a, S x) {
    re.add_prod(a.x, x.x); re.add_prod(-a.y, x.y);
    im.add_prod(a.x, x.y); im.add_prod(a.y, x.x);
  }
  __device__ __forceinline__ void shfl_combine(int m) {
    R oh = __shfl_xor_sync(0xffffffffu, re.hi, m), ol = __shfl_xor_sync(0xffffffffu, re.lo, m);
    re.add_comp(oh, ol);
    oh = __shfl_xor_sync(0xffffffffu, im.hi, m);
    ol = __shfl_xor_sync(0xffffffffu, im.lo, m);
    im.add_comp(oh, ol);
  }
  __device__ __forceinline__ S result() const { S s; s.x = re.value(); s.y = im.value(); return s; }
};

template <int DT, typename IT, typename PT, bool VEC>
__global__ void __launch_bounds__(256)
k_bsr_spmv(const typename VT<DT>::Store* __restrict__ blocks, const IT* __restrict__ bcol,
           const PT* __restrict__ bptr, int64_t n_block_rows, int bd, const typename VT<DT>::Store* __restrict__ x,
           typename VT<DT>::Store* __restrict__ y) {
  using S = typename VT<DT>::Store;
  constexpr int E = Vec16<S>::N;
  const int64_t row = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (row >= n_block_rows * bd) return;
  const int64_t br = row / bd;
  const int r = static_cast<int>(row - br * bd);
  const int64_t k0 = ld_ptr(bptr, br), k1 = ld_ptr(bptr, br + 1);
  const int64_t bb = int64_t(bd) * bd;
  BsrAcc<DT> acc;
  acc.zero();
  int64_t k = k0;
  for (; k + 1 < k1; k += 2) {
    const int64_t c0 = static_cast<int64_t>(__ldg(bcol + k)), c1 = static_cast<int64_t>(__ldg(bcol + k + 1));
    const S* a0 = blocks + k * bb + int64_t(r) * bd;
    const S* a1 = a0 + bb;
    const S* x0 = x + c0 * bd;
    const S* x1 = x + c1 * bd;
    if constexpr (VEC) {
      for (int c = 0; c < bd; c += E) {
        const Vec16<S> va0 = ld_vec_stream(a0 + c), va1 = ld_vec_stream(a1 + c);
        const Vec16<S> vx0 = ld_vec(x0 + c), vx1 = ld_vec(x1 + c);
#pragma unroll
        for (int e = 0; e < E; ++e) acc.add(va0.v[e], vx0.v[e]);
#pragma unroll
        for (int e = 0; e < E; ++e) acc.add(va1.v[e], vx1.v[e]);
      }
    } else {
      for (int c = 0; c < bd; ++c) acc.add(ld_one(a0 + c), __ldg(x0 + c));
      for (int c = 0; c < bd; ++c) acc.add(ld_one(a1 + c), __ldg(x1 + c));
    }
  }
  if (k < k1) {
    const int64_t c0 = static_cast<int64_t>(__ldg(bcol + k));
    const S* a0 = blocks + k * bb + int64_t(r) * bd;
    const S* x0 = x + c0 * bd;
    if constexpr (VEC) {
      for (int c = 0; c < bd; c += E) {
        const Vec16<S> va0 = ld_vec_stream(a0 + c);
        const Vec16<S> vx0 = ld_vec(x0 + c);
#pragma unroll
        for (int e = 0; e < E; ++e) acc.add(va0.v[e], vx0.v[e]);
      }
    } else {
      for (int c = 0; c < bd; ++c) acc.add(ld_one(a0 + c), __ldg(x0 + c));
    }
  }
  y[row] = acc.result();
}

// Wide blocks (bd * sizeof(value) of 64 or 128 bytes and bd >= 32 / CPR):
// one warp per block row.  A block row's block is CPR = bd * s / 16 chunks of
// 16 bytes per row; lane l owns chunk column l % CPR and rows
// l / CPR + p * (32 / CPR) for the P = bd * CPR / 32 passes, so each pass is
// one fully coalesced 512-byte load of the block and the lane's x chunk is
// loaded once per block.  The CPR lanes of a row are reduced by xor shuffles
// at the end, in a fixed order.
template <int DT, int BD, typename IT, typename PT>
__global__ void __launch_bounds__(256)
k_bsr_spmv_warp(const typename VT<DT>::Store* __restrict__ blocks, const IT* __restrict__ bcol,
                const PT* __restrict__ bptr, int64_t n_block_rows, const typename VT<DT>::Store* __restrict__ x,
                typename VT<DT>::Store* __restrict__ y) {
  using S = typename VT<DT>::Store;
  constexpr int E = Vec16<S>::N;
  constexpr int CPR = BD / E;           // 16-byte chunks per block row
  constexpr int RPP = 32 / CPR;         // rows per pass
  constexpr int P = BD / RPP;           // passes per block
  static_assert(CPR >= 1 && 32 % CPR == 0 && BD % RPP == 0 && P >= 1, "unsupported wide-block shape");
  const int lane = threadIdx.x & 31;
  const int64_t br = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (br >= n_block_rows) return;
  const int cc = lane % CPR, r0 = lane / CPR;
  const int64_t k0 = ld_ptr(bptr, br), k1 = ld_ptr(bptr, br + 1);
  constexpr int64_t BB = int64_t(BD) * BD;
  BsrAcc<DT> acc[P];
#pragma unroll
  for (int p = 0; p < P; ++p) acc[p].zero();
  // two blocks per step while the loads of both fit in registers
  constexpr bool kPair = P <= 2;
  int64_t k = k0;
  for (; kPair && k + 1 < k1; k += 2) {
    const int64_t c0 = static_cast<int64_t>(__ldg(bcol + k)), c1 = static_cast<int64_t>(__ldg(bcol + k + 1));
    const Vec16<S> vx0 = ld_vec(x + c0 * BD + cc * E), vx1 = ld_vec(x + c1 * BD + cc * E);
    const S* a0 = blocks + k * BB + int64_t(r0) * BD + cc * E;
    Vec16<S> va0[P], va1[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      va0[p] = ld_vec_stream(a0 + p * RPP * BD);
      va1[p] = ld_vec_stream(a0 + BB + p * RPP * BD);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
      for (int e = 0; e < E; ++e) acc[p].add(va0[p].v[e], vx0.v[e]);
#pragma unroll
      for (int e = 0; e < E; ++e) acc[p].add(va1[p].v[e], vx1.v[e]);
    }
  }
  for (; k < k1; ++k) {
    const int64_t c0 = static_cast<int64_t>(__ldg(bcol + k));
    const Vec16<S> vx0 = ld_vec(x + c0 * BD + cc * E);
    const S* a0 = blocks + k * BB + int64_t(r0) * BD + cc * E;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const Vec16<S> va = ld_vec_stream(a0 + p * RPP * BD);
#pragma unroll
      for (int e = 0; e < E; ++e) acc[p].add(va.v[e], vx0.v[e]);
    }
  }
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int m = 1; m < CPR; m <<= 1) acc[p].shfl_combine(m);
    if (cc == 0) y[br * BD + p * RPP + r0] = acc[p].result();
  }
}

// dst[j][r][c] = src[perm[j]][c][r] (conjugated when CONJ): the values of A^T's
// blocks, in the order of the transposed block pattern.
template <typename S, bool CONJ>
__global__ void k_bsr_transpose_values(const S* __restrict__ src, const int64_t* __restrict__ perm, int64_t nnzb,
                                       int bd, S* __restrict__ dst) {
  const int64_t bb = int64_t(bd) * bd;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nnzb * bb) return;
  const int64_t j = i / bb;
  const int rc = static_cast<int>(i - j * bb);
  const int r = rc / bd, c = rc - r * bd;
  S v = src[perm[j] * bb + int64_t(c) * bd + r];
  if constexpr (CONJ) v.y = -v.y;
  dst[i] = v;
}

static inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <int DT, typename IT, typename PT>
static int bsr_spmv_launch(const void* blocks, const void* idx, const void* ptr, int64_t n_block_rows, int bd,
                           const void* x, void* y, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  const int64_t rows = n_block_rows * bd;
  if (rows == 0) return FSB_OK;
  const unsigned B = 256;
  const unsigned G = (unsigned)ceil_div(rows, B);
  const bool vec = (int64_t(bd) * int64_t(sizeof(S))) % 16 == 0 && aligned16(blocks) && aligned16(x);
  if (vec) {
    // wide blocks: one warp per block row
    const unsigned GW = (unsigned)ceil_div(n_block_rows * 32, B);
    auto wide = [&](auto kern) {
      kern<<<GW, B, 0, st>>>(static_cast<const S*>(blocks), static_cast<const IT*>(idx), static_cast<const PT*>(ptr),
                             n_block_rows, static_cast<const S*>(x), static_cast<S*>(y));
      return true;
    };
    bool done = false;
    if constexpr (sizeof(S) == 4 && !VT<DT>::kComplex) {
      if (bd == 16) done = wide(k_bsr_spmv_warp<DT, 16, IT, PT>);
      else if (bd == 32) done = wide(k_bsr_spmv_warp<DT, 32, IT, PT>);
    } else if constexpr (sizeof(S) == 8) {
      if (bd == 8) done = wide(k_bsr_spmv_warp<DT, 8, IT, PT>);
      else if (bd == 16) done = wide(k_bsr_spmv_warp<DT, 16, IT, PT>);
    } else if constexpr (sizeof(S) == 16) {
      if (bd == 8) done = wide(k_bsr_spmv_warp<DT, 8, IT, PT>);
    }
    if (done) {
      FSB_LAUNCH_CHECK();
      return FSB_OK;
    }
  }
  if (vec) {
    k_bsr_spmv<DT, IT, PT, true><<<G, B, 0, st>>>(static_cast<const S*>(blocks), static_cast<const IT*>(idx),
                                                   static_cast<const PT*>(ptr), n_block_rows, bd,
                                                   static_cast<const S*>(x), static_cast<S*>(y));
  } else {
    k_bsr_spmv<DT, IT, PT, false><<<G, B, 0, st>>>(static_cast<const S*>(blocks), static_cast<const IT*>(idx),
                                                    static_cast<const PT*>(ptr), n_block_rows, bd,
                                                    static_cast<const S*>(x), static_cast<S*>(y));
  }
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

template <int DT>
static int bsr_spmv_dispatch(const void* blocks, const void* idx, int i64, const void* ptr, int p64,
                             int64_t n_block_rows, int bd, const void* x, void* y, cudaStream_t st) {
  if (i64) {
    return p64 ? bsr_spmv_launch<DT, int64_t, int64_t>(blocks, idx, ptr, n_block_rows, bd, x, y, st)
               : bsr_spmv_launch<DT, int64_t, int32_t>(blocks, idx, ptr, n_block_rows, bd, x, y, st);
  }
  return p64 ? bsr_spmv_launch<DT, int32_t, int64_t>(blocks, idx, ptr, n_block_rows, bd, x, y, st)
             : bsr_spmv_launch<DT, int32_t, int32_t>(blocks, idx, ptr, n_block_rows, bd, x, y, st);
}

}  // namespace fsb

using namespace fsb;

extern "C" {

int fsb_bsr_spmv(int dtype, const void* blocks, const void* indices, int idx_is_64, const void* indptr,
                 int ptr_is_64, int64_t n_block_rows, int64_t n_block_cols, int block_dim, const void* x, void* y,
                 void* stream) {
  if (n_block_rows < 0 || n_block_cols < 0 || block_dim < 1 || !indptr || (n_block_rows > 0 && !y))
    return FSB_ERR_INVALID_ARG;
  if (n_block_rows * int64_t(block_dim) >= INT32_MAX * int64_t(256)) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16: return bsr_spmv_dispatch<FSB_F16>(blocks, indices, idx_is_64, indptr, ptr_is_64, n_block_rows, block_dim, x, y, st);
    case FSB_BF16: return bsr_spmv_dispatch<FSB_BF16>(blocks, indices, idx_is_64, indptr, ptr_is_64, n_block_rows, block_dim, x, y, st);
    case FSB_F32: return bsr_spmv_dispatch<FSB_F32>(blocks, indices, idx_is_64, indptr, ptr_is_64, n_block_rows, block_dim, x, y, st);
    case FSB_F64: return bsr_spmv_dispatch<FSB_F64>(blocks, indices, idx_is_64, indptr, ptr_is_64, n_block_rows, block_dim, x, y, st);
    case FSB_C64: return bsr_spmv_dispatch<FSB_C64>(blocks, indices, idx_is_64, indptr, ptr_is_64, n_block_rows, block_dim, x, y, st);
    case FSB_C128: return bsr_spmv_dispatch<FSB_C128>(blocks, indices, idx_is_64, indptr, ptr_is_64, n_block_rows, block_dim, x, y, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

int fsb_bsr_transpose_values(int dtype, const void* src, const int64_t* perm, int64_t nnzb, int block_dim, int conj,
                             void* dst, void* stream) {
  if (nnzb < 0 || block_dim < 1 || (nnzb > 0 && (!src || !perm || !dst))) return FSB_ERR_INVALID_ARG;
  if (nnzb == 0) return FSB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = nnzb * int64_t(block_dim) * block_dim;
  const unsigned B = 256;
  const unsigned G = (unsigned)ceil_div(n, B);
  switch (dtype) {
    case FSB_F16: case FSB_BF16:
      k_bsr_transpose_values<uint16_t, false><<<G, B, 0, st>>>(static_cast<const uint16_t*>(src), perm, nnzb,
                                                                block_dim, static_cast<uint16_t*>(dst));
      break;
    case FSB_F32:
      k_bsr_transpose_values<float, false><<<G, B, 0, st>>>(static_cast<const float*>(src), perm, nnzb, block_dim,
                                                             static_cast<float*>(dst));
      break;
    case FSB_F64:
      k_bsr_transpose_values<double, false><<<G, B, 0, st>>>(static_cast<const double*>(src), perm, nnzb, block_dim,
                                                              static_cast<double*>(dst));
      break;
    case FSB_C64:
      if (conj)
        k_bsr_transpose_values<float2, true><<<G, B, 0, st>>>(static_cast<const float2*>(src), perm, nnzb, block_dim,
                                                               static_cast<float2*>(dst));
      else
        k_bsr_transpose_values<float2, false><<<G, B, 0, st>>>(static_cast<const float2*>(src), perm, nnzb,
                                                                block_dim, static_cast<float2*>(dst));
      break;
    case FSB_C128:
      if (conj)
        k_bsr_transpose_values<double2, true><<<G, B, 0, st>>>(static_cast<const double2*>(src), perm, nnzb,
                                                                block_dim, static_cast<double2*>(dst));
      else
        k_bsr_transpose_values<double2, false><<<G, B, 0, st>>>(static_cast<const double2*>(src), perm, nnzb,
                                                                 block_dim, static_cast<double2*>(dst));
      break;
    default: return FSB_ERR_UNSUPPORTED;
  }
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

}  // extern "C"

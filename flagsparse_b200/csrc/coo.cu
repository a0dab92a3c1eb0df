// COO -> CSR conversion for sm_100a: the on-ramp that feeds COO triples to
// the CSR SpMV.
//
//  * fsb_coo_inspect: one pass over the (row, col) pairs counting pairs out of
//    (row, col) order and indices outside the matrix.
//  * fsb_coo_to_csr: for ordered input, the column indices are narrowed to
//    int32 and the row pointers are read off the row boundaries; otherwise a
//    stable LSD radix sort of the packed key row * 2^cbits + col (CUB
//    DeviceRadixSort over rbits + cbits bits) gives the CSR order, its
//    permutation (source position of every CSR entry, applied to the values by
//    fsb_gather_values) and, from the sorted rows, the row pointers.
//
// Replaces coo_to_csr_for_spmv / _coo_is_sorted_lex
// (sparse_operations/spmv_csr.py:948-984) of flagos-ai/FlagSparse, whose
// argsort + bincount + cumsum give the same CSR for distinct (row, col)
// pairs; for repeated pairs the stable sort keeps their input order.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>

#include "fsb_common.cuh"

namespace fsb {

template <typename T>
__device__ __forceinline__ int64_t ld_idx(const T* p, int64_t i) {
  return static_cast<int64_t>(__ldg(p + i));
}

// out[0] += pairs (i-1, i) out of (row, col) order, out[1] += rows outside
// [0, n_rows), out[2] += columns outside [0, n_cols).
template <typename RT, typename CT>
__global__ void k_coo_inspect(const RT* row, const CT* col, int64_t nnz, int64_t n_rows, int64_t n_cols,
                              unsigned long long* out) {
  unsigned long long unsorted = 0, bad_r = 0, bad_c = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = ld_idx(row, i), c = ld_idx(col, i);
    bad_r += (r < 0 || r >= n_rows);
    bad_c += (c < 0 || c >= n_cols);
    if (i > 0) {
      const int64_t rp = ld_idx(row, i - 1), cp = ld_idx(col, i - 1);
      unsorted += (r < rp || (r == rp && c < cp));
    }
  }
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    unsorted += __shfl_xor_sync(0xffffffffu, unsorted, m);
    bad_r += __shfl_xor_sync(0xffffffffu, bad_r, m);
    bad_c += __shfl_xor_sync(0xffffffffu, bad_c, m);
  }
  if ((threadIdx.x & 31) == 0) {
    if (unsorted) atomicAdd(out + 0, unsorted);
    if (bad_r) atomicAdd(out + 1, bad_r);
    if (bad_c) atomicAdd(out + 2, bad_c);
  }
}

template <typename RT, typename CT>
__global__ void k_coo_keys(const RT* row, const CT* col, int64_t nnz, int cbits, uint64_t* keys, int32_t* pos) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nnz) {
    const uint64_t cmask = (uint64_t(1) << cbits) - 1;
    keys[i] = (uint64_t(ld_idx(row, i)) << cbits) | (uint64_t(ld_idx(col, i)) & cmask);
    pos[i] = static_cast<int32_t>(i);
  }
}

// Sorted order: CSR columns and the source positions.
__global__ void k_coo_sorted_cols(const uint64_t* keys, const int32_t* pos, int64_t nnz, int cbits, int32_t* out_col,
                                  int64_t* perm) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nnz) {
    out_col[i] = static_cast<int32_t>(keys[i] & ((uint64_t(1) << cbits) - 1));
    perm[i] = pos[i];
  }
}

template <typename CT>
__global__ void k_coo_copy_cols(const CT* col, int64_t nnz, int32_t* out_col) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nnz) out_col[i] = static_cast<int32_t>(ld_idx(col, i));
}

// Row pointers from non-decreasing row ids: boundary i (between entries i-1
// and i, i in [0, nnz]) owns rows (row[i-1], row[i]] and writes ptr[r] = i for
// them; rows are clamped to [0, n_rows], so no store leaves the array.
struct RowsFromKeys {
  const uint64_t* keys;
  int cbits;
  __device__ __forceinline__ int64_t operator()(int64_t i) const { return int64_t(keys[i] >> cbits); }
};
template <typename RT>
struct RowsFromArray {
  const RT* row;
  __device__ __forceinline__ int64_t operator()(int64_t i) const { return ld_idx(row, i); }
};

template <typename Rows>
__global__ void k_coo_row_ptr(Rows rows, int64_t nnz, int64_t n_rows, int64_t* ptr) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i > nnz) return;
  int64_t lo = (i == 0) ? 0 : rows(i - 1) + 1;
  int64_t hi = (i == nnz) ? n_rows : rows(i);
  lo = lo < 0 ? 0 : lo;
  hi = hi > n_rows ? n_rows : hi;
  for (int64_t r = lo; r <= hi; ++r) ptr[r] = i;
}

static int coo_bits(int64_t n) {
  int b = 1;
  while (b < 62 && (int64_t(1) << b) < n) ++b;
  return b;
}

struct CooWs {
  uint64_t* keys_in; uint64_t* keys_out; int32_t* pos_in; int32_t* pos_out;
  void* cub_tmp; size_t cub_bytes; int64_t total;
};

static inline int64_t coo_align256(int64_t b) { return (b + 255) & ~int64_t(255); }

static int coo_layout(int64_t nnz, int64_t n_rows, int64_t n_cols, void* base, CooWs& ws) {
  size_t cub_bytes = 0;
  const int bits = coo_bits(n_rows) + coo_bits(n_cols);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                                  (const int32_t*)nullptr, (int32_t*)nullptr, (int)nnz, 0, bits);
  if (e != cudaSuccess) return FSB_ERR_CUDA;
  char* p = static_cast<char*>(base);
  int64_t off = 0;
  auto take = [&](int64_t bytes) { char* q = p ? p + off : nullptr; off += coo_align256(bytes); return q; };
  ws.keys_in = reinterpret_cast<uint64_t*>(take(8 * nnz));
  ws.keys_out = reinterpret_cast<uint64_t*>(take(8 * nnz));
  ws.pos_in = reinterpret_cast<int32_t*>(take(4 * nnz));
  ws.pos_out = reinterpret_cast<int32_t*>(take(4 * nnz));
  ws.cub_tmp = take(int64_t(cub_bytes));
  ws.cub_bytes = cub_bytes;
  ws.total = off;
  return FSB_OK;
}

template <typename RT, typename CT>
static int coo_inspect_impl(const void* row, const void* col, int64_t nnz, int64_t n_rows, int64_t n_cols,
                            int64_t* d_out, cudaStream_t st) {
  if (cudaMemsetAsync(d_out, 0, 3 * sizeof(int64_t), st) != cudaSuccess) {
    (void)cudaGetLastError();
    return FSB_ERR_CUDA;
  }
  if (nnz == 0) return FSB_OK;
  const int64_t blocks = std::min<int64_t>(ceil_div(nnz, 256), int64_t(148) * 8);
  k_coo_inspect<RT, CT><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const RT*>(row), static_cast<const CT*>(col),
                                                           nnz, n_rows, n_cols,
                                                           reinterpret_cast<unsigned long long*>(d_out));
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

template <typename RT, typename CT>
static int coo_to_csr_impl(const void* row_v, const void* col_v, int64_t nnz, int64_t n_rows, int64_t n_cols,
                           int sorted, void* workspace, int64_t workspace_bytes, int32_t* out_col, int64_t* out_ptr,
                           int64_t* perm, cudaStream_t st) {
  const RT* row = static_cast<const RT*>(row_v);
  const CT* col = static_cast<const CT*>(col_v);
  const unsigned B = 256;
  if (sorted || nnz == 0) {
    if (nnz > 0) {
      k_coo_copy_cols<CT><<<(unsigned)ceil_div(nnz, B), B, 0, st>>>(col, nnz, out_col);
      FSB_LAUNCH_CHECK();
    }
    k_coo_row_ptr<RowsFromArray<RT>><<<(unsigned)ceil_div(nnz + 1, B), B, 0, st>>>(RowsFromArray<RT>{row}, nnz,
                                                                                    n_rows, out_ptr);
    FSB_LAUNCH_CHECK();
    return FSB_OK;
  }
  if (!perm || !workspace) return FSB_ERR_INVALID_ARG;
  CooWs ws;
  int rc = coo_layout(nnz, n_rows, n_cols, workspace, ws);
  if (rc != FSB_OK) return rc;
  if (workspace_bytes < ws.total) return FSB_ERR_WORKSPACE;
  const int cbits = coo_bits(n_cols);
  const int bits = coo_bits(n_rows) + cbits;
  k_coo_keys<RT, CT><<<(unsigned)ceil_div(nnz, B), B, 0, st>>>(row, col, nnz, cbits, ws.keys_in, ws.pos_in);
  FSB_LAUNCH_CHECK();
  size_t tmp = ws.cub_bytes;
  if (cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.keys_in, ws.keys_out, ws.pos_in, ws.pos_out, (int)nnz, 0,
                                      bits, st) != cudaSuccess) {
    (void)cudaGetLastError();
    return FSB_ERR_CUDA;
  }
  k_coo_sorted_cols<<<(unsigned)ceil_div(nnz, B), B, 0, st>>>(ws.keys_out, ws.pos_out, nnz, cbits, out_col, perm);
  FSB_LAUNCH_CHECK();
  k_coo_row_ptr<RowsFromKeys><<<(unsigned)ceil_div(nnz + 1, B), B, 0, st>>>(RowsFromKeys{ws.keys_out, cbits}, nnz,
                                                                             n_rows, out_ptr);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

}  // namespace fsb

using namespace fsb;

extern "C" {

int fsb_coo_inspect(const void* row, int row_is_64, const void* col, int col_is_64, int64_t nnz, int64_t n_rows,
                    int64_t n_cols, int64_t* d_out, void* stream) {
  if (!d_out || nnz < 0 || n_rows < 0 || n_cols < 0 || (nnz > 0 && (!row || !col))) return FSB_ERR_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (row_is_64) {
    return col_is_64 ? coo_inspect_impl<int64_t, int64_t>(row, col, nnz, n_rows, n_cols, d_out, st)
                     : coo_inspect_impl<int64_t, int32_t>(row, col, nnz, n_rows, n_cols, d_out, st);
  }
  return col_is_64 ? coo_inspect_impl<int32_t, int64_t>(row, col, nnz, n_rows, n_cols, d_out, st)
                   : coo_inspect_impl<int32_t, int32_t>(row, col, nnz, n_rows, n_cols, d_out, st);
}

int64_t fsb_coo_to_csr_workspace_bytes(int64_t nnz, int64_t n_rows, int64_t n_cols) {
  if (nnz < 0 || nnz > INT32_MAX || n_rows < 0 || n_cols < 0) return -1;
  if (nnz == 0) return 0;
  CooWs ws;
  if (coo_layout(nnz, n_rows, n_cols, nullptr, ws) != FSB_OK) return -1;
  return ws.total;
}

int fsb_coo_to_csr(const void* row, int row_is_64, const void* col, int col_is_64, int64_t nnz, int64_t n_rows,
                   int64_t n_cols, int sorted, void* workspace, int64_t workspace_bytes, int32_t* out_col,
                   int64_t* out_ptr, int64_t* perm, void* stream) {
  if (nnz < 0 || n_rows < 0 || n_cols < 0 || !out_ptr || (nnz > 0 && (!row || !col || !out_col)))
    return FSB_ERR_INVALID_ARG;
  if (nnz > INT32_MAX || n_rows >= INT32_MAX || n_cols >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (row_is_64) {
    return col_is_64 ? coo_to_csr_impl<int64_t, int64_t>(row, col, nnz, n_rows, n_cols, sorted, workspace,
                                                         workspace_bytes, out_col, out_ptr, perm, st)
                     : coo_to_csr_impl<int64_t, int32_t>(row, col, nnz, n_rows, n_cols, sorted, workspace,
                                                         workspace_bytes, out_col, out_ptr, perm, st);
  }
  return col_is_64 ? coo_to_csr_impl<int32_t, int64_t>(row, col, nnz, n_rows, n_cols, sorted, workspace,
                                                       workspace_bytes, out_col, out_ptr, perm, st)
                   : coo_to_csr_impl<int32_t, int32_t>(row, col, nnz, n_rows, n_cols, sorted, workspace,
                                                       workspace_bytes, out_col, out_ptr, perm, st);
}

}  // extern "C"

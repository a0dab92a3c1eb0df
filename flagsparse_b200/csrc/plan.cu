// Plan building for the CSR hot path: inspection, the SpMV unit plan,
// stable row-length bucketing, the stable CSR transpose and value gathers.
//
// Everything here runs once per prepared matrix (the reference's prepare_*
// step); the per-call kernels live in spmv_csr.cu / spmm_csr.cu / sddmm_csr.cu.
#include <climits>

#include <cub/device/device_radix_sort.cuh>

#include "fsb_common.cuh"
#include "scan.cuh"

namespace fsb {

// ---------------------------------------------------------------------------
// fsb_csr_inspect
// ---------------------------------------------------------------------------
__global__ void k_inspect_init(int64_t* out) {
  out[0] = 0; out[1] = 0; out[2] = 0; out[3] = LLONG_MAX; out[4] = -1; out[5] = 0;
}

template <typename IT, typename PT>
__global__ void __launch_bounds__(256) k_inspect(const IT* idx, const PT* ptr, int64_t n_rows, int64_t nnz,
                                                 int64_t* out) {
  int64_t bad = 0, mn = LLONG_MAX, mx = -1, mlen = 0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int64_t r = t0; r < n_rows; r += stride) {
    int64_t a = ld_ptr(ptr, r), b = ld_ptr(ptr, r + 1);
    if (b < a) ++bad;
    mlen = max(mlen, b - a);
  }
  for (int64_t i = t0; i < nnz; i += stride) {
    int64_t c = static_cast<int64_t>(__ldg(idx + i));
    mn = min(mn, c);
    mx = max(mx, c);
  }
  // warp reduce then one atomic per warp
  for (int m = 16; m > 0; m >>= 1) {
    bad += __shfl_xor_sync(0xffffffffu, bad, m);
    mn = min(mn, (int64_t)__shfl_xor_sync(0xffffffffu, mn, m));
    mx = max(mx, (int64_t)__shfl_xor_sync(0xffffffffu, mx, m));
    mlen = max(mlen, (int64_t)__shfl_xor_sync(0xffffffffu, mlen, m));
  }
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicAdd(reinterpret_cast<unsigned long long*>(out + 2), (unsigned long long)bad);
    if (mn != LLONG_MAX) atomicMin(reinterpret_cast<long long*>(out + 3), (long long)mn);
    if (mx >= 0) atomicMax(reinterpret_cast<long long*>(out + 4), (long long)mx);
    if (mlen > 0) atomicMax(reinterpret_cast<long long*>(out + 5), (long long)mlen);
  }
  if (t0 == 0) {
    out[0] = ld_ptr(ptr, 0);
    out[1] = ld_ptr(ptr, n_rows);
  }
}

template <typename IT, typename PT>
static int inspect_impl(const void* idx, const void* ptr, int64_t n_rows, int64_t nnz, int64_t* out,
                        cudaStream_t st) {
  k_inspect_init<<<1, 1, 0, st>>>(out);
  FSB_LAUNCH_CHECK();
  int64_t work = n_rows > nnz ? n_rows : nnz;
  int64_t blocks = ceil_div(work, 256 * 8);
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_inspect<IT, PT><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const IT*>(idx), static_cast<const PT*>(ptr),
                                                      n_rows, nnz, out);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

// ---------------------------------------------------------------------------
// SpMV unit plan.  Row r starts a segment when it is long (len > cap), follows
// a long row, is row 0, or when its window key (ptr[r] + r) / cap differs from
// the previous row's.  A long segment is one row and owns ceil(len/chunk)
// units; every other segment owns one row-block unit.  Row-block units come
// first in the unit list (in row order), long-row chunks after them (in row
// order), so the two kinds run as separate launches.  Channel 0 counts
// segments, channel 1 row-block units, channel 2 scratch slots (one per chunk
// of a row of two or more chunks: only those chunks publish a partial sum),
// channel 3 long-row chunks.
// ---------------------------------------------------------------------------
template <typename PT>
struct SpmvSegFlags {
  const PT* ptr;
  int64_t cap, chunk;
  __device__ __forceinline__ Vec<4> operator()(int64_t r) const {
    int64_t a = ld_ptr(ptr, r), b = ld_ptr(ptr, r + 1);
    int64_t len = b - a;
    bool is_long = len > cap;
    bool start;
    if (r == 0 || is_long) {
      start = true;
    } else {
      int64_t pa = ld_ptr(ptr, r - 1);
      bool prev_long = (a - pa) > cap;
      start = prev_long || ((pa + r - 1) / cap != (a + r) / cap);
    }
    const int64_t nch = is_long ? ceil_div(len, chunk) : 0;
    Vec<4> v;
    v.v[0] = start ? 1 : 0;
    v.v[1] = (start && !is_long) ? 1 : 0;
    v.v[2] = nch > 1 ? nch : 0;
    v.v[3] = nch;
    return v;
  }
};

// Records every segment start and writes the chunk descriptors of long rows
// (k_spmv_units writes the row-block descriptors).
template <typename PT>
struct SpmvSegWriter {
  const PT* ptr;
  int64_t cap, chunk;
  int32_t* seg_row0;
  int32_t* seg_unit0;
  fsb_spmv_unit* units;
  const int64_t* totals;  // scan totals: [1] = row-block units, which precede the long-row chunks
  __device__ __forceinline__ void operator()(int64_t r, const Vec<4>& pre, const Vec<4>& val) const {
    if (val.v[0] == 0) return;
    const int64_t a = ld_ptr(ptr, r), len = ld_ptr(ptr, r + 1) - a;
    const int64_t first_unit = len <= cap ? pre.v[1] : totals[1] + pre.v[3];
    seg_row0[pre.v[0]] = static_cast<int32_t>(r);
    seg_unit0[pre.v[0]] = static_cast<int32_t>(first_unit);
    if (len <= cap) return;
    const int32_t nch = static_cast<int32_t>(val.v[3]);
    for (int32_t k = 0; k < nch; ++k) {
      fsb_spmv_unit d;
      d.nnz_begin = a + int64_t(k) * chunk;
      d.nnz_end = min(a + int64_t(k + 1) * chunk, a + len);
      d.row = static_cast<int32_t>(r);
      d.tag = -(k + 1);
      d.n_chunks = nch;
      d.slot = nch > 1 ? static_cast<int32_t>(pre.v[2] + k) : -1;
      units[first_unit + k] = d;
    }
  }
};

__global__ void k_spmv_plan_sentinel(const int64_t* totals, int64_t n_rows, int32_t* seg_row0, int32_t* seg_unit0) {
  seg_row0[totals[0]] = static_cast<int32_t>(n_rows);
  seg_unit0[totals[0]] = static_cast<int32_t>(totals[1] + totals[3]);
}

// One thread per row-block segment writes that segment's descriptor.
template <typename PT>
__global__ void k_spmv_units(const PT* ptr, const int64_t* totals, const int32_t* seg_row0, const int32_t* seg_unit0,
                             int64_t cap, fsb_spmv_unit* units) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= totals[0]) return;
  const int32_t r0 = seg_row0[s], r1 = seg_row0[s + 1];
  const int64_t a = ld_ptr(ptr, r0);
  if (r1 - r0 == 1 && ld_ptr(ptr, r0 + 1) - a > cap) return;  // long row: written by the scan
  fsb_spmv_unit d;
  d.nnz_begin = a;
  d.nnz_end = ld_ptr(ptr, r1);
  d.row = r0;
  d.tag = r1;
  d.n_chunks = 1;
  d.slot = -1;
  units[seg_unit0[s]] = d;
}

template <typename PT>
static int spmv_plan_build_impl(const PT* ptr, int64_t n_rows, int64_t cap, int64_t chunk, const int64_t* ws,
                                int32_t* seg_row0, int32_t* seg_unit0, fsb_spmv_unit* units, cudaStream_t st) {
  const int64_t* totals = scan_totals<4>(ws, n_rows);
  int rc = scan_apply<4>(SpmvSegFlags<PT>{ptr, cap, chunk},
                         SpmvSegWriter<PT>{ptr, cap, chunk, seg_row0, seg_unit0, units, totals}, n_rows, ws, st);
  if (rc != FSB_OK) return rc;
  k_spmv_plan_sentinel<<<1, 1, 0, st>>>(totals, n_rows, seg_row0, seg_unit0);
  FSB_LAUNCH_CHECK();
  // at most one segment per row
  const unsigned blocks = (unsigned)ceil_div(n_rows > 0 ? n_rows : 1, 256);
  k_spmv_units<PT><<<blocks, 256, 0, st>>>(ptr, totals, seg_row0, seg_unit0, cap, units);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

__global__ void k_copy_totals(const int64_t* src, int64_t* dst, int n) {
  if (threadIdx.x < n) dst[threadIdx.x] = src[threadIdx.x];
}

// public totals of the SpMV plan: n_segs, n_units, n_slots, n_block_units
__global__ void k_spmv_totals(const int64_t* t, int64_t* out) {
  if (threadIdx.x == 0) {
    out[0] = t[0];
    out[1] = t[1] + t[3];
    out[2] = t[2];
    out[3] = t[1];
  }
}

// ---------------------------------------------------------------------------
// Stable bucketing (NV = 8 channels, one per bucket).
// ---------------------------------------------------------------------------
constexpr int kMaxBuckets = 8;
struct BucketBounds { int64_t ub[kMaxBuckets]; int n; };

template <typename PT>
struct BucketFlags {
  const PT* ptr;
  BucketBounds bb;
  __device__ __forceinline__ int bucket_of(int64_t r) const {
    int64_t len = ld_ptr(ptr, r + 1) - ld_ptr(ptr, r);
    for (int b = 0; b < bb.n; ++b) {
      if (bb.ub[b] < 0 || len <= bb.ub[b]) return b;
    }
    return -1;  // longer than every bound: in no bucket
  }
  __device__ __forceinline__ Vec<kMaxBuckets> operator()(int64_t r) const {
    Vec<kMaxBuckets> v; v.zero();
    int b = bucket_of(r);
    if (b >= 0) v.v[b] = 1;
    return v;
  }
};

struct BucketWriter {
  int32_t* rows_out;
  const int64_t* totals;
  int nb;
  __device__ __forceinline__ void operator()(int64_t r, const Vec<kMaxBuckets>& pre,
                                             const Vec<kMaxBuckets>& val) const {
    int64_t base = 0;
    for (int b = 0; b < nb; ++b) {
      if (val.v[b]) { rows_out[base + pre.v[b]] = static_cast<int32_t>(r); return; }
      base += totals[b];
    }
  }
};

// ---------------------------------------------------------------------------
// Transpose helpers.
// ---------------------------------------------------------------------------
template <typename IT>
__global__ void k_keys_from_cols(const IT* idx, int64_t nnz, uint32_t* keys, int32_t* pos) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nnz) {
    keys[i] = static_cast<uint32_t>(__ldg(idx + i));
    pos[i] = static_cast<int32_t>(i);
  }
}

// one warp per row writes the row id over the row's nonzeros
template <typename PT>
__global__ void k_row_ids(const PT* ptr, int64_t n_rows, int32_t* row_ids) {
  int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= n_rows) return;
  int64_t a = ld_ptr(ptr, w), b = ld_ptr(ptr, w + 1);
  for (int64_t i = a + lane; i < b; i += 32) row_ids[i] = static_cast<int32_t>(w);
}

template <typename OIT>
__global__ void k_transpose_fill(const int32_t* sorted_pos, const int32_t* row_ids, int64_t nnz, OIT* t_idx,
                                 int64_t* perm) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nnz) {
    int32_t p = sorted_pos[i];
    perm[i] = p;
    t_idx[i] = static_cast<OIT>(row_ids[p]);
  }
}

// t_ptr[c] = first position whose key >= c, for c in [0, n_cols]
template <typename OPT>
__global__ void k_transpose_ptr(const uint32_t* sorted_keys, int64_t nnz, int64_t n_cols, OPT* t_ptr) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i > nnz) return;
  int64_t lo = (i == 0) ? 0 : int64_t(sorted_keys[i - 1]) + 1;   // first column owned by boundary i
  int64_t hi = (i == nnz) ? n_cols : int64_t(sorted_keys[i]);    // last column owned by boundary i
  for (int64_t c = lo; c <= hi; ++c) t_ptr[c] = static_cast<OPT>(i);
}

template <typename S>
__global__ void k_gather(const S* src, const int64_t* perm, int64_t n, S* dst) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[perm[i]];
}
template <typename S>
__global__ void k_gather_conj(const S* src, const int64_t* perm, int64_t n, S* dst) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) { S v = src[perm[i]]; v.y = -v.y; dst[i] = v; }
}

static int bits_for(int64_t n_cols) {
  int b = 1;
  while (b < 32 && (int64_t(1) << b) < n_cols) ++b;
  return b;
}

struct TransposeWs {
  uint32_t* keys_in; uint32_t* keys_out; int32_t* pos_in; int32_t* pos_out; int32_t* row_ids;
  void* cub_tmp; size_t cub_bytes; int64_t total;
};

static inline int64_t align256(int64_t b) { return (b + 255) & ~int64_t(255); }

static int transpose_layout(int64_t nnz, int64_t n_cols, void* base, TransposeWs& ws) {
  size_t cub_bytes = 0;
  int bits = bits_for(n_cols);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                                  (const int32_t*)nullptr, (int32_t*)nullptr, (int)nnz, 0, bits);
  if (e != cudaSuccess) return FSB_ERR_CUDA;
  char* p = static_cast<char*>(base);
  int64_t off = 0;
  auto take = [&](int64_t bytes) { char* q = p ? p + off : nullptr; off += align256(bytes); return q; };
  ws.keys_in = reinterpret_cast<uint32_t*>(take(4 * nnz));
  ws.keys_out = reinterpret_cast<uint32_t*>(take(4 * nnz));
  ws.pos_in = reinterpret_cast<int32_t*>(take(4 * nnz));
  ws.pos_out = reinterpret_cast<int32_t*>(take(4 * nnz));
  ws.row_ids = reinterpret_cast<int32_t*>(take(4 * nnz));
  ws.cub_tmp = take(int64_t(cub_bytes));
  ws.cub_bytes = cub_bytes;
  ws.total = off;
  return FSB_OK;
}

template <typename IT, typename PT, typename OIT, typename OPT>
static int transpose_impl(const void* idx, const void* ptr, int64_t n_rows, int64_t n_cols, int64_t nnz,
                          TransposeWs& ws, void* t_idx, void* t_ptr, int64_t* perm, cudaStream_t st) {
  const unsigned B = 256;
  if (nnz > 0) {
    k_keys_from_cols<IT><<<(unsigned)ceil_div(nnz, B), B, 0, st>>>(static_cast<const IT*>(idx), nnz, ws.keys_in,
                                                                     ws.pos_in);
    FSB_LAUNCH_CHECK();
    if (n_rows > 0) {
      k_row_ids<PT><<<(unsigned)ceil_div(n_rows * 32, B), B, 0, st>>>(static_cast<const PT*>(ptr), n_rows,
                                                                        ws.row_ids);
      FSB_LAUNCH_CHECK();
    }
    size_t tmp = ws.cub_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.keys_in, ws.keys_out, ws.pos_in, ws.pos_out,
                                                    (int)nnz, 0, bits_for(n_cols), st);
    if (e != cudaSuccess) return FSB_ERR_CUDA;
    k_transpose_fill<OIT><<<(unsigned)ceil_div(nnz, B), B, 0, st>>>(ws.pos_out, ws.row_ids, nnz,
                                                                      static_cast<OIT*>(t_idx), perm);
    FSB_LAUNCH_CHECK();
  }
  k_transpose_ptr<OPT><<<(unsigned)ceil_div(nnz + 1, B), B, 0, st>>>(ws.keys_out, nnz, n_cols,
                                                                       static_cast<OPT*>(t_ptr));
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

}  // namespace fsb

using namespace fsb;

extern "C" {

int fsb_version(void) { return 100; }

const char* fsb_status_string(int status) {
  switch (status) {
    case FSB_OK: return "ok";
    case FSB_ERR_INVALID_ARG: return "invalid argument";
    case FSB_ERR_UNSUPPORTED: return "unsupported dtype or index combination";
    case FSB_ERR_LAUNCH: return "kernel launch failed";
    case FSB_ERR_TIMEOUT: return "bounded device wait expired";
    case FSB_ERR_CUDA: return "CUDA runtime error";
    case FSB_ERR_WORKSPACE: return "workspace too small";
    case FSB_ERR_TOO_LARGE: return "plan needs more scratch slots than the built-in scratch holds";
    default: return "unknown status";
  }
}

int fsb_csr_inspect(const void* indices, int idx_is_64, const void* indptr, int ptr_is_64, int64_t n_rows,
                    int64_t nnz, int64_t* d_out, void* stream) {
  if (!indptr || !d_out || n_rows < 0 || nnz < 0 || (nnz > 0 && !indices)) return FSB_ERR_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (idx_is_64) {
    return ptr_is_64 ? inspect_impl<int64_t, int64_t>(indices, indptr, n_rows, nnz, d_out, st)
                     : inspect_impl<int64_t, int32_t>(indices, indptr, n_rows, nnz, d_out, st);
  }
  return ptr_is_64 ? inspect_impl<int32_t, int64_t>(indices, indptr, n_rows, nnz, d_out, st)
                   : inspect_impl<int32_t, int32_t>(indices, indptr, n_rows, nnz, d_out, st);
}

// A row-block unit of a warp holds < 2*cap nonzeros: 14 per lane for the 2- and
// 4-byte real types (cap 224), 8 per lane for the wider types (cap 128).
int32_t fsb_spmv_default_cap(int dtype) { return (dtype == FSB_F16 || dtype == FSB_BF16 || dtype == FSB_F32) ? 224 : 128; }

// Long rows are cut into chunks of 256-nonzero batches per warp: four for the
// 2- and 4-byte real types (fewer tickets on the gather-bound long rows), two
// for the wider types.
int32_t fsb_spmv_default_chunk(int dtype) { return (dtype == FSB_F16 || dtype == FSB_BF16 || dtype == FSB_F32) ? 1024 : 512; }

int64_t fsb_spmv_plan_workspace_bytes(int64_t n_rows) { return scan_workspace_bytes<4>(n_rows); }

int fsb_spmv_plan_analyze(const void* indptr, int ptr_is_64, int64_t n_rows, int32_t cap, int32_t chunk_nnz,
                          void* workspace, int64_t workspace_bytes, int64_t* d_totals, void* stream) {
  if (!indptr || !workspace || !d_totals || n_rows < 0 || cap < 1 || chunk_nnz < 1) return FSB_ERR_INVALID_ARG;
  if (n_rows >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  if (workspace_bytes < fsb_spmv_plan_workspace_bytes(n_rows)) return FSB_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int64_t* ws = static_cast<int64_t*>(workspace);
  int rc;
  if (ptr_is_64) {
    rc = scan_analyze<4>(SpmvSegFlags<int64_t>{static_cast<const int64_t*>(indptr), cap, chunk_nnz}, n_rows, ws, st);
  } else {
    rc = scan_analyze<4>(SpmvSegFlags<int32_t>{static_cast<const int32_t*>(indptr), cap, chunk_nnz}, n_rows, ws, st);
  }
  if (rc != FSB_OK) return rc;
  k_spmv_totals<<<1, 32, 0, st>>>(scan_totals<4>(ws, n_rows), d_totals);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

int fsb_spmv_plan_build(const void* indptr, int ptr_is_64, int64_t n_rows, int32_t cap, int32_t chunk_nnz,
                        const void* workspace, int64_t workspace_bytes, int32_t* seg_row0, int32_t* seg_unit0,
                        fsb_spmv_unit* units, void* stream) {
  if (!indptr || !workspace || !seg_row0 || !seg_unit0 || !units || n_rows < 0 || cap < 1 || chunk_nnz < 1)
    return FSB_ERR_INVALID_ARG;
  if (workspace_bytes < fsb_spmv_plan_workspace_bytes(n_rows)) return FSB_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t* ws = static_cast<const int64_t*>(workspace);
  if (ptr_is_64)
    return spmv_plan_build_impl(static_cast<const int64_t*>(indptr), n_rows, cap, chunk_nnz, ws, seg_row0, seg_unit0,
                                units, st);
  return spmv_plan_build_impl(static_cast<const int32_t*>(indptr), n_rows, cap, chunk_nnz, ws, seg_row0, seg_unit0,
                              units, st);
}

int64_t fsb_csr_bucketize_workspace_bytes(int64_t n_rows, int n_buckets) {
  (void)n_buckets;
  return scan_workspace_bytes<kMaxBuckets>(n_rows);
}

int fsb_csr_bucketize(const void* indptr, int ptr_is_64, int64_t n_rows, const int64_t* upper_bounds, int n_buckets,
                      void* workspace, int64_t workspace_bytes, int32_t* rows_out, int64_t* d_counts, void* stream) {
  if (!indptr || !upper_bounds || !workspace || !d_counts || n_rows < 0 || n_buckets < 1 ||
      n_buckets > kMaxBuckets || (n_rows > 0 && !rows_out))
    return FSB_ERR_INVALID_ARG;
  if (n_rows >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  if (workspace_bytes < fsb_csr_bucketize_workspace_bytes(n_rows, n_buckets)) return FSB_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  BucketBounds bb;
  bb.n = n_buckets;
  for (int b = 0; b < kMaxBuckets; ++b) bb.ub[b] = b < n_buckets ? upper_bounds[b] : -1;
  int64_t* ws = static_cast<int64_t*>(workspace);
  const int64_t* totals = scan_totals<kMaxBuckets>(ws, n_rows);
  BucketWriter w{rows_out, totals, n_buckets};
  int rc;
  if (ptr_is_64) {
    BucketFlags<int64_t> f{static_cast<const int64_t*>(indptr), bb};
    rc = scan_analyze<kMaxBuckets>(f, n_rows, ws, st);
    if (rc == FSB_OK) rc = scan_apply<kMaxBuckets>(f, w, n_rows, ws, st);
  } else {
    BucketFlags<int32_t> f{static_cast<const int32_t*>(indptr), bb};
    rc = scan_analyze<kMaxBuckets>(f, n_rows, ws, st);
    if (rc == FSB_OK) rc = scan_apply<kMaxBuckets>(f, w, n_rows, ws, st);
  }
  if (rc != FSB_OK) return rc;
  k_copy_totals<<<1, 32, 0, st>>>(totals, d_counts, n_buckets);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

int64_t fsb_csr_transpose_workspace_bytes(int64_t nnz, int64_t n_rows, int64_t n_cols) {
  (void)n_rows;
  if (nnz < 0 || nnz >= INT32_MAX) return -1;
  TransposeWs ws;
  if (transpose_layout(nnz, n_cols, nullptr, ws) != FSB_OK) return -1;
  return ws.total;
}

int fsb_csr_transpose(const void* indices, int idx_is_64, const void* indptr, int ptr_is_64, int64_t n_rows,
                      int64_t n_cols, int64_t nnz, void* workspace, int64_t workspace_bytes, void* t_indices,
                      int t_idx_is_64, void* t_indptr, int t_ptr_is_64, int64_t* perm, void* stream) {
  if (!indptr || !t_indptr || n_rows < 0 || n_cols < 0 || nnz < 0) return FSB_ERR_INVALID_ARG;
  if (nnz > 0 && (!indices || !t_indices || !perm || !workspace)) return FSB_ERR_INVALID_ARG;
  if (nnz >= INT32_MAX || n_cols > (int64_t(1) << 32) || n_rows >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  TransposeWs ws;
  if (nnz == 0) {
    // every transposed row is empty
    ws.keys_out = nullptr;
  } else {
    int rc = transpose_layout(nnz, n_cols, workspace, ws);
    if (rc != FSB_OK) return rc;
    if (workspace_bytes < ws.total) return FSB_ERR_WORKSPACE;
  }
#define FSB_T(IT, PT, OIT, OPT) \
  return transpose_impl<IT, PT, OIT, OPT>(indices, indptr, n_rows, n_cols, nnz, ws, t_indices, t_indptr, perm, st)
  if (idx_is_64) {
    if (ptr_is_64) {
      if (t_idx_is_64) { if (t_ptr_is_64) FSB_T(int64_t, int64_t, int64_t, int64_t); else FSB_T(int64_t, int64_t, int64_t, int32_t); }
      else { if (t_ptr_is_64) FSB_T(int64_t, int64_t, int32_t, int64_t); else FSB_T(int64_t, int64_t, int32_t, int32_t); }
    } else {
      if (t_idx_is_64) { if (t_ptr_is_64) FSB_T(int64_t, int32_t, int64_t, int64_t); else FSB_T(int64_t, int32_t, int64_t, int32_t); }
      else { if (t_ptr_is_64) FSB_T(int64_t, int32_t, int32_t, int64_t); else FSB_T(int64_t, int32_t, int32_t, int32_t); }
    }
  } else {
    if (ptr_is_64) {
      if (t_idx_is_64) { if (t_ptr_is_64) FSB_T(int32_t, int64_t, int64_t, int64_t); else FSB_T(int32_t, int64_t, int64_t, int32_t); }
      else { if (t_ptr_is_64) FSB_T(int32_t, int64_t, int32_t, int64_t); else FSB_T(int32_t, int64_t, int32_t, int32_t); }
    } else {
      if (t_idx_is_64) { if (t_ptr_is_64) FSB_T(int32_t, int32_t, int64_t, int64_t); else FSB_T(int32_t, int32_t, int64_t, int32_t); }
      else { if (t_ptr_is_64) FSB_T(int32_t, int32_t, int32_t, int64_t); else FSB_T(int32_t, int32_t, int32_t, int32_t); }
    }
  }
#undef FSB_T
}

int fsb_gather_values(int dtype, const void* src, const int64_t* perm, int64_t n, int conj, void* dst, void* stream) {
  if (n < 0 || (n > 0 && (!src || !perm || !dst))) return FSB_ERR_INVALID_ARG;
  if (n == 0) return FSB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned B = 256;
  const unsigned G = (unsigned)ceil_div(n, B);
  switch (dtype) {
    case FSB_F16: case FSB_BF16:
      k_gather<uint16_t><<<G, B, 0, st>>>(static_cast<const uint16_t*>(src), perm, n, static_cast<uint16_t*>(dst));
      break;
    case FSB_F32:
      k_gather<float><<<G, B, 0, st>>>(static_cast<const float*>(src), perm, n, static_cast<float*>(dst));
      break;
    case FSB_F64:
      k_gather<double><<<G, B, 0, st>>>(static_cast<const double*>(src), perm, n, static_cast<double*>(dst));
      break;
    case FSB_C64:
      if (conj) k_gather_conj<float2><<<G, B, 0, st>>>(static_cast<const float2*>(src), perm, n, static_cast<float2*>(dst));
      else k_gather<float2><<<G, B, 0, st>>>(static_cast<const float2*>(src), perm, n, static_cast<float2*>(dst));
      break;
    case FSB_C128:
      if (conj) k_gather_conj<double2><<<G, B, 0, st>>>(static_cast<const double2*>(src), perm, n, static_cast<double2*>(dst));
      else k_gather<double2><<<G, B, 0, st>>>(static_cast<const double2*>(src), perm, n, static_cast<double2*>(dst));
      break;
    default:
      return FSB_ERR_UNSUPPORTED;
  }
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

}  // extern "C"

// BSR SpMM with 16 x 16 blocks on the sm_100a tensor cores (tcgen05).
//
// C (M x N) = A (M x K in 16 x 16 blocks, bf16 or f16) * B (K x N, row-major),
// fp32 accumulation in tensor memory, C written in the value type.
//
// Each block contributes C[16 rows][N] += A_blk (16 x 16) * B[16 rows of the
// block column][N].  The MMA computes the transpose, so the dense columns fill
// the 128-row M dimension of one tcgen05.mma:
//
//     D (128 x 16, TMEM) += B_slab^T (128 x 16, MN-major smem) * A_blk^T (16 x 16, K-major smem)
//
// with M = 128 dense columns of one column tile, N = the block row's 16 rows
// and K = the block's 16 columns: one instruction per block.  A CTA owns a
// contiguous range of block rows and one column tile; its warps specialise:
//  * warp 4 (one thread) streams blocks through a 4-deep shared-memory ring:
//    two TMA tile loads per B slab (64 columns x 16 rows each, 128-byte
//    swizzle = the MMA's SWIZZLE_128B MN-major layout) and one bulk copy of the
//    block, pre-packed into the MMA's K-major core-matrix layout
//    (fsb_bsr16_pack), all completing on the slot's "full" mbarrier;
//  * warp 5 allocates 32 TMEM columns (two 16-column fp32 accumulators) and
//    one thread issues one tcgen05.mma per block, tcgen05.commit-ing the
//    slot's "empty" mbarrier and, after a block row's last block, the
//    accumulator's "full" mbarrier;
//  * warps 0-3 read their 32 TMEM lanes (= 32 dense columns) with tcgen05.ld,
//    release the accumulator and store 16 output rows.
// N may be any multiple of 64: in a last tile with only 64 columns left, the
// upper half of each B slab is not loaded (its MMA rows compute unused values
// from whatever that half of the slot holds, and are never stored).
// Every mbarrier wait is bounded.  On expiry a role records the error (in the
// caller's error word and in a shared abort flag that every other wait polls)
// and stops; before TMEM is freed the producer waits (bounded) for the copies
// it issued to land and the MMA thread commits a drain barrier and waits
// (bounded) for its issued MMAs, so no copy or MMA is left in flight.
#include <cstdint>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "fsb_common.cuh"
#include "fsb_tma.cuh"

namespace fsb {
namespace {

constexpr int kBsrThreads = 192;                      // warps 0-3 epilogue, 4 producer, 5 MMA
// 7 CTAs per SM with a 4-deep ring each: more independent block pipelines per
// SM measured faster than fewer, deeper ones (N = 64: 0.23 ms against 0.32 ms
// with 4 CTAs x 8 stages; N = 128: 0.362 against 0.366 ms).  Products of at
// most 64 columns (one half-filled tile, half-size slab copies) run 8 per SM:
// 0.222 against 0.242 ms on 65,536^2 blocks, where N = 128 measured 0.369
// against 0.366 ms (6 stages at 7 per SM: 0.248 / 0.384 ms).
constexpr int kBsrCtasPerSm = 7;
constexpr int kBsrCtasPerSmNarrow = 8;
constexpr int kBsrStages = 4;
constexpr int kBsrTileM = 128;                        // dense columns per MMA
constexpr int kSlabBytes = 16 * kBsrTileM * 2;        // B slab: 16 rows x 128 columns, 2-byte values
constexpr int kBlkBytes = 16 * 16 * 2;                // one 16 x 16 block
constexpr int kTmemCols = 32;                         // two 16-column fp32 accumulators

// Shared-memory operand layouts:
//   slab (MMA A, MN-major, SWIZZLE_128B): two 64-column halves 2048 bytes apart
//     (LBO = 2048, the MN-atom stride); each half is 16 rows of 128 bytes as
//     written by TMA, i.e. two 8-row swizzle atoms 1024 bytes apart (SBO = 1024)
//   block (MMA B, K-major, no swizzle): element (n, k) at
//     (n/8)*256 + (k/8)*128 + (n%8)*16 + (k%8)*2 -> SBO 256, LBO 128
constexpr uint32_t kSlabLBO = 2048, kSlabSBO = 1024, kBlkSBO = 256, kBlkLBO = 128;
constexpr uint32_t kLayoutNone = 0, kLayoutSw128 = 2;

// UMMA shared-memory descriptor: start address, leading / stride byte offsets
// (all >> 4), version 1, base offset 0 (swizzle atoms are 1024-byte aligned),
// layout type (0 = no swizzle, 2 = 128-byte swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  d |= uint64_t(layout & 7u) << 61;
  return d;
}

// Instruction descriptor, kind::f16: fp32 accumulator, A and B of the same
// 16-bit type (bf16 = 1, f16 = 0), A MN-major, B K-major, N = 16, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t ab_format) {
  return (1u << 4) | (ab_format << 7) | (ab_format << 10) | (1u << 15) | (0u << 16) | ((16u >> 3) << 17) |
         ((uint32_t(kBsrTileM) >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on the mbarrier once every previously issued tcgen05 op of this thread completes
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}


__device__ __forceinline__ void store_out(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void store_out(__half* p, float v) { *p = __float2half_rn(v); }

// Shared-memory map (from a 1024-byte aligned base): slabs [S][4096] | blocks
// [S][512] | mbarriers full[S], empty[S], acc_full[2], acc_empty[2], drain |
// TMEM address | abort flag.
constexpr int kSmemSlabs = 0;
constexpr int kSmemBlocks = kBsrStages * kSlabBytes;
constexpr int kSmemBars = kSmemBlocks + kBsrStages * kBlkBytes;
constexpr int kNumBars = 2 * kBsrStages + 5;
constexpr int kSmemTmemSlot = kSmemBars + kNumBars * 8;
constexpr int kSmemAbort = kSmemTmemSlot + 4;
constexpr int kSmemBytes = 1024 + kSmemTmemSlot + 16;  // 1024: alignment slack for the base

// A bounded wait expired: record it for the host (err may be device memory or
// mapped pinned host memory, so a plain store) and tell the other roles.
__device__ __forceinline__ void bsr_fail(int* err, volatile int* abort) {
  *reinterpret_cast<volatile int*>(err) = 1;
  *abort = 1;
}

// grid: x = CTAs over contiguous block-row ranges, y = 128-column tiles of C.
template <typename S>
__global__ void __launch_bounds__(kBsrThreads, kBsrCtasPerSmNarrow)
k_bsr16_spmm(const __grid_constant__ CUtensorMap tmap_b, const S* __restrict__ packed, const int32_t* __restrict__ bcol,
             const int64_t* __restrict__ bptr, int64_t n_brows, int64_t rows_per_cta, S* __restrict__ C, int64_t ldc,
             int64_t n, uint32_t idesc, int tile_cols, int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_addr(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* smem = smem_raw + (base - raw);
  const uint32_t full0 = base + kSmemBars, empty0 = full0 + 8 * kBsrStages;
  const uint32_t accf0 = empty0 + 8 * kBsrStages, acce0 = accf0 + 16, drain = acce0 + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kSmemTmemSlot);
  volatile int* abort = reinterpret_cast<volatile int*>(smem + kSmemAbort);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_cta;
  const int64_t r1 = r0 + rows_per_cta < n_brows ? r0 + rows_per_cta : n_brows;
  if (r0 >= r1) return;  // the whole CTA, before any allocation
  const int64_t col0 = int64_t(blockIdx.y) * tile_cols;
  const int64_t b0 = bptr[r0], total = bptr[r1] - b0;

  // a tile's upper 64 columns may lie past N (N a multiple of 64), or the tile
  // is 64 columns wide: that half of the B slab is neither loaded nor stored
  const bool upper = tile_cols == kBsrTileM && col0 + 64 < n;
  if (warp < 4 && tid < tile_cols && col0 + tid < n) {  // block rows without blocks get zero rows
    for (int64_t r = r0; r < r1; ++r) {
      if (bptr[r] == bptr[r + 1]) {
        S* c = C + r * 16 * ldc + col0 + tid;
        for (int n = 0; n < 16; ++n) store_out(c + n * ldc, 0.0f);
      }
    }
  }
  if (total == 0) return;

  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 128) {
    for (int i = 0; i < kBsrStages; ++i) {
      mbar_init(full0 + 8 * i, 1);
      mbar_init(empty0 + 8 * i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(accf0 + 8 * i, 1);
      mbar_init(acce0 + 8 * i, 4);  // one arrival per epilogue warp
    }
    mbar_init(drain, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int64_t issued = 0;
      for (int64_t j = 0; j < total; ++j) {
        const int s = static_cast<int>(j % kBsrStages);
        const uint32_t use = static_cast<uint32_t>(j / kBsrStages);
        if (!mbar_wait(empty0 + 8 * s, (use & 1u) ^ 1u, abort)) {  // slot released by the MMA of block j-S
          bsr_fail(err, abort);
          break;
        }
        const int64_t blk = b0 + j;
        const int32_t krow = __ldg(bcol + blk) * 16;
        const uint32_t full = full0 + 8 * s;
        const uint32_t slab = base + kSmemSlabs + s * kSlabBytes;
        mbar_arrive_expect_tx(full, (upper ? kSlabBytes : kSlabBytes / 2) + kBlkBytes);
        tma_load_2d(slab, &tmap_b, static_cast<int32_t>(col0), krow, full);
        if (upper) tma_load_2d(slab + 2048, &tmap_b, static_cast<int32_t>(col0 + 64), krow, full);
        bulk_load(base + kSmemBlocks + s * kBlkBytes, packed + blk * 256, kBlkBytes, full);
        issued = j + 1;
      }
      // drain: the copies of the last (up to S) blocks issued have landed once
      // their slot's phase for that use completed (bounded, ignores abort)
      for (int64_t j = issued > kBsrStages ? issued - kBsrStages : 0; j < issued; ++j)
        if (!mbar_wait(full0 + 8 * static_cast<int>(j % kBsrStages), static_cast<uint32_t>(j / kBsrStages) & 1u))
          bsr_fail(err, abort);
    }
  } else if (warp == 5) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int64_t row = r0, row_begin = bptr[r0], row_end = bptr[r0 + 1];
      int64_t rr = 0;  // index of the current row among the CTA's non-empty rows
      for (int64_t j = 0; j < total; ++j) {
        const int s = static_cast<int>(j % kBsrStages);
        const uint32_t use = static_cast<uint32_t>(j / kBsrStages);
        const int64_t blk = b0 + j;
        while (blk >= row_end) {
          ++row;
          row_begin = row_end;
          row_end = bptr[row + 1];
        }
        const bool first = blk == row_begin, last = blk == row_end - 1;
        const int buf = static_cast<int>(rr & 1);
        if (first && !mbar_wait(acce0 + 8 * buf, static_cast<uint32_t>(((rr >> 1) & 1) ^ 1), abort)) {
          bsr_fail(err, abort);  // accumulator not released
          break;
        }
        if (!mbar_wait(full0 + 8 * s, use & 1u, abort)) {  // block j landed
          bsr_fail(err, abort);
          break;
        }
        tc_fence_after();
        const uint32_t slab = base + kSmemSlabs + s * kSlabBytes;
        const uint32_t blkp = base + kSmemBlocks + s * kBlkBytes;
        tc_mma(tmem + uint32_t(buf * 16), umma_desc(slab, kSlabLBO, kSlabSBO, kLayoutSw128),
               umma_desc(blkp, kBlkLBO, kBlkSBO, kLayoutNone), idesc, first ? 0u : 1u);
        tc_commit(empty0 + 8 * s);
        if (last) {
          tc_commit(accf0 + 8 * buf);
          ++rr;
        }
      }
      // drain: every MMA this thread issued has completed once this commit arrives
      tc_commit(drain);
      if (!mbar_wait(drain, 0u)) bsr_fail(err, abort);
    }
  } else {
    // ------------------------------------------------------------ epilogue (warps 0-3)
    int64_t rr = 0;
    for (int64_t r = r0; r < r1; ++r) {
      if (bptr[r] == bptr[r + 1]) continue;
      const int buf = static_cast<int>(rr & 1);
      // warp-uniform outcome: tcgen05.ld below is .sync.aligned
      if (!__all_sync(0xffffffffu, mbar_wait(accf0 + 8 * buf, static_cast<uint32_t>((rr >> 1) & 1), abort))) {
        if (lane == 0) bsr_fail(err, abort);
        break;
      }
      tc_fence_after();
      uint32_t v[16];
      tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(buf * 16), v);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * buf);
      if (warp * 32 + lane < tile_cols && col0 + warp * 32 + lane < n) {
        S* c = C + r * 16 * ldc + col0 + warp * 32 + lane;
#pragma unroll
        for (int q = 0; q < 16; ++q) store_out(c + q * ldc, __uint_as_float(v[q]));
      }
      ++rr;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 5) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// packed[b] = block b rearranged into the K-major core-matrix layout: chunk
// (n, k8) of 16 bytes at (n/8)*256 + k8*128 + (n%8)*16.
__global__ void k_bsr16_pack(const uint4* __restrict__ src, uint4* __restrict__ dst, int64_t nnzb) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nnzb * 32; i += stride) {
    const int64_t b = i >> 5;
    const int a = static_cast<int>(i & 31), n = a >> 1, k8 = a & 1;
    dst[b * 32 + ((n >> 3) * 256 + k8 * 128 + (n & 7) * 16) / 16] = src[i];
  }
}

template <typename S>
int bsr_launch(CUtensorMapDataType tdt, uint32_t ab_format, const void* packed, const int32_t* bcol,
               const int64_t* bptr, int64_t n_brows, int64_t k_rows, const void* B, int64_t ldb, int64_t n, void* C,
               int64_t ldc, int* err, cudaStream_t st) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = encode_fn();
  if (!encode) return FSB_ERR_CUDA;
  alignas(64) CUtensorMap map;
  const cuuint64_t dims[2] = {cuuint64_t(n), cuuint64_t(k_rows)};
  const cuuint64_t strides[1] = {cuuint64_t(ldb) * 2};
  const cuuint32_t box[2] = {64, 16};
  const cuuint32_t estr[2] = {1, 1};
  if (encode(&map, tdt, 2, const_cast<void*>(B), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return FSB_ERR_UNSUPPORTED;
  // 128-column tiles.  (64-column tiles when B exceeds L2, so that only half of
  // B is gathered at a time, measured slower on 65,536^2 blocks with N = 128:
  // 0.53 against 0.36 ms, the blocks being read once per tile.)
  const int tile_cols = kBsrTileM;
  const int64_t tiles = ceil_div(n, tile_cols);
  if (tiles > 65535) return FSB_ERR_UNSUPPORTED;
  const int64_t target = 148 * (n <= 64 ? kBsrCtasPerSmNarrow : kBsrCtasPerSm);  // resident CTAs
  const int64_t rows_per_cta = ceil_div(n_brows, target);
  const int64_t grid_x = ceil_div(n_brows, rows_per_cta);
  dim3 grid((unsigned)grid_x, (unsigned)tiles);
  k_bsr16_spmm<S><<<grid, kBsrThreads, kSmemBytes, st>>>(map, static_cast<const S*>(packed), bcol, bptr, n_brows,
                                                         rows_per_cta, static_cast<S*>(C), ldc, n,
                                                         umma_idesc(ab_format), tile_cols, err);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

}  // namespace
}  // namespace fsb

using namespace fsb;

extern "C" {

int fsb_bsr16_pack(int dtype, const void* blocks, int64_t nnzb, void* packed, void* stream) {
  if (nnzb < 0 || (nnzb > 0 && (!blocks || !packed))) return FSB_ERR_INVALID_ARG;
  if (dtype != FSB_BF16 && dtype != FSB_F16) return FSB_ERR_UNSUPPORTED;
  if (reinterpret_cast<uintptr_t>(blocks) % 16 || reinterpret_cast<uintptr_t>(packed) % 16) return FSB_ERR_UNSUPPORTED;
  if (nnzb == 0) return FSB_OK;
  int64_t grid = ceil_div(nnzb * 32, 256);
  if (grid > 148 * 32) grid = 148 * 32;
  k_bsr16_pack<<<(unsigned)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const uint4*>(blocks),
                                                                              static_cast<uint4*>(packed), nnzb);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

int fsb_bsr16_spmm(int dtype, const void* packed, const int32_t* bcol, const int64_t* bptr, int64_t n_brows,
                   int64_t n_bcols, const void* B, int64_t ldb, int64_t n, void* C, int64_t ldc, int* d_error,
                   void* stream) {
  if (n_brows < 0 || n_bcols < 0 || n < 0 || ldb < n || ldc < n) return FSB_ERR_INVALID_ARG;
  if (n_brows == 0 || n == 0) return FSB_OK;
  if (!bptr || !C || !d_error || (n_bcols > 0 && (!B || !packed || !bcol))) return FSB_ERR_INVALID_ARG;
  // TMA and bulk copies: B and the packed blocks 16-byte aligned, row stride a
  // multiple of 16 bytes, whole 64-column TMA boxes
  if (n % 64 != 0 || ldb % 8 != 0 || reinterpret_cast<uintptr_t>(B) % 16 != 0 ||
      reinterpret_cast<uintptr_t>(packed) % 16 != 0 || n_bcols * 16 > INT32_MAX || n > INT32_MAX)
    return FSB_ERR_UNSUPPORTED;
  if (ceil_div(n, 64) > 65535) return FSB_ERR_UNSUPPORTED;
  if (n_bcols == 0) {  // every block row is empty: C = 0 (no tensor map over an empty B)
    return cudaMemset2DAsync(C, size_t(ldc) * 2, 0, size_t(n) * 2, size_t(n_brows) * 16,
                             static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? FSB_OK
               : FSB_ERR_CUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t k_rows = n_bcols * 16;
  switch (dtype) {
    case FSB_BF16:
      return bsr_launch<__nv_bfloat16>(CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 1u, packed, bcol, bptr, n_brows, k_rows, B,
                                       ldb, n, C, ldc, d_error, st);
    case FSB_F16:
      return bsr_launch<__half>(CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 0u, packed, bcol, bptr, n_brows, k_rows, B, ldb, n, C,
                                ldc, d_error, st);
    default:
      return FSB_ERR_UNSUPPORTED;
  }
}

}  // extern "C"

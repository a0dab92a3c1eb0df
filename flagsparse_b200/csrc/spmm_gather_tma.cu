// The B-row gather floor of the CSR SpMM through the tensor memory
// accelerator: a measurement kernel, not a product path.
//
// B (k_rows x n, row-major, ldb) is a 2-D tensor map whose box is one row of
// RB = n * sizeof(value) bytes (256 or 512).  One
// cp.async.bulk.tensor.2d ... tile::gather4 copies four B rows, named by four
// column indices of A, into shared memory.  Each warp keeps its own ring of
// 16 KB: stages of 8 rows (two gather4 copies completing on one mbarrier),
// 4 stages of 512-byte rows or 8 of 256-byte rows in flight.  Lane 0 issues;
// after a stage has landed every lane reads its RB / 32 bytes of each row from
// shared memory and adds value * row to fp32 sums.  Warp w covers nonzeros
// [w * per, (w + 1) * per) and writes its n sums to out[w]; there are no rows
// of A, so the time is what the B-row gathers alone take when TMA moves them.
//
// On the 1,000,000 x 1,000,000 power-law matrix (29.7 M nonzeros) the floor
// takes about as long for 256- as for 512-byte rows and scales inversely with
// the warps per SM, which is what ruled TMA gathers out for the SpMM kernels.
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "flagsparse_b200.h"
#include "fsb_common.cuh"
#include "fsb_tma.cuh"

namespace fsb {
namespace {

constexpr int kGtWarps = 4;              // warps per CTA
constexpr int kGtRingBytes = 16384;      // ring per warp
constexpr int kGtStageRows = 8;          // two gather4 copies per stage

template <typename S> __device__ __forceinline__ float gt_real(S v);
template <> __device__ __forceinline__ float gt_real<float>(float v) { return v; }
template <> __device__ __forceinline__ float gt_real<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float gt_real<__half>(__half v) { return __half2float(v); }

template <typename S, int RB>
__global__ void __launch_bounds__(kGtWarps * 32)
k_spmm_gather_tma(const __grid_constant__ CUtensorMap tmap, const S* __restrict__ vals,
                  const int32_t* __restrict__ cols, int64_t nnz, int64_t per_warp, float* __restrict__ out, int* err) {
  constexpr int kStageBytes = kGtStageRows * RB;
  constexpr int R = kGtRingBytes / kStageBytes;  // stages in flight
  constexpr int E = RB / 32 / int(sizeof(S));    // elements per lane
  static_assert(E >= 1 && R >= 2, "rows of 256 or 512 bytes");
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t gw = int64_t(blockIdx.x) * kGtWarps + warp;
  unsigned char* ring = smem + warp * kGtRingBytes;
  const uint32_t ring_a = smem_addr(ring);
  const uint32_t bar_a = smem_addr(smem + kGtWarps * kGtRingBytes) + uint32_t(warp * R * 8);
  const int64_t s0 = gw * per_warp, s1 = s0 + per_warp < nnz ? s0 + per_warp : nnz;
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  if (s0 < s1) {
    if (lane == 0) {
      for (int i = 0; i < R; ++i) mbar_init(bar_a + 8 * i, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    const int64_t nst = (s1 - s0 + kGtStageRows - 1) / kGtStageRows;
    int32_t icol = 0;   // lane l: column of nonzero l of the 4-stage window being issued
    float cval = 0.f;   // lane l: value of nonzero l of the 4-stage window being summed
    auto issue = [&](int64_t t) {  // stage t: nonzeros s0 + 8t .. s0 + 8t + 7
      const int64_t b = s0 + kGtStageRows * t;
      if ((t & 3) == 0) icol = b + lane < s1 ? __ldcs(cols + b + lane) : 0;
      int32_t c[kGtStageRows];
#pragma unroll
      for (int i = 0; i < kGtStageRows; ++i) c[i] = __shfl_sync(0xffffffffu, icol, int(t & 3) * kGtStageRows + i);
      const int valid = s1 - b < kGtStageRows ? int(s1 - b) : kGtStageRows;
#pragma unroll
      for (int i = 1; i < kGtStageRows; ++i)
        if (i >= valid) c[i] = c[0];  // padding rows: copied, never summed
      if (lane == 0) {
        const int ops = (valid + 3) / 4;
        const uint32_t bar = bar_a + 8 * uint32_t(t % R);
        const uint32_t dst = ring_a + uint32_t(t % R) * kStageBytes;
        mbar_arrive_expect_tx(bar, uint32_t(ops) * 4 * RB);
        tma_gather4(dst, &tmap, 0, c[0], c[1], c[2], c[3], bar);
        if (ops > 1) tma_gather4(dst + 4 * RB, &tmap, 0, c[4], c[5], c[6], c[7], bar);
      }
    };
    for (int64_t t = 0; t < R && t < nst; ++t) issue(t);
    int64_t t = 0;
    bool ok = true;
    for (; t < nst; ++t) {
      if (!mbar_wait(bar_a + 8 * uint32_t(t % R), uint32_t((t / R) & 1))) {
        ok = false;
        break;
      }
      const int64_t b = s0 + kGtStageRows * t;
      if ((t & 3) == 0) cval = b + lane < s1 ? gt_real<S>(__ldcs(vals + b + lane)) : 0.f;
      const int valid = s1 - b < kGtStageRows ? int(s1 - b) : kGtStageRows;
      const unsigned char* st = ring + (t % R) * kStageBytes + lane * (RB / 32);
#pragma unroll
      for (int i = 0; i < kGtStageRows; ++i) {
        const float a = __shfl_sync(0xffffffffu, cval, int(t & 3) * kGtStageRows + i);
        if (i < valid) {
          S v[E];
          if constexpr (RB / 32 == 16) *reinterpret_cast<uint4*>(v) = *reinterpret_cast<const uint4*>(st + i * RB);
          else *reinterpret_cast<uint2*>(v) = *reinterpret_cast<const uint2*>(st + i * RB);
#pragma unroll
          for (int e = 0; e < E; ++e) acc[e] = fmaf(a, gt_real<S>(v[e]), acc[e]);
        }
      }
      __syncwarp();  // every lane is done with the slot before the next copy into it
      if (t + R < nst) {
        if (lane == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(t + R);
      }
    }
    if (!ok) {  // a copy did not land in time: flag it, let the copies in flight finish
      if (lane == 0) atomicExch(err, 1);
      for (int64_t u = t; u < nst && u < t + R; ++u) (void)mbar_wait(bar_a + 8 * uint32_t(u % R), uint32_t((u / R) & 1));
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) out[(gw * 32 + lane) * E + e] = acc[e];
}

template <typename S, int RB>
int gather_tma_launch(CUtensorMapDataType tdt, const void* vals, const int32_t* cols, int64_t nnz, const void* B,
                      int64_t k_rows, int64_t ldb, float* out, int64_t out_rows, int* err, cudaStream_t st) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = encode_fn();
  if (!encode) return FSB_ERR_CUDA;
  alignas(64) CUtensorMap map;
  const cuuint64_t dims[2] = {cuuint64_t(RB / sizeof(S)), cuuint64_t(k_rows)};
  const cuuint64_t strides[1] = {cuuint64_t(ldb) * sizeof(S)};
  const cuuint32_t box[2] = {cuuint32_t(RB / sizeof(S)), 1};  // one row high: the gather4 box
  const cuuint32_t estr[2] = {1, 1};
  if (encode(&map, tdt, 2, const_cast<void*>(B), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
      CUDA_SUCCESS)
    return FSB_ERR_UNSUPPORTED;
  const int64_t blocks = out_rows / kGtWarps;
  const int64_t per_warp = ceil_div(nnz, out_rows);
  const size_t smem = size_t(kGtWarps) * kGtRingBytes + size_t(kGtWarps) * (kGtRingBytes / (kGtStageRows * RB)) * 8;
  auto kern = k_spmm_gather_tma<S, RB>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
    (void)cudaGetLastError();
    return FSB_ERR_CUDA;
  }
  kern<<<(unsigned)blocks, kGtWarps * 32, smem, st>>>(map, static_cast<const S*>(vals), cols, nnz, per_warp, out, err);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

template <typename S>
int gather_tma_rows(CUtensorMapDataType tdt, int64_t rb, const void* vals, const int32_t* cols, int64_t nnz,
                    const void* B, int64_t k_rows, int64_t ldb, float* out, int64_t out_rows, int* err,
                    cudaStream_t st) {
  if (rb == 512) return gather_tma_launch<S, 512>(tdt, vals, cols, nnz, B, k_rows, ldb, out, out_rows, err, st);
  if (rb == 256) return gather_tma_launch<S, 256>(tdt, vals, cols, nnz, B, k_rows, ldb, out, out_rows, err, st);
  return FSB_ERR_UNSUPPORTED;
}

}  // namespace
}  // namespace fsb

int fsb_spmm_gather_floor_tma(int dtype, const void* data, const int32_t* indices, int64_t nnz, const void* B,
                              int64_t k_rows, int64_t ldb, int64_t n, float* out, int64_t out_rows, int* err,
                              void* stream) {
  using namespace fsb;
  if (nnz < 0 || k_rows < 1 || k_rows > INT32_MAX || n < 1 || out_rows < kGtWarps || out_rows % kGtWarps != 0 ||
      out_rows / kGtWarps > INT32_MAX || ldb < n || !out || !err || (nnz > 0 && (!data || !indices || !B)))
    return FSB_ERR_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int64_t elem = 0;
  CUtensorMapDataType tdt;
  switch (dtype) {
    case FSB_F32: elem = 4; tdt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; break;
    case FSB_BF16: elem = 2; tdt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; break;
    case FSB_F16: elem = 2; tdt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; break;
    default: return FSB_ERR_UNSUPPORTED;
  }
  const int64_t rb = n * elem;
  if ((rb != 256 && rb != 512) || reinterpret_cast<uintptr_t>(B) % 16 != 0 || (ldb * elem) % 16 != 0)
    return FSB_ERR_UNSUPPORTED;
  switch (dtype) {
    case FSB_F32: return gather_tma_rows<float>(tdt, rb, data, indices, nnz, B, k_rows, ldb, out, out_rows, err, st);
    case FSB_BF16:
      return gather_tma_rows<__nv_bfloat16>(tdt, rb, data, indices, nnz, B, k_rows, ldb, out, out_rows, err, st);
    default: return gather_tma_rows<__half>(tdt, rb, data, indices, nnz, B, k_rows, ldb, out, out_rows, err, st);
  }
}

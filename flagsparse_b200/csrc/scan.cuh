// Deterministic device-wide exclusive scans for plan building.
//
// A scan over n items runs as three launches: per-tile sums, one block that
// scans the tile sums, and a pass that recomputes each item, scans it inside
// its tile and hands (index, exclusive prefix, value) to a writer functor.
// Items are produced by a functor, so flag arrays are never materialised.
// Every channel is an int64 counter; NV channels are scanned together.
#pragma once

#include "fsb_common.cuh"

namespace fsb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <int NV>
struct Vec {
  int64_t v[NV];
  __host__ __device__ __forceinline__ void zero() {
#pragma unroll
    for (int c = 0; c < NV; ++c) v[c] = 0;
  }
  __host__ __device__ __forceinline__ void add(const Vec& o) {
#pragma unroll
    for (int c = 0; c < NV; ++c) v[c] += o.v[c];
  }
};

// Exclusive scan of one Vec per thread across a kScanThreads block.
// Returns the exclusive prefix of this thread; `total` gets the block sum.
template <int NV>
__device__ __forceinline__ Vec<NV> block_exclusive_scan(Vec<NV> x, Vec<NV>& total) {
  __shared__ int64_t warp_tot[kScanThreads / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Vec<NV> inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      int64_t o = __shfl_up_sync(0xffffffffu, inc.v[c], d);
      if (lane >= d) inc.v[c] += o;
    }
  }
  if (lane == 31) {
#pragma unroll
    for (int c = 0; c < NV; ++c) warp_tot[warp][c] = inc.v[c];
  }
  __syncthreads();
  Vec<NV> base; base.zero();
  total.zero();
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      int64_t t = warp_tot[w][c];
      if (w < warp) base.v[c] += t;
      total.v[c] += t;
    }
  }
  __syncthreads();  // warp_tot may be reused by the caller's next scan
  Vec<NV> exc;
#pragma unroll
  for (int c = 0; c < NV; ++c) exc.v[c] = base.v[c] + inc.v[c] - x.v[c];
  return exc;
}

// Pass 1: tile sums. tile_sums layout: [NV][ntiles].
template <int NV, class F>
__global__ void __launch_bounds__(kScanThreads) k_scan_tile_reduce(F f, int64_t n, int64_t* tile_sums,
                                                                    int64_t ntiles) {
  const int64_t tile = blockIdx.x;
  const int64_t i0 = tile * kScanTile + int64_t(threadIdx.x) * kScanItems;
  Vec<NV> s; s.zero();
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = i0 + k;
    if (i < n) s.add(f(i));
  }
  Vec<NV> tot;
  block_exclusive_scan<NV>(s, tot);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < NV; ++c) tile_sums[c * ntiles + tile] = tot.v[c];
  }
}

// Pass 2: one block scans tile sums in place (exclusive) and writes totals[NV].
template <int NV>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int64_t* tile_sums, int64_t ntiles, int64_t* totals) {
  Vec<NV> carry; carry.zero();
  for (int64_t base = 0; base < ntiles; base += kScanThreads) {
    int64_t t = base + threadIdx.x;
    Vec<NV> x;
#pragma unroll
    for (int c = 0; c < NV; ++c) x.v[c] = (t < ntiles) ? tile_sums[c * ntiles + t] : 0;
    Vec<NV> tot;
    Vec<NV> exc = block_exclusive_scan<NV>(x, tot);
    if (t < ntiles) {
#pragma unroll
      for (int c = 0; c < NV; ++c) tile_sums[c * ntiles + t] = carry.v[c] + exc.v[c];
    }
    carry.add(tot);
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < NV; ++c) totals[c] = carry.v[c];
  }
}

// Pass 3: recompute, scan inside the tile, call w(i, prefix, value).
template <int NV, class F, class W>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(F f, W w, int64_t n, const int64_t* tile_offsets,
                                                              int64_t ntiles) {
  const int64_t tile = blockIdx.x;
  const int64_t i0 = tile * kScanTile + int64_t(threadIdx.x) * kScanItems;
  Vec<NV> vals[kScanItems];
  Vec<NV> s; s.zero();
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = i0 + k;
    if (i < n) vals[k] = f(i); else vals[k].zero();
    s.add(vals[k]);
  }
  Vec<NV> tot;
  Vec<NV> pre = block_exclusive_scan<NV>(s, tot);
#pragma unroll
  for (int c = 0; c < NV; ++c) pre.v[c] += tile_offsets[c * ntiles + tile];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = i0 + k;
    if (i < n) w(i, pre, vals[k]);
    pre.add(vals[k]);
  }
}

inline int64_t scan_ntiles(int64_t n) { return ceil_div(n, kScanTile); }
// Workspace of a scan: NV*ntiles tile sums + NV totals.
template <int NV>
inline int64_t scan_workspace_bytes(int64_t n) { return int64_t(sizeof(int64_t)) * NV * (scan_ntiles(n) + 1); }

// Runs passes 1 and 2; afterwards ws holds tile offsets followed by totals.
template <int NV, class F>
inline int scan_analyze(F f, int64_t n, int64_t* ws, cudaStream_t st) {
  const int64_t nt = scan_ntiles(n);
  if (nt == 0) {
    cudaMemsetAsync(ws, 0, sizeof(int64_t) * NV, st);
    FSB_LAUNCH_CHECK();
    return FSB_OK;
  }
  k_scan_tile_reduce<NV><<<(unsigned)nt, kScanThreads, 0, st>>>(f, n, ws, nt);
  FSB_LAUNCH_CHECK();
  k_scan_tiles<NV><<<1, kScanThreads, 0, st>>>(ws, nt, ws + NV * nt);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

template <int NV, class F, class W>
inline int scan_apply(F f, W w, int64_t n, const int64_t* ws, cudaStream_t st) {
  const int64_t nt = scan_ntiles(n);
  if (nt == 0) return FSB_OK;
  k_scan_apply<NV><<<(unsigned)nt, kScanThreads, 0, st>>>(f, w, n, ws, nt);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

template <int NV>
__host__ __device__ inline const int64_t* scan_totals(const int64_t* ws, int64_t n) { return ws + NV * ((n + kScanTile - 1) / kScanTile); }

}  // namespace fsb

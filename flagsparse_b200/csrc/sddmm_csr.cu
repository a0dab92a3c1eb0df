// CSR SDDMM  out[p] = alpha * <x[row(p)], y[col(p)]> + beta * in[p]  for sm_100a.
//
// x is M x K and y is N x K, both row-major; the sparsity pattern comes as the
// per-nonzero row ids and column indices (the reference's own prepared
// layout).  Every warp owns 32 consecutive nonzeros: it loads their row ids
// and columns with one coalesced read each, then walks them four at a time.
// The lanes own consecutive K-slices of V elements (16-byte loads when K and
// the leading dimensions allow it); the x and y slices of four nonzeros are
// loaded before any product is formed, and the four dot products are reduced
// together with a transpose butterfly (6 shuffles for 4 results instead of
// 20).  Consecutive nonzeros mostly share a row, so the x slice is an L1 hit.
//
// That generic kernel serves every shape; rows of 5 to 64 aligned 16-byte
// slices take the team kernel below, which caches the x row per team.
//
// Accumulation: fp32 for half / bfloat16 / fp32, fp64 for fp64 (fp64 for every
// type with FSB_SDDMM_ACC64, which the reference's "acc64" variants select),
// in a fixed order, so results are bitwise reproducible.
//
// Replaces _sddmm_csr_real_kernel (sparse_operations/sddmm_csr.py:121-162)
// launched by _run_sddmm_prepared (sddmm_csr.py:291-384) of flagos-ai/FlagSparse.
#include <cstring>
#include <type_traits>

#include "fsb_common.cuh"

namespace fsb {
namespace {

constexpr int kSddmmWarps = 8;
constexpr int kSddmmGroup = 4;  // nonzeros reduced together

template <int BYTES> struct SRaw;
template <> struct SRaw<2> { using T = unsigned short; };
template <> struct SRaw<4> { using T = unsigned int; };
template <> struct SRaw<8> { using T = uint2; };
template <> struct SRaw<16> { using T = uint4; };

template <typename S, int V>
__device__ __forceinline__ void sload(const S* p, int nv, S (&out)[V]) {
  if (nv == V) {
    using Raw = typename SRaw<int(sizeof(S)) * V>::T;
    Raw r = __ldg(reinterpret_cast<const Raw*>(p));
    memcpy(out, &r, sizeof(Raw));
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if (j < nv) out[j] = p[j];
      else memset(&out[j], 0, sizeof(S));
    }
  }
}

__device__ __forceinline__ __half sddmm_out(float v, const __half*) { return __float2half_rn(v); }
__device__ __forceinline__ __nv_bfloat16 sddmm_out(float v, const __nv_bfloat16*) { return __float2bfloat16_rn(v); }
__device__ __forceinline__ float sddmm_out(float v, const float*) { return v; }
__device__ __forceinline__ double sddmm_out(double v, const double*) { return v; }
__device__ __forceinline__ __half sddmm_out(double v, const __half*) { return __double2half(v); }
__device__ __forceinline__ __nv_bfloat16 sddmm_out(double v, const __nv_bfloat16*) { return __double2bfloat16(v); }
__device__ __forceinline__ float sddmm_out(double v, const float*) { return __double2float_rn(v); }

__device__ __forceinline__ double to_acc64(float v) { return static_cast<double>(v); }
__device__ __forceinline__ double to_acc64(double v) { return v; }

// grid: one warp per 32 nonzeros.  ACC64: accumulate in fp64 whatever the
// value type; OUT64: write fp64 results (only with ACC64).
template <int DT, int V, bool ACC64, bool OUT64>
__global__ void __launch_bounds__(kSddmmWarps * 32)
k_sddmm_csr(const int32_t* __restrict__ row_ids, const int32_t* __restrict__ col, int64_t nnz,
            const typename VT<DT>::Store* __restrict__ x, int64_t ldx, const typename VT<DT>::Store* __restrict__ y,
            int64_t ldy, int64_t k, const typename VT<DT>::Store* __restrict__ in, double alpha, double beta,
            typename std::conditional<OUT64, double, typename VT<DT>::Store>::type* __restrict__ out) {
  using S = typename VT<DT>::Store;
  using R = typename std::conditional<ACC64, double, typename VT<DT>::Real>::type;
  const int lane = threadIdx.x & 31;
  const int64_t base = (int64_t(blockIdx.x) * kSddmmWarps + (threadIdx.x >> 5)) * 32;
  if (base >= nnz) return;  // whole warp leaves together
  const int cnt = nnz - base < 32 ? static_cast<int>(nnz - base) : 32;
  int my_r = 0, my_c = 0;
  if (lane < cnt) {
    my_r = __ldcs(row_ids + base + lane);
    my_c = __ldcs(col + base + lane);
  }
  const R a = static_cast<R>(alpha), b = static_cast<R>(beta);
  const int64_t tile_w = int64_t(32) * V;
  const int n_tiles = static_cast<int>((k + tile_w - 1) / tile_w);

  for (int g = 0; g < cnt; g += kSddmmGroup) {
    R part[kSddmmGroup];
#pragma unroll
    for (int q = 0; q < kSddmmGroup; ++q) part[q] = R(0);
    int rq[kSddmmGroup], cq[kSddmmGroup];
#pragma unroll
    for (int q = 0; q < kSddmmGroup; ++q) {
      const int src = g + q < cnt ? g + q : g;
      rq[q] = __shfl_sync(0xffffffffu, my_r, src);
      cq[q] = __shfl_sync(0xffffffffu, my_c, src);
    }
    for (int t = 0; t < n_tiles; ++t) {
      const int64_t j0 = int64_t(t) * tile_w + int64_t(lane) * V;
      const int nv = static_cast<int>(k - j0 >= V ? int64_t(V) : (k > j0 ? k - j0 : int64_t(0)));
      S xs[kSddmmGroup][V], ys[kSddmmGroup][V];
#pragma unroll
      for (int q = 0; q < kSddmmGroup; ++q) {
        const int w = g + q < cnt ? nv : 0;
        sload<S, V>(x + int64_t(rq[q]) * ldx + j0, w, xs[q]);
        sload<S, V>(y + int64_t(cq[q]) * ldy + j0, w, ys[q]);
      }
#pragma unroll
      for (int q = 0; q < kSddmmGroup; ++q)
#pragma unroll
        for (int j = 0; j < V; ++j) {
          if constexpr (ACC64) part[q] = fma(to_acc64(to_real(xs[q][j])), to_acc64(to_real(ys[q][j])), part[q]);
          else part[q] = fma(to_real(xs[q][j]), to_real(ys[q][j]), part[q]);
        }
    }
    // Transpose butterfly: after the xor-16 step lanes 0-15 hold items {0,1}
    // and lanes 16-31 items {2,3}; after xor-8 each quarter of the warp holds
    // one item (quarter index = item index); xor 4, 2, 1 finish the sums.
    const bool hi16 = lane & 16, hi8 = lane & 8;
    R s0 = hi16 ? part[2] : part[0], s1 = hi16 ? part[3] : part[1];
    const R o0 = hi16 ? part[0] : part[2], o1 = hi16 ? part[1] : part[3];
    s0 += __shfl_xor_sync(0xffffffffu, o0, 16);
    s1 += __shfl_xor_sync(0xffffffffu, o1, 16);
    R v = hi8 ? s1 : s0;
    v += __shfl_xor_sync(0xffffffffu, hi8 ? s0 : s1, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    const int q = lane >> 3;
    if ((lane & 7) == 0 && g + q < cnt) {
      const int64_t p = base + g + q;
      R res = v * a;
      if (in) res += static_cast<R>(to_real(in[p])) * b;
      out[p] = sddmm_out(res, out);
    }
  }
}

// ---------------------------------------------------------------------------
// Fast path: teams of T lanes (8, 16 or 32) own 16-byte slices of a K-row,
// TILES (1 or 2) slices per lane, so T * VW * TILES >= K.  A team walks U = 4
// consecutive nonzeros per round; it keeps its current x row in registers as
// fp32 and reloads it only when the row changes, so each nonzero costs one
// 16-byte y load per lane.  The four dot products are reduced across the team
// by a transpose butterfly: after the T/2 step a lane holds 2 items, after
// T/4 one, then log2(T/4) plain steps.
// ---------------------------------------------------------------------------
constexpr int kTeamU = 4;

template <typename S> struct Widen;
template <> struct Widen<__nv_bfloat16> {
  static constexpr int VW = 8;
  __device__ __forceinline__ static void run(const uint4& w, float (&f)[8]) {
    const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      f[2 * i] = __uint_as_float(u[i] << 16);
      f[2 * i + 1] = __uint_as_float(u[i] & 0xffff0000u);
    }
  }
};
template <> struct Widen<__half> {
  static constexpr int VW = 8;
  __device__ __forceinline__ static void run(const uint4& w, float (&f)[8]) {
    const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      __half2 h;
      memcpy(&h, &u[i], 4);
      const float2 p = __half22float2(h);
      f[2 * i] = p.x;
      f[2 * i + 1] = p.y;
    }
  }
};
template <> struct Widen<float> {
  static constexpr int VW = 4;
  __device__ __forceinline__ static void run(const uint4& w, float (&f)[4]) {
    f[0] = __uint_as_float(w.x); f[1] = __uint_as_float(w.y);
    f[2] = __uint_as_float(w.z); f[3] = __uint_as_float(w.w);
  }
};
template <> struct Widen<double> {
  static constexpr int VW = 2;
  __device__ __forceinline__ static void run(const uint4& w, double (&f)[2]) {
    f[0] = __hiloint2double(int(w.y), int(w.x));
    f[1] = __hiloint2double(int(w.w), int(w.z));
  }
};

// acc += lo(x) * lo(y), then acc += hi(x) * hi(y) for two packed 16-bit
// values each: sm_100a's mixed-precision fma.rn.f32.{bf16,f16} multiplies the
// 16-bit inputs exactly (their product fits fp32) and rounds the sum once,
// so the result equals widening both to fp32 and calling fmaf, in the same
// order, with no widening instructions.
template <typename S>
__device__ __forceinline__ float fma_pair16(unsigned xw, unsigned yw, float acc) {
  if constexpr (std::is_same<S, __nv_bfloat16>::value) {
    asm("{\n .reg .b16 xl, xh, yl, yh;\n mov.b32 {xl, xh}, %1;\n mov.b32 {yl, yh}, %2;\n"
        " fma.rn.f32.bf16 %0, xl, yl, %0;\n fma.rn.f32.bf16 %0, xh, yh, %0;\n}"
        : "+f"(acc) : "r"(xw), "r"(yw));
  } else {
    asm("{\n .reg .b16 xl, xh, yl, yh;\n mov.b32 {xl, xh}, %1;\n mov.b32 {yl, yh}, %2;\n"
        " fma.rn.f32.f16 %0, xl, yl, %0;\n fma.rn.f32.f16 %0, xh, yh, %0;\n}"
        : "+f"(acc) : "r"(xw), "r"(yw));
  }
  return acc;
}

// 16-byte slice at p, or only its first nv elements (the rest zero).
template <typename S>
__device__ __forceinline__ uint4 slice16(const S* p, int nv) {
  constexpr int VW = 16 / int(sizeof(S));
  if (nv == VW) return __ldg(reinterpret_cast<const uint4*>(p));
  S tmp[VW];
#pragma unroll
  for (int j = 0; j < VW; ++j) {
    if (j < nv) tmp[j] = p[j];
    else memset(&tmp[j], 0, sizeof(S));
  }
  uint4 r;
  memcpy(&r, tmp, 16);
  return r;
}

template <int DT, int T, int TILES>
__global__ void __launch_bounds__(kSddmmWarps * 32, TILES == 1 ? 4 : 3)
k_sddmm_team(const int32_t* __restrict__ row_ids, const int32_t* __restrict__ col, int64_t nnz,
             const typename VT<DT>::Store* __restrict__ x, int64_t ldx, const typename VT<DT>::Store* __restrict__ y,
             int64_t ldy, int64_t k, const typename VT<DT>::Store* __restrict__ in, double alpha, double beta,
             typename VT<DT>::Store* __restrict__ out) {
  using S = typename VT<DT>::Store;
  using R = typename VT<DT>::Real;
  using W = Widen<S>;
  constexpr int VW = W::VW;
  constexpr int G = 32 / T;                 // teams per warp
  constexpr int PER_ROUND = G * kTeamU;     // nonzeros per warp round
  static_assert(T >= 8 && T <= 32, "team size");
  const int lane = threadIdx.x & 31;
  const int team = lane / T, tl = lane % T;
  const int64_t base = (int64_t(blockIdx.x) * kSddmmWarps + (threadIdx.x >> 5)) * 32;
  if (base >= nnz) return;  // whole warp leaves together
  const int cnt = nnz - base < 32 ? static_cast<int>(nnz - base) : 32;
  int my_r = -1, my_c = 0;
  if (lane < cnt) {
    my_r = __ldcs(row_ids + base + lane);
    my_c = __ldcs(col + base + lane);
  }
  int nvt[TILES];
  int64_t off[TILES];
#pragma unroll
  for (int t = 0; t < TILES; ++t) {
    off[t] = (int64_t(t) * T + tl) * VW;
    nvt[t] = static_cast<int>(k - off[t] >= VW ? int64_t(VW) : (k > off[t] ? k - off[t] : int64_t(0)));
  }
  const R a = static_cast<R>(alpha), b = static_cast<R>(beta);
  // 16-bit values: x rows stay packed and multiply through fma_pair16
  constexpr bool kMixed = sizeof(S) == 2;
  int cur = -1;
  R xf[TILES][VW];
  uint4 xw[TILES];
#pragma unroll
  for (int t = 0; t < TILES; ++t) {
    xw[t] = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int j = 0; j < VW; ++j) xf[t][j] = R(0);
  }

  for (int r0 = 0; r0 < cnt; r0 += PER_ROUND) {
    const int first = r0 + team * kTeamU;  // this team's items: first .. first+3
    int rq[kTeamU], cq[kTeamU];
#pragma unroll
    for (int u = 0; u < kTeamU; ++u) {
      rq[u] = __shfl_sync(0xffffffffu, my_r, (first + u) & 31);
      cq[u] = __shfl_sync(0xffffffffu, my_c, (first + u) & 31);
    }
    uint4 yw[kTeamU][TILES];
#pragma unroll
    for (int u = 0; u < kTeamU; ++u) {
      const bool valid = first + u < cnt;
#pragma unroll
      for (int t = 0; t < TILES; ++t)
        yw[u][t] = slice16<S>(y + int64_t(cq[u]) * ldy + off[t], valid ? nvt[t] : 0);
    }
    R part[kTeamU];
#pragma unroll
    for (int u = 0; u < kTeamU; ++u) {
      part[u] = R(0);
      if (first + u < cnt) {
        if (rq[u] != cur) {  // uniform inside the team
          cur = rq[u];
#pragma unroll
          for (int t = 0; t < TILES; ++t) {
            if constexpr (kMixed) xw[t] = slice16<S>(x + int64_t(cur) * ldx + off[t], nvt[t]);
            else W::run(slice16<S>(x + int64_t(cur) * ldx + off[t], nvt[t]), xf[t]);
          }
        }
#pragma unroll
        for (int t = 0; t < TILES; ++t) {
          if constexpr (kMixed) {
            part[u] = fma_pair16<S>(xw[t].x, yw[u][t].x, part[u]);
            part[u] = fma_pair16<S>(xw[t].y, yw[u][t].y, part[u]);
            part[u] = fma_pair16<S>(xw[t].z, yw[u][t].z, part[u]);
            part[u] = fma_pair16<S>(xw[t].w, yw[u][t].w, part[u]);
          } else {
            R yf[VW];
            W::run(yw[u][t], yf);
#pragma unroll
            for (int j = 0; j < VW; ++j) part[u] = fma(xf[t][j], yf[j], part[u]);
          }
        }
      }
    }
    // transpose butterfly inside the team
    constexpr int H = T / 2, Q = T / 4;
    const bool hb = tl & H, qb = tl & Q;
    R s0 = hb ? part[2] : part[0], s1 = hb ? part[3] : part[1];
    const R o0 = hb ? part[0] : part[2], o1 = hb ? part[1] : part[3];
    s0 += __shfl_xor_sync(0xffffffffu, o0, H);
    s1 += __shfl_xor_sync(0xffffffffu, o1, H);
    R v = qb ? s1 : s0;
    v += __shfl_xor_sync(0xffffffffu, qb ? s0 : s1, Q);
#pragma unroll
    for (int m = Q / 2; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    const int item = first + (hb ? 2 : 0) + (qb ? 1 : 0);
    if ((tl & (Q - 1)) == 0 && item < cnt) {
      const int64_t p = base + item;
      R res = v * a;
      if (in) res += to_real(in[p]) * b;
      out[p] = sddmm_out(res, out);
    }
  }
}

template <int DT, int T, int TILES>
int sddmm_launch_team(const int32_t* row_ids, const int32_t* col, int64_t nnz, const void* x, int64_t ldx,
                      const void* y, int64_t ldy, int64_t k, const void* in, double alpha, double beta, void* out,
                      cudaStream_t st) {
  using S = typename VT<DT>::Store;
  const int64_t blocks = ceil_div(ceil_div(nnz, 32), kSddmmWarps);
  if (blocks > INT32_MAX) return FSB_ERR_UNSUPPORTED;
  k_sddmm_team<DT, T, TILES><<<(unsigned)blocks, kSddmmWarps * 32, 0, st>>>(
      row_ids, col, nnz, static_cast<const S*>(x), ldx, static_cast<const S*>(y), ldy, k, static_cast<const S*>(in),
      alpha, beta, static_cast<S*>(out));
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

// Fast path when x / y rows are 16-byte aligned and K fits two 16-byte
// slices per lane of a 32-lane team; returns 1 when it launched (rc set).
template <int DT>
int sddmm_try_team(const int32_t* row_ids, const int32_t* col, int64_t nnz, const void* x, int64_t ldx,
                   const void* y, int64_t ldy, int64_t k, const void* in, double alpha, double beta, void* out,
                   int* rc, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  constexpr int VW = 16 / int(sizeof(S));
  if (reinterpret_cast<uintptr_t>(x) % 16 || reinterpret_cast<uintptr_t>(y) % 16 || ldx % VW || ldy % VW) return 0;
  const int64_t slices = ceil_div(k, VW);  // 16-byte slices per row
  if (slices < 5 || slices > 64) return 0;
  if (slices <= 8) *rc = sddmm_launch_team<DT, 8, 1>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
  else if (slices <= 16) *rc = sddmm_launch_team<DT, 16, 1>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
  else if (slices <= 32) *rc = sddmm_launch_team<DT, 32, 1>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
  else *rc = sddmm_launch_team<DT, 32, 2>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
  return 1;
}

template <int DT, int V, bool ACC64, bool OUT64>
int sddmm_launch_mode(const int32_t* row_ids, const int32_t* col, int64_t nnz, const void* x, int64_t ldx,
                      const void* y, int64_t ldy, int64_t k, const void* in, double alpha, double beta, void* out,
                      cudaStream_t st) {
  using S = typename VT<DT>::Store;
  using O = typename std::conditional<OUT64, double, S>::type;
  const int64_t blocks = ceil_div(ceil_div(nnz, 32), kSddmmWarps);
  if (blocks > INT32_MAX) return FSB_ERR_UNSUPPORTED;
  k_sddmm_csr<DT, V, ACC64, OUT64><<<(unsigned)blocks, kSddmmWarps * 32, 0, st>>>(
      row_ids, col, nnz, static_cast<const S*>(x), ldx, static_cast<const S*>(y), ldy, k,
      static_cast<const S*>(in), alpha, beta, static_cast<O*>(out));
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

template <int DT, int V>
int sddmm_launch_v(const int32_t* row_ids, const int32_t* col, int64_t nnz, const void* x, int64_t ldx,
                   const void* y, int64_t ldy, int64_t k, const void* in, double alpha, double beta, void* out,
                   int flags, cudaStream_t st) {
  if constexpr (DT != FSB_F64) {
    if (flags & FSB_SDDMM_OUT64)
      return sddmm_launch_mode<DT, V, true, true>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
    if (flags & FSB_SDDMM_ACC64)
      return sddmm_launch_mode<DT, V, true, false>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
  }
  return sddmm_launch_mode<DT, V, false, false>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, st);
}

template <int DT>
int sddmm_dispatch(const int32_t* row_ids, const int32_t* col, int64_t nnz, const void* x, int64_t ldx,
                   const void* y, int64_t ldy, int64_t k, const void* in, double alpha, double beta, void* out,
                   int flags, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  constexpr int kVmax = 16 / int(sizeof(S));
  if (!(flags & (FSB_SDDMM_ACC64 | FSB_SDDMM_OUT64)) || DT == FSB_F64) {
    int rc = FSB_OK;
    if (sddmm_try_team<DT>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, &rc, st)) return rc;
  }
  int v = 1;
  while (v < kVmax && int64_t(32) * v < k) v *= 2;
  auto ok = [&](int w) {
    const uintptr_t al = uintptr_t(w) * sizeof(S);
    return reinterpret_cast<uintptr_t>(x) % al == 0 && reinterpret_cast<uintptr_t>(y) % al == 0 && ldx % w == 0 &&
           ldy % w == 0;
  };
  while (v > 1 && !ok(v)) v /= 2;
  if constexpr (kVmax >= 8)
    if (v == 8) return sddmm_launch_v<DT, 8>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
  if constexpr (kVmax >= 4)
    if (v == 4) return sddmm_launch_v<DT, 4>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
  if constexpr (kVmax >= 2)
    if (v == 2) return sddmm_launch_v<DT, 2>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
  return sddmm_launch_v<DT, 1>(row_ids, col, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
}

// row_ids[p] = the row of nonzero p: one thread per nonzero, upper bound on indptr.
template <typename PT>
__global__ void k_csr_row_ids(const PT* __restrict__ ptr, int64_t n_rows, int64_t nnz, int32_t* __restrict__ rows) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += stride) {
    int64_t lo = 0, hi = n_rows - 1;  // last row r with ptr[r] <= p
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (ld_ptr(ptr, mid) <= p) lo = mid; else hi = mid - 1;
    }
    rows[p] = static_cast<int32_t>(lo);
  }
}

}  // namespace
}  // namespace fsb

using namespace fsb;

extern "C" {

int fsb_csr_row_ids(const void* indptr, int ptr_is_64, int64_t n_rows, int64_t nnz, int32_t* row_ids, void* stream) {
  if (!indptr || n_rows < 0 || nnz < 0 || (nnz > 0 && (!row_ids || n_rows == 0))) return FSB_ERR_INVALID_ARG;
  if (n_rows > INT32_MAX) return FSB_ERR_UNSUPPORTED;
  if (nnz == 0) return FSB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int64_t blocks = ceil_div(nnz, 256);
  if (blocks > 148 * 64) blocks = 148 * 64;
  if (ptr_is_64)
    k_csr_row_ids<int64_t><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const int64_t*>(indptr), n_rows, nnz, row_ids);
  else
    k_csr_row_ids<int32_t><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const int32_t*>(indptr), n_rows, nnz, row_ids);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

int fsb_sddmm_csr(int dtype, const int32_t* row_ids, const int32_t* indices, int64_t nnz, const void* x, int64_t ldx,
                  const void* y, int64_t ldy, int64_t k, const void* in, double alpha, double beta, void* out,
                  int flags, void* stream) {
  if ((flags & FSB_SDDMM_OUT64) && !(flags & FSB_SDDMM_ACC64)) return FSB_ERR_INVALID_ARG;
  if (nnz < 0 || k < 0 || ldx < k || ldy < k) return FSB_ERR_INVALID_ARG;
  if (nnz == 0) return FSB_OK;
  if (!row_ids || !indices || !out || (k > 0 && (!x || !y))) return FSB_ERR_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16: return sddmm_dispatch<FSB_F16>(row_ids, indices, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
    case FSB_BF16: return sddmm_dispatch<FSB_BF16>(row_ids, indices, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
    case FSB_F32: return sddmm_dispatch<FSB_F32>(row_ids, indices, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
    case FSB_F64: return sddmm_dispatch<FSB_F64>(row_ids, indices, nnz, x, ldx, y, ldy, k, in, alpha, beta, out, flags, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

}  // extern "C"

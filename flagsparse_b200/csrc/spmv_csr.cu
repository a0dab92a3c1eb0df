// CSR SpMV y = A x for sm_100a.
//
// Every warp executes work units of the plan built by fsb_spmv_plan_build
// (plan.cu); a unit's 32-byte descriptor carries its nonzero range, so the
// warp issues its value / column loads immediately.  The plan lists the two
// kinds of unit apart, and each kind runs as its own launch:
//
//  * row-block units: a run of rows with < 2*cap nonzeros.  Persistent warps
//    stride over the units, loading the next unit's descriptor and
//    prefetching its values and columns into L2 while the current unit runs.
//    Lanes load up to 14 nonzeros each with coalesced evict-first loads,
//    gather x, park the products in the warp's shared-memory slice in
//    compensated form, then a lane-level merge path sums the rows and a
//    segmented shuffle scan joins rows that span lanes.
//  * long-row chunks: `chunk_nnz` nonzeros of one row with > cap nonzeros, in
//    256-nonzero batches whose column loads are issued one batch ahead; no
//    shared memory; launched as a programmatic dependent of the row-block
//    launch so it overlaps that grid's tail.  A one-chunk row is written directly; otherwise the warp
//    publishes a partial sum and the warp whose atomic ticket completes the
//    row adds all partials in a fixed order and resets the ticket, so results
//    are deterministic.
//
// x is gathered with L2-only loads (ld.global.cg): the gathers have no reuse
// in L1, and where the row-block staging takes most of L1 they run faster
// without L1 allocation.
//
// Replaces _spmv_csr_real_kernel / _spmv_csr_complex_kernel
// (sparse_operations/spmv_csr.py:179-240) and the bucketed CSR-vector kernels
// (spmv_csr.py:247-368) of flagos-ai/FlagSparse.
#include <algorithm>
#include <mutex>

#include <cuda.h>
#include <type_traits>

#include "fsb_common.cuh"

namespace fsb {

// Per-nonzero contribution, one (hi, lo) pair per real component when the
// sum is compensated.  For the half types the fp32 product is exact, so lo
// stays 0 and is not stored.
template <int DT>
struct SpmvTraits {
  using V = VT<DT>;
  using S = typename V::Store;
  using R = typename V::Real;
  static constexpr int kComp = V::kComplex ? 2 : 1;
  static constexpr bool kLo = !V::kExactProduct;
};

template <typename S> __device__ __forceinline__ S to_store(float v);
template <> __device__ __forceinline__ __half to_store<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ float to_store<float>(float v) { return v; }
template <typename S> __device__ __forceinline__ S to_store(double v) { return v; }

// Row accumulator.  COMP = true: Dot2 compensated sums (Comp); COMP = false:
// plain sums in the real type (Plain), used only where the caller opts in.
template <int DT, bool COMP, bool CPLX = VT<DT>::kComplex>
struct SpmvAcc;

template <int DT, bool COMP>
struct SpmvAcc<DT, COMP, false> {
  using Tr = SpmvTraits<DT>;
  using S = typename Tr::S;
  using R = typename Tr::R;
  static constexpr bool kLo = COMP && Tr::kLo;   // stored products carry their rounding error
  static constexpr int kPartialReals = 2;
  using Sum = typename std::conditional<COMP, Comp<R>, Plain<R>>::type;
  Sum c;
  __device__ __forceinline__ void zero() { c.zero(); }
  // contribution of a*x; with kLo, hi + lo == a*x exactly
  __device__ __forceinline__ static void prod(S a, S x, R* hi, R* lo) {
    R ar = to_real(a), xr = to_real(x);
    R p = mul_rn(ar, xr);
    hi[0] = p;
    if constexpr (kLo) lo[0] = fma_rn(ar, xr, -p);
  }
  __device__ __forceinline__ void add_prod(S a, S x) {
    if constexpr (COMP) {
      if constexpr (Tr::kLo) c.add_prod(to_real(a), to_real(x));
      else c.add(mul_rn(to_real(a), to_real(x)));
    } else {
      c.add_prod(to_real(a), to_real(x));
    }
  }
  __device__ __forceinline__ void add_rec(const R* hi, const R* lo) {
    if constexpr (COMP) c.add_comp(hi[0], kLo ? lo[0] : R(0));
    else c.add(hi[0]);
  }
  __device__ __forceinline__ void combine(const SpmvAcc& o) {
    if constexpr (COMP) c.add_comp(o.c.hi, o.c.lo);
    else c.add(o.c.hi);
  }
  __device__ __forceinline__ void shfl_combine(int m) {
    SpmvAcc o = *this;
    o.c.hi = __shfl_xor_sync(0xffffffffu, c.hi, m);
    if constexpr (COMP) o.c.lo = __shfl_xor_sync(0xffffffffu, c.lo, m);
    combine(o);
  }
  __device__ __forceinline__ void shfl_up(int o) {
    c.hi = __shfl_up_sync(0xffffffffu, c.hi, o);
    if constexpr (COMP) c.lo = __shfl_up_sync(0xffffffffu, c.lo, o);
  }
  __device__ __forceinline__ S result() const { return to_store<S>(c.value()); }
  __device__ __forceinline__ void store(R* p) const {
    p[0] = c.hi;
    if constexpr (COMP) p[1] = c.lo;
  }
  __device__ __forceinline__ void load_cg(const R* p) {
    c.hi = __ldcg(p);
    if constexpr (COMP) c.lo = __ldcg(p + 1);
  }
};

// Short rows of the fp32 SpMV: fp64 sums of the exact products (an fp32
// product is exact in fp64, and the fp64 sum of a row-block row is far inside
// the Dot2 bound), staged as the two words of the double in the hi / lo
// slots.  One DADD per term instead of Dot2's six additions: the row-block
// launch is issue-bound, and the SpMV of the 2M x 2M Zipf(2) matrix took
// 0.200 against 0.204 ms.
struct SpmvWideF32 {
  static constexpr bool kLo = true;
  double c;
  __device__ __forceinline__ void zero() { c = 0.0; }
  __device__ __forceinline__ static void prod(float a, float x, float* hi, float* lo) {
    const double p = __dmul_rn(double(a), double(x));
    hi[0] = __int_as_float(__double2loint(p));
    lo[0] = __int_as_float(__double2hiint(p));
  }
  __device__ __forceinline__ void add_rec(const float* hi, const float* lo) {
    c = __dadd_rn(c, __hiloint2double(__float_as_int(lo[0]), __float_as_int(hi[0])));
  }
  __device__ __forceinline__ void combine(const SpmvWideF32& o) { c = __dadd_rn(c, o.c); }
  __device__ __forceinline__ void shfl_up(int o) { c = __shfl_up_sync(0xffffffffu, c, o); }
  __device__ __forceinline__ float result() const { return __double2float_rn(c); }
};

template <int DT, bool COMP>
struct SpmvAcc<DT, COMP, true> {
  using Tr = SpmvTraits<DT>;
  using S = typename Tr::S;
  using R = typename Tr::R;
  static constexpr bool kLo = COMP;
  static constexpr int kPartialReals = 4;
  using Sum = typename std::conditional<COMP, Comp<R>, Plain<R>>::type;
  Sum re, im;
  __device__ __forceinline__ void zero() { re.zero(); im.zero(); }
  // (ar + i ai)(xr + i xi): re = ar*xr - ai*xi, im = ar*xi + ai*xr.  With
  // COMP each part is a compensated pair built from the exact products.
  __device__ __forceinline__ static void prod(S a, S x, R* hi, R* lo) {
    if constexpr (COMP) {
      Comp<R> r, i;
      r.zero(); i.zero();
      r.add_prod(a.x, x.x); r.add_prod(-a.y, x.y);
      i.add_prod(a.x, x.y); i.add_prod(a.y, x.x);
      hi[0] = r.hi; lo[0] = r.lo; hi[1] = i.hi; lo[1] = i.lo;
    } else {
      hi[0] = fma_rn(a.x, x.x, -mul_rn(a.y, x.y));
      hi[1] = fma_rn(a.x, x.y, mul_rn(a.y, x.x));
    }
  }
  __device__ __forceinline__ void add_prod(S a, S x) {
    re.add_prod(a.x, x.x); re.add_prod(-a.y, x.y);
    im.add_prod(a.x, x.y); im.add_prod(a.y, x.x);
  }
  __device__ __forceinline__ void add_rec(const R* hi, const R* lo) {
    if constexpr (COMP) { re.add_comp(hi[0], lo[0]); im.add_comp(hi[1], lo[1]); }
    else { re.add(hi[0]); im.add(hi[1]); }
  }
  __device__ __forceinline__ void combine(const SpmvAcc& o) {
    if constexpr (COMP) { re.add_comp(o.re.hi, o.re.lo); im.add_comp(o.im.hi, o.im.lo); }
    else { re.add(o.re.hi); im.add(o.im.hi); }
  }
  __device__ __forceinline__ void shfl_combine(int m) {
    SpmvAcc o = *this;
    o.re.hi = __shfl_xor_sync(0xffffffffu, re.hi, m);
    o.im.hi = __shfl_xor_sync(0xffffffffu, im.hi, m);
    if constexpr (COMP) {
      o.re.lo = __shfl_xor_sync(0xffffffffu, re.lo, m);
      o.im.lo = __shfl_xor_sync(0xffffffffu, im.lo, m);
    }
    combine(o);
  }
  __device__ __forceinline__ void shfl_up(int o) {
    re.hi = __shfl_up_sync(0xffffffffu, re.hi, o);
    im.hi = __shfl_up_sync(0xffffffffu, im.hi, o);
    if constexpr (COMP) {
      re.lo = __shfl_up_sync(0xffffffffu, re.lo, o);
      im.lo = __shfl_up_sync(0xffffffffu, im.lo, o);
    }
  }
  __device__ __forceinline__ S result() const {
    S s; s.x = re.value(); s.y = im.value(); return s;
  }
  __device__ __forceinline__ void store(R* p) const {
    p[0] = re.hi; p[1] = re.lo; p[2] = im.hi; p[3] = im.lo;
  }
  __device__ __forceinline__ void load_cg(const R* p) {
    re.hi = __ldcg(p); re.lo = __ldcg(p + 1); im.hi = __ldcg(p + 2); im.lo = __ldcg(p + 3);
  }
};

template <typename T> __device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }
template <> __device__ __forceinline__ __half ld_stream<__half>(const __half* p) {
  unsigned short v = __ldcs(reinterpret_cast<const unsigned short*>(p));
  return __ushort_as_half(v);
}
template <> __device__ __forceinline__ __nv_bfloat16 ld_stream<__nv_bfloat16>(const __nv_bfloat16* p) {
  unsigned short v = __ldcs(reinterpret_cast<const unsigned short*>(p));
  return __ushort_as_bfloat16(v);
}
// Gather of x: L2-only, no L1 allocation.
template <typename T> __device__ __forceinline__ T ld_x(const T* p) { return __ldcg(p); }
template <> __device__ __forceinline__ __half ld_x<__half>(const __half* p) {
  return __ushort_as_half(__ldcg(reinterpret_cast<const unsigned short*>(p)));
}
template <> __device__ __forceinline__ __nv_bfloat16 ld_x<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __ushort_as_bfloat16(__ldcg(reinterpret_cast<const unsigned short*>(p)));
}

// One 128-byte line into L2; the address must lie inside the buffer.
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

constexpr int kSpmvWarps = 8;     // warps per block; one unit per warp
constexpr int kSpmvItems = 8;     // nonzeros per lane per long-row batch
constexpr int kSpmvBatch = 32 * kSpmvItems;

// Row-block units: nonzero slots per lane.  A unit holds < 2*cap nonzeros, so
// the largest window is cap = 16 * slots.  Units carry a fixed cost (their
// descriptor, row-pointer and first loads are dependent round trips), so the
// 2- and 4-byte real types use 14 slots (cap 224); the wider types keep 8.
// 14 rather than 16: the smaller staging slice leaves more of each SM's L1 to
// the long-row launch that overlaps this one's tail (199.7 against 210 us on
// a 2 M-row Zipf matrix).
template <int DT>
struct SpmvRow {
  static constexpr int kItems = (DT == FSB_F16 || DT == FSB_BF16 || DT == FSB_F32) ? 14 : 8;
  static constexpr int kBatch = 32 * kItems;
  static constexpr int kCap = kBatch / 2;
};

struct UnitRegs { int64_t s0, s1; int32_t row, tag, nch, slot; };

__device__ __forceinline__ UnitRegs load_unit(const fsb_spmv_unit* u) {
  const int4* p = reinterpret_cast<const int4*>(u);
  int4 a = __ldg(p), b = __ldg(p + 1);
  UnitRegs r;
  r.s0 = (int64_t)(uint32_t)a.x | ((int64_t)a.y << 32);
  r.s1 = (int64_t)(uint32_t)a.z | ((int64_t)a.w << 32);
  r.row = b.x;
  r.tag = b.y;
  r.nch = b.z;
  r.slot = b.w;
  return r;
}

// Per-warp shared-memory slice, rounded to 16 bytes so every warp's slice
// starts on a boundary that suits its widest element (double2 for c128).
template <int DT, bool SHORT_COMP>
static constexpr int spmv_warp_smem_bytes() {
  using Tr = SpmvTraits<DT>;
  constexpr bool lo = SpmvAcc<DT, SHORT_COMP>::kLo;
  return (Tr::kComp * int(sizeof(typename Tr::R)) * (lo ? 2 : 1) * SpmvRow<DT>::kBatch + 4 * (SpmvRow<DT>::kCap + 1) +
          15) & ~15;
}

// Resident blocks per SM the register budget is sized for: 8-byte reals and
// complex values need more registers per thread than fp32 / half types.
template <int DT>
struct SpmvMinBlocks { static constexpr int value = (DT == FSB_C128) ? 2 : (DT == FSB_F64 || DT == FSB_C64) ? 3 : 4; };
// The long-row kernel keeps fewer values live (no staging, columns one batch
// ahead): the 2- and 4-byte real types with 32-bit columns fit 5 blocks per SM
// without spills.
template <int DT, typename IT>
struct SpmvLongMinBlocks {
  static constexpr int value =
      ((DT == FSB_F16 || DT == FSB_BF16 || DT == FSB_F32) && sizeof(IT) == 4) ? 5 : SpmvMinBlocks<DT>::value;
};

// The long-row launch may start while the row-block launch before it still
// runs (programmatic dependent launch); pdl_join_primary makes its grid
// complete only after both have, so work later in the stream sees every y row.
__device__ __forceinline__ void spmv_long_join() { pdl_join_primary(); }

// LONG = true: the long-row chunks units[unit0, unit1), no shared memory (the
// gathers of long rows run faster with the L1 capacity that row-block staging
// would take); LONG = false: the row-block units.
template <int DT, typename IT, typename PT, bool SHORT_COMP, bool LONG>
__global__ void __launch_bounds__(kSpmvWarps * 32, LONG ? SpmvLongMinBlocks<DT, IT>::value : SpmvMinBlocks<DT>::value)
k_spmv_csr(const typename VT<DT>::Store* __restrict__ data, const IT* __restrict__ col,
           const PT* __restrict__ ptr, const typename VT<DT>::Store* __restrict__ x,
           typename VT<DT>::Store* __restrict__ y, fsb_spmv_plan plan, int64_t unit0, int64_t unit1) {
  using Tr = SpmvTraits<DT>;
  using S = typename Tr::S;
  using R = typename Tr::R;
  using Acc = SpmvAcc<DT, true>;  // long rows: always compensated
  constexpr int NC = Tr::kComp;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t unit = unit0 + int64_t(blockIdx.x) * kSpmvWarps + warp;
  if (unit >= unit1) return;  // whole warp leaves together

  if constexpr (LONG) {
    const UnitRegs u = load_unit(plan.units + unit);
    // ------------------------------------------------------ long-row chunk
    // Offsets within the chunk are 32-bit (chunk_nnz < 2^31).  Columns run one
    // batch ahead; values are loaded beside the x gathers they pair with.
    Acc acc;
    acc.zero();
    const S* dp = data + u.s0;
    const IT* cp = col + u.s0;
    const int n = static_cast<int>(u.s1 - u.s0);
    IT cv[kSpmvItems];
#pragma unroll
    for (int k = 0; k < kSpmvItems; ++k) {
      const int i = k * 32 + lane;
      if (i < n) cv[k] = ld_stream(cp + i);
    }
    for (int base = 0; base < n; base += kSpmvBatch) {
      S av[kSpmvItems], xv[kSpmvItems];
#pragma unroll
      for (int k = 0; k < kSpmvItems; ++k) {
        const int i = base + k * 32 + lane;
        if (i < n) { xv[k] = ld_x(x + cv[k]); av[k] = ld_stream(dp + i); }
      }
      IT cn[kSpmvItems];
#pragma unroll
      for (int k = 0; k < kSpmvItems; ++k) {
        const int i = base + kSpmvBatch + k * 32 + lane;
        if (i < n) cn[k] = ld_stream(cp + i);
      }
#pragma unroll
      for (int k = 0; k < kSpmvItems; ++k) {
        if (base + k * 32 + lane < n) acc.add_prod(av[k], xv[k]);
      }
#pragma unroll
      for (int k = 0; k < kSpmvItems; ++k) cv[k] = cn[k];
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) acc.shfl_combine(m);
    if (u.nch == 1) {
      if (lane == 0) y[u.row] = acc.result();
      spmv_long_join();
      return;
    }
    const int64_t s0 = int64_t(u.slot) + (u.tag + 1);  // slot of this row's first chunk
    R* part = static_cast<R*>(plan.partials);
    int ticket = 0;
    if (lane == 0) {
      acc.store(part + int64_t(u.slot) * Acc::kPartialReals);
      __threadfence();
      ticket = atomicAdd(plan.counters + s0, 1);
    }
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    if (ticket != u.nch - 1) {
      spmv_long_join();
      return;
    }
    __threadfence();
    Acc fin;
    fin.zero();
    for (int64_t c = lane; c < u.nch; c += 32) {
      Acc p;
      p.load_cg(part + (s0 + c) * Acc::kPartialReals);
      fin.combine(p);
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) fin.shfl_combine(m);
    if (lane == 0) {
      y[u.row] = fin.result();
      plan.counters[s0] = 0;  // ready for the next call
    }
    spmv_long_join();
  } else {
  // The long-row launch that follows is independent of this one (other rows,
  // its own scratch): let it start on the SMs this grid leaves.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // -------------------------------------------------------------- row block
  // Persistent warps: units unit, unit + stride, ...; the next unit's
  // descriptor is loaded while the current one is processed, so only the
  // value / column loads and the x gathers remain on each unit's critical path.
  const int64_t stride = int64_t(gridDim.x) * kSpmvWarps;
  UnitRegs u = load_unit(plan.units + unit);
  for (int64_t uid = unit; uid < unit1; uid += stride) {
  UnitRegs nxt = u;
  if (uid + stride < unit1) nxt = load_unit(plan.units + uid + stride);
  using SAcc = typename std::conditional<DT == FSB_F32 && SHORT_COMP, SpmvWideF32, SpmvAcc<DT, SHORT_COMP>>::type;
  constexpr bool kLo = SAcc::kLo;
  const int64_t r0 = u.row;
  const int nr = u.tag - u.row;
  const int n = static_cast<int>(u.s1 - u.s0);
  unsigned char* wbase = smem_raw + warp * spmv_warp_smem_bytes<DT, SHORT_COMP>();
  R* sh_hi = reinterpret_cast<R*>(wbase);
  constexpr int kRowItems = SpmvRow<DT>::kItems, kRowBatch = SpmvRow<DT>::kBatch;
  R* sh_lo = sh_hi + NC * kRowBatch;
  int32_t* sh_off = reinterpret_cast<int32_t*>(sh_hi + NC * kRowBatch * (kLo ? 2 : 1));

  // Units average about cap nonzeros against 2*cap slots: slots past n are
  // skipped by a warp-uniform test instead of being issued predicated off.
  S av[kRowItems];
  IT cv[kRowItems];
#pragma unroll
  for (int k = 0; k < kRowItems; ++k) {
    if (k * 32 >= n) break;
    const int i = k * 32 + lane;
    if (i < n) { av[k] = ld_stream(data + u.s0 + i); cv[k] = ld_stream(col + u.s0 + i); }
  }
  for (int i = lane; i <= nr; i += 32) sh_off[i] = static_cast<int32_t>(ld_ptr(ptr, r0 + i) - u.s0);
  if (uid + stride < unit1) {
    // the next unit's values (lanes 0-15) and columns (lanes 16-31) into L2,
    // one line per lane: 16 lines of each cover a whole unit of the 2- and
    // 4-byte types and the first part of a unit of the wider types
    const int64_t nn = nxt.s1 - nxt.s0;
    const int li = lane & 15;
    if (lane < 16) {
      constexpr int kPer = 128 / int(sizeof(S));
      if (int64_t(li) * kPer < nn) prefetch_l2(data + nxt.s0 + int64_t(li) * kPer);
    } else {
      constexpr int kPer = 128 / int(sizeof(IT));
      if (int64_t(li) * kPer < nn) prefetch_l2(col + nxt.s0 + int64_t(li) * kPer);
    }
  }
#pragma unroll
  for (int k = 0; k < kRowItems; ++k) {
    if (k * 32 >= n) break;
    const int i = k * 32 + lane;
    if (i < n) {
      R hi[NC], lo[NC];
      SAcc::prod(av[k], ld_x(x + cv[k]), hi, lo);
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        sh_hi[q * kRowBatch + i] = hi[q];
        if constexpr (kLo) sh_lo[q * kRowBatch + i] = lo[q];
      }
    }
  }
  __syncwarp();

  // Lane-level merge path over the unit's merged list of L = nr row ends and
  // n nonzeros: row i's end sits at position off[i+1] + i.  Lane l walks
  // positions [l*K, (l+1)*K) -- every lane does the same number of steps,
  // whatever the row lengths -- summing nonzeros and emitting a row at its end.
  const int L = nr + n;
  const int K = (L + 31) >> 5;
  const int d = min(lane * K, L);
  int lo_i = max(0, d - n), hi_i = min(d, nr);
  while (lo_i < hi_i) {  // i = number of row ends before position d
    const int mid = (lo_i + hi_i) >> 1;
    if (sh_off[mid + 1] + mid < d) lo_i = mid + 1; else hi_i = mid;
  }
  int i = lo_i, j = d - lo_i;
  const int stop = min(d + K, L);
  int next_end = i < nr ? sh_off[i + 1] : 0x7fffffff;
  SAcc acc, first;
  acc.zero();
  first.zero();
  int first_row = -1;
  for (int pos = d; pos < stop; ++pos) {
    if (j >= next_end) {
      if (first_row < 0) {
        first_row = i;   // may continue a row begun by earlier lanes: finish after the scan
        first = acc;
      } else {
        y[r0 + i] = acc.result();
      }
      acc.zero();
      ++i;
      next_end = i < nr ? sh_off[i + 1] : 0x7fffffff;
    } else {
      R hi[NC], lo[NC];
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        hi[q] = sh_hi[q * kRowBatch + j];
        lo[q] = kLo ? sh_lo[q * kRowBatch + j] : R(0);
      }
      acc.add_rec(hi, lo);
      ++j;
    }
  }
  // The partial a lane holds at its end belongs to row i, which the next lane
  // starts in.  A segmented inclusive scan over lanes (keys are non-decreasing
  // row indices) totals the partials of rows spanning several lanes.
  const int key = i;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    SAcc other = acc;
    other.shfl_up(o);
    const int okey = __shfl_up_sync(0xffffffffu, key, o);
    if (lane >= o && okey == key) acc.combine(other);
  }
  SAcc carry = acc;
  carry.shfl_up(1);
  if (first_row >= 0) {
    if (lane > 0) first.combine(carry);
    y[r0 + first_row] = first.result();
  }
  __syncwarp();  // the staging slice is rewritten by the next unit
  u = nxt;
  }  // units of this warp
  }  // row block
}

template <int DT, typename IT, typename PT, bool SHORT_COMP>
static int spmv_launch_mode(const void* data, const void* idx, const void* ptr, const void* x, void* y,
                            const fsb_spmv_plan& plan, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  const int64_t nb = plan.n_block_units, nu = plan.n_units;
  if (nb > 0) {  // row blocks: per-warp staging in shared memory
    const size_t smem = size_t(spmv_warp_smem_bytes<DT, SHORT_COMP>()) * kSpmvWarps;
    auto kern = k_spmv_csr<DT, IT, PT, SHORT_COMP, false>;
    if (smem > 48 * 1024) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return FSB_ERR_CUDA;
    }
    // persistent: at most the resident blocks (SpmvMinBlocks per SM on 148 SMs)
    const int64_t blocks = std::min<int64_t>(ceil_div(nb, kSpmvWarps), int64_t(148) * SpmvMinBlocks<DT>::value);
    kern<<<(unsigned)blocks, kSpmvWarps * 32, smem, st>>>(
        static_cast<const S*>(data), static_cast<const IT*>(idx), static_cast<const PT*>(ptr),
        static_cast<const S*>(x), static_cast<S*>(y), plan, 0, nb);
    FSB_LAUNCH_CHECK();
  }
  if (nu > nb) {  // long-row chunks: no shared memory
    // after a row-block launch: a programmatic dependent launch, so its blocks
    // fill the SMs the row-block grid's tail leaves (see spmv_long_join)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ceil_div(nu - nb, kSpmvWarps));
    cfg.blockDim = dim3(kSpmvWarps * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = nb > 0 ? 1 : 0;
    if (cudaLaunchKernelEx(&cfg, k_spmv_csr<DT, IT, PT, SHORT_COMP, true>, static_cast<const S*>(data),
                           static_cast<const IT*>(idx), static_cast<const PT*>(ptr), static_cast<const S*>(x),
                           static_cast<S*>(y), plan, nb, nu) != cudaSuccess) {
      (void)cudaGetLastError();
      return FSB_ERR_LAUNCH;
    }
  }
  return FSB_OK;
}

template <int DT, typename IT, typename PT>
static int spmv_launch(const void* data, const void* idx, const void* ptr, const void* x, void* y,
                       const fsb_spmv_plan& plan, cudaStream_t st) {
  // any window up to the type's cap fits a row-block unit's staging (<= cap rows, < 2*cap nonzeros)
  if (plan.cap < 1 || plan.cap > SpmvRow<DT>::kCap || plan.chunk_nnz % kSpmvBatch != 0) return FSB_ERR_INVALID_ARG;
  if (plan.flags & FSB_SPMV_FAST_SHORT_ROWS) return spmv_launch_mode<DT, IT, PT, false>(data, idx, ptr, x, y, plan, st);
  return spmv_launch_mode<DT, IT, PT, true>(data, idx, ptr, x, y, plan, st);
}

template <int DT>
static int spmv_dispatch_idx(const void* data, const void* idx, int i64, const void* ptr, int p64, const void* x,
                             void* y, const fsb_spmv_plan& plan, cudaStream_t st) {
  if (i64) {
    return p64 ? spmv_launch<DT, int64_t, int64_t>(data, idx, ptr, x, y, plan, st)
               : spmv_launch<DT, int64_t, int32_t>(data, idx, ptr, x, y, plan, st);
  }
  return p64 ? spmv_launch<DT, int32_t, int64_t>(data, idx, ptr, x, y, plan, st)
             : spmv_launch<DT, int32_t, int32_t>(data, idx, ptr, x, y, plan, st);
}

// ---------------------------------------------------------------------------
// The x-gather floor of a CSR SpMV (measurement only): out[b] = sum of
// data[i] * x[col[i]] over block b's grid-stride share of all nnz nonzeros,
// fp64 sums.  It moves the SpMV's values, columns and x gathers with the same
// load flavours (streaming values / columns, L2-only x) and 8 gathers in
// flight per thread, without the row structure: its time bounds what any
// CSR SpMV of the same pattern can reach.
// ---------------------------------------------------------------------------
constexpr int kFloorThreads = 256;
constexpr int kFloorItems = 8;

template <int DT, typename IT>
__global__ void __launch_bounds__(kFloorThreads)
k_gather_floor(const typename VT<DT>::Store* __restrict__ data, const IT* __restrict__ col, int64_t nnz,
               const typename VT<DT>::Store* __restrict__ x, double* __restrict__ out) {
  using S = typename VT<DT>::Store;
  __shared__ double red[kFloorThreads / 32];
  double acc = 0.0;
  const int64_t step = int64_t(gridDim.x) * kFloorThreads * kFloorItems;
  for (int64_t base = int64_t(blockIdx.x) * kFloorThreads * kFloorItems; base < nnz; base += step) {
    S av[kFloorItems], xv[kFloorItems];
#pragma unroll
    for (int q = 0; q < kFloorItems; ++q) {
      const int64_t i = base + q * kFloorThreads + threadIdx.x;
      if (i < nnz) {
        av[q] = ld_stream(data + i);
        xv[q] = ld_x(x + ld_stream(col + i));
      }
    }
#pragma unroll
    for (int q = 0; q < kFloorItems; ++q)
      if (base + q * kFloorThreads + threadIdx.x < nnz) acc = fma(double(to_real(av[q])), double(to_real(xv[q])), acc);
  }
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kFloorThreads / 32; ++w) t += red[w];
    out[blockIdx.x] = t;
  }
}

template <int DT>
static int gather_floor_launch(const void* data, const void* idx, int i64, int64_t nnz, const void* x, double* out,
                               int64_t blocks, cudaStream_t st) {
  using S = typename VT<DT>::Store;
  if (i64)
    k_gather_floor<DT, int64_t><<<(unsigned)blocks, kFloorThreads, 0, st>>>(
        static_cast<const S*>(data), static_cast<const int64_t*>(idx), nnz, static_cast<const S*>(x), out);
  else
    k_gather_floor<DT, int32_t><<<(unsigned)blocks, kFloorThreads, 0, st>>>(
        static_cast<const S*>(data), static_cast<const int32_t*>(idx), nnz, static_cast<const S*>(x), out);
  FSB_LAUNCH_CHECK();
  return FSB_OK;
}

// ---------------------------------------------------------------------------
// Built-in long-row scratch of fsb_spmv_csr_static_scratch: partial sums of
// the widest type (c128, 32 bytes) for every slot, then one int32 ticket per
// slot.  Zero at module load; every call clears the tickets it uses.
// ---------------------------------------------------------------------------
constexpr int64_t kStaticSlots = FSB_SPMV_STATIC_MAX_SLOTS;
constexpr int64_t kStaticPartialBytes = 4 * sizeof(double);
constexpr int64_t kStaticTicketOffset = kStaticSlots * kStaticPartialBytes;
static __device__ __align__(256) unsigned char g_spmv_static_scratch[kStaticTicketOffset + kStaticSlots * sizeof(int32_t)];

constexpr int kStaticMaxDevices = 256;
struct StaticScratchEntry {
  unsigned long long ctx_id;  // the context the address was resolved in (0: none yet)
  void* addr;
};
static StaticScratchEntry g_static_cache[kStaticMaxDevices];
static std::mutex g_static_mu;

// Unique id of the calling thread's current context, 0 if there is none or the
// driver cannot tell.  A device reset (or a new primary context) gives a new
// id, so an address resolved in an earlier context is never reused.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);
static unsigned long long current_context_id() {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PfnCtxGetCurrent>(p);
    else
      (void)cudaGetLastError();
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PfnCtxGetId>(p);
    else
      (void)cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the current device's scratch.  cudaGetSymbolAddress runs
// once per device and context: on the first call, and again only after the
// device's context changed (a device reset).  `st` must belong to the current
// device: the scratch of another device is not reachable through it.
static int static_scratch_address(cudaStream_t st, void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return FSB_ERR_CUDA;
  }
  if (dev < 0 || dev >= kStaticMaxDevices) return FSB_ERR_UNSUPPORTED;
  int sdev = -1;
  if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
    (void)cudaGetLastError();
    return FSB_ERR_INVALID_ARG;
  }
  if (sdev != dev) return FSB_ERR_INVALID_ARG;
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_static_mu);
  StaticScratchEntry& e = g_static_cache[dev];
  if (!e.addr || (ctx != 0 && e.ctx_id != ctx)) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_spmv_static_scratch) != cudaSuccess || !p) {
      (void)cudaGetLastError();
      return FSB_ERR_CUDA;
    }
    e.addr = p;
    e.ctx_id = current_context_id();  // the symbol lookup made the device's context current
  }
  *out = e.addr;
  return FSB_OK;
}

}  // namespace fsb

using namespace fsb;

extern "C" {

int64_t fsb_spmv_partial_bytes(int dtype) {
  switch (dtype) {
    case FSB_F16: case FSB_BF16: case FSB_F32: return 2 * sizeof(float);
    case FSB_F64: return 2 * sizeof(double);
    case FSB_C64: return 4 * sizeof(float);
    case FSB_C128: return 4 * sizeof(double);
    default: return -1;
  }
}

int fsb_spmv_csr(int dtype, const void* data, const void* indices, int idx_is_64, const void* indptr, int ptr_is_64,
                 int64_t n_rows, int64_t n_cols, const void* x, void* y, const fsb_spmv_plan* plan, void* stream) {
  if (!plan || n_rows < 0 || n_cols < 0) return FSB_ERR_INVALID_ARG;
  if (n_rows == 0 || plan->n_units == 0) return FSB_OK;
  if (!indptr || !y || !plan->units || plan->cap < 1 || plan->chunk_nnz < 1 || plan->n_slots < 0 ||
      plan->n_block_units < 0 || plan->n_block_units > plan->n_units ||
      (plan->n_slots > 0 && (!plan->partials || !plan->counters)))
    return FSB_ERR_INVALID_ARG;
  if (plan->n_units >= INT32_MAX) return FSB_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16: return spmv_dispatch_idx<FSB_F16>(data, indices, idx_is_64, indptr, ptr_is_64, x, y, *plan, st);
    case FSB_BF16: return spmv_dispatch_idx<FSB_BF16>(data, indices, idx_is_64, indptr, ptr_is_64, x, y, *plan, st);
    case FSB_F32: return spmv_dispatch_idx<FSB_F32>(data, indices, idx_is_64, indptr, ptr_is_64, x, y, *plan, st);
    case FSB_F64: return spmv_dispatch_idx<FSB_F64>(data, indices, idx_is_64, indptr, ptr_is_64, x, y, *plan, st);
    case FSB_C64: return spmv_dispatch_idx<FSB_C64>(data, indices, idx_is_64, indptr, ptr_is_64, x, y, *plan, st);
    case FSB_C128: return spmv_dispatch_idx<FSB_C128>(data, indices, idx_is_64, indptr, ptr_is_64, x, y, *plan, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

int fsb_spmv_gather_floor(int dtype, const void* data, const void* indices, int idx_is_64, int64_t nnz,
                          const void* x, double* out, int64_t n_out, void* stream) {
  if (nnz < 0 || n_out < 1 || !out || (nnz > 0 && (!data || !indices || !x))) return FSB_ERR_INVALID_ARG;
  const int64_t blocks = std::min<int64_t>(n_out, int64_t(148) * 8);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FSB_F16: return gather_floor_launch<FSB_F16>(data, indices, idx_is_64, nnz, x, out, blocks, st);
    case FSB_BF16: return gather_floor_launch<FSB_BF16>(data, indices, idx_is_64, nnz, x, out, blocks, st);
    case FSB_F32: return gather_floor_launch<FSB_F32>(data, indices, idx_is_64, nnz, x, out, blocks, st);
    case FSB_F64: return gather_floor_launch<FSB_F64>(data, indices, idx_is_64, nnz, x, out, blocks, st);
    default: return FSB_ERR_UNSUPPORTED;
  }
}

int fsb_spmv_csr_static_scratch(int dtype, const void* data, const void* indices, int idx_is_64, const void* indptr,
                                int ptr_is_64, int64_t n_rows, int64_t n_cols, const void* x, void* y,
                                const fsb_spmv_plan* plan, void* stream) {
  if (!plan || n_rows < 0 || n_cols < 0 || plan->n_slots < 0) return FSB_ERR_INVALID_ARG;
  if (plan->n_slots > kStaticSlots) return FSB_ERR_TOO_LARGE;
  if (fsb_spmv_partial_bytes(dtype) < 0) return FSB_ERR_UNSUPPORTED;
  if (n_rows == 0 || plan->n_units == 0) return FSB_OK;
  fsb_spmv_plan p = *plan;
  p.partials = nullptr;
  p.counters = nullptr;
  if (p.n_slots > 0) {
    void* base = nullptr;
    const int rc = static_scratch_address(static_cast<cudaStream_t>(stream), &base);
    if (rc != FSB_OK) return rc;
    p.partials = base;
    p.counters = reinterpret_cast<int32_t*>(static_cast<unsigned char*>(base) + kStaticTicketOffset);
    if (cudaMemsetAsync(p.counters, 0, size_t(p.n_slots) * sizeof(int32_t), static_cast<cudaStream_t>(stream)) !=
        cudaSuccess) {
      (void)cudaGetLastError();
      return FSB_ERR_CUDA;
    }
  }
  return fsb_spmv_csr(dtype, data, indices, idx_is_64, indptr, ptr_is_64, n_rows, n_cols, x, y, &p, stream);
}

}  // extern "C"

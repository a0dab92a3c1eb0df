/*
 * flagsparse_b200 C ABI.
 *
 * Plain-C entry points of the sm_100a CSR SpMV / SpMM / SDDMM library.  Every
 * function takes raw device pointers, sizes, dtype codes and a cudaStream_t
 * passed as `void*`; none allocates device memory, none throws, none aborts.
 * Each returns FSB_OK (0) or a negative FSB_ERR_* status.  Work is enqueued
 * on `stream`; the functions return without synchronising unless stated.
 *
 * Every entry point names the flagos-ai/FlagSparse interface it replaces
 * (paths relative to the FlagSparse source tree).  The Python host mirror in
 * flagsparse_b200/sparse_operations binds these with ctypes.
 */
#ifndef FLAGSPARSE_B200_H_
#define FLAGSPARSE_B200_H_

#include <stdint.h>

#if defined(__GNUC__)
#define FSB_API __attribute__((visibility("default")))
#else
#define FSB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FSB_OK 0
#define FSB_ERR_INVALID_ARG (-1)   /* bad size, null pointer, bad enum          */
#define FSB_ERR_UNSUPPORTED (-2)   /* dtype / index combination not built       */
#define FSB_ERR_LAUNCH (-3)        /* kernel launch failed                      */
#define FSB_ERR_TIMEOUT (-4)       /* a bounded device wait gave up             */
#define FSB_ERR_CUDA (-5)          /* other CUDA runtime error                  */
#define FSB_ERR_WORKSPACE (-6)     /* caller workspace too small                */
#define FSB_ERR_TOO_LARGE (-7)     /* plan exceeds a fixed built-in scratch     */

/* ---- value dtype codes (torch dtype -> code mapping lives in _native.py) -- */
#define FSB_F16 0
#define FSB_BF16 1
#define FSB_F32 2
#define FSB_F64 3
#define FSB_C64 4
#define FSB_C128 5

/* Library version (major*10000 + minor*100 + patch). */
FSB_API int fsb_version(void);

/* Human-readable text of a status code (static storage). */
FSB_API const char* fsb_status_string(int status);

/* ------------------------------------------------------------------------
 * CSR inspection.  One pass over indptr and indices that gathers every fact
 * the host-side validation needs, so the host reads one small vector instead
 * of issuing a synchronising reduction per check.
 * Replaces the chain of .item() checks in
 *   sparse_operations/spmv_csr.py:569-586 (_prepare_spmv_csr_matrix),
 *   sparse_operations/spmm_csr.py:371-403 (_prepare_spmm_csr_matrix),
 *   sparse_operations/sddmm_csr.py:79-92 (_prepare_sddmm_csr_pattern).
 * d_out (device, int64[6]) receives:
 *   [0] indptr[0]  [1] indptr[n_rows]  [2] count of i with indptr[i+1] < indptr[i]
 *   [3] min column index (INT64_MAX if nnz == 0)  [4] max column index (-1 if nnz == 0)
 *   [5] max row length (0 if n_rows == 0)
 * ------------------------------------------------------------------------ */
FSB_API int fsb_csr_inspect(const void* indices, int idx_is_64, const void* indptr, int ptr_is_64,
                    int64_t n_rows, int64_t nnz, int64_t* d_out, void* stream);

/* ------------------------------------------------------------------------
 * Stable row-length bucketing.  Bucket b holds the rows whose length lies in
 * (upper_bounds[b-1], upper_bounds[b]]; bucket 0 also holds empty rows and an
 * upper bound < 0 means "no bound".  Rows of a bucket keep ascending order, so
 * the result is identical to torch.nonzero on each bucket mask.
 * Replaces _build_spmv_opt_buckets (sparse_operations/spmv_csr.py:371-417)
 * and the count/compact kernels of sparse_operations/spmm_csr.py:3022-3153.
 * rows_out: int32[n_rows], all buckets concatenated in bucket order.
 * d_counts: int64[n_buckets] rows per bucket.  n_buckets <= 8.
 * ------------------------------------------------------------------------ */
FSB_API int64_t fsb_csr_bucketize_workspace_bytes(int64_t n_rows, int n_buckets);
FSB_API int fsb_csr_bucketize(const void* indptr, int ptr_is_64, int64_t n_rows,
                      const int64_t* upper_bounds, int n_buckets,
                      void* workspace, int64_t workspace_bytes,
                      int32_t* rows_out, int64_t* d_counts, void* stream);

/* ------------------------------------------------------------------------
 * CSR transpose (CSR of A -> CSR of A^T), stable in the original nonzero
 * order, so entries of one transposed row keep ascending source-row order.
 * Bit-identical to _transpose_csr_for_spmv (sparse_operations/spmv_csr.py:498-536)
 * and _transpose_csr_for_spmm (sparse_operations/spmm_csr.py:407-445), which
 * use a stable argsort by column, bincount and cumsum.
 * perm (int64[nnz]) receives, for every transposed entry, the position of its
 * value in the source arrays; fsb_gather_values applies it to any values.
 * Requires nnz < 2^31 and n_cols < 2^32.
 * ------------------------------------------------------------------------ */
FSB_API int64_t fsb_csr_transpose_workspace_bytes(int64_t nnz, int64_t n_rows, int64_t n_cols);
FSB_API int fsb_csr_transpose(const void* indices, int idx_is_64, const void* indptr, int ptr_is_64,
                      int64_t n_rows, int64_t n_cols, int64_t nnz,
                      void* workspace, int64_t workspace_bytes,
                      void* t_indices, int t_idx_is_64, void* t_indptr, int t_ptr_is_64,
                      int64_t* perm, void* stream);

/* dst[i] = src[perm[i]] (conjugated when conj != 0 and dtype is complex). */
FSB_API int fsb_gather_values(int dtype, const void* src, const int64_t* perm, int64_t n, int conj,
                      void* dst, void* stream);

/* ------------------------------------------------------------------------
 * COO -> CSR, the on-ramp for COO inputs (replaces coo_to_csr_for_spmv and
 * _coo_is_sorted_lex, sparse_operations/spmv_csr.py:948-984).
 *
 * fsb_coo_inspect: d_out (device int64[3]) receives the number of adjacent
 * pairs out of (row, col) order, of rows outside [0, n_rows) and of columns
 * outside [0, n_cols).
 *
 * fsb_coo_to_csr: out_col (int32[nnz]) and out_ptr (int64[n_rows + 1]) of
 * the CSR with entries in (row, col) order.  sorted != 0 states that the
 * input is already in that order (no workspace, perm untouched); otherwise a
 * stable radix sort of the packed (row, col) key runs in the workspace and
 * perm (int64[nnz]) receives the source position of every CSR entry, for
 * fsb_gather_values.  Repeated (row, col) pairs keep their input order.
 * Indices must lie inside the matrix (fsb_coo_inspect); nnz, n_rows and
 * n_cols must be < 2^31.
 * ------------------------------------------------------------------------ */
FSB_API int fsb_coo_inspect(const void* row, int row_is_64, const void* col, int col_is_64, int64_t nnz,
                      int64_t n_rows, int64_t n_cols, int64_t* d_out, void* stream);
FSB_API int64_t fsb_coo_to_csr_workspace_bytes(int64_t nnz, int64_t n_rows, int64_t n_cols);
FSB_API int fsb_coo_to_csr(const void* row, int row_is_64, const void* col, int col_is_64, int64_t nnz,
                      int64_t n_rows, int64_t n_cols, int sorted, void* workspace, int64_t workspace_bytes,
                      int32_t* out_col, int64_t* out_ptr, int64_t* perm, void* stream);

/* ------------------------------------------------------------------------
 * BSR SpMV  y = A x, any block dimension bd (replaces the BSR SpMV kernels of
 * sparse_operations/spmv_bsr.py:183-446).  blocks: [nnzb][bd][bd] row-major;
 * indices: block columns; indptr: [n_block_rows + 1] block row pointers.  x
 * has the padded length n_block_cols * bd, y receives all
 * n_block_rows * bd padded rows (empty block rows give 0).  Compensated
 * sums in block order: deterministic.  dtype: any of the six value types.
 * A^T x runs on the transposed matrix: fsb_csr_transpose of the block
 * pattern (n_cols = n_block_cols) gives its indices, row pointers and perm;
 * fsb_bsr_transpose_values gives its blocks (conjugated when conj != 0).
 * ------------------------------------------------------------------------ */
FSB_API int fsb_bsr_spmv(int dtype, const void* blocks, const void* indices, int idx_is_64, const void* indptr,
                      int ptr_is_64, int64_t n_block_rows, int64_t n_block_cols, int block_dim, const void* x,
                      void* y, void* stream);
FSB_API int fsb_bsr_transpose_values(int dtype, const void* src, const int64_t* perm, int64_t nnzb, int block_dim,
                      int conj, void* dst, void* stream);

/* ------------------------------------------------------------------------
 * CSR SpMV  y = A x.
 *
 * A launch plan splits the matrix into work units of one warp each:
 *  - row-block units: maximal runs of rows whose (row index + first nonzero
 *    index) falls in one window of `cap`; every row of the run has at most
 *    `cap` nonzeros, so a unit holds <= cap rows and < 2*cap nonzeros.  The
 *    warp streams them with coalesced loads, parks the products in shared
 *    memory and reduces each row with a team of lanes;
 *  - long-row units: a row with more than `cap` nonzeros is cut into chunks of
 *    `chunk_nnz` nonzeros; a row of one chunk is finished by its warp, a row of
 *    several chunks leaves one partial sum per chunk in its scratch slot of
 *    `partials` and the warp that finishes last (a ticket in the counter of
 *    the row's first slot) adds them in chunk order.
 * All sums use compensated (Dot2) accumulation in the value's real type, so
 * results do not depend on the unit split.
 * Replaces _triton_spmv_csr_impl_prepared / _spmv_csr_real_kernel
 * (sparse_operations/spmv_csr.py:702-746, 179-240) and the bucketed
 * _triton_spmv_csr_impl_opt_prepared (spmv_csr.py:433-482).
 * ------------------------------------------------------------------------ */
typedef struct fsb_spmv_unit {
  int64_t nnz_begin;         /* first nonzero of the unit                              */
  int64_t nnz_end;           /* one past its last nonzero                              */
  int32_t row;               /* first row (row block) / the row (long-row chunk)       */
  int32_t tag;               /* >= 0: row block ending before row `tag`;
                                < 0: chunk -(tag+1) of a long row                      */
  int32_t n_chunks;          /* chunks of that long row (1 for row blocks)             */
  int32_t slot;              /* scratch slot of a chunk of a row of >= 2 chunks; the
                                row's slots are consecutive.  -1 for other units       */
} fsb_spmv_unit;

typedef struct fsb_spmv_plan {
  const int32_t* seg_row0;   /* [n_segs + 1] first row of each segment; last entry == n_rows */
  const int32_t* seg_unit0;  /* [n_segs + 1] first work unit of each segment                */
  const fsb_spmv_unit* units;/* [n_units]    unit descriptors                                */
  int64_t n_segs;
  int64_t n_units;
  int64_t n_slots;           /* scratch slots, see fsb_spmv_unit.slot                        */
  int64_t n_block_units;     /* units[0, n_block_units) are row blocks, the rest long-row
                                chunks (fsb_spmv_csr launches the two kinds separately)      */
  int32_t cap;               /* row-block window, see above                                  */
  int32_t chunk_nnz;         /* nonzeros per long-row chunk                                  */
  void* partials;            /* scratch: n_slots * fsb_spmv_partial_bytes(dtype) bytes       */
  int32_t* counters;         /* scratch: n_slots int32, zero before the first call; every
                                call leaves them zero again                                  */
  int32_t flags;             /* FSB_SPMV_* / FSB_SPMM_* bits                                 */
  int32_t tile_bytes;        /* SpMM only: column tile of the team kernel in bytes (rounded
                                up to a power of two, 16 .. 512); 0 = the library's choice    */
} fsb_spmv_plan;

/* Sum the rows of row-block units (rows of <= cap nonzeros) with plain
 * accumulation in the value's real type instead of Dot2.  Long rows stay
 * compensated.  Off by default. */
#define FSB_SPMV_FAST_SHORT_ROWS 1

/* Row-block window: 224 for f16 / bf16 / f32 (14 nonzeros per lane), 128 for
 * the wider types; any smaller window is accepted. */
FSB_API int32_t fsb_spmv_default_cap(int dtype);
/* Long-row chunk: 1024 nonzeros for f16 / bf16 / f32, 512 for the wider types;
 * any positive multiple of 256 is accepted. */
FSB_API int32_t fsb_spmv_default_chunk(int dtype);
FSB_API int64_t fsb_spmv_partial_bytes(int dtype);
FSB_API int64_t fsb_spmv_plan_workspace_bytes(int64_t n_rows);
/* d_totals (device int64[4]) receives n_segs, n_units, n_slots and n_block_units. */
FSB_API int fsb_spmv_plan_analyze(const void* indptr, int ptr_is_64, int64_t n_rows, int32_t cap,
                          int32_t chunk_nnz, void* workspace, int64_t workspace_bytes,
                          int64_t* d_totals, void* stream);
FSB_API int fsb_spmv_plan_build(const void* indptr, int ptr_is_64, int64_t n_rows, int32_t cap,
                        int32_t chunk_nnz, const void* workspace, int64_t workspace_bytes,
                        int32_t* seg_row0, int32_t* seg_unit0, fsb_spmv_unit* units, void* stream);

FSB_API int fsb_spmv_csr(int dtype, const void* data, const void* indices, int idx_is_64,
                 const void* indptr, int ptr_is_64, int64_t n_rows, int64_t n_cols,
                 const void* x, void* y, const fsb_spmv_plan* plan, void* stream);

/* ------------------------------------------------------------------------
 * The x-gather floor of a CSR SpMV, for measurement: out[b] (b < the number
 * of blocks, min(n_out, 1184)) receives the fp64 sum of data[i] * x[indices[i]]
 * over block b's share of all nnz nonzeros, read with the SpMV's own load
 * kinds.  Its time is what any SpMV of that pattern needs for its values,
 * columns and x gathers alone.  Real dtypes (f16, bf16, f32, f64).
 * No FlagSparse counterpart: a measurement kernel of this library.
 * ------------------------------------------------------------------------ */
FSB_API int fsb_spmv_gather_floor(int dtype, const void* data, const void* indices, int idx_is_64, int64_t nnz,
                          const void* x, double* out, int64_t n_out, void* stream);

/* ------------------------------------------------------------------------
 * The B-row gather floor of the CSR SpMM through TMA (measurement kernel).
 *
 * out[w * n + j] = sum over nonzeros i in [w * per, min(nnz, (w + 1) * per))
 * of data[i] * B[indices[i] * ldb + j], fp32 sums, for w < out_rows and
 * j < n, per = ceil(nnz / out_rows): every nonzero's B row and no row
 * structure.  Rows of B are copied four at a time by cp.async.bulk.tensor
 * tile::gather4 into per-warp shared-memory rings (one CTA per 4 warps,
 * out_rows / 4 CTAs).  dtype f32, bf16 or f16 with n * sizeof(value) = 256
 * or 512 bytes (else FSB_ERR_UNSUPPORTED); indices int32 in [0, k_rows);
 * B 16-byte aligned with ldb * sizeof(value) a
 * multiple of 16; out_rows a positive multiple of 4.  *err (device int) is
 * set to 1 if a copy did not land within the wait limit, leaving out
 * partial.  No FlagSparse counterpart: a measurement kernel of this library.
 * ------------------------------------------------------------------------ */
FSB_API int fsb_spmm_gather_floor_tma(int dtype, const void* data, const int32_t* indices, int64_t nnz,
                                      const void* B, int64_t k_rows, int64_t ldb, int64_t n, float* out,
                                      int64_t out_rows, int* err, void* stream);

/* ------------------------------------------------------------------------
 * CSR SpMV with built-in scratch: allocates nothing on any call.
 *
 * No counterpart in flagos-ai/FlagSparse, whose SpMV allocates its output and
 * temporaries with torch on every call.  This entry point serves callers that
 * must not allocate device memory on the call path: code running where an
 * allocation could block or fail at the wrong time (a real-time loop with a
 * fixed memory budget, a caller that owns no allocator, a stream about to be
 * captured).
 *
 * Same arguments and results as fsb_spmv_csr (bit-identical output), except
 * that plan->partials and plan->counters are ignored (they may be NULL): the
 * long-row scratch is one file-scope device array of this library,
 * FSB_SPMV_STATIC_MAX_SLOTS slots (32 bytes of partial sum + one int32 ticket
 * each, 2.25 MiB per device).  A plan with n_slots > FSB_SPMV_STATIC_MAX_SLOTS
 * is rejected with FSB_ERR_TOO_LARGE before any work is enqueued; use
 * fsb_spmv_csr with caller scratch for it.  65536 slots cover every plan whose
 * multi-chunk long rows hold at most 65536 * chunk_nnz nonzeros (33.5 M at the
 * default chunk).
 *
 * The scratch is the current device's: `stream` must belong to the device
 * current on the calling thread (checked with cudaStreamGetDevice; a stream
 * of another device gives FSB_ERR_INVALID_ARG).  The first call on a device
 * resolves the scratch address with cudaGetSymbolAddress (once per device,
 * device current, status checked; failure returns FSB_ERR_CUDA); make that
 * first call before any stream capture begins.  The address is kept per
 * device and context: after a device reset the next call resolves it again
 * (and is then again a first call).  Every call clears the n_slots tickets
 * the plan uses (cudaMemsetAsync on `stream`) before its kernel.
 *
 * One scratch per device: calls whose kernels can overlap on the GPU (other
 * streams, other threads, other plans) race on it and give wrong results.
 * Serialise them, e.g. by issuing all such calls on one stream.
 * ------------------------------------------------------------------------ */
#define FSB_SPMV_STATIC_MAX_SLOTS 65536
FSB_API int fsb_spmv_csr_static_scratch(int dtype, const void* data, const void* indices, int idx_is_64,
                                const void* indptr, int ptr_is_64, int64_t n_rows, int64_t n_cols,
                                const void* x, void* y, const fsb_spmv_plan* plan, void* stream);

/* ------------------------------------------------------------------------
 * CSR SpMM  C = A B  (A: n_rows x n_cols CSR with int32 column indices and
 * int64 row pointers; B: n_cols x n row-major with row stride ldb; C: n_rows x
 * n row-major with row stride ldc; every element of C is written).
 *
 * Uses an fsb_spmv_plan built by fsb_spmv_plan_analyze / _build with
 * cap = fsb_spmm_default_cap (<= 64) and chunk_nnz = fsb_spmm_default_chunk
 * (a multiple of 128).  Rows made of whole 16-byte slices (16-byte aligned B
 * and C, n, ldb and ldc multiples of the slice) run on teams of lanes that own
 * whole rows (512-byte column tiles beyond 512 bytes); otherwise one warp
 * handles one (unit, column tile) and its lanes own consecutive column groups,
 * with loads as wide as B, C, ldb and ldc allow.  Rows of several chunks reduce
 * through the plan's
 * scratch, sized per slot by fsb_spmm_scratch_layout for this n:
 * partials = n_slots * partial_bytes_per_slot bytes, counters = n_slots *
 * tickets_per_slot int32 (zero before the first call; left zero).
 * Accumulation: fp32 for f16 / bf16 / f32, fp64 for f64, componentwise for
 * complex; plan->flags & FSB_SPMM_COMPENSATED selects Dot2 compensated sums.
 * Results are bitwise reproducible.
 * Replaces _triton_spmm_csr_impl / _spmm_csr_real_kernel and the complex
 * kernel (sparse_operations/spmm_csr.py:3373-3466, 144-339), which
 * flagsparse_spmm_csr (spmm_csr.py:3981-4137) and every registered route
 * (spmm_csr.py:2452-2544) launch.
 * ------------------------------------------------------------------------ */
#define FSB_SPMM_COMPENSATED 2
/* Team kernel (rows of whole 16-byte slices): a persistent grid of the
 * resident blocks whose warps stride over the work items, instead of one work
 * item per warp.  Results are identical either way; the batched step's
 * autotuner times both. */
#define FSB_SPMM_PERSISTENT 4

FSB_API int32_t fsb_spmm_default_cap(int dtype);
FSB_API int32_t fsb_spmm_default_chunk(int dtype);
FSB_API int fsb_spmm_scratch_layout(int dtype, int64_t n, int64_t* partial_bytes_per_slot,
                            int64_t* tickets_per_slot);
FSB_API int fsb_spmm_csr(int dtype, const void* data, const int32_t* indices, const int64_t* indptr,
                 int64_t n_rows, int64_t n_cols, const void* B, int64_t ldb, int64_t n,
                 void* C, int64_t ldc, const fsb_spmv_plan* plan, void* stream);

/* C = A B and y = A x in one launch (one pass over A's values and columns):
 * the narrow-row SpMM kernel whose team leaders also sum y, compensated, from
 * x[col] gathered beside B's row.  Real dtypes only; needs n * sizeof(value)
 * <= 256, n a multiple of 16 / sizeof(value), 16-byte aligned B and C with
 * such leading dimensions, and n not a multiple of 256 (y's long-row partial
 * takes column n of the slot scratch that fsb_spmm_scratch_layout sizes for
 * n).  Returns FSB_ERR_UNSUPPORTED otherwise, with nothing launched; the
 * caller then runs fsb_spmm_csr and fsb_spmv_csr.  plan as for fsb_spmm_csr. */
FSB_API int fsb_spmm_spmv_csr(int dtype, const void* data, const int32_t* indices, const int64_t* indptr,
                      int64_t n_rows, int64_t n_cols, const void* B, int64_t ldb, int64_t n, void* C, int64_t ldc,
                      const void* x, void* y, const fsb_spmv_plan* plan, void* stream);

/* Backward of Y = A X (A: n_rows x n_cols CSR with values vals[nnz]) in one
 * launch over the transposed pattern (t_indices int32[nnz], t_indptr
 * int64[n_cols + 1], and perm int32[nnz] with perm[q] = A's position of A^T's
 * nonzero q, as fsb_csr_transpose gives them):
 *   dX    = A^T dY                         (n_cols x n, row stride lddx)
 *   dvals[p] = <dY[row(p)], X[col(p)]>     (when dvals is not NULL)
 * dY is n_rows x n (stride lddy), X is n_cols x n (stride ldx).  Each dY row
 * slice is gathered once for both sums, and A's values are read through perm
 * (no transposed copy).  Real dtypes; needs 1 <= n, n * sizeof(value) <= 512,
 * n a multiple of 16 / sizeof(value), 16-byte aligned dY, dX (and X) with such
 * leading dimensions, and t_plan without FSB_SPMM_COMPENSATED.  Returns
 * FSB_ERR_UNSUPPORTED otherwise, with nothing launched; the caller then runs
 * fsb_gather_values + fsb_spmm_csr and fsb_sddmm_csr.  t_plan: A^T's SpMM plan
 * with scratch for this n (as for fsb_spmm_csr).  dX sums in fp32 (fp64 for
 * f64) in a fixed order, A^T rows of more than 1,024 nonzeros in fp64 from
 * exact products (f16, bf16, f32); each dvals entry sums in fp32 (fp64) over
 * a fixed tree.  No FlagSparse counterpart: it has no autograd for CSR SpMM. */
FSB_API int fsb_spmm_csr_backward(int dtype, const void* vals, const int32_t* perm, const int32_t* t_indices,
                          const int64_t* t_indptr, int64_t n_rows, int64_t n_cols, const void* dY, int64_t lddy,
                          const void* X, int64_t ldx, int64_t n, void* dX, int64_t lddx, void* dvals,
                          const fsb_spmv_plan* t_plan, void* stream);

/* ------------------------------------------------------------------------
 * CSR SDDMM  out[p] = alpha * <x[row(p)], y[col(p)]> + beta * in[p].
 *
 * x: M x k row-major (row stride ldx); y: N x k row-major (row stride ldy);
 * row_ids / indices: int32[nnz] row and column of every nonzero (CSR order);
 * in: nnz values or NULL (then beta is ignored); out: nnz values.  dtype is
 * f16, bf16, f32 or f64; the dot products accumulate in fp32 (fp64 for f64)
 * in a fixed order, or in fp64 with FSB_SDDMM_ACC64; FSB_SDDMM_OUT64 (with
 * ACC64) writes fp64 results.  Each warp owns 32 nonzeros and reduces four
 * dot products at a time.
 * Replaces _sddmm_csr_real_kernel / _run_sddmm_prepared
 * (sparse_operations/sddmm_csr.py:121-162, 291-384); fsb_csr_row_ids
 * replaces _build_row_ids (sddmm_csr.py:95-104).
 * ------------------------------------------------------------------------ */
FSB_API int fsb_csr_row_ids(const void* indptr, int ptr_is_64, int64_t n_rows, int64_t nnz,
                    int32_t* row_ids, void* stream);
#define FSB_SDDMM_ACC64 1
#define FSB_SDDMM_OUT64 2
FSB_API int fsb_sddmm_csr(int dtype, const int32_t* row_ids, const int32_t* indices, int64_t nnz,
                  const void* x, int64_t ldx, const void* y, int64_t ldy, int64_t k,
                  const void* in, double alpha, double beta, void* out, int flags, void* stream);

/* ------------------------------------------------------------------------
 * BSR SpMM with 16 x 16 blocks on the tensor cores (tcgen05.mma, fp32
 * accumulation in tensor memory):  C = A B, A = n_brows x n_bcols blocks.
 *
 * fsb_bsr16_pack rearranges blocks ([nnzb][16][16] row-major, FSB_BF16 or
 * FSB_F16) into the MMA's shared-memory layout, once per matrix; `packed`
 * (same size, 16-byte aligned) is what fsb_bsr16_spmm reads.
 * bcol: int32 block columns; bptr: int64 block row pointers [n_brows + 1];
 * B: (16 n_bcols) x n row-major, row stride ldb, 16-byte aligned, read with
 * TMA; C: (16 n_brows) x n, row stride ldc, written in the value type (block
 * rows without blocks give zero rows).  n must be a multiple of 64 (a
 * 128-column tile whose upper half lies past n loads and stores only its
 * lower half) and ldb of 8.  d_error is set to 1 if a bounded wait inside
 * the kernel expired (the kernel then stops, lets its copies and MMAs finish
 * and frees its tensor memory; C is not valid).  It is written with a plain
 * store and never cleared, so it may be device memory or mapped pinned host
 * memory that the host polls without synchronising.
 * No FlagSparse counterpart: its BSR support is SpMV (spmv_bsr.py).
 * ------------------------------------------------------------------------ */
FSB_API int fsb_bsr16_pack(int dtype, const void* blocks, int64_t nnzb, void* packed, void* stream);
FSB_API int fsb_bsr16_spmm(int dtype, const void* packed, const int32_t* bcol, const int64_t* bptr,
                   int64_t n_brows, int64_t n_bcols, const void* B, int64_t ldb, int64_t n,
                   void* C, int64_t ldc, int* d_error, void* stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* FLAGSPARSE_B200_H_ */

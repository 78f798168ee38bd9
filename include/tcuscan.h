/*
 * tcuscan.h -- C ABI of the B200 (sm_100a) tcuscan scan family.
 *
 * Plain pointers and sizes only: no torch types cross this boundary.  Every
 * device pointer must be 16-byte aligned; every call is asynchronous on the
 * given stream (a cudaStream_t passed as void*, NULL = legacy default stream)
 * and returns a status code.  Kernels that need a decoupled look-back take a
 * workspace from tcu_workspace_bytes()/tcu_workspace_init(); a workspace must
 * not be shared by launches that can overlap on the GPU.  Device-side errors
 * (a bounded wait that ran out) are recorded in the workspace and read back
 * with tcu_workspace_error().
 *
 * Each entry point names the reference interface it replaces (path:line in
 * huawei-csl/pytorch-tcuscan).
 */
#ifndef TCUSCAN_H_
#define TCUSCAN_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TCU_API __attribute__((visibility("default")))
#else
#define TCU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tcu_status {
  TCU_OK = 0,
  TCU_ERR_ARG = 1,        /* bad size / S / shape argument */
  TCU_ERR_DTYPE = 2,      /* unsupported dtype combination */
  TCU_ERR_LAUNCH = 3,     /* CUDA launch or API error */
  TCU_ERR_TIMEOUT = 4,    /* a device-side bounded wait ran out */
  TCU_ERR_OOM = 5,        /* allocation failed / budget exceeded */
  TCU_ERR_ALIGN = 6,      /* pointer not 16-byte aligned */
  TCU_ERR_DEVICE = 7,     /* no sm_100 device / driver entry point missing */
  TCU_ERR_WORKSPACE = 8   /* workspace missing or too small */
} tcu_status_t;

typedef enum tcu_dtype {
  TCU_INT8 = 1,
  TCU_INT16 = 2,
  TCU_INT32 = 3,
  TCU_INT64 = 4,
  TCU_FLOAT16 = 5,
  TCU_BFLOAT16 = 6,
  TCU_FLOAT32 = 7,
  TCU_FLOAT64 = 8,
  TCU_UINT32 = 9,
  TCU_UINT8 = 10
} tcu_dtype_t;

/* ---- library / workspace ------------------------------------------------ */
TCU_API int tcu_version(void);
TCU_API const char* tcu_status_string(int status);
/* Message of the last CUDA error seen by this thread (empty if none). */
TCU_API const char* tcu_last_error_message(void);
/* Timeout of every device-side bounded wait, in nanoseconds (default 4 s). */
TCU_API void tcu_set_timeout_ns(uint64_t ns);
TCU_API uint64_t tcu_get_timeout_ns(void);
/* Bytes of workspace needed by the look-back kernels for n elements at tile
 * parameter S (covers every entry point below for that n and S). */
TCU_API size_t tcu_workspace_bytes(int64_t n, int S);
/* Zero a freshly allocated workspace (once; later launches self-reset it). */
TCU_API tcu_status_t tcu_workspace_init(void* ws, size_t ws_bytes, void* stream);
/* Synchronise `stream`, copy out the sticky device error of a workspace:
 * info[0] = status code, info[1] = site, info[2] = chunk.  clear != 0 resets
 * it.  Returns info[0]. */
TCU_API tcu_status_t tcu_workspace_error(void* ws, uint32_t info[3], int clear, void* stream);
/* Diagnostics: when enabled, the scan kernels add per-phase device time (ns)
 * to eight counters in the workspace: 0 epilogue wait for the MMA, 1 row
 * totals, 2 look-back, 3 drain, 4 producer stage waits, 5 summer warp (its
 * waits included), 6 summer waits for landed data, 7 tiles.  Read (and
 * optionally clear) them with tcu_workspace_phase_ns (synchronises the
 * stream).  Off by default. */
TCU_API void tcu_set_phase_profile(int enable);
/* Self-test of device-side failure detection (no reference counterpart):
 * one warp waits, with the kernels' own bounded-wait code, on an mbarrier
 * phase (which = 0) or a look-back descriptor (which = 1) that nothing
 * completes, gives up after timeout_ns (<= 2 s), records TCU_ERR_TIMEOUT in
 * `ws` (read it with tcu_workspace_error) and returns.  Nothing faults. */
TCU_API tcu_status_t tcu_selftest_wait_timeout(int which, uint64_t timeout_ns, void* ws, size_t ws_bytes,
                                               void* stream);
/* Tuning: CTAs of the persistent scan and compaction launches (0 = one per
 * SM, the default; smaller values leave SMs to concurrent launches).
 * Process-wide; the autotuner sets it per size class. */
TCU_API void tcu_set_max_ctas(int n);
TCU_API int tcu_get_max_ctas(void);
/* Tuning: full scans of n elements run with one 128 x S block per look-back
 * tile (instead of 32768-element tiles) when ceil(n / 32768) < `tiles`, so
 * small inputs spread over every SM.  Default (or a negative value): the SM
 * count; 0 disables the small tiles.  Process-wide. */
TCU_API void tcu_set_small_tile_limit(int tiles);
TCU_API int tcu_get_small_tile_limit(void);
/* Tuning: full scans of at most `n` elements run in one SIMT pass -- 32
 * input bytes per thread, a block scan, a one-warp look-back -- instead of
 * on the tensor cores, whose per-tile chain of steps bounds small launches.
 * Default (a negative value; tcu_get_simt_scan_limit then returns -1): 2^18
 * fp16 / fp32 elements, 2^20 int8; 0 = never.  Same results up to FP32
 * rounding inside a tile (exact for int8).  Process-wide; no reference
 * counterpart (a launch-size choice inside run_scan_single_core /
 * run_scan_multi_core, src/torch/torch_scan.h:47-110, 184-241). */
TCU_API void tcu_set_simt_scan_limit(int64_t n);
TCU_API int64_t tcu_get_simt_scan_limit(void);
TCU_API tcu_status_t tcu_workspace_phase_ns(void* ws, uint64_t out[8], int clear, void* stream);

/* ---- scans ---------------------------------------------------------------
 * Inclusive prefix sum z = cumsum(x) + start.  x: int8 -> z int32 (exact,
 * two's-complement wrap like torch.cumsum(dtype=int32)); x: fp16 -> z fp32
 * (FP32 tensor-core rows, FP64 carry chain); x: fp32 -> z fp32 (each value
 * split into bf16 hi = RN(x) and lo = RN(x - hi), two MMAs into one FP32
 * accumulator, FP64 carry chain; S is fixed to 64).  S in {16,32,64,128} is the row
 * length of the S x S triangular tile multiplied on the tensor cores.
 * Replaces run_scan_multi_core (src/torch/torch_scan.h:184-241),
 * run_scan_multi_core_no_l2 (:253-304), run_scan_single_core (:47-110,
 * start = starting_sum) and run_scan_multi_cube (:416-466).              */
TCU_API tcu_status_t tcu_scan(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start, void* z, void* ws,
                      size_t ws_bytes, void* stream);

/* tcu_scan whose starting value also includes one element read from device
 * memory when the kernel runs (start_dev: int32 for int8 inputs, fp32
 * otherwise; NULL = none).  Chunks of a long input scanned one after another
 * on one stream, each given the previous chunk's last output as start_dev,
 * give the scan of the whole input without a host round trip between them
 * (used to overlap host copies with the scan, tcuscan_b200.stream).        */
TCU_API tcu_status_t tcu_scan_chained(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start,
                                      const void* start_dev, void* z, void* ws, size_t ws_bytes, void* stream);

/* tcu_scan_chained with the device start value's type given: start_dtype
 * TCU_INT32, TCU_INT64, TCU_FLOAT32 or TCU_FLOAT64 (start_dev aligned to its
 * size).  No reference counterpart: the sharded scan passes the exclusive
 * prefix of the ranks' totals as int64 (int8 input) or FP64 (fp16 / fp32
 * input), so the carry between ranks keeps the precision of the carry chain
 * inside one GPU.                                                          */
TCU_API tcu_status_t tcu_scan_chained_typed(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start,
                                            const void* start_dev, tcu_dtype_t start_dtype, void* z, void* ws,
                                            size_t ws_bytes, void* stream);

/* Sum of all n elements of x into *out (8-byte aligned device memory):
 * int8 -> int64 (exact), fp16 / fp32 -> FP64, in a fixed order (the same
 * bits on every call).  ws: a workspace of at least tcu_workspace_bytes(n, S)
 * bytes for any S (its scratch is zeroed again by the call).  No reference
 * counterpart: the exchange step of the sharded scan (one total per rank). */
TCU_API tcu_status_t tcu_total(const void* x, tcu_dtype_t dtype, int64_t n, void* out, void* ws, size_t ws_bytes,
                               void* stream);

/* Inclusive scan that allocates nothing.  No counterpart in the reference.
 * Same arguments and results as tcu_scan, minus the workspace, for callers
 * that cannot allocate device memory where they scan (inside an allocator or
 * memory-pool callback, under a fixed device budget owned by a host program,
 * or on a path that must not reach cudaMalloc).  Its look-back scratch is a
 * fixed 1 MiB array inside the library, held by every GPU that loads it
 * until exit; so n is limited to 2,147,221,504 elements and larger n returns
 * TCU_ERR_ARG.  The first call on a device looks the array up and zeroes it
 * on `stream`: make that first call before any stream capture.  The address
 * is kept for the life of the process, so do not call this entry point on a
 * device after cudaDeviceReset has been called on it.  All calls share the
 * array and it keeps the last call's contents, so calls that can overlap on
 * the GPU (other streams, other threads) race -- serialise them.
 * A device-side wait that ran out leaves its error in the shared array (each
 * call clears it first); read it with tcu_scan_noalloc_error after the call
 * and before the next one on that device.                                  */
TCU_API tcu_status_t tcu_scan_noalloc(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start, void* z,
                                      void* stream);
/* Error words of the last tcu_scan_noalloc call on the current device:
 * synchronises `stream`, copies them into info (info[0] = status code,
 * info[1] = site, info[2] = chunk; all zero when the call succeeded) with no
 * allocation, clears them when clear != 0, and returns info[0].  No
 * counterpart in the reference.                                            */
TCU_API tcu_status_t tcu_scan_noalloc_error(uint32_t info[3], int clear, void* stream);

/* Host-side inclusive scan of a host array (x and z in host memory; no GPU
 * work): int8 -> int32 (two's-complement wrap), fp16 / fp32 -> fp32.  The
 * input is cut into min(threads, n) contiguous blocks, each scanned
 * sequentially in the output type, the block totals scanned serially and
 * each block's offset added (skipped where it is zero), so the results are
 * bit-identical to the reference's for the same block count (it uses
 * omp_get_max_threads()).  n <= 2^32 - 1.  Synchronous.
 * Replaces run_scan_cpu (src/torch/torch_scan_cpu.h:24-107).              */
TCU_API tcu_status_t tcu_scan_cpu(const void* x, tcu_dtype_t x_dtype, int64_t n, void* z, int threads);

/* Per-row scans of n_rows rows of S elements (z has n_rows*S elements).
 * Replaces run_row_scan (src/torch/torch_scan.h:312-351).                 */
TCU_API tcu_status_t tcu_row_scan(const void* x, tcu_dtype_t x_dtype, int64_t n_rows, int S, void* z, void* ws,
                          size_t ws_bytes, void* stream);

/* Scan of every consecutive S*S block (n must be a multiple of S*S).
 * Replaces run_block_scan (src/torch/torch_scan.h:362-405).               */
TCU_API tcu_status_t tcu_block_scan(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, void* z, void* ws,
                            size_t ws_bytes, void* stream);

/* Block scan in the reference's tensor-only formulation: for every S x S
 * tile A of fp16 x (S = 64 or 128; n a multiple of S*S) z = A.upper +
 * lower_strict.(A.J) with J all ones, every product on the tensor cores
 * (the row totals A.J go back in as a three-term fp16 operand on a per-block
 * power-of-two scale, FP32 accumulation).  upper / lower_strict: the
 * caller's S x S fp16 row-major matrices on the device, used as given.
 * ws: a workspace (device-side wait errors are recorded there).  Replaces
 * run_block_scan (src/torch/torch_scan.h:362-405) with the reference's
 * multi-cube kernel (src/kernels/kernel_block_scan.h:23-40).              */
TCU_API tcu_status_t tcu_block_scan_tensor(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, const void* upper,
                                           const void* lower_strict, void* z, void* ws, size_t ws_bytes,
                                           void* stream);

/* ---- segmented scans (tensor cores) ---------------------------------------
 * Segmented inclusive scan of x (int8 -> int32 exact, fp16 -> fp32, fp32 ->
 * fp32 via split-precision bf16 hi + lo operands).
 * flags_are_ends = 0: flags[i] != 0 starts a segment at i (run_seg_scan,
 * src/torch/torch_seg_ops.h:165-193); 1: flags[i] != 0 ends a segment at i,
 * the building block of run_seg_sum (:85-107).  S in {16,32,64,128} (tiles of
 * 32 or 64 columns are used; results do not depend on S).                  */
TCU_API tcu_status_t tcu_seg_scan(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, const int8_t* flags,
                                  int flags_are_ends, void* z, void* ws, size_t ws_bytes, void* stream);
/* Segments given by a non-decreasing start array bounds[0..nbounds) (int32 or
 * int64; a CSR indptr).  out_sums = 1: out[k] = sum x[bounds[k]:bounds[k+1]]
 * for k < nbounds-1 (empty segments give 0) -- run_seg_sum_multi_core
 * (src/torch/torch_seg_ops.h:333-426), _single_core (:211-266), _multi_cube
 * (:443-522), _single_cube (:278-322, starts + n).  out_sums = 0: out is the
 * segmented scan of all n elements (uneven batched rows).                  */
TCU_API tcu_status_t tcu_seg_bounds(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, const void* bounds,
                                    tcu_dtype_t bounds_dtype, int64_t nbounds, int out_sums, void* out, void* ws,
                                    size_t ws_bytes, void* stream);
/* CSR SpMV y = A x with y fp32: products vals[i] * x[cols[i]] formed in fp32
 * (fp16 products exact) and written to the caller's prod_tmp (roundup(nnz,
 * 64) floats, 16-byte aligned) already split into the bf16 hi + lo operand
 * rows of the tensor-core segmented sum (64 hi then 64 lo per 64 products),
 * then indptr segment sums on the tensor cores (FP32 accumulation, FP64
 * carries across tiles).  indptr has rows + 1 entries
 * (int32 or int64).  Replaces run_spmv_v2 (src/torch/torch_spmv.h:112-209),
 * run_spmv_v2_multi_cube (:235-302), run_spmv (:63-94) and
 * run_spmv_multi_cube (:32-46).                                           */
TCU_API tcu_status_t tcu_spmv_csr(const void* vals, tcu_dtype_t dtype, const void* indptr, tcu_dtype_t indptr_dtype,
                                  int64_t rows, const int32_t* cols, int64_t nnz, const void* x, int64_t x_len, int S,
                                  float* y, float* prod_tmp, void* ws, size_t ws_bytes, void* stream);
/* Segment sums and SpMV split by elements on the SIMT cores (the
 * tensor-core segmented sum is bound by segment starts when segments are
 * short): 128 bytes of input per thread (32 elements for SpMV), segment
 * starts and ends marked in per-tile bitmaps, segments crossing threads
 * combined by a segmented scan and segments crossing CTAs by an in-order
 * fix-up, so each segment is summed in a fixed order (FP32 for fp16 / fp32
 * input, exact int32 for int8), independent of the launch.  Bounds must be
 * non-decreasing; empty segments give 0.  ws: a workspace of at least
 * tcu_rows_workspace_bytes(n) bytes (its scratch is zeroed again before the
 * call returns).
 * tcu_seg_sum_rows: out[k] = sum x[bounds[k]:bounds[k+1]] (bounds clamped to
 * [0, n]) -- the out_sums form of tcu_seg_bounds.
 * tcu_spmv_rows: y = A x with fp32 products vals[i] * x[cols[i]]; columns
 * outside [0, x_len) read 0 and are recorded in ws.  Same replacements as
 * tcu_seg_bounds / tcu_spmv_csr; the drop-in picks these for short mean
 * segment lengths.                                                          */
TCU_API size_t tcu_rows_workspace_bytes(int64_t n);
TCU_API tcu_status_t tcu_seg_sum_rows(const void* x, tcu_dtype_t x_dtype, int64_t n, const void* bounds,
                                      tcu_dtype_t bounds_dtype, int64_t nbounds, void* out, void* ws, size_t ws_bytes,
                                      void* stream);
TCU_API tcu_status_t tcu_spmv_rows(const void* vals, tcu_dtype_t dtype, const void* indptr, tcu_dtype_t indptr_dtype,
                                   int64_t rows, const int32_t* cols, int64_t nnz, const void* x, int64_t x_len,
                                   float* y, void* ws, size_t ws_bytes, void* stream);
/* The product step of tcu_spmv_csr on its own (fp16 / fp32 inputs). */
TCU_API tcu_status_t tcu_spmv_products(const void* values, tcu_dtype_t dtype, const int32_t* cols, int64_t nnz,
                                       const void* x, int64_t x_len, float* prod, void* ws, void* stream);
/* Row-wise scan of a row-major [batch, len] matrix (int8 / fp16 / fp32).
 * Replaces run_scan_batch (src/torch/torch_scan.h:119-175).               */
TCU_API tcu_status_t tcu_scan_batch(const void* x, tcu_dtype_t x_dtype, int64_t batch, int64_t len, int S, void* z,
                                    void* ws, size_t ws_bytes, void* stream);

/* ---- stream compaction ---------------------------------------------------
 * Stable compaction of x[mask != 0] (elem_bytes = 1, 2, 4 or 8; int8 mask):
 * a count pass over the mask, a scan of the tile counts, then one streaming
 * compaction pass; selected elements beyond `capacity` are dropped.  idx_mode 0: values only; 1: also gather idx_in
 * (idx_bytes = 4 or 8); 2: also write the selected positions (int32 when
 * idx_bytes = 4, int64 when 8).  count_dev (optional, 8-byte aligned device
 * int64) receives the number selected.
 * Replaces run_compress (src/torch/torch_compress.h:41-98), run_compress_pos
 * (:109-161, capacity = output_len), run_compress_ind (:172-239) and
 * run_compress_ind_no_arange (:249-309).                                   */
TCU_API tcu_status_t tcu_compress(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in,
                                  int idx_bytes, int idx_mode, void* out, void* idx_out, int64_t capacity,
                                  void* count_dev, void* ws, size_t ws_bytes, void* stream);
/* The two halves of tcu_compress, for callers that size the output from
 * the count first (run_compress reads the count back to the host, as the
 * reference does, src/torch/torch_compress.h:62-64): tcu_compress_count
 * counts the selected elements per tile, leaves the tile offsets in `ws` and
 * writes the total (int64) to count_dev; tcu_compress_counted then compacts
 * with those offsets.  The two calls take the same workspace, stream and
 * element / index sizes, with no other use of the workspace between them. */
TCU_API tcu_status_t tcu_compress_count(const int8_t* mask, int64_t n, int elem_bytes, int idx_mode, int idx_bytes,
                                        void* count_dev, void* ws, size_t ws_bytes, void* stream);
TCU_API tcu_status_t tcu_compress_counted(const void* x, int elem_bytes, const int8_t* mask, int64_t n,
                                          const void* idx_in, int idx_bytes, int idx_mode, void* out, void* idx_out,
                                          int64_t capacity, void* ws, size_t ws_bytes, void* stream);
/* Compaction of several independent requests packed into one buffer (the
 * serving loop batches compress calls this way): the stable compaction of
 * x[mask != 0] over all n elements, plus seg_pos[i] = number of selected
 * elements before seg_starts[i] (sorted int64 element offsets, one per
 * request) and seg_pos[nseg] = the total.  Request i's result is
 * out[seg_pos[i] : seg_pos[i+1]].  Batched form of run_compress
 * (src/torch/torch_compress.h:41-98). */
TCU_API tcu_status_t tcu_compress_segments(const void* x, int elem_bytes, const int8_t* mask, int64_t n,
                                           const int64_t* seg_starts, int64_t nseg, void* out, int64_t capacity,
                                           int64_t* seg_pos, void* ws, size_t ws_bytes, void* stream);
/* Stable partition: out[0, k) = x[mask != 0] and out[k, n) = x[mask == 0],
 * both in input order (k = number selected, written to count_dev as int64
 * when given).  idx_mode 0: values only; 1: idx_in (idx_bytes 4 or 8)
 * permuted the same way into idx_out.  out / idx_out hold n elements.  Same
 * passes and workspace as tcu_compress.  Replaces run_split
 * (src/torch/torch_split.h:33-79) and run_split_ind (:91-142), which take
 * 16-bit elements only; any of 1, 2, 4 or 8 bytes here.                   */
TCU_API tcu_status_t tcu_split(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in,
                               int idx_bytes, int idx_mode, void* out, void* idx_out, void* count_dev, void* ws,
                               size_t ws_bytes, void* stream);
/* Number of mask != 0 into a device uint64 (the reference sizes compress
 * outputs with run_reduce_tiles + .sum(), src/torch/torch_compress.h:62-64). */
TCU_API tcu_status_t tcu_mask_count(const int8_t* mask, int64_t n, void* count_dev, void* stream);

/* ---- CSR gather ------------------------------------------------------------
 * z[i] = values[i] * x[cols[i]] in the values dtype (fp16, int16, fp32).
 * Out-of-range columns read 0 and record TCU_ERR_ARG in ws (optional).
 * Replaces run_csr_gather (src/torch/torch_gather.h:92-172).               */
TCU_API tcu_status_t tcu_csr_gather(const void* values, tcu_dtype_t dtype, const int32_t* cols, int64_t nnz,
                                    const void* x, int64_t x_len, void* z, void* ws, void* stream);

/* z[i] = values[idxs[i] - 1] (elements of 2, 4 or 8 bytes), 0 where
 * idxs[i] == 0; idxs int32 / uint32 / int64.  An index past the values is
 * recorded in `ws` (if given) and gives 0.  Replaces run_gather_spmv
 * (src/torch/torch_gather.h:182-213), the row-pointer gather of the
 * reference's v1 SpMV.                                                     */
TCU_API tcu_status_t tcu_gather_spmv(const void* values, int elem_bytes, int64_t n_values, const void* idxs,
                                     tcu_dtype_t idx_dtype, int64_t n_idx, void* z, void* ws, void* stream);

/* ---- radix sort and top-k ------------------------------------------------
 * Ascending stable sort with int32 positions: out = sorted x, idx_out[i] =
 * position in x of out[i] (0-based), n <= 2^31 - 1.  Keys of 1, 2 or 4
 * bytes (int8/uint8, int16/fp16/bf16, int32/uint32/fp32) in byte-digit LSD
 * passes.  Floats are ordered by the reference's encoding: negatives below
 * positives, -0 below +0, NaNs with the sign bit first and NaNs without it
 * last.  tmp: device scratch of tcu_radix_sort_tmp_bytes(dtype, n) bytes,
 * 256-byte aligned, no initialisation needed.  Replaces run_radix_sort
 * (src/torch/torch_sort.h:30-82; fp16 / int16 there).                     */
TCU_API size_t tcu_radix_sort_tmp_bytes(tcu_dtype_t dtype, int64_t n);
TCU_API tcu_status_t tcu_radix_sort(const void* x, tcu_dtype_t dtype, int64_t n, void* out, int32_t* idx_out,
                                    void* tmp, size_t tmp_bytes, void* stream);
/* The k largest elements of x (int16, fp16 or bf16) and their int32
 * positions, in input order: every element above the k-th largest value
 * and, of the elements equal to it, the lowest-positioned ones.  NaN ranks
 * above every number and -0 equals +0 (value comparisons, as the reference's
 * x <= pivot splits).  0 <= k <= n.  tmp: tcu_topk_tmp_bytes(n) bytes,
 * 256-byte aligned.  Replaces run_topk_int16 / run_topk_fp16
 * (src/torch/torch_topk.h:86-211), which return the same set band by band;
 * their x_min / x_max bisection bounds are not needed here.               */
TCU_API size_t tcu_topk_tmp_bytes(int64_t n);
TCU_API tcu_status_t tcu_topk(const void* x, tcu_dtype_t dtype, int64_t n, int64_t k, void* out, int32_t* idx_out,
                              void* tmp, size_t tmp_bytes, void* stream);
/* Lower-bound estimates of the k-th largest value, one per block (fp16):
 * tcu_topk_pivot_blocks(n, num_samples) blocks = min(SM count, tiles of
 * num_samples * 32 elements); block b samples 8 tiles from tile
 * b * ceil(tiles / blocks); per tile the k_outer-th largest of the groups'
 * k_inner-th largest values (32-element groups).  Replaces
 * run_topk_pivot_fp16 (src/torch/torch_topk.h:35-73, k_inner 8 and
 * k_outer 4 there).                                                        */
TCU_API int tcu_topk_pivot_blocks(int64_t n, int num_samples);
TCU_API tcu_status_t tcu_topk_pivot(const void* x, tcu_dtype_t dtype, int64_t n, int num_samples, int k_inner,
                                    int k_outer, void* out, void* stream);

/* ---- scan phases as standalone operators ----------------------------------
 * reduce_tiles: z[b] = sum of block b, block = tile_len * ceil(ceil(n /
 * tile_len) / num_blocks) elements; int8 -> int32, fp16 -> fp32.  Needs
 * 128 + 8 * num_blocks * 64 bytes of workspace.
 * Replaces run_reduce_tiles (src/torch/torch_reduce.h:42-75).             */
TCU_API tcu_status_t tcu_reduce_tiles(const void* x, tcu_dtype_t dtype, int64_t n, int64_t tile_len, int num_blocks,
                                      void* z, void* ws, size_t ws_bytes, void* stream);
/* complete_rows: block b (n / num_blocks elements) starts from sum(sums[:b]);
 * each `width`-long row gets the running carry added, and the carry becomes
 * the updated row's last element.  fp32 or int32.  Workspace: 128 + 8 *
 * num_blocks * ceil(block / width) bytes.
 * Replaces run_complete_rows (src/torch/torch_reduce.h:143-182).          */
TCU_API tcu_status_t tcu_complete_rows(const void* x, tcu_dtype_t dtype, int64_t n, const void* sums, int num_blocks,
                                       int64_t width, void* z, void* ws, size_t ws_bytes, void* stream);
/* complete_blocks: z[block b] = x[block b] + sum(sums[:b]); fp32 or int32.
 * Replaces run_complete_blocks (src/torch/torch_reduce.h:197-231).        */
TCU_API tcu_status_t tcu_complete_blocks(const void* x, tcu_dtype_t dtype, int64_t n, const void* sums,
                                         int num_blocks, void* z, void* stream);
/* z = tril(ones(s, s)) in int8 / fp16 / bf16 / fp32 / int32.
 * Replaces run_gen_lower (src/torch/torch_gen_lower.h:31-59).            */
TCU_API tcu_status_t tcu_gen_lower(int64_t s, tcu_dtype_t dtype, void* z, void* stream);

/* ---- request packing (serving loop) ----------------------------------------
 * The reference has no serving layer: each request is one run_* call
 * (src/torch/torch_scan.h, torch_seg_ops.h, torch_compress.h).  The serving
 * loop batches requests by packing them into one buffer and running one
 * segmented launch; tcu_pack is the packing step.  `items` (device memory,
 * sorted by dst, contiguous: items[0].dst == 0, items[i+1].dst == items[i].dst
 * + items[i].len, total == sum of len) each copy n elements from src into
 * dst[item.dst : item.dst + n] and zero the rest of the item's len.  src_bytes
 * == dst_bytes copies elements of 1, 2, 4 or 8 bytes; src 4 -> dst 8 widens
 * int32 to int64.  For 4- and 8-byte integer elements `add` is added to every
 * copied element (rebasing row pointers by the request's offset); it must be
 * zero for floating-point data.                                            */
typedef struct tcu_pack_item {
  const void* src;
  int64_t dst;
  int64_t n;
  int64_t len;
  int64_t add;
} tcu_pack_item_t;
TCU_API tcu_status_t tcu_pack(const tcu_pack_item_t* items, int64_t nitems, int src_bytes, int dst_bytes, void* dst,
                              int64_t total, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TCUSCAN_H_ */

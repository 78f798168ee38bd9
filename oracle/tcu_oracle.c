/*
 * tcu_oracle.c -- CPU restatement of the tcuscan scan family, used ONLY as
 * test infrastructure (the reference of the parity tests and the timed CPU
 * "port" baseline).
 * Nothing in the product links or calls this file.
 *
 * Every function states the reference file:line whose semantics it restates.
 * Float data is accumulated in FP64 and integer data in int64 so the oracle is
 * the exact answer the CUDA path is compared against; callers cast to the
 * reference's output dtype (fp32 / int32 with two's-complement wrap).
 *
 * Parity pin: tests/golden/ holds fixtures produced by the reference's own
 * run_scan_cpu (compiled from src/torch/torch_scan_cpu.h) and by the
 * reference's own test oracles (ref_segsum, ref_segscan, ref_complete_rows,
 * ref_complete_blocks, ref_reduce_tiles, masked_select, values * x[cols],
 * scipy A @ x); tests/test_oracle_golden.py checks this file against them.
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* Blocked three-phase scan, restating parallel_inclusive_scan_blocked
 * (src/torch/torch_scan_cpu.h:24-80) in fp32/int32 arithmetic with the same
 * block partition, executed serially.  With `blocks` equal to the reference's
 * omp_get_max_threads() it reproduces run_scan_cpu bit-for-bit.            */
#define BLOCKED_SCAN(NAME, T)                                                  \
  EXPORT void NAME(T* a, int64_t n, int64_t threads) {                         \
    if (n <= 0) return;                                                        \
    int64_t blocks = threads < 1 ? 1 : threads;                                \
    if (blocks > n) blocks = n;                                                \
    const int64_t bs = (n + blocks - 1) / blocks;                              \
    T running = (T)0;                                                          \
    /* phase 1 + 2 fused serially: block-local scans, then block prefixes */   \
    T totals[4096];                                                            \
    if (blocks > 4096) blocks = 4096; /* caller bound */                       \
    for (int64_t b = 0; b < blocks; ++b) {                                     \
      const int64_t s = b * bs, e = (s + bs < n) ? s + bs : n;                 \
      if (s >= e) { totals[b] = (T)0; continue; }                              \
      T sum = a[s];                                                            \
      for (int64_t i = s + 1; i < e; ++i) { sum += a[i]; a[i] = sum; }         \
      totals[b] = sum;                                                         \
    }                                                                          \
    for (int64_t b = 0; b < blocks; ++b) {                                     \
      const T off = running;                                                   \
      running += totals[b];                                                    \
      if (off == (T)0) continue; /* torch_scan_cpu.h:72 skips zero offsets */  \
      const int64_t s = b * bs, e = (s + bs < n) ? s + bs : n;                 \
      for (int64_t i = s; i < e; ++i) a[i] += off;                             \
    }                                                                          \
  }
BLOCKED_SCAN(tcuo_blocked_scan_f32, float)
BLOCKED_SCAN(tcuo_blocked_scan_i32, int32_t)

/* ------------------------------------------------------------------------ */
/* Inclusive prefix sum with a starting value.
 * Semantics: tests/test_scan_multi_core.py:45 (torch.cumsum) and
 * run_scan_single_core's starting_sum (src/torch/torch_scan.h:47-110).      */
EXPORT void tcuo_cumsum_f64(const double* x, double* out, int64_t n, double start) {
  double acc = start;
  for (int64_t i = 0; i < n; ++i) { acc += x[i]; out[i] = acc; }
}
EXPORT void tcuo_cumsum_i64(const int64_t* x, int64_t* out, int64_t n, int64_t start) {
  int64_t acc = start;
  for (int64_t i = 0; i < n; ++i) { acc += x[i]; out[i] = acc; }
}

/* Per-row scan of length-S rows: z[r*S+j] = sum_{k<=j} x[r*S+k].
 * Semantics: KernelRowScan (src/kernels/kernel_row_scan.h:47-176),
 * tests/test_row_scan.py:34-40 (F.linear(A, tril)).  Also the block scan
 * (per S*S tile, src/kernels/kernel_block_scan.h:23-40,
 * tests/test_block_scan.py:28-38) with seg = S*S, and run_scan_batch
 * (src/torch/torch_scan.h:119-175) with seg = L.                            */
EXPORT void tcuo_segment_scan_fixed_f64(const double* x, double* out, int64_t n, int64_t seg) {
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (i % seg == 0) acc = 0.0;
    acc += x[i];
    out[i] = acc;
  }
}
EXPORT void tcuo_segment_scan_fixed_i64(const int64_t* x, int64_t* out, int64_t n, int64_t seg) {
  int64_t acc = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (i % seg == 0) acc = 0;
    acc += x[i];
    out[i] = acc;
  }
}

/* Batched scan over uneven rows given by offsets[0..B] (row b is
 * x[offsets[b]:offsets[b+1]]).  Extends run_scan_batch
 * (src/torch/torch_scan.h:119-175) from uniform L to uneven rows.          */
EXPORT void tcuo_scan_offsets_f64(const double* x, double* out, const int64_t* offsets, int64_t B) {
  for (int64_t b = 0; b < B; ++b) {
    double acc = 0.0;
    for (int64_t i = offsets[b]; i < offsets[b + 1]; ++i) { acc += x[i]; out[i] = acc; }
  }
}

/* Flag segmented scan, f[i] != 0 => a segment starts at i.
 * Semantics: ref_segscan (tests/test_seg_scan_single_core.py:40-63) and the
 * sequential baseline scripts/baselines/segscan_cpu/randomdata/baseline_random_cpu.cpp:7-18. */
EXPORT void tcuo_seg_scan_flags_f64(const double* x, const int8_t* f, double* out, int64_t n) {
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (f[i]) acc = 0.0;
    acc += x[i];
    out[i] = acc;
  }
}

/* Flag segmented sum, f[i] != 0 => a segment ENDS at i; one output per end
 * flag; elements after the last end flag are dropped.
 * Semantics: run_seg_sum (src/torch/torch_seg_ops.h:85-107: scan, compress
 * at the flags, prepend 0, diff) as exercised by
 * tests/test_segmented_sum.py:39-75.  Returns the number of outputs.       */
EXPORT int64_t tcuo_seg_sum_flags_f64(const double* x, const int8_t* f, double* out, int64_t n) {
  double acc = 0.0;
  int64_t k = 0;
  for (int64_t i = 0; i < n; ++i) {
    acc += x[i];
    if (f[i]) { out[k++] = acc; acc = 0.0; }
  }
  return k;
}

/* indptr segmented sum: out[r] = sum x[indptr[r] : indptr[r+1]].
 * Semantics: run_seg_sum_multi_core (src/torch/torch_seg_ops.h:333-426),
 * KernelSegSumVecRevert (src/kernels/kernel_seg_sum_vec_revert.h:17-25),
 * tests/test_seg_sum_multi_core.py:82-97 (scipy A @ ones).                 */
EXPORT void tcuo_seg_sum_indptr_f64(const double* x, const int64_t* indptr, int64_t nseg, double* out) {
  for (int64_t r = 0; r < nseg; ++r) {
    double acc = 0.0;
    for (int64_t i = indptr[r]; i < indptr[r + 1]; ++i) acc += x[i];
    out[r] = acc;
  }
}
EXPORT void tcuo_seg_sum_indptr_i64(const int64_t* x, const int64_t* indptr, int64_t nseg, int64_t* out) {
  for (int64_t r = 0; r < nseg; ++r) {
    int64_t acc = 0;
    for (int64_t i = indptr[r]; i < indptr[r + 1]; ++i) acc += x[i];
    out[r] = acc;
  }
}

/* complete_rows: per block b (block = n / nblocks elements) start from the
 * exclusive prefix of sums, add the carry to each width-long row and carry
 * the updated row's last element forward.
 * Semantics: ref_complete_rows (tests/test_complete_rows.py:27-55),
 * KernelCompleteRows (src/kernels/kernel_complete_rows.h:99-161).          */
EXPORT void tcuo_complete_rows_f64(const double* x, const double* sums, int64_t n,
                                   int64_t nblocks, int64_t width, double* out) {
  const int64_t bl = n / nblocks;
  double pre = 0.0;
  for (int64_t b = 0; b < nblocks; ++b) {
    double acc = pre;
    pre += sums[b];
    for (int64_t h = 0; h * width < bl; ++h) {
      const int64_t s = b * bl + h * width;
      int64_t e = s + width;
      if (e > (b + 1) * bl) e = (b + 1) * bl;
      for (int64_t i = s; i < e; ++i) out[i] = x[i] + acc;
      acc = out[e - 1];
    }
  }
}
EXPORT void tcuo_complete_rows_i64(const int64_t* x, const int64_t* sums, int64_t n,
                                   int64_t nblocks, int64_t width, int64_t* out) {
  const int64_t bl = n / nblocks;
  int64_t pre = 0;
  for (int64_t b = 0; b < nblocks; ++b) {
    int64_t acc = pre;
    pre += sums[b];
    for (int64_t h = 0; h * width < bl; ++h) {
      const int64_t s = b * bl + h * width;
      int64_t e = s + width;
      if (e > (b + 1) * bl) e = (b + 1) * bl;
      for (int64_t i = s; i < e; ++i) out[i] = x[i] + acc;
      acc = out[e - 1];
    }
  }
}

/* complete_blocks: out[block b] = x[block b] + sum(sums[:b]).
 * Semantics: ref_complete_blocks (tests/test_complete_blocks.py:27-49).    */
EXPORT void tcuo_complete_blocks_f64(const double* x, const double* sums, int64_t n,
                                     int64_t nblocks, double* out) {
  const int64_t bl = n / nblocks;
  double pre = 0.0;
  for (int64_t b = 0; b < nblocks; ++b) {
    for (int64_t i = b * bl; i < (b + 1) * bl; ++i) out[i] = x[i] + pre;
    pre += sums[b];
  }
}
EXPORT void tcuo_complete_blocks_i64(const int64_t* x, const int64_t* sums, int64_t n,
                                     int64_t nblocks, int64_t* out) {
  const int64_t bl = n / nblocks;
  int64_t pre = 0;
  for (int64_t b = 0; b < nblocks; ++b) {
    for (int64_t i = b * bl; i < (b + 1) * bl; ++i) out[i] = x[i] + pre;
    pre += sums[b];
  }
}

/* reduce_tiles: block_len = tile_len * ceil(ceil(n / tile_len) / nblocks);
 * out[i] = sum x[i*block_len : min((i+1)*block_len, n)].
 * Semantics: ref_reduce_tiles (tests/test_reduce_tiles.py), run_reduce_tiles
 * (src/torch/torch_reduce.h:42-75).                                        */
static int64_t reduce_tiles_block_len(int64_t n, int64_t tile_len, int64_t nblocks) {
  const int64_t tiles = (n + tile_len - 1) / tile_len;
  return tile_len * ((tiles + nblocks - 1) / nblocks);
}
EXPORT void tcuo_reduce_tiles_f64(const double* x, int64_t n, int64_t tile_len, int64_t nblocks, double* out) {
  const int64_t bl = reduce_tiles_block_len(n, tile_len, nblocks);
  for (int64_t b = 0; b < nblocks; ++b) {
    double acc = 0.0;
    for (int64_t i = b * bl; i < (b + 1) * bl && i < n; ++i) acc += x[i];
    out[b] = acc;
  }
}
EXPORT void tcuo_reduce_tiles_i64(const int64_t* x, int64_t n, int64_t tile_len, int64_t nblocks, int64_t* out) {
  const int64_t bl = reduce_tiles_block_len(n, tile_len, nblocks);
  for (int64_t b = 0; b < nblocks; ++b) {
    int64_t acc = 0;
    for (int64_t i = b * bl; i < (b + 1) * bl && i < n; ++i) acc += x[i];
    out[b] = acc;
  }
}

/* Stream compaction: stable x[mask != 0], optionally with the matching
 * entries of idx_in (or the positions themselves when idx_in is NULL).
 * Semantics: torch.masked_select as used by tests/test_compress.py:44,
 * tests/test_compress_ind.py:46-47 and tests/test_compress_ind_no_arange.py;
 * run_compress / run_compress_ind / run_compress_ind_no_arange
 * (src/torch/torch_compress.h:41-309).  Returns the number selected.      */
EXPORT int64_t tcuo_compress(const void* x, int64_t elem_bytes, const int8_t* mask, int64_t n,
                             void* out, const void* idx_in, int64_t idx_bytes, void* idx_out) {
  const uint8_t* xs = (const uint8_t*)x;
  uint8_t* os = (uint8_t*)out;
  int64_t k = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (!mask[i]) continue;
    if (os) memcpy(os + k * elem_bytes, xs + i * elem_bytes, (size_t)elem_bytes);
    if (idx_out) {
      if (idx_in) {
        memcpy((uint8_t*)idx_out + k * idx_bytes, (const uint8_t*)idx_in + i * idx_bytes, (size_t)idx_bytes);
      } else if (idx_bytes == 4) {
        ((int32_t*)idx_out)[k] = (int32_t)i;
      } else {
        ((int64_t*)idx_out)[k] = i;
      }
    }
    ++k;
  }
  return k;
}

/* CSR SpMV y = A @ x in FP64.
 * Semantics: run_spmv_v2 (src/torch/torch_spmv.h:112-209) as checked by
 * tests/test_spmv_v2.py:59-98 (scipy B @ vector).                          */
EXPORT void tcuo_spmv_f64(const double* vals, const int64_t* indptr, const int64_t* cols,
                          const double* x, int64_t rows, double* y) {
  for (int64_t r = 0; r < rows; ++r) {
    double acc = 0.0;
    for (int64_t i = indptr[r]; i < indptr[r + 1]; ++i) acc += vals[i] * x[cols[i]];
    y[r] = acc;
  }
}

// tcu_rows.cu -- per-segment sums and CSR SpMV split by elements.
//
// Reference: run_seg_sum_multi_core (src/torch/torch_seg_ops.h:333-426) and
// run_spmv_v2 (src/torch/torch_spmv.h:112-209) sum each CSR row with the
// matrix-unit scan and a per-segment revert walk.  The tensor-core segmented
// sum here (scan_tc_kernel<..., kSegBounds>) is bound by segment starts when
// rows are short (an SpMV row of 16 nonzeros gives ~2000 starts per 32768-
// element tile).  A segment SUM needs no prefix output, so this path splits
// the elements -- not the rows -- evenly and stays bound by HBM for any mix
// of row lengths:
//   nz_rowrange_kernel   one warp per tile of 4096 elements: the row holding
//                        the tile's first element (a 32-way search of the
//                        bounds, four rounds for 2^20 rows);
//   nz_split_kernel      one CTA per tile, 16 consecutive elements per thread
//                        (16-byte loads; SpMV gathers x from L2 and multiplies
//                        in FP32).  Each thread sums its elements in order and
//                        writes every row that starts and ends inside its 16;
//                        a row that crosses threads is finished by the thread
//                        where it ends, with the partial sums of the threads
//                        before it from one segmented scan over the CTA; a row
//                        that crosses tiles leaves its partial sums per tile;
//   nz_fixup_kernel      one thread per tile whose first row started in an
//                        earlier tile adds those partials in tile order.
// Every row is summed in a fixed order, so results do not depend on the
// launch.  Empty rows are zeroed up front.  No kernel waits on another CTA.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

constexpr int kNzThreads = 256;
constexpr int kNzWarps = kNzThreads / 32;
constexpr int kNzTile = kNzThreads * 16;  // the smallest tile (SpMV): workspace sizing
constexpr int kNzStageCap = 4096 + 2;      // row starts staged in shared memory per tile

template <typename T>
__device__ __forceinline__ float elem_f32(const T* p);
template <>
__device__ __forceinline__ float elem_f32<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <>
__device__ __forceinline__ float elem_f32<float>(const float* p) { return __ldg(p); }

template <typename IT>
__device__ __forceinline__ int64_t bound_at(const IT* b, int64_t i, int64_t n) {
  const int64_t v = (int64_t)b[i];
  return v < 0 ? 0 : (v > n ? n : v);
}

// Rows are numbered internally ri = 0 .. nseg + 1: ri = 0 holds the elements
// before bounds[0], ri = 1 .. nseg are the segments, ri = nseg + 1 holds the
// elements from bounds[nseg] on; only 1 .. nseg are written (out[ri - 1]).
// row_start(ri) for ri in [0, nseg + 2].
template <typename IT>
__device__ __forceinline__ int64_t row_start(const IT* b, int64_t ri, int64_t nseg, int64_t n) {
  if (ri <= 0) return 0;
  if (ri > nseg + 1) return n;
  return bound_at(b, ri - 1, n);
}

// Per-tile carries, in the caller's workspace scratch.
template <typename ACC>
struct NzCarry {
  long long head_row;  // internal id of the tile's first row if it began in an earlier tile and ends here, else -1
  long long tail_row;  // internal id of the row that continues past the tile's end, else -1
  ACC head_val;        // this tile's part of head_row
  ACC tail_val;        // this tile's part of tail_row (the whole tile when span)
  int span;            // the tile lies inside one row that continues on both sides
};

// The internal row holding the first element of each tile: the largest ri in
// [0, nseg + 1] with row_start(ri) <= tile start (bounds assumed
// non-decreasing; any bounds keep every access in range).
template <typename IT>
__global__ void __launch_bounds__(256) nz_rowrange_kernel(const IT* __restrict__ bounds, int64_t nseg, int64_t n,
                                                          int64_t tiles, int tile, long long* __restrict__ row_lo) {
  const int lane = threadIdx.x & 31;
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= tiles) return;  // warp-uniform
  const int64_t key = t * tile;
  int64_t lo = 0, hi = nseg + 1;  // answer in [lo, hi]: row_start(lo) <= key
  while (hi - lo > 31) {
    const int64_t step = (hi - lo + 31) / 32;
    const int64_t p = lo + lane * step;
    const bool ok = p <= hi && row_start(bounds, p, nseg, n) <= key;
    const unsigned m = __ballot_sync(0xffffffffu, ok);  // lane 0 always true
    const int L = 31 - __clz(m);
    const int64_t nlo = lo + L * step;
    const int64_t nhi = L == 31 ? hi : (lo + (L + 1) * step - 1 < hi ? lo + (L + 1) * step - 1 : hi);
    lo = nlo;
    hi = nhi;
  }
  const int64_t p = lo + lane;
  const bool ok = p <= hi && row_start(bounds, p, nseg, n) <= key;
  const unsigned m = __ballot_sync(0xffffffffu, ok);
  if (lane == 0) row_lo[t] = lo + (31 - __clz(m));
}

// Segmented inclusive scan over the CTA's threads: a thread with reset = 1
// starts a new segment.  Returns the thread's inclusive value; `sv`/`sr` are
// kNzWarps-entry scratch.
template <typename ACC>
__device__ __forceinline__ ACC block_seg_scan(ACC v, int reset, ACC* sv, int* sr) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int r = reset;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const ACC ov = __shfl_up_sync(0xffffffffu, v, d);
    const int orr = __shfl_up_sync(0xffffffffu, r, d);
    if (lane >= d) {
      if (!r) v += ov;
      r |= orr;
    }
  }
  if (lane == 31) {
    sv[w] = v;
    sr[w] = r;
  }
  __syncthreads();
  if (!r) {  // no reset in this warp up to this lane: add the warps before, back to the last reset
    for (int k = w - 1; k >= 0; --k) {
      v += sv[k];
      if (sr[k]) break;
    }
  }
  __syncthreads();
  return v;
}

// VT: element type; ACC: accumulator / output type; SPMV: element i is
// vals[i] * x[cols[i]] (FP32 product), else vals[i].  Segment r covers
// [bounds[r], bounds[r + 1]) (clamped); the tiles cover all n elements.
template <typename VT, typename ACC, bool SPMV, typename IT, int ITEMS>
__global__ void __launch_bounds__(kNzThreads, 4) nz_split_kernel(const VT* __restrict__ vals,
                                                              const int32_t* __restrict__ cols,
                                                              const VT* __restrict__ x, int64_t x_len,
                                                              const IT* __restrict__ bounds, int64_t nseg, int64_t n,
                                                              const long long* __restrict__ row_lo,
                                                              ACC* __restrict__ out, NzCarry<ACC>* __restrict__ carry,
                                                              WsHeader* ws) {
  constexpr int TILE = kNzThreads * ITEMS;
  __shared__ ACC sv[kNzWarps];
  __shared__ int sr[kNzWarps];
  const int64_t c = blockIdx.x;
  const int64_t t_lo = c * TILE;
  const int64_t t_hi = t_lo + TILE < n ? t_lo + TILE : n;
  const int64_t j0 = t_lo + (int64_t)threadIdx.x * ITEMS;
  const int64_t j_end = j0 + ITEMS < t_hi ? j0 + ITEMS : t_hi;  // this thread's [j0, j_end)
  const bool has_items = j0 < t_hi;
  const int64_t r_tile = row_lo[c];
  const int64_t r_last = c + 1 < gridDim.x ? row_lo[c + 1] : nseg + 1;  // rows of this tile lie in [r_tile, r_last]

  // ---- the thread's elements: SpMV products, or the packed input words ----
  const bool full = j0 + ITEMS <= t_hi;
  const bool vec_v = full && ((reinterpret_cast<uintptr_t>(vals + j0) & 15u) == 0);
  constexpr int WORDS = SPMV ? 1 : ITEMS * (int)sizeof(VT) / 4;
  float p[SPMV ? ITEMS : 1];
  uint32_t raw[WORDS];
  if constexpr (SPMV) {
    // Coalesced: lane L of warp w loads elements w*512 + q*128 + 4L .. +3
    // (q = 0..3), so every load instruction covers whole 128-byte lines; the
    // products then go through padded shared memory (16 bytes of padding per
    // 32 products: conflict-free both ways) into each thread's 16
    // consecutive elements, the order the row logic below needs.
    static_assert(ITEMS == 16, "the SpMV transpose assumes 16 elements per thread");
    __shared__ __align__(16) float s_prod[kNzWarps][512 + 64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t wbase = t_lo + (int64_t)w * 512;
    const bool aligned = ((reinterpret_cast<uintptr_t>(cols) | reinterpret_cast<uintptr_t>(vals)) & 15u) == 0 &&
                         (sizeof(VT) == 4 || (reinterpret_cast<uintptr_t>(vals) & 7u) == 0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t e0 = wbase + q * 128 + 4 * lane;
      int32_t cc[4];
      float va[4];
      if (aligned && e0 + 4 <= t_hi) {
        const int4 c4 = __ldg(reinterpret_cast<const int4*>(cols + e0));
        cc[0] = c4.x; cc[1] = c4.y; cc[2] = c4.z; cc[3] = c4.w;
        if constexpr (sizeof(VT) == 4) {
          const float4 v4 = __ldg(reinterpret_cast<const float4*>(vals + e0));
          va[0] = v4.x; va[1] = v4.y; va[2] = v4.z; va[3] = v4.w;
        } else {
          const uint2 u = __ldg(reinterpret_cast<const uint2*>(vals + e0));
          const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
          const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
          va[0] = f0.x; va[1] = f0.y; va[2] = f1.x; va[3] = f1.y;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const bool in = e0 + i < t_hi;
          cc[i] = in ? __ldg(cols + e0 + i) : 0;
          va[i] = in ? elem_f32<VT>(vals + e0 + i) : 0.f;
        }
      }
      float pr[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        float xv = 0.f;
        if ((unsigned long long)(unsigned)cc[i] < (unsigned long long)x_len) xv = elem_f32<VT>(x + cc[i]);
        else if (e0 + i < t_hi && ws) record_error(ws, TCU_ERR_ARG, 301, (uint32_t)(e0 + i));
        pr[i] = __fmul_rn(va[i], xv);
      }
      const int el = q * 128 + 4 * lane;  // element within the warp's 512
      *reinterpret_cast<float4*>(&s_prod[w][el + (el >> 5) * 4]) = make_float4(pr[0], pr[1], pr[2], pr[3]);
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int el = 16 * lane + 4 * c;
      const float4 f = *reinterpret_cast<const float4*>(&s_prod[w][el + (el >> 5) * 4]);
      p[4 * c] = f.x; p[4 * c + 1] = f.y; p[4 * c + 2] = f.z; p[4 * c + 3] = f.w;
    }
  } else {
    if (vec_v) {
#pragma unroll
      for (int q = 0; q < WORDS / 4; ++q) {
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(vals + j0) + q);
        raw[4 * q] = u.x;
        raw[4 * q + 1] = u.y;
        raw[4 * q + 2] = u.z;
        raw[4 * q + 3] = u.w;
      }
    } else {  // ragged or unaligned: element by element, packed the same way
#pragma unroll
      for (int w = 0; w < WORDS; ++w) raw[w] = 0;
      const uint8_t* vb = reinterpret_cast<const uint8_t*>(vals + j0);
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        if (j0 + i < t_hi) {
          uint32_t bits;
          if constexpr (sizeof(VT) == 1) bits = vb[i];
          else if constexpr (sizeof(VT) == 2) bits = reinterpret_cast<const uint16_t*>(vb)[i];
          else bits = reinterpret_cast<const uint32_t*>(vb)[i];
          raw[i * (int)sizeof(VT) / 4] |= bits << (8 * ((i * (int)sizeof(VT)) & 3));
        }
      }
    }
  }
  // element i of the thread as ACC (constant i after unrolling)
  auto elem = [&](int i) -> ACC {
    if constexpr (SPMV) {
      return p[i];
    } else if constexpr (sizeof(VT) == 1) {
      return (ACC)(int8_t)(raw[i >> 2] >> (8 * (i & 3)));
    } else if constexpr (sizeof(VT) == 2) {
      return (ACC)__half2float(__ushort_as_half((unsigned short)(raw[i >> 1] >> (16 * (i & 1)))));
    } else {
      return (ACC)__uint_as_float(raw[i]);
    }
  };

  // ---- fast path: the next tile's first element is in this tile's first row,
  // so the whole tile lies in one row that goes on past it (block-uniform) ----
  if (c + 1 < gridDim.x && r_tile == r_last) {
    ACC part = (ACC)0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) part += elem(i);  // every thread of this tile is full
    part = warp_sum_any(part);
    if ((threadIdx.x & 31) == 0) sv[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      ACC tot = (ACC)0;
#pragma unroll
      for (int k = 0; k < kNzWarps; ++k) tot += sv[k];
      const bool began_before = row_start(bounds, r_tile, nseg, n) < t_lo;
      carry[c].head_row = -1;
      carry[c].tail_row = r_tile;  // the row goes on into the next tile
      carry[c].tail_val = tot;
      carry[c].span = began_before ? 1 : 0;  // else the row begins here (a tail)
    }
    return;
  }

  // ---- the starts of the tile's rows [r_tile, r_last + 1], relative to the
  // tile start and clamped to [-1, kNzTile + 1], staged in shared memory ----
  __shared__ int s_st[kNzStageCap];
  const int64_t cnt = r_last - r_tile + 2;
  const bool staged = cnt <= kNzStageCap;  // block-uniform; else read from global memory
  if (staged) {
    for (int i = threadIdx.x; i < (int)cnt; i += kNzThreads) {
      const int64_t v = row_start(bounds, r_tile + i, nseg, n) - t_lo;
      s_st[i] = v < -1 ? -1 : (v > TILE ? TILE + 1 : (int)v);
    }
  }
  __syncthreads();
  auto S = [&](int64_t ri) -> int {
    const int64_t k = ri - r_tile;
    if (staged) return k < 0 ? -1 : (k < cnt ? s_st[k] : TILE + 1);
    const int64_t v = row_start(bounds, ri, nseg, n) - t_lo;
    return v < -1 ? -1 : (v > TILE ? TILE + 1 : (int)v);
  };
  const int j0r = (int)(j0 - t_lo), j_endr = (int)(j_end - t_lo);  // tile-relative

  // ---- the thread's first row: largest ri in [r_tile, r_last] with start <= j0 ----
  int64_t row = r_tile;
  if (has_items) {
    int64_t lo = r_tile, hi = r_last;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (S(mid) <= j0r) lo = mid;
      else hi = mid - 1;
    }
    row = lo;
  }
  const int row_begin = S(row);
  const bool tile_head_row = has_items && row_begin < 0;  // the thread's first row began before the tile
  bool head_open = has_items && row_begin < j0r;          // it began before this thread
  const int64_t head_row = row;
  ACC head_val = (ACC)0;
  bool has_head = false;
  ACC acc = (ACC)0;
  int next = has_items ? S(row + 1) : 0;
  if (has_items) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int j = j0r + i;
      if (j < j_endr) {
        while (next <= j) {  // the current row ends before element j (empty rows pass through)
          if (head_open) {
            has_head = true;
            head_val = acc;
            head_open = false;
          } else if (row >= 1 && row <= nseg) {
            out[row - 1] = acc;
          }
          acc = (ACC)0;
          ++row;
          next = S(row + 1);
        }
        acc += elem(i);
      }
    }
  }
  // the last row: ends exactly at j_end, or continues past it
  bool carry_out = false, span = false;
  if (has_items) {
    if (next == j_endr) {
      if (head_open) {
        has_head = true;
        head_val = acc;
        head_open = false;
      } else if (row >= 1 && row <= nseg) {
        out[row - 1] = acc;
      }
    } else {
      carry_out = true;
      span = head_open;  // inside one row from the thread's first element to its last
    }
  }
  // partial sums of rows crossing threads: segmented scan, a segment per starting row
  const ACC scanned = block_seg_scan<ACC>(carry_out ? acc : (ACC)0, carry_out ? (span ? 0 : 1) : 1, sv, sr);
  // carry into this thread's head row = the previous thread's scanned value
  const ACC carry_in = __shfl_up_sync(0xffffffffu, scanned, 1);
  __shared__ ACC s_last[kNzWarps];
  if ((threadIdx.x & 31) == 31) s_last[threadIdx.x >> 5] = scanned;
  __syncthreads();
  const ACC prev = (threadIdx.x & 31) ? carry_in : (threadIdx.x ? s_last[(threadIdx.x >> 5) - 1] : (ACC)0);
  const int t_last = (int)((t_hi - t_lo - 1) / ITEMS);
  if (threadIdx.x == 0) {
    carry[c].head_row = -1;
    carry[c].span = 0;
  }
  __syncthreads();
  if (has_head) {
    const ACC v = (threadIdx.x ? prev : (ACC)0) + head_val;
    if (tile_head_row) {  // began in an earlier tile: the fix-up adds the earlier tiles' parts
      carry[c].head_row = head_row;
      carry[c].head_val = v;
    } else if (head_row >= 1 && head_row <= nseg) {
      out[head_row - 1] = v;
    }
  }
  if ((int)threadIdx.x == t_last) {
    carry[c].tail_row = carry_out ? row : -1;
    carry[c].tail_val = scanned;
    // the whole tile inside one row that began earlier and goes on
    carry[c].span = (carry_out && span && S(row) < 0) ? 1 : 0;
  }
}

// One thread per tile: a tile whose head row began in an earlier tile adds
// the parts of the tiles before it (back to the tile where the row began).
template <typename ACC>
__global__ void __launch_bounds__(256) nz_fixup_kernel(const NzCarry<ACC>* __restrict__ carry, int64_t tiles,
                                                       int64_t nseg, ACC* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= tiles) return;
  const long long r = carry[c].head_row;
  if (r < 1 || r > nseg) return;  // none, or a range outside the segments
  ACC total = carry[c].head_val;
  for (int64_t k = c - 1; k >= 0; --k) {
    if (carry[k].tail_row != r) break;
    total += carry[k].tail_val;
    if (!carry[k].span) break;
  }
  out[r - 1] = total;
}

// Scratch in the workspace's descriptor region: row_lo[tiles + 1], then the
// per-tile carries (64-byte aligned).
static size_t nz_scratch_bytes(int64_t tiles) {
  return (size_t)(tiles + 1) * 8 + 64 + (size_t)tiles * sizeof(NzCarry<double>);
}

template <typename VT, typename ACC, bool SPMV, typename IT>
static tcu_status_t nz_run(const VT* vals, const int32_t* cols, const VT* x, int64_t x_len, const IT* bounds,
                           int64_t nseg, int64_t n, ACC* out, void* ws, size_t ws_bytes, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, (size_t)nseg * sizeof(ACC), st);  // empty rows
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(row sums)");
  if (n == 0) return TCU_OK;
  // 16 elements per thread (64 per thread for sums -- 4x fewer tiles -- was
  // measured no faster at 2^28 and slower for short segments)
  constexpr int ITEMS = 16;
  constexpr int TILE = kNzThreads * ITEMS;
  const int64_t tiles = (n + TILE - 1) / TILE;
  if (tiles > 0x7FFFFFFF) return TCU_ERR_ARG;
  const size_t need = nz_scratch_bytes(tiles);
  if (!ws || ws_capacity(ws_bytes) * 16 < (int64_t)need) return TCU_ERR_WORKSPACE;
  long long* row_lo = reinterpret_cast<long long*>(ws_descs(ws));
  NzCarry<ACC>* carry = reinterpret_cast<NzCarry<ACC>*>(
      (reinterpret_cast<uintptr_t>(row_lo + tiles + 1) + 63) & ~(uintptr_t)63);
  WsHeader* h = static_cast<WsHeader*>(ws);
  nz_rowrange_kernel<IT><<<(unsigned)((tiles * 32 + 255) / 256), 256, 0, st>>>(bounds, nseg, n, tiles, TILE, row_lo);
  nz_split_kernel<VT, ACC, SPMV, IT, ITEMS><<<(unsigned)tiles, kNzThreads, 0, st>>>(vals, cols, x, x_len, bounds, nseg,
                                                                                    n, row_lo, out, carry, h);
  nz_fixup_kernel<ACC><<<(unsigned)((tiles + 255) / 256), 256, 0, st>>>(carry, tiles, nseg, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "nz_split launch");
  // the scratch lives in the look-back descriptor region, which must hold only
  // descriptors or zeros between launches
  e = cudaMemsetAsync(row_lo, 0, need, st);
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(row scratch)");
}

template <typename VT, typename ACC, bool SPMV>
static tcu_status_t nz_dispatch(const VT* vals, const int32_t* cols, const VT* x, int64_t x_len, const void* bounds,
                                tcu_dtype_t bdt, int64_t nseg, int64_t n, ACC* out, void* ws, size_t ws_bytes,
                                cudaStream_t st) {
  if (bdt == TCU_INT64)
    return nz_run<VT, ACC, SPMV, long long>(vals, cols, x, x_len, static_cast<const long long*>(bounds), nseg, n, out,
                                            ws, ws_bytes, st);
  if (bdt == TCU_UINT32)
    return nz_run<VT, ACC, SPMV, unsigned>(vals, cols, x, x_len, static_cast<const unsigned*>(bounds), nseg, n, out, ws,
                                           ws_bytes, st);
  return nz_run<VT, ACC, SPMV, int>(vals, cols, x, x_len, static_cast<const int*>(bounds), nseg, n, out, ws, ws_bytes,
                                    st);
}

static tcu_status_t check_bounds(const void* bounds, tcu_dtype_t bdt) {
  if (bdt != TCU_INT32 && bdt != TCU_UINT32 && bdt != TCU_INT64) return TCU_ERR_DTYPE;
  if (reinterpret_cast<uintptr_t>(bounds) & (bdt == TCU_INT64 ? 7u : 3u)) return TCU_ERR_ALIGN;
  return TCU_OK;
}

}  // namespace tcu

using namespace tcu;

extern "C" {

size_t tcu_rows_workspace_bytes(int64_t n) {
  const int64_t tiles = (n + kNzTile - 1) / kNzTile;
  return 128 + nz_scratch_bytes(tiles) + 16;
}

tcu_status_t tcu_seg_sum_rows(const void* x, tcu_dtype_t x_dtype, int64_t n, const void* bounds,
                              tcu_dtype_t bounds_dtype, int64_t nbounds, void* out, void* ws, size_t ws_bytes,
                              void* stream) {
  if (n < 0 || nbounds < 0) return TCU_ERR_ARG;
  if (nbounds < 2) return TCU_OK;
  if (!bounds || !out || (n > 0 && !x)) return TCU_ERR_ARG;
  tcu_status_t s = check_bounds(bounds, bounds_dtype);
  if (s != TCU_OK) return s;
  const int64_t nseg = nbounds - 1;
  cudaStream_t st = (cudaStream_t)stream;
  switch (x_dtype) {
    case TCU_INT8:
      return nz_dispatch<int8_t, int, false>((const int8_t*)x, nullptr, nullptr, 0, bounds, bounds_dtype, nseg, n,
                                             (int*)out, ws, ws_bytes, st);
    case TCU_FLOAT16:
      return nz_dispatch<__half, float, false>((const __half*)x, nullptr, nullptr, 0, bounds, bounds_dtype, nseg, n,
                                               (float*)out, ws, ws_bytes, st);
    case TCU_FLOAT32:
      return nz_dispatch<float, float, false>((const float*)x, nullptr, nullptr, 0, bounds, bounds_dtype, nseg, n,
                                              (float*)out, ws, ws_bytes, st);
    default:
      return TCU_ERR_DTYPE;
  }
}

tcu_status_t tcu_spmv_rows(const void* vals, tcu_dtype_t dtype, const void* indptr, tcu_dtype_t indptr_dtype,
                           int64_t rows, const int32_t* cols, int64_t nnz, const void* x, int64_t x_len, float* y,
                           void* ws, size_t ws_bytes, void* stream) {
  if (rows < 0 || nnz < 0 || x_len < 0) return TCU_ERR_ARG;
  if (rows == 0) return TCU_OK;
  if (!y || !indptr || (nnz > 0 && (!vals || !cols || !x))) return TCU_ERR_ARG;
  tcu_status_t s = check_bounds(indptr, indptr_dtype);
  if (s != TCU_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == TCU_FLOAT16)
    return nz_dispatch<__half, float, true>((const __half*)vals, cols, (const __half*)x, x_len, indptr, indptr_dtype,
                                            rows, nnz, y, ws, ws_bytes, st);
  if (dtype == TCU_FLOAT32)
    return nz_dispatch<float, float, true>((const float*)vals, cols, (const float*)x, x_len, indptr, indptr_dtype,
                                           rows, nnz, y, ws, ws_bytes, st);
  return TCU_ERR_DTYPE;
}

}  // extern "C"

// tcu_rows.cu -- per-segment sums and CSR SpMV split by elements.
//
// Reference: run_seg_sum_multi_core (src/torch/torch_seg_ops.h:333-426) and
// run_spmv_v2 (src/torch/torch_spmv.h:112-209) sum each CSR row with the
// matrix-unit scan and a per-segment revert walk.  A segment SUM needs no
// prefix output, so this path splits the elements -- not the segments --
// evenly and marks the segment boundaries in per-tile bitmaps, which keeps
// every element's work to a few branch-free instructions for any mix of
// segment lengths:
//   bm_tile_first_kernel  one warp per tile: the first bound at or after the
//                         tile start (a 32-way search);
//   bm_segsum_kernel      one CTA per tile, 64 bytes of input per thread
//                         (32 elements for fp32 and for SpMV: it gathers x[cols] and
//                         multiplies in FP32), loads issued first.  The
//                         tile's bounds set two bitmaps in shared memory, one
//                         bit per element: segment starts and segment ends
//                         (the last element of every non-empty segment).
//                         Each thread takes its elements 32 at a time: their
//                         inclusive prefix P goes to the thread's padded row
//                         of shared memory, and every end e, visited by bit,
//                         gets P[e] - P[s - 1] for the last start s <= e (or
//                         P[e] plus the sum carried in from before).  An end's
//                         output index is the tile's first segment index plus
//                         the end's ordinal (a popcount prefix of the end
//                         bitmap) -- or, in a tile whose bounds hold an empty
//                         segment, a search of the tile's bounds.  Threads
//                         are chained by one segmented scan of their tails;
//                         empty segments get 0 from the tile holding their
//                         bound;
//   bm_fixup_kernel       one thread per tile whose first end closes a segment
//                         that began in an earlier tile: adds the tails of the
//                         tiles before it, in tile order, in FP64.
// Every segment is summed in a fixed order, so results do not depend on the
// launch, and no kernel waits on another CTA.  Bounds must be non-decreasing
// (values are clamped to [0, n]).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

constexpr int kBmThreads = 256;
constexpr int kBmWarps = kBmThreads / 32;
// Elements per thread: 64 bytes of input (fp16 32, int8 64), 32 elements
// for fp32 and SpMV (whose products take a register each).  Fewer bytes per
// thread leave fewer registers per thread and more CTAs per SM, which hide
// the per-tile chain of dependent loads better: 128 bytes per thread at 4
// CTAs per SM measured 0.71 / 0.25 / 0.20 ms at mean segment 4 / 64 / 1024
// (2^28 fp16), 64 bytes at up to 6 CTAs per SM 0.62 / 0.22 / 0.19 ms.  The
// boundary bitmaps give every element one bit: thread t owns words
// [t * IPT / 32, ...).
template <typename VT, bool SPMV>
struct BmCfg {
  static constexpr int IPT = SPMV ? 32 : (64 / (int)sizeof(VT) < 32 ? 32 : 64 / (int)sizeof(VT));
  static constexpr int WPT = IPT / 32;  // bitmap words per thread
  static constexpr int TILE = kBmThreads * IPT;
};
constexpr int kBmMinTile = kBmThreads * 32;  // the smallest tile (workspace sizing)

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

// Per-tile record for the cross-tile fix-up (CT: FP64 for floating sums,
// int32 for int8 sums).
template <typename CT>
struct BmCarry {
  CT tail;           // sum of the tile's elements after its last segment start (the whole tile without one)
  long long head_k;  // output index of the tile's first segment end when that segment began earlier, else -1
  int has_start;     // the tile holds a segment start
  int pad;
};

// tile_first[c] = first index i in [0, nb] with clamp(bounds[i]) >= c * tile,
// for c in [0, tiles); tile_first[tiles] = nb.  One warp per entry.
template <typename IT>
__global__ void __launch_bounds__(256) bm_tile_first_kernel(const IT* __restrict__ bounds, int64_t nb, int64_t n,
                                                            int64_t tiles, int tile, long long* __restrict__ tile_first) {
  const int lane = threadIdx.x & 31;
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (c > tiles) return;  // warp-uniform
  if (c == tiles) {
    if (lane == 0) tile_first[c] = nb;
    return;
  }
  const int64_t key = c * tile;
  int64_t lo = 0, hi = nb;  // the answer lies in [lo, hi]
  while (hi - lo > 32) {
    const int64_t step = (hi - lo + 31) / 32;
    const int64_t p = lo + lane * step;
    const bool below = p < hi && bound_at(bounds, p, n) < key;
    const int cnt = __popc(__ballot_sync(0xffffffffu, below));  // probes below the key: a prefix of the lanes
    const int64_t nlo = cnt == 0 ? lo : lo + (int64_t)(cnt - 1) * step + 1;
    const int64_t nhi = lo + (int64_t)cnt * step < hi ? lo + (int64_t)cnt * step : hi;
    lo = nlo;
    hi = nhi;
  }
  const int64_t p = lo + lane;
  const bool below = p < hi && bound_at(bounds, p, n) < key;
  const int cnt = __popc(__ballot_sync(0xffffffffu, below));
  if (lane == 0) tile_first[c] = lo + cnt;
}

// First index in [lo, hi) with clamp(bounds[i]) >= key (hi if none).
template <typename IT>
__device__ __forceinline__ int64_t bm_lower_bound(const IT* bounds, int64_t lo, int64_t hi, int64_t key, int64_t n) {
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (bound_at(bounds, mid, n) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// VT: element type; ACC: per-tile accumulator and output type (FP32, or
// int32 for int8); CT: cross-tile carry type; SPMV: element i is
// vals[i] * x[cols[i]] (FP32 product), else vals[i].
template <typename VT, typename ACC, typename CT, bool SPMV, typename IT>
__global__ void __launch_bounds__(kBmThreads, SPMV ? 3 : (sizeof(VT) == 4 ? 4 : 6)) bm_segsum_kernel(const VT* __restrict__ vals,
                                                                  const int32_t* __restrict__ cols,
                                                                  const VT* __restrict__ x, int64_t x_len,
                                                                  const IT* __restrict__ bounds, int64_t nb,
                                                                  int64_t n, const long long* __restrict__ tile_first,
                                                                  ACC* __restrict__ out, BmCarry<CT>* __restrict__ carry,
                                                                  WsHeader* ws) {
  using C = BmCfg<VT, SPMV>;
  constexpr int IPT = C::IPT, WPT = C::WPT, TILE = C::TILE;
  __shared__ uint32_t sS[kBmThreads * WPT];  // segment-start bits
  __shared__ uint32_t sE[kBmThreads * WPT];  // segment-end bits (the last element of every non-empty segment)
  __shared__ ACC swv[kBmWarps];
  __shared__ int swf[kBmWarps], swc[kBmWarps];
  __shared__ __align__(16) ACC sP[kBmThreads * 32];  // per-thread word prefixes (row of 32, chunks swizzled)
  __shared__ unsigned long long s_kfirst;  // output index of the tile's first end
  __shared__ int s_empty;                  // the tile's bounds hold an empty segment
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t c = blockIdx.x;
  const int64_t t0 = c * TILE;
  const int64_t t1 = t0 + TILE < n ? t0 + TILE : n;
  const int64_t j0 = t0 + (int64_t)t * IPT;
  const int nvalid = j0 >= t1 ? 0 : (j0 + IPT <= t1 ? IPT : (int)(t1 - j0));

  // ---- the thread's elements: loads issued before the bounds work ----
  constexpr int WORDS = SPMV ? 1 : IPT * (int)sizeof(VT) / 4;
  uint32_t raw[WORDS];
  int32_t cc[SPMV ? IPT : 1];
  float pv[SPMV ? IPT : 1];
  const bool vec = nvalid == IPT && ((reinterpret_cast<uintptr_t>(vals) & 15u) == 0) &&
                   (!SPMV || (reinterpret_cast<uintptr_t>(cols) & 15u) == 0);
  if constexpr (SPMV) {
    if (vec) {
#pragma unroll
      for (int q = 0; q < IPT / 4; ++q) {
        const int4 c4 = __ldg(reinterpret_cast<const int4*>(cols + j0) + q);
        cc[4 * q] = c4.x; cc[4 * q + 1] = c4.y; cc[4 * q + 2] = c4.z; cc[4 * q + 3] = c4.w;
      }
      if constexpr (sizeof(VT) == 4) {
#pragma unroll
        for (int q = 0; q < IPT / 4; ++q) {
          const float4 v4 = __ldg(reinterpret_cast<const float4*>(vals + j0) + q);
          pv[4 * q] = v4.x; pv[4 * q + 1] = v4.y; pv[4 * q + 2] = v4.z; pv[4 * q + 3] = v4.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < IPT / 8; ++q) {
          const uint4 u = __ldg(reinterpret_cast<const uint4*>(vals + j0) + q);
          const uint32_t uu[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&uu[h]));
            pv[8 * q + 2 * h] = f.x;
            pv[8 * q + 2 * h + 1] = f.y;
          }
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const bool in = i < nvalid;
        cc[i] = in ? __ldg(cols + j0 + i) : 0;
        pv[i] = in ? elem_f32<VT>(vals + j0 + i) : 0.f;
      }
    }
  } else {
    if (vec) {
#pragma unroll
      for (int q = 0; q < WORDS / 4; ++q) {
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(vals + j0) + q);
        raw[4 * q] = u.x; raw[4 * q + 1] = u.y; raw[4 * q + 2] = u.z; raw[4 * q + 3] = u.w;
      }
    } else {  // ragged or unaligned: element by element, packed the same way (zeros past the end)
#pragma unroll
      for (int q = 0; q < WORDS; ++q) raw[q] = 0;
      const uint8_t* vb = reinterpret_cast<const uint8_t*>(vals + j0);
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        if (i < nvalid) {
          uint32_t bits;
          if constexpr (sizeof(VT) == 1) bits = vb[i];
          else if constexpr (sizeof(VT) == 2) bits = reinterpret_cast<const uint16_t*>(vb)[i];
          else bits = reinterpret_cast<const uint32_t*>(vb)[i];
          raw[i * (int)sizeof(VT) / 4] |= bits << (8 * ((i * (int)sizeof(VT)) & 3));
        }
      }
    }
  }

  // ---- SpMV: gather x[cols] (FP32 products), issued before the bounds
  // work so their L2 latency overlaps the chain first bound index ->
  // bounds -> bitmaps ----
  if constexpr (SPMV) {
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      float xv = 0.f;
      if ((unsigned long long)(unsigned)cc[i] < (unsigned long long)x_len) xv = elem_f32<VT>(x + cc[i]);
      else if (i < nvalid && ws) record_error(ws, TCU_ERR_ARG, 301, (uint32_t)(j0 + i));
      pv[i] = __fmul_rn(pv[i], xv);
    }
  }
  // ---- boundary bitmaps from the tile's bounds ----
#pragma unroll
  for (int q = 0; q < WPT; ++q) {
    sS[t * WPT + q] = 0u;
    sE[t * WPT + q] = 0u;
  }
  if (t == 0) {
    s_kfirst = ~0ull;
    s_empty = 0;
  }
  __syncthreads();
  const int64_t i_lo = tile_first[c];
  const int64_t i_own = tile_first[c + 1];            // bounds [i_lo, i_own) lie in [t0, t1) (the last tile: [t0, n])
  const int64_t i_end = i_own < nb ? i_own + 1 : nb;  // + the first later bound: it may end a segment at t1 - 1
  for (int64_t i = i_lo + t; i < i_end; i += kBmThreads) {
    const int64_t b = bound_at(bounds, i, n);
    const int64_t bp = i >= 1 ? bound_at(bounds, i - 1, n) : -1;
    if (i < i_own) {
      if (b >= t0 && b < t1) atomicOr(&sS[(b - t0) >> 5], 1u << ((b - t0) & 31));
      if (i >= 1 && b == bp) {  // an empty segment
        out[i - 1] = ACC(0);
        s_empty = 1;
      }
    }
    if (i >= 1 && b > bp && b - 1 >= t0 && b - 1 < t1) {  // segment i - 1 ends at b - 1, in this tile
      const int64_t e = b - 1 - t0;
      atomicOr(&sE[e >> 5], 1u << (e & 31));
      atomicMin(&s_kfirst, (unsigned long long)(i - 1));
    }
  }
  __syncthreads();
  uint32_t Sw[WPT], Ew[WPT];
  int ec = 0;
#pragma unroll
  for (int q = 0; q < WPT; ++q) {
    Sw[q] = sS[t * WPT + q];
    Ew[q] = sE[t * WPT + q];
    ec += __popc(Ew[q]);
  }
  // ends before this thread's words: block exclusive scan of the popcounts
  int ecs = ec;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, ecs, d);
    if (lane >= d) ecs += o;
  }
  if (lane == 31) swc[w] = ecs;
  const int64_t kfirst = (int64_t)s_kfirst;  // read before the barrier below
  const bool direct = s_empty == 0;          // no empty segment: the ends' outputs are consecutive
  __syncthreads();
  int wpre = 0;
#pragma unroll
  for (int k = 0; k < kBmWarps; ++k) wpre += k < w ? swc[k] : 0;
  int ord = wpre + ecs - ec;

  auto elem = [&](int i) -> ACC {
    if constexpr (SPMV) {
      return pv[i];
    } else if constexpr (sizeof(VT) == 1) {
      return (ACC)(int8_t)(raw[i >> 2] >> (8 * (i & 3)));
    } else if constexpr (sizeof(VT) == 2) {
      return (ACC)__half2float(__ushort_as_half((unsigned short)(raw[i >> 1] >> (16 * (i & 1)))));
    } else {
      return (ACC)__uint_as_float(raw[i]);
    }
  };
  // output index of the end with ordinal o at tile element e
  auto out_index = [&](int o, int e) -> int64_t {
    if (direct) return kfirst + o;
    return bm_lower_bound(bounds, i_lo, i_end, t0 + e + 1, n) - 1;
  };

  // ---- the thread's segmented sums, a word (32 elements) at a time: the
  // word's inclusive prefix P goes to the thread's row of shared memory
  // (32 entries; 16-byte chunk c of row t at c ^ (t & 7), so the 16-byte
  // stores of 8 lanes hit distinct banks without padding the rows -- 32 KB
  // per CTA instead of 36 KB, one more CTA per SM), then every end e takes
  // P[e] - P[s - 1] for the last
  // start s <= e in the word, or P[e] plus the sum carried in from before
  // the word.  No per-element branch: the ends are visited by bit. ----
  ACC* myP = sP + t * 32;
  const int sx = t & 7;
  auto pat = [&](int i) -> ACC { return myP[(((i >> 2) ^ sx) << 2) | (i & 3)]; };
  ACC running = ACC(0);  // sum since the thread's last start (everything so far without one)
  bool open = true;      // no start seen yet in this thread
  int open_ord = -1, open_e = 0;
  ACC open_val = ACC(0);
#pragma unroll
  for (int q = 0; q < WPT; ++q) {
    const uint32_t sw = Sw[q];
    uint32_t em = Ew[q];
    const bool need = (sw | em) != 0u;
    ACC pfx = ACC(0);
#pragma unroll
    for (int i4 = 0; i4 < 8; ++i4) {
      const ACC a0 = pfx + elem(q * 32 + 4 * i4);
      const ACC a1 = a0 + elem(q * 32 + 4 * i4 + 1);
      const ACC a2 = a1 + elem(q * 32 + 4 * i4 + 2);
      const ACC a3 = a2 + elem(q * 32 + 4 * i4 + 3);
      if (need) {
        if constexpr (sizeof(ACC) == 4) {
          uint4 u;
          u.x = *reinterpret_cast<const uint32_t*>(&a0);
          u.y = *reinterpret_cast<const uint32_t*>(&a1);
          u.z = *reinterpret_cast<const uint32_t*>(&a2);
          u.w = *reinterpret_cast<const uint32_t*>(&a3);
          *reinterpret_cast<uint4*>(myP + 4 * (i4 ^ sx)) = u;
        }
      }
      pfx = a3;
    }
    while (em) {
      const int i = __ffs(em) - 1;
      em &= em - 1u;
      const uint32_t sb = sw & (0xFFFFFFFFu >> (31 - i));  // starts at or before i
      const ACC pe = pat(i);
      const int e = t * IPT + q * 32 + i;
      if (sb) {
        const int ls = 31 - __clz(sb);
        out[out_index(ord, e)] = pe - (ls ? pat(ls - 1) : ACC(0));
      } else if (!open) {
        out[out_index(ord, e)] = running + pe;
      } else {  // the segment began before this thread: finished after the carry scan
        open_ord = ord;
        open_e = e;
        open_val = running + pe;
      }
      ++ord;
    }
    if (sw) {
      const int ls = 31 - __clz(sw);
      running = pfx - (ls ? pat(ls - 1) : ACC(0));
      open = false;
    } else {
      running += pfx;
    }
  }
  const ACC acc = running;
  // ---- carries between threads: segmented scan of the threads' tails ----
  ACC v = acc;  // the sum after this thread's last start (all of it without one)
  int f = 0;
#pragma unroll
  for (int q = 0; q < WPT; ++q) f |= Sw[q] != 0u;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const ACC ov = __shfl_up_sync(0xffffffffu, v, d);
    const int of = __shfl_up_sync(0xffffffffu, f, d);
    if (lane >= d) {
      if (!f) v += ov;
      f |= of;
    }
  }
  if (lane == 31) {
    swv[w] = v;
    swf[w] = f;
  }
  __syncthreads();
  ACC pv_w = ACC(0);  // the warps before this one, back to the last start
  int pf_w = 0;
  for (int k = w - 1; k >= 0; --k) {
    pv_w += swv[k];
    if (swf[k]) {
      pf_w = 1;
      break;
    }
  }
  const ACC vi = f ? v : pv_w + v;  // inclusive over the tile's threads
  const int fi = f | pf_w;
  ACC ve = __shfl_up_sync(0xffffffffu, vi, 1);
  int fe = __shfl_up_sync(0xffffffffu, fi, 1);
  if (lane == 0) {
    ve = pv_w;
    fe = pf_w;
  }
  if (t == kBmThreads - 1) {
    carry[c].tail = (CT)vi;
    carry[c].has_start = fi;
  }
  long long head_k = -1;
  if (open_ord >= 0) {
    const int64_t k = out_index(open_ord, open_e);
    out[k] = open_val + ve;
    if (!fe) head_k = k;  // no start before it in the tile: the tile's first end, finished by the fix-up
  }
  // the tile's first end is in the first thread holding an end; exactly one
  // thread writes head_k (the value, or -1)
  if (ord > 0 && ord - ec == 0 && ec > 0) carry[c].head_k = head_k;
  if (t == kBmThreads - 1 && ord == 0) carry[c].head_k = -1;  // no end in the tile
}

// One thread per tile: a tile whose first end closes a segment that began in
// an earlier tile adds the tails of the tiles before it (back to the tile
// holding the segment's start), in tile order.
template <typename ACC, typename CT>
__global__ void __launch_bounds__(256) bm_fixup_kernel(const BmCarry<CT>* __restrict__ carry, int64_t tiles,
                                                       ACC* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= tiles) return;
  const long long k = carry[c].head_k;
  if (k < 0) return;
  CT tot = CT(0);
  for (int64_t q = c - 1; q >= 0; --q) {
    tot += carry[q].tail;
    if (carry[q].has_start) break;
  }
  out[k] = (ACC)((CT)out[k] + tot);
}

// Scratch in the workspace's descriptor region: tile_first[tiles + 1], then
// the per-tile carries (64-byte aligned).
static size_t bm_scratch_bytes(int64_t tiles) {  // tiles of kBmMinTile elements or more
  return (size_t)(tiles + 1) * 8 + 64 + (size_t)tiles * sizeof(BmCarry<double>);
}

template <typename VT, typename ACC, typename CT, bool SPMV, typename IT>
static tcu_status_t bm_run(const VT* vals, const int32_t* cols, const VT* x, int64_t x_len, const IT* bounds,
                           int64_t nb, int64_t n, ACC* out, void* ws, size_t ws_bytes, cudaStream_t st) {
  const int64_t nseg = nb - 1;
  if (n == 0) {  // every segment is empty
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)nseg * sizeof(ACC), st);
    return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(segment sums)");
  }
  constexpr int TILE = BmCfg<VT, SPMV>::TILE;
  const int64_t tiles = (n + TILE - 1) / TILE;
  if (tiles > 0x7FFFFFFF) return TCU_ERR_ARG;
  const size_t need = bm_scratch_bytes(tiles);
  if (!ws || ws_capacity(ws_bytes) * 16 < (int64_t)need) return TCU_ERR_WORKSPACE;
  long long* tile_first = reinterpret_cast<long long*>(ws_descs(ws));
  BmCarry<CT>* carry = reinterpret_cast<BmCarry<CT>*>(
      (reinterpret_cast<uintptr_t>(tile_first + tiles + 1) + 63) & ~(uintptr_t)63);
  WsHeader* h = static_cast<WsHeader*>(ws);
  bm_tile_first_kernel<IT><<<(unsigned)(((tiles + 1) * 32 + 255) / 256), 256, 0, st>>>(bounds, nb, n, tiles, TILE,
                                                                                       tile_first);
  bm_segsum_kernel<VT, ACC, CT, SPMV, IT><<<(unsigned)tiles, kBmThreads, 0, st>>>(vals, cols, x, x_len, bounds, nb, n,
                                                                                  tile_first, out, carry, h);
  bm_fixup_kernel<ACC, CT><<<(unsigned)((tiles + 255) / 256), 256, 0, st>>>(carry, tiles, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "segment sum launch");
  // the scratch lives in the look-back descriptor region, which must hold only
  // descriptors or zeros between launches
  e = cudaMemsetAsync(tile_first, 0, need, st);
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(row scratch)");
}

template <typename VT, typename ACC, typename CT, bool SPMV>
static tcu_status_t bm_dispatch(const VT* vals, const int32_t* cols, const VT* x, int64_t x_len, const void* bounds,
                                tcu_dtype_t bdt, int64_t nb, int64_t n, ACC* out, void* ws, size_t ws_bytes,
                                cudaStream_t st) {
  if (bdt == TCU_INT64)
    return bm_run<VT, ACC, CT, SPMV, long long>(vals, cols, x, x_len, static_cast<const long long*>(bounds), nb, n,
                                                out, ws, ws_bytes, st);
  if (bdt == TCU_UINT32)
    return bm_run<VT, ACC, CT, SPMV, unsigned>(vals, cols, x, x_len, static_cast<const unsigned*>(bounds), nb, n, out,
                                               ws, ws_bytes, st);
  return bm_run<VT, ACC, CT, SPMV, int>(vals, cols, x, x_len, static_cast<const int*>(bounds), nb, n, out, ws,
                                        ws_bytes, st);
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
  const int64_t tiles = (n + kBmMinTile - 1) / kBmMinTile;
  return 128 + bm_scratch_bytes(tiles) + 16;
}

tcu_status_t tcu_seg_sum_rows(const void* x, tcu_dtype_t x_dtype, int64_t n, const void* bounds,
                              tcu_dtype_t bounds_dtype, int64_t nbounds, void* out, void* ws, size_t ws_bytes,
                              void* stream) {
  if (n < 0 || nbounds < 0) return TCU_ERR_ARG;
  if (nbounds < 2) return TCU_OK;
  if (!bounds || !out || (n > 0 && !x)) return TCU_ERR_ARG;
  tcu_status_t s = check_bounds(bounds, bounds_dtype);
  if (s != TCU_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  switch (x_dtype) {
    case TCU_INT8:
      return bm_dispatch<int8_t, int, int, false>((const int8_t*)x, nullptr, nullptr, 0, bounds, bounds_dtype, nbounds,
                                                  n, (int*)out, ws, ws_bytes, st);
    case TCU_FLOAT16:
      return bm_dispatch<__half, float, double, false>((const __half*)x, nullptr, nullptr, 0, bounds, bounds_dtype,
                                                       nbounds, n, (float*)out, ws, ws_bytes, st);
    case TCU_FLOAT32:
      return bm_dispatch<float, float, double, false>((const float*)x, nullptr, nullptr, 0, bounds, bounds_dtype,
                                                      nbounds, n, (float*)out, ws, ws_bytes, st);
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
    return bm_dispatch<__half, float, double, true>((const __half*)vals, cols, (const __half*)x, x_len, indptr,
                                                    indptr_dtype, rows + 1, nnz, y, ws, ws_bytes, st);
  if (dtype == TCU_FLOAT32)
    return bm_dispatch<float, float, double, true>((const float*)vals, cols, (const float*)x, x_len, indptr,
                                                   indptr_dtype, rows + 1, nnz, y, ws, ws_bytes, st);
  return TCU_ERR_DTYPE;
}

}  // extern "C"

// tcu_lookback.cuh -- decoupled look-back across tiles (Merrill & Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016), B200
// variant: one 16-byte descriptor per tile, one warp inspects a 512-tile
// window per round (16 independent loads in flight per lane), and the carry
// chain is FP64 (floating scans) or int64 (integer scans).
#pragma once

#include "tcu_device.cuh"

namespace tcu {

// Descriptor word: value bits | (epoch << 3 | seg << 2 | state).  Written and
// read with single 16-byte accesses so a reader never sees a state without
// its value.
struct alignas(16) TileDesc {
  unsigned long long value;
  uint32_t flag;
  uint32_t pad;
};

__device__ __forceinline__ void desc_store(TileDesc* d, unsigned long long value, uint32_t flag) {
  asm volatile("st.relaxed.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(d), "l"(value),
               "l"((unsigned long long)flag)
               : "memory");
}
__device__ __forceinline__ void desc_load(const TileDesc* d, unsigned long long& value, uint32_t& flag) {
  unsigned long long f;
  asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];" : "=l"(value), "=l"(f) : "l"(d) : "memory");
  flag = (uint32_t)f;
}

template <typename V>
__device__ __forceinline__ unsigned long long v_bits(V v) {
  if constexpr (__is_same(V, double)) return (unsigned long long)__double_as_longlong(v);
  else return (unsigned long long)v;
}
template <typename V>
__device__ __forceinline__ V v_from_bits(unsigned long long b) {
  if constexpr (__is_same(V, double)) return __longlong_as_double((long long)b);
  else return (V)(long long)b;
}

// Run by one full warp.  Publishes the tile's aggregate (agg; agg_seg = the
// tile contains a segment start, so its aggregate is a complete carry) and
// returns the exclusive prefix of tile `tid` (with `start` added before tile
// 0); then publishes the tile's inclusive prefix.  Each lane inspects 16
// predecessors per round (a 512-tile window), so one round normally reaches
// an inclusive prefix.  Waits are bounded; on timeout the abort flag is
// raised and the launch reports TCU_ERR_TIMEOUT.
template <typename V>
__device__ __forceinline__ void publish_aggregate(int64_t tid, V agg, int agg_seg, V start, TileDesc* descs,
                                                  uint32_t epoch) {
  const uint32_t tag = (epoch & 0x1FFFFFFFu) << 3;
  const uint32_t segbit = agg_seg ? LB_SEGSTART : 0u;
  if (tid == 0) desc_store(descs, v_bits<V>(agg_seg ? agg : start + agg), tag | segbit | LB_INC);
  else desc_store(descs + tid, v_bits<V>(agg), tag | segbit | LB_AGG);
}

// publish_agg = false when another warp already published the aggregate
// with publish_aggregate() (tile 0's inclusive prefix included).
template <typename V>
__device__ __forceinline__ V warp_lookback(int64_t tid, V agg, int agg_seg, V start, TileDesc* descs, uint32_t epoch,
                                           const WaitCtx& wc, bool publish_agg = true) {
  const int lane = threadIdx.x & 31;
  const uint32_t tag = (epoch & 0x1FFFFFFFu) << 3;
  const uint32_t segbit = agg_seg ? LB_SEGSTART : 0u;
  if (tid == 0) {
    if (lane == 0 && publish_agg) desc_store(descs, v_bits<V>(agg_seg ? agg : start + agg), tag | segbit | LB_INC);
    return start;
  }
  if (lane == 0 && publish_agg) desc_store(descs + tid, v_bits<V>(agg), tag | segbit | LB_AGG);
  constexpr int K = 16;
  V acc = V(0);
  int64_t base = tid - 1;
  while (true) {
    V val[K];
    unsigned long long vb[K];
    uint32_t fl[K];
    uint32_t stop_d = 0xFFFFFFFFu;
#pragma unroll
    for (int k = 0; k < K; ++k) {  // issue every load first
      const int64_t idx = base - (int64_t)(lane + 32 * k);
      if (idx >= 0) desc_load(descs + idx, vb[k], fl[k]);
      else { vb[k] = 0; fl[k] = tag | LB_INC; }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t d = (uint32_t)(lane + 32 * k);
      const int64_t idx = base - d;
      if (idx < 0) {
        val[k] = (idx == -1) ? start : V(0);
        stop_d = min(stop_d, d);
        continue;
      }
      uint32_t f = fl[k];
      if ((f & ~7u) != tag || (f & 3u) == 0u) {
        const uint64_t t0 = globaltimer();
        uint32_t it = 0;
        while (true) {
          desc_load(descs + idx, vb[k], f);
          if ((f & ~7u) == tag && (f & 3u) != 0u) break;
          if (aborted(wc)) { f = tag | LB_INC; vb[k] = 0; break; }
          if ((++it & 15u) == 0u && globaltimer() - t0 > wc.timeout_ns) {
            raise_abort(wc, 100, (uint32_t)tid);
            f = tag | LB_INC;
            vb[k] = 0;
            break;
          }
        }
      }
      val[k] = v_from_bits<V>(vb[k]);
      if ((f & 3u) == LB_INC || (f & LB_SEGSTART)) stop_d = min(stop_d, d);
    }
    // nearest stop: an inclusive prefix, a tile holding a segment start, or
    // the start of the input
    const uint32_t dmin = __reduce_min_sync(0xffffffffu, stop_d);
    V part = V(0);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if ((uint32_t)(lane + 32 * k) <= dmin) part += val[k];
    acc += warp_sum_any(part);
    if (dmin != 0xFFFFFFFFu) break;
    base -= 32 * K;
  }
  if (lane == 0) desc_store(descs + tid, v_bits<V>(agg_seg ? agg : acc + agg), tag | segbit | LB_INC);
  return acc;
}

// Per-warpgroup scratch for the warpgroup look-back reductions.
struct LbScratch {
  unsigned long long sum[4];
  uint32_t dmin[4];
};

// Warpgroup variant: the tile's aggregate was already published by another
// warp; this publishes the inclusive prefix agg_inc + exclusive prefix.  The
// first warp of the warpgroup looks back, one predecessor per lane per round
// (a 32-tile window), and hands the prefix to the other three warps through
// `sc` at one named barrier.  Tiles finish nearly in order, so the nearest
// inclusive prefix is normally a few tiles back: a 1024-tile window (eight
// loads on every thread) measured 1-11% slower end to end on 2^28-element
// scans, its extra loads and instructions landing on every tile.
template <typename V>
__device__ __forceinline__ V wg_lookback(int64_t tid, V agg_inc, V start, TileDesc* descs, uint32_t epoch,
                                         const WaitCtx& wc, LbScratch* sc, int wg_thread, uint32_t bar_id,
                                         int agg_seg = 0) {
  if (tid == 0) return start;
  if (wg_thread < 32) {
    const int lane = wg_thread;
    const uint32_t tag = (epoch & 0x1FFFFFFFu) << 3;
    V acc = V(0);
    int64_t base = tid - 1;
    while (true) {
      const int64_t idx = base - lane;
      V val = V(0);
      uint32_t stop_d = 0xFFFFFFFFu;
      if (idx < 0) {
        val = (idx == -1) ? start : V(0);
        stop_d = (uint32_t)lane;
      } else {
        unsigned long long vb;
        uint32_t f;
        desc_load(descs + idx, vb, f);
        if ((f & ~7u) != tag || (f & 3u) == 0u) {
          const uint64_t t0 = globaltimer();
          uint32_t it = 0;
          while (true) {
            desc_load(descs + idx, vb, f);
            if ((f & ~7u) == tag && (f & 3u) != 0u) break;
            if (aborted(wc)) { f = tag | LB_INC; vb = 0; break; }
            if ((++it & 15u) == 0u && globaltimer() - t0 > wc.timeout_ns) {
              raise_abort(wc, 100, (uint32_t)tid);
              f = tag | LB_INC;
              vb = 0;
              break;
            }
          }
        }
        val = v_from_bits<V>(vb);
        if ((f & 3u) == LB_INC || (f & LB_SEGSTART)) stop_d = (uint32_t)lane;
      }
      const uint32_t dmin = __reduce_min_sync(0xffffffffu, stop_d);
      acc += warp_sum_any(((uint32_t)lane <= dmin) ? val : V(0));
      if (dmin != 0xFFFFFFFFu) break;
      base -= 32;
    }
    if (lane == 0) {
      desc_store(descs + tid, v_bits<V>(agg_seg ? agg_inc : acc + agg_inc),
                 tag | (agg_seg ? LB_SEGSTART : 0u) | LB_INC);
      sc->sum[0] = v_bits<V>(acc);
    }
  }
  named_bar_sync(bar_id, 128);
  const V pre = v_from_bits<V>(sc->sum[0]);
  named_bar_sync(bar_id, 128);  // scratch reused by the next tile
  return pre;
}

}  // namespace tcu

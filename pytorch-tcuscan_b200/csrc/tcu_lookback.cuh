// tcu_lookback.cuh -- decoupled look-back across tiles (Merrill & Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016), B200
// variant: one 16-byte descriptor per tile, a 128-thread warpgroup inspects a
// 512-tile window per round, and the carry chain is FP64 (floating scans) or
// int64 (integer scans).
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

// Per-warpgroup scratch for the look-back reductions (in shared memory).
struct LbScratch {
  double sum_f[4];
  long long sum_i[4];
  uint32_t dmin[4];
};

template <typename V>
__device__ __forceinline__ V wg_sum(V v, LbScratch* sc, int q, int lane, uint32_t bar_id) {
  v = warp_sum_any(v);
  if (lane == 0) {
    if constexpr (__is_same(V, double)) sc->sum_f[q] = v; else sc->sum_i[q] = v;
  }
  named_bar_sync(bar_id, 128);
  V t;
  if constexpr (__is_same(V, double)) t = (sc->sum_f[0] + sc->sum_f[1]) + (sc->sum_f[2] + sc->sum_f[3]);
  else t = (sc->sum_i[0] + sc->sum_i[1]) + (sc->sum_i[2] + sc->sum_i[3]);
  named_bar_sync(bar_id, 128);
  return t;
}

// Run by all 128 threads of one epilogue warpgroup.  Publishes the tile's
// aggregate (agg, agg_seg = the tile contains a segment start) and returns
// the exclusive prefix of tile `tid` (with `start` added before tile 0), then
// publishes the tile's inclusive prefix.  Waits are bounded; on timeout the
// abort flag is raised and the result is meaningless (the launch reports
// TCU_ERR_TIMEOUT).
template <typename V>
__device__ __forceinline__ V tile_lookback(int64_t tid, V agg, int agg_seg, V start, TileDesc* descs, uint32_t epoch,
                                           const WaitCtx& wc, LbScratch* sc, int wg_thread, uint32_t bar_id) {
  const int lane = wg_thread & 31, q = wg_thread >> 5;
  const uint32_t tag = (epoch & 0x1FFFFFFFu) << 3;
  const uint32_t segbit = agg_seg ? LB_SEGSTART : 0u;
  if (tid == 0) {
    if (wg_thread == 0) desc_store(descs, v_bits<V>(agg_seg ? agg : start + agg), tag | segbit | LB_INC);
    return start;
  }
  if (wg_thread == 0) desc_store(descs + tid, v_bits<V>(agg), tag | segbit | LB_AGG);
  V acc = V(0);
  int64_t base = tid - 1;
  while (true) {
    V val[4];
    uint32_t stop_d = 0xFFFFFFFFu;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t d = (uint32_t)(wg_thread + 128 * k);
      const int64_t idx = base - d;
      if (idx < 0) {
        val[k] = (idx == -1) ? start : V(0);
        stop_d = min(stop_d, d);
        continue;
      }
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
      val[k] = v_from_bits<V>(vb);
      if ((f & 3u) == LB_INC || (f & LB_SEGSTART)) stop_d = min(stop_d, d);
    }
    // nearest stop (an inclusive prefix, a tile holding a segment start, or
    // the start of the input) over the warpgroup
    uint32_t m = __reduce_min_sync(0xffffffffu, stop_d);
    if (lane == 0) sc->dmin[q] = m;
    named_bar_sync(bar_id, 128);
    const uint32_t dmin = min(min(sc->dmin[0], sc->dmin[1]), min(sc->dmin[2], sc->dmin[3]));
    V part = V(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t d = (uint32_t)(wg_thread + 128 * k);
      if (d <= dmin) part += val[k];
    }
    acc += wg_sum<V>(part, sc, q, lane, bar_id);
    if (dmin != 0xFFFFFFFFu) break;
    base -= 512;
  }
  if (wg_thread == 0) desc_store(descs + tid, v_bits<V>(agg_seg ? agg : acc + agg), tag | segbit | LB_INC);
  return acc;
}

}  // namespace tcu

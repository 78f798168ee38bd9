// tcu_serve.cu -- device side of the serving loop's batching.
//
// The serving loop (tcuscan_b200/serve.py) answers many independent scan,
// seg_sum and compress requests with one launch per batch: the requests of a
// batch are packed back to back into one device buffer and scanned as the
// segments of one segmented launch (tcu_seg_bounds, tcu_compress_segments).
// tcu_pack is that packing step: one launch gathers every request's elements
// (and, for seg_sum requests, rebases every request's row pointers by the
// request's offset in the packed buffer), with coalesced 16-byte stores and
// zero padding between requests.  The reference has no serving layer; its
// per-request entry points are the run_* calls of src/torch/*.h.
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

template <int SB, int DB>
__device__ __forceinline__ void pack_load(const tcu_pack_item_t& it, int64_t local, int64_t add, uint8_t* out) {
  if constexpr (SB == 4 && DB == 8) {
    const long long v = (long long)static_cast<const int32_t*>(it.src)[local] + add;
    *reinterpret_cast<long long*>(out) = v;
  } else if constexpr (SB == 8) {
    *reinterpret_cast<long long*>(out) = static_cast<const long long*>(it.src)[local] + add;
  } else if constexpr (SB == 4) {
    *reinterpret_cast<int32_t*>(out) = (int32_t)(static_cast<const int32_t*>(it.src)[local] + (int32_t)add);
  } else if constexpr (SB == 2) {
    *reinterpret_cast<uint16_t*>(out) = static_cast<const uint16_t*>(it.src)[local];
  } else {
    *out = static_cast<const uint8_t*>(it.src)[local];
  }
}

// Index of the last item whose dst is <= d (items sorted by dst), within [lo, hi].
__device__ __forceinline__ int64_t pack_find(const tcu_pack_item_t* items, int64_t lo, int64_t hi, int64_t d) {
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (items[mid].dst <= d) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Same, searching forward from `from` (galloping: O(log distance) loads, one
// or two when d lies in the same or the next item).
__device__ __forceinline__ int64_t pack_gallop(const tcu_pack_item_t* items, int64_t nitems, int64_t from, int64_t d) {
  int64_t lo = from, step = 1;
  while (lo + step < nitems && items[lo + step].dst <= d) {
    lo += step;
    step <<= 1;
  }
  const int64_t hi = (lo + step < nitems ? lo + step : nitems) - 1;
  return pack_find(items, lo, hi, d);
}

// Each CTA copies one contiguous range of the destination, chunk by chunk,
// walking the (sorted) items forward; a chunk's first and last items are
// found by thread 0 and each thread searches only between them.
template <int SB, int DB>
__global__ void __launch_bounds__(256) pack_kernel(const tcu_pack_item_t* __restrict__ items, int64_t nitems,
                                                   uint8_t* __restrict__ dst, int64_t total, int64_t per_cta) {
  constexpr int VEC = 16 / DB;              // destination elements per 16-byte store
  constexpr int64_t CH = 256 * 4 * VEC;     // elements per chunk
  __shared__ int64_t s_range[2];
  const int64_t r0 = (int64_t)blockIdx.x * per_cta;
  const int64_t r1 = r0 + per_cta < total ? r0 + per_cta : total;
  int64_t cursor = 0;  // thread 0: first item of the current chunk
  if (threadIdx.x == 0 && r0 < r1) cursor = pack_find(items, 0, nitems - 1, r0);
  for (int64_t c0 = r0; c0 < r1; c0 += CH) {
    const int64_t c1 = c0 + CH < r1 ? c0 + CH : r1;
    if (threadIdx.x == 0) {
      cursor = pack_gallop(items, nitems, cursor, c0);
      s_range[0] = cursor;
      s_range[1] = pack_gallop(items, nitems, cursor, c1 - 1);
    }
    __syncthreads();
    const int64_t lo = s_range[0], hi = s_range[1];
    if (lo == hi && SB == DB) {
      // the whole chunk lies in one item: one item read, then all of this
      // thread's 16-byte loads in flight before its stores
      const tcu_pack_item_t it = items[lo];
      const int64_t a = c0 - it.dst;
      const uintptr_t sa = reinterpret_cast<uintptr_t>(it.src) + (uintptr_t)(a * SB);
      if (a >= 0 && c1 - it.dst <= it.n && (sa & 15u) == 0 && it.add == 0 && ((c1 - c0) % VEC) == 0) {
        const uint4* src = reinterpret_cast<const uint4*>(sa);
        uint4* out = reinterpret_cast<uint4*>(dst + c0 * DB);
        const int nv = (int)((c1 - c0) / VEC);
        uint4 r[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int vi = k * 256 + threadIdx.x;
          if (vi < nv) r[k] = __ldg(src + vi);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int vi = k * 256 + threadIdx.x;
          if (vi < nv) out[vi] = r[k];
        }
        __syncthreads();  // s_range is rewritten for the next chunk
        continue;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t d0 = c0 + ((int64_t)k * 256 + threadIdx.x) * VEC;
      if (d0 >= c1) break;
      int64_t r = lo < hi ? pack_find(items, lo, hi, d0) : lo;
      tcu_pack_item_t it = items[r];
      const int64_t local0 = d0 - it.dst;
      const bool whole = d0 + VEC <= c1 && local0 >= 0 && local0 + VEC <= it.n;
      const uintptr_t sa = reinterpret_cast<uintptr_t>(it.src) + (uintptr_t)(local0 * SB);
      if (whole && SB == DB && (sa & 15u) == 0 && it.add == 0) {
        *reinterpret_cast<uint4*>(dst + d0 * DB) = __ldg(reinterpret_cast<const uint4*>(sa));
        continue;
      }
      alignas(16) uint8_t buf[16];
#pragma unroll
      for (int e = 0; e < VEC; ++e) {
        const int64_t d = d0 + e;
        uint8_t* o = buf + e * DB;
#pragma unroll
        for (int b = 0; b < DB; ++b) o[b] = 0;
        if (d >= c1) continue;
        while (r + 1 < nitems && d >= it.dst + it.len) it = items[++r];
        const int64_t local = d - it.dst;
        if (local >= 0 && local < it.n) pack_load<SB, DB>(it, local, it.add, o);
      }
      if (d0 + VEC <= c1) {
        *reinterpret_cast<uint4*>(dst + d0 * DB) = *reinterpret_cast<const uint4*>(buf);
      } else {
        for (int e = 0; e < VEC && d0 + e < c1; ++e)
          for (int b = 0; b < DB; ++b) dst[(d0 + e) * DB + b] = buf[e * DB + b];
      }
    }
    __syncthreads();  // s_range is rewritten for the next chunk
  }
}

template <int SB, int DB>
static tcu_status_t launch_pack(const tcu_pack_item_t* items, int64_t nitems, void* dst, int64_t total,
                                cudaStream_t st) {
  constexpr int64_t CH = 256 * 4 * (16 / DB);
  const int64_t chunks = (total + CH - 1) / CH;
  const int64_t cap = (int64_t)sm_count() * 8;
  const int64_t grid = chunks < cap ? chunks : cap;
  const int64_t per_cta = (chunks + grid - 1) / grid * CH;  // whole chunks: 16-byte aligned ranges
  pack_kernel<SB, DB><<<(int)grid, 256, 0, st>>>(items, nitems, static_cast<uint8_t*>(dst), total, per_cta);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "pack_kernel launch");
}

}  // namespace tcu

using namespace tcu;

extern "C" {

tcu_status_t tcu_pack(const tcu_pack_item_t* items, int64_t nitems, int src_bytes, int dst_bytes, void* dst,
                      int64_t total, void* stream) {
  if (nitems < 0 || total < 0) return TCU_ERR_ARG;
  if (total == 0) return TCU_OK;
  if (nitems == 0 || !items || !dst) return TCU_ERR_ARG;
  if (!aligned16(dst) || (reinterpret_cast<uintptr_t>(items) & 7u)) return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  if (src_bytes == dst_bytes) {
    switch (src_bytes) {
      case 1: return launch_pack<1, 1>(items, nitems, dst, total, st);
      case 2: return launch_pack<2, 2>(items, nitems, dst, total, st);
      case 4: return launch_pack<4, 4>(items, nitems, dst, total, st);
      case 8: return launch_pack<8, 8>(items, nitems, dst, total, st);
      default: return TCU_ERR_DTYPE;
    }
  }
  if (src_bytes == 4 && dst_bytes == 8) return launch_pack<4, 8>(items, nitems, dst, total, st);
  return TCU_ERR_DTYPE;
}

}  // extern "C"

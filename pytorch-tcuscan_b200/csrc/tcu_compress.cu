// tcu_compress.cu -- single-pass stream compaction on B200.
//
// Reference: run_compress / run_compress_pos / run_compress_ind /
// run_compress_ind_no_arange (src/torch/torch_compress.h:41-309) count the
// mask per block with reduce_tiles, read the total back to the host, then
// gather with the vector GatherMask instruction (kernel_compress.h:97-208).
//
// Here compaction is byte/integer work bound by HBM, so it stays on the SIMT
// cores: each CTA takes 256 x E elements per tile (tile ids from a global
// counter), builds a 32-bit selection mask per thread from 16-byte mask
// loads, publishes the tile's count at once, prefetches its x (and index)
// values, looks back across tiles (int64 decoupled look-back) for its output
// offset, compacts through shared memory and writes the compacted run with
// coalesced stores.  The last tile writes the total count to device memory
// so callers that cannot synchronise (CUDA graphs, the serving loop) never
// need a host round trip.
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

struct CompressParams {
  const void* x;
  const int8_t* mask;
  const void* idx_in;   // optional gathered indices (compress_ind)
  void* out;
  void* idx_out;        // optional
  int64_t n;
  int64_t capacity;     // elements the outputs can hold (compress_pos output_len)
  int64_t num_tiles;
  long long* count_out; // optional: total selected (device)
  WsHeader* ws;
  TileDesc* descs;
  uint64_t timeout_ns;
};

constexpr int kCmpThreads = 256;

template <int EB>
struct ElemT;
template <>
struct ElemT<1> { using T = uint8_t; };
template <>
struct ElemT<2> { using T = uint16_t; };
template <>
struct ElemT<4> { using T = uint32_t; };
template <>
struct ElemT<8> { using T = unsigned long long; };

// Element j of a run of 16-byte vectors held in registers (constant j after
// unrolling, so the extraction is shifts and selects).
template <int EB>
__device__ __forceinline__ typename ElemT<EB>::T vec_elem(const uint4* v, int j) {
  constexpr int PER = 16 / EB;
  const uint4 w = v[j / PER];
  const int b = (j % PER) * EB;  // byte offset inside the vector
  const uint32_t word = (b < 4) ? w.x : (b < 8) ? w.y : (b < 12) ? w.z : w.w;
  if constexpr (EB == 8) {
    const uint32_t hi = (b < 8) ? w.y : w.w;
    return ((unsigned long long)hi << 32) | word;
  } else if constexpr (EB == 4) {
    return word;
  } else {
    return (typename ElemT<EB>::T)(word >> (8 * (b % 4)));
  }
}

// IDX: 0 none, 1 gather idx_in (IB bytes), 2 positions (int32 when IB == 4,
// int64 when IB == 8).
template <int EB, int IDX, int IB, int E>
__global__ void __launch_bounds__(kCmpThreads) compress_kernel(const CompressParams p) {
  using T = typename ElemT<EB>::T;
  using I = typename ElemT<(IB > 0 ? IB : 4)>::T;
  constexpr int TILE = kCmpThreads * E;
  extern __shared__ __align__(16) uint8_t s_dyn[];  // compacted values | indices
  T* s_val = reinterpret_cast<T*>(s_dyn);
  I* s_idx = reinterpret_cast<I*>(s_dyn + TILE * EB);
  __shared__ uint32_t s_tid;
  __shared__ int s_wsum[kCmpThreads / 32];
  __shared__ long long s_prefix;
  __shared__ uint32_t s_epoch;
  __shared__ int s_abort;

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  WaitCtx wc{p.ws, &s_abort, p.timeout_ns};
  if (t == 0) {
    s_abort = 0;
    s_epoch = *(volatile uint32_t*)&p.ws->epoch;
  }
  __syncthreads();
  const uint32_t epoch = s_epoch;

  while (true) {
    if (t == 0) s_tid = atomicAdd(&p.ws->tile_counter, 1u);
    __syncthreads();
    const uint32_t tid = s_tid;
    if ((int64_t)tid >= p.num_tiles || s_abort) break;
    const int64_t e0 = (int64_t)tid * TILE + (int64_t)t * E;

    // ---- mask -> selection bits ----
    uint32_t sel = 0;
    if (e0 + E <= p.n) {
      const uint4* mv = reinterpret_cast<const uint4*>(p.mask + e0);
#pragma unroll
      for (int v = 0; v < E / 16; ++v) {
        const uint4 w = __ldg(mv + v);
        sel |= (sel4(w.x) | (sel4(w.y) << 4) | (sel4(w.z) << 8) | (sel4(w.w) << 12)) << (16 * v);
      }
    } else {
      for (int j = 0; j < E; ++j)
        if (e0 + j < p.n && p.mask[e0 + j] != 0) sel |= 1u << j;
    }
    const int cnt = __popc(sel);

    // ---- prefetch x / indices of selected elements ----
    constexpr int XV = E * EB / 16;
    constexpr int IV = (IDX == 1) ? E * IB / 16 : 1;
    uint4 xv[XV];
    uint4 iv[IV];
    const bool full = e0 + E <= p.n;
    if (sel && full) {
      const uint4* xs = reinterpret_cast<const uint4*>(static_cast<const T*>(p.x) + e0);
#pragma unroll
      for (int v = 0; v < XV; ++v) xv[v] = __ldg(xs + v);
      if constexpr (IDX == 1) {
        const uint4* is = reinterpret_cast<const uint4*>(static_cast<const I*>(p.idx_in) + e0);
#pragma unroll
        for (int v = 0; v < IV; ++v) iv[v] = __ldg(is + v);
      }
    }
    // ---- tile count: exclusive scan over threads ----
    int inc = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += o;
    }
    if (lane == 31) s_wsum[warp] = inc;
    __syncthreads();
    int wpre = 0, total = 0;
#pragma unroll
    for (int k = 0; k < kCmpThreads / 32; ++k) {
      const int ws = s_wsum[k];
      if (k < warp) wpre += ws;
      total += ws;
    }
    const int local = wpre + inc - cnt;  // exclusive offset inside the tile

    // ---- publish the count at once, then look back for the tile offset ----
    if (warp == 0) {
      if (lane == 0) publish_aggregate<long long>((int64_t)tid, (long long)total, 0, 0ll, p.descs, epoch);
      const long long pre = warp_lookback<long long>((int64_t)tid, (long long)total, 0, 0ll, p.descs, epoch, wc, false);
      if (lane == 0) {
        s_prefix = pre;
        if ((int64_t)tid == p.num_tiles - 1 && p.count_out) *p.count_out = pre + total;
      }
    }
    // ---- compact into shared memory ----
    {
      int o = local;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        if (sel & (1u << j)) {
          if (full) {
            s_val[o] = vec_elem<EB>(xv, j);
            if constexpr (IDX == 1) s_idx[o] = (I)vec_elem<(IB > 0 ? IB : 4)>(iv, j);
          } else {  // ragged end of the input: scalar loads
            s_val[o] = static_cast<const T*>(p.x)[e0 + j];
            if constexpr (IDX == 1) s_idx[o] = static_cast<const I*>(p.idx_in)[e0 + j];
          }
          if constexpr (IDX == 2) s_idx[o] = (I)(e0 + j);
          ++o;
        }
      }
    }
    __syncthreads();
    const long long pre = s_prefix;
    // ---- coalesced write of the compacted run ----
    for (int i = t; i < total; i += kCmpThreads) {
      const long long gpos = pre + i;
      if (gpos < p.capacity) {
        static_cast<T*>(p.out)[gpos] = s_val[i];
        if constexpr (IDX != 0) static_cast<I*>(p.idx_out)[gpos] = s_idx[i];
      }
    }
    __syncthreads();  // shared buffers are reused by the next tile
  }

  // ---- teardown: the last CTA resets the counters and bumps the epoch ----
  __syncthreads();
  if (t == 0) {
    __threadfence();
    const uint32_t prev = atomicAdd(&p.ws->done_ctas, 1u);
    if (prev == gridDim.x - 1) {
      p.ws->tile_counter = 0;
      p.ws->done_ctas = 0;
      __threadfence();
      atomicAdd(&p.ws->epoch, 1u);
    }
  }
}

// Count of mask != 0 (the reference's reduce_tiles + .sum() used to size the
// output, src/torch/torch_compress.h:62-64).  *count must be zero on entry.
__global__ void __launch_bounds__(256) mask_count_kernel(const int8_t* mask, int64_t n, unsigned long long* count) {
  unsigned long long c = 0;
  const int64_t nv = n / 16;
  const uint4* mv = reinterpret_cast<const uint4*>(mask);
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const uint4 w = __ldg(mv + v);
    c += __popc(sel4(w.x) | (sel4(w.y) << 4) | (sel4(w.z) << 8) | (sel4(w.w) << 12));
  }
  if (blockIdx.x == 0) {
    for (int64_t i = nv * 16 + threadIdx.x; i < n; i += blockDim.x) c += mask[i] != 0;
  }
  c = warp_sum_any(c);
  __shared__ unsigned long long s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tsum = 0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) tsum += s[k];
    if (tsum) atomicAdd(count, tsum);
  }
}

template <int EB, int IDX, int IB>
static tcu_status_t launch_compress(CompressParams& p, cudaStream_t st) {
  // elements per thread: keep the shared staging (256*E*(EB+IB) bytes) <= 32 KB
  constexpr int E = (EB + IB) <= 4 ? 32 : 16;
  constexpr int TILE = kCmpThreads * E;
  p.num_tiles = (p.n + TILE - 1) / TILE;
  const int smem = TILE * EB + (IDX ? TILE * IB : 0);
  auto kern = compress_kernel<EB, IDX, IB, E>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(compress)");
    attr_set = true;
  }
  int grid = sm_count() * 3;
  if (p.num_tiles < grid) grid = (int)p.num_tiles;
  kern<<<grid, kCmpThreads, smem, st>>>(p);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "compress_kernel launch");
}

}  // namespace tcu

using namespace tcu;

extern "C" {

tcu_status_t tcu_mask_count(const int8_t* mask, int64_t n, void* count_dev, void* stream) {
  if (n < 0 || !count_dev) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(count_dev, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(count)");
  if (n == 0) return TCU_OK;
  if (!mask || !aligned16(mask) || !aligned16(count_dev)) return mask ? TCU_ERR_ALIGN : TCU_ERR_ARG;
  int64_t blocks = (n / 16 + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 4;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  mask_count_kernel<<<(int)blocks, 256, 0, st>>>(mask, n, static_cast<unsigned long long*>(count_dev));
  e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "mask_count_kernel launch");
}

tcu_status_t tcu_compress(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in,
                          int idx_bytes, int idx_mode, void* out, void* idx_out, int64_t capacity, void* count_dev,
                          void* ws, size_t ws_bytes, void* stream) {
  if (n < 0 || capacity < 0) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) {
    if (count_dev) {
      cudaError_t e = cudaMemsetAsync(count_dev, 0, sizeof(long long), st);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(count)");
    }
    return TCU_OK;
  }
  if (!x || !mask || !out) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(mask) || !aligned16(out)) return TCU_ERR_ALIGN;
  if (idx_mode < 0 || idx_mode > 2) return TCU_ERR_ARG;
  if (idx_mode != 0 && (!idx_out || (idx_bytes != 4 && idx_bytes != 8))) return TCU_ERR_ARG;
  if (idx_mode == 1 && (!idx_in || !aligned16(idx_in))) return idx_in ? TCU_ERR_ALIGN : TCU_ERR_ARG;
  CompressParams p{};
  p.x = x;
  p.mask = mask;
  p.idx_in = idx_in;
  p.out = out;
  p.idx_out = idx_out;
  p.n = n;
  p.capacity = capacity;
  p.count_out = static_cast<long long*>(count_dev);
  p.timeout_ns = timeout_ns();
  const int64_t tiles_needed = (n + 4095) / 4096;
  if (!ws || ws_capacity(ws_bytes) < tiles_needed) return TCU_ERR_WORKSPACE;
  p.ws = static_cast<WsHeader*>(ws);
  p.descs = ws_descs(ws);
#define TCU_CMP(EB, IDX, IB) return launch_compress<EB, IDX, IB>(p, st)
  switch (elem_bytes) {
    case 1:
      if (idx_mode == 0) TCU_CMP(1, 0, 0);
      if (idx_mode == 1) { if (idx_bytes == 4) TCU_CMP(1, 1, 4); TCU_CMP(1, 1, 8); }
      if (idx_bytes == 4) TCU_CMP(1, 2, 4);
      TCU_CMP(1, 2, 8);
    case 2:
      if (idx_mode == 0) TCU_CMP(2, 0, 0);
      if (idx_mode == 1) { if (idx_bytes == 4) TCU_CMP(2, 1, 4); TCU_CMP(2, 1, 8); }
      if (idx_bytes == 4) TCU_CMP(2, 2, 4);
      TCU_CMP(2, 2, 8);
    case 4:
      if (idx_mode == 0) TCU_CMP(4, 0, 0);
      if (idx_mode == 1) { if (idx_bytes == 4) TCU_CMP(4, 1, 4); TCU_CMP(4, 1, 8); }
      if (idx_bytes == 4) TCU_CMP(4, 2, 4);
      TCU_CMP(4, 2, 8);
    case 8:
      if (idx_mode == 0) TCU_CMP(8, 0, 0);
      if (idx_mode == 1) { if (idx_bytes == 4) TCU_CMP(8, 1, 4); TCU_CMP(8, 1, 8); }
      if (idx_bytes == 4) TCU_CMP(8, 2, 4);
      TCU_CMP(8, 2, 8);
    default:
      return TCU_ERR_DTYPE;
  }
#undef TCU_CMP
}

}  // extern "C"

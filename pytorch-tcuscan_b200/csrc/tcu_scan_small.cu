// tcu_scan_small.cu -- full scans of small inputs on the SIMT cores.
//
// The tensor-core engine (tcu_scan_tc.cuh) streams large inputs at HBM speed,
// but every tile passes a chain of steps (TMA load, conversion / summing,
// MMA into TMEM, epilogue, look-back, TMA store) that costs several
// microseconds however small the tile, so below a few million elements the
// launch is bound by that chain, not by bytes.  This kernel takes the same
// scan (reference: run_scan_single_core / run_scan_multi_core,
// src/torch/torch_scan.h:47-110, 184-241) in one short chain per CTA:
//   16-byte loads of 32 bytes per thread -> the thread's inclusive scan (FP32,
//   int32 for int8) -> a block scan through warp shuffles -> the tile
//   aggregate published at once and a one-warp decoupled look-back (FP64 /
//   int64 carries, the workspace's epoch-tagged descriptors, bounded waits)
//   -> 16-byte stores of carry + local prefix.
// Tiles are taken in launch order from the workspace counter, so a look-back
// only ever waits on a CTA that has started.  Results equal the tensor-core
// path's up to FP32 rounding inside a tile (exactly, for int8).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

constexpr int kSmThreads = 256;
constexpr int kSmWarps = kSmThreads / 32;

template <typename InT>
struct SmallCfg {
  static constexpr bool IS_INT = sizeof(InT) == 1;
  static constexpr int IPT = 32 / (int)sizeof(InT);  // 32 input bytes per thread
  static constexpr int TILE = kSmThreads * IPT;
};

struct SmallParams {
  const void* x;
  void* z;
  int64_t n;
  int64_t num_tiles;
  double start_f;
  long long start_i;
  const void* start_dev;  // optional device start value (added to the host one)
  int start_dev_kind;     // 0 int32, 1 fp32, 2 int64, 3 fp64
  uint64_t timeout_ns;
  WsHeader* ws;
  TileDesc* descs;
};

template <typename InT>
__global__ void __launch_bounds__(kSmThreads) scan_small_kernel(const SmallParams p) {
  using C = SmallCfg<InT>;
  constexpr bool IS_INT = C::IS_INT;
  constexpr int IPT = C::IPT;
  using A = typename std::conditional<IS_INT, int, float>::type;         // in-tile arithmetic
  using V = typename std::conditional<IS_INT, long long, double>::type;  // carries
  __shared__ uint32_t s_tid, s_epoch;
  __shared__ int s_abort;
  __shared__ A s_warp[kSmWarps];
  __shared__ unsigned long long s_pre;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) {
    s_tid = atomicAdd(&p.ws->tile_counter, 1u);
    s_epoch = *(volatile uint32_t*)&p.ws->epoch;
    s_abort = 0;
  }
  __syncthreads();
  const uint32_t tid = s_tid;
  const uint32_t epoch = s_epoch;
  const int64_t j0 = (int64_t)tid * C::TILE + (int64_t)t * IPT;
  const int nvalid = j0 >= p.n ? 0 : (j0 + IPT <= p.n ? IPT : (int)(p.n - j0));

  // ---- the thread's elements ----
  uint32_t raw[8];
  const InT* xs = static_cast<const InT*>(p.x) + j0;
  if (nvalid == IPT) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(xs));
    const uint4 b = __ldg(reinterpret_cast<const uint4*>(xs) + 1);
    raw[0] = a.x; raw[1] = a.y; raw[2] = a.z; raw[3] = a.w;
    raw[4] = b.x; raw[5] = b.y; raw[6] = b.z; raw[7] = b.w;
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) raw[q] = 0u;
    const uint8_t* vb = reinterpret_cast<const uint8_t*>(xs);
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      if (i < nvalid) {
        uint32_t bits;
        if constexpr (sizeof(InT) == 1) bits = vb[i];
        else if constexpr (sizeof(InT) == 2) bits = reinterpret_cast<const uint16_t*>(vb)[i];
        else bits = reinterpret_cast<const uint32_t*>(vb)[i];
        raw[i * (int)sizeof(InT) / 4] |= bits << (8 * ((i * (int)sizeof(InT)) & 3));
      }
    }
  }
  A v[IPT];
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    if constexpr (sizeof(InT) == 1) v[i] = (A)(int8_t)(raw[i >> 2] >> (8 * (i & 3)));
    else if constexpr (sizeof(InT) == 2)
      v[i] = (A)__half2float(__ushort_as_half((unsigned short)(raw[i >> 1] >> (16 * (i & 1)))));
    else v[i] = (A)__uint_as_float(raw[i]);
  }
#pragma unroll
  for (int i = 1; i < IPT; ++i) v[i] += v[i - 1];

  // ---- block scan of the thread totals ----
  A tot = v[IPT - 1];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const A o = __shfl_up_sync(0xffffffffu, tot, d);
    if (lane >= d) tot += o;
  }
  if (lane == 31) s_warp[w] = tot;
  __syncthreads();
  A wpre = A(0), agg = A(0);
#pragma unroll
  for (int k = 0; k < kSmWarps; ++k) {
    const A s = s_warp[k];
    wpre += k < w ? s : A(0);
    agg += s;
  }
  A texcl = __shfl_up_sync(0xffffffffu, tot, 1);
  if (lane == 0) texcl = A(0);
  texcl += wpre;  // the sum of the tile's elements before this thread's

  // ---- carry from the tiles before: one warp looks back ----
  if (w == 0) {
    V start = IS_INT ? (V)p.start_i : (V)p.start_f;
    if (p.start_dev) {
      switch (p.start_dev_kind) {
        case 0: start += (V)*static_cast<const int*>(p.start_dev); break;
        case 1: start += (V)*static_cast<const float*>(p.start_dev); break;
        case 2: start += (V)*static_cast<const long long*>(p.start_dev); break;
        default: start += (V)*static_cast<const double*>(p.start_dev); break;
      }
    }
    const WaitCtx wc{p.ws, &s_abort, p.timeout_ns};
    const V pre = warp_lookback<V>((int64_t)tid, (V)agg, 0, start, p.descs, epoch, wc, true);
    if (lane == 0) s_pre = v_bits<V>(pre);
  }
  __syncthreads();
  const V pre = v_from_bits<V>(s_pre);

  // ---- outputs: carry + prefix, 16-byte stores ----
  uint32_t o[IPT];
  if constexpr (IS_INT) {
    const uint32_t c = (uint32_t)(long long)pre + (uint32_t)texcl;  // int32 wrap, like the reference
#pragma unroll
    for (int i = 0; i < IPT; ++i) o[i] = c + (uint32_t)v[i];
  } else {
    const double c = pre + (double)texcl;
#pragma unroll
    for (int i = 0; i < IPT; ++i) o[i] = __float_as_uint((float)(c + (double)v[i]));
  }
  uint32_t* zs = static_cast<uint32_t*>(p.z) + j0;
  if (nvalid == IPT) {
#pragma unroll
    for (int q = 0; q < IPT / 4; ++q)
      reinterpret_cast<uint4*>(zs)[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < IPT; ++i)
      if (i < nvalid) zs[i] = o[i];
  }

  // ---- the last CTA resets the tile counter and advances the epoch ----
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

template <typename InT>
static tcu_status_t launch_small(const void* x, int64_t n, void* z, double start_f, long long start_i, void* ws,
                                 size_t ws_bytes, cudaStream_t st, const void* start_dev, int start_dev_kind) {
  using C = SmallCfg<InT>;
  SmallParams p{};
  p.x = x;
  p.z = z;
  p.n = n;
  p.num_tiles = (n + C::TILE - 1) / C::TILE;
  p.start_f = start_f;
  p.start_i = start_i;
  p.start_dev = start_dev;
  p.start_dev_kind = start_dev_kind;
  p.timeout_ns = timeout_ns();
  if (ws == nullptr || ws_capacity(ws_bytes) < p.num_tiles) return TCU_ERR_WORKSPACE;
  if (p.num_tiles > 0x7FFFFFFF) return TCU_ERR_ARG;
  p.ws = static_cast<WsHeader*>(ws);
  p.descs = ws_descs(ws);
  scan_small_kernel<InT><<<(unsigned)p.num_tiles, kSmThreads, 0, st>>>(p);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "scan_small_kernel launch");
}

tcu_status_t scan_small(const void* x, tcu_dtype_t dt, int64_t n, void* z, double start, void* ws, size_t ws_bytes,
                        cudaStream_t st, const void* start_dev, int start_dev_kind) {
  if (!aligned16(x) || !aligned16(z)) return TCU_ERR_ALIGN;
  switch (dt) {
    case TCU_INT8:
      return launch_small<int8_t>(x, n, z, 0.0, (long long)start, ws, ws_bytes, st, start_dev, start_dev_kind);
    case TCU_FLOAT16:
      return launch_small<__half>(x, n, z, start, 0, ws, ws_bytes, st, start_dev, start_dev_kind);
    case TCU_FLOAT32:
      return launch_small<float>(x, n, z, start, 0, ws, ws_bytes, st, start_dev, start_dev_kind);
    default:
      return TCU_ERR_DTYPE;
  }
}

}  // namespace tcu

// tcu_sort.cu -- radix sort, top-k and the top-k pivot estimator on B200.
//
// Reference: run_radix_sort (src/torch/torch_sort.h:30-82, kernels in
// src/radix_sort.cpp:37-175) sorts 16-bit keys with sixteen one-bit stable
// split passes; run_topk_int16 / run_topk_fp16 (src/torch/torch_topk.h:86-211,
// src/kernels/kernel_topk.h:35-140) bisect the value range with repeated
// splits; run_topk_pivot_fp16 (torch_topk.h:35-73,
// src/kernels/kernel_topk_pivot.h:22-160) estimates a lower bound of the k-th
// largest value from sampled 32-element groups.
//
// Here the same results come from byte-digit passes bound by HBM:
//   radix sort   8-bit LSD passes (2 for 16-bit keys).  Each pass: digit
//                counts per chunk of tiles (rs_hist_kernel, one CTA per
//                chunk), one scan of the chunk counts (rs_chunk_scan_kernel),
//                and a scatter pass over the same chunks (rs_scatter_kernel)
//                that ranks each tile's keys stably per digit with warp
//                ballots, sorts the tile by digit in shared memory and writes
//                each digit's run at the chunk's running position, so stores
//                are runs of consecutive addresses.
//   top-k        a radix select: 256-bin histograms of the key's high byte,
//                then of the low byte inside the chosen high byte, fix the
//                k-th largest key t; a count pass, one offset scan and an
//                emit pass then write every element with key > t and the
//                lowest-indexed elements with key == t, in index order.
//                That is the set the reference's bisection returns (its
//                splits are stable, so the ties it keeps are the first ones
//                in input order); the reference emits it band by band.
//   pivot        one CTA per block of tiles, one warp per 32-element group.
// Keys are order-preserving unsigned images of the input bits: signed
// integers flip the sign bit, floats flip all bits of negatives and set the
// sign bit of positives (the reference's encoding, kernel_radix_enc.h:17-28,
// followed by its reversed sign pass, radix_sort.cpp:71-84).
// None of these kernels waits on another CTA.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsEpt = 16;
constexpr int kRsTile = kRsThreads * kRsEpt;  // 4096 keys per tile
constexpr int kRsDigits = 256;

enum KeyCodec { kCodecUnsigned = 0, kCodecSigned = 1, kCodecFloat = 2 };

template <typename K>
__device__ __forceinline__ K sign_bit() {
  return (K)((K)1 << (8 * sizeof(K) - 1));
}

// Order-preserving unsigned image of the input bits, and its inverse.
template <typename K, int CODEC>
__device__ __forceinline__ K key_enc(K b) {
  if constexpr (CODEC == kCodecSigned) return (K)(b ^ sign_bit<K>());
  else if constexpr (CODEC == kCodecFloat) return (b & sign_bit<K>()) ? (K)~b : (K)(b | sign_bit<K>());
  else return b;
}
template <typename K, int CODEC>
__device__ __forceinline__ K key_dec(K k) {
  if constexpr (CODEC == kCodecSigned) return (K)(k ^ sign_bit<K>());
  else if constexpr (CODEC == kCodecFloat) return (k & sign_bit<K>()) ? (K)(k ^ sign_bit<K>()) : (K)~k;
  else return k;
}

// Exclusive scan of one int per thread over a 256-thread block; returns the
// block total through *total.  `sw` holds 8 ints.
__device__ __forceinline__ int block_excl_scan256(int v, int* sw, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) sw[w] = inc;
  __syncthreads();
  int pre = 0, tot = 0;
#pragma unroll
  for (int k = 0; k < kRsWarps; ++k) {
    const int s = sw[k];
    pre += k < w ? s : 0;
    tot += s;
  }
  __syncthreads();
  *total = tot;
  return pre + inc - v;
}

// ---------------------------------------------------------------------------
// Radix sort.  The tiles are split into contiguous chunks, one per CTA, the
// same for the counting and the scatter kernel of a pass, so a CTA carries
// its running per-digit output positions from tile to tile and no per-tile
// offsets are stored.

// Lanes of the warp whose digit equals this lane's: one match instruction
// (eight ballots and masks per key, the earlier form, kept the scatter
// bound by ranking instructions).
__device__ __forceinline__ unsigned digit_peers(int d) { return __match_any_sync(0xffffffffu, d); }

__host__ __device__ inline int64_t chunk_tiles(int64_t num_tiles, int chunks) {
  return (num_tiles + chunks - 1) / chunks;
}

// 256-bin histograms in shared memory: four counter copies per warp
// (lane % 4), so equal digits in one warp spread over four addresses.
constexpr int kHistCopies = kRsWarps * 4;

__device__ __forceinline__ int* hist_slot(int* s_h) {
  return s_h + (((threadIdx.x >> 5) << 2) + (threadIdx.x & 3)) * kRsDigits;
}

// Counts digit(key) >= 0 of keys[lo, hi) into s_h (kHistCopies x 256 ints):
// per round every thread has four 16-byte loads in flight (VEC: keys 16-byte
// aligned; lo a multiple of the vector length).  Called by all threads.
template <typename K, bool VEC, typename DigitF>
__device__ __forceinline__ void smem_hist_range(const K* __restrict__ keys, int64_t lo, int64_t hi, int* s_h,
                                                DigitF digit) {
  constexpr int KPV = 16 / (int)sizeof(K);
  constexpr int VPT = 4;
  constexpr int PER = KPV * VPT;
  int* slot = hist_slot(s_h);
  for (int64_t b = lo; b < hi; b += (int64_t)kRsThreads * PER) {  // block-uniform
    union {
      uint4 u[VPT];
      K k[PER];
    } kv;
#pragma unroll
    for (int v = 0; v < VPT; ++v) {
      const int64_t e = b + ((int64_t)v * kRsThreads + threadIdx.x) * KPV;
      if (VEC && e + KPV <= hi) {
        kv.u[v] = __ldg(reinterpret_cast<const uint4*>(keys + e));
      } else {
#pragma unroll
        for (int i = 0; i < KPV; ++i) kv.k[v * KPV + i] = e + i < hi ? keys[e + i] : (K)0;
      }
    }
#pragma unroll
    for (int v = 0; v < VPT; ++v) {
      const int64_t e = b + ((int64_t)v * kRsThreads + threadIdx.x) * KPV;
#pragma unroll
      for (int i = 0; i < KPV; ++i) {
        const int d = digit(kv.k[v * KPV + i]);
        if (e + i < hi && d >= 0) atomicAdd(slot + d, 1);
      }
    }
  }
}

// Thread d: the total of digit d over the copies (after a barrier).
__device__ __forceinline__ int smem_hist_total(const int* s_h) {
  int c = 0;
#pragma unroll
  for (int k = 0; k < kHistCopies; ++k) c += s_h[k * kRsDigits + threadIdx.x];
  return c;
}

template <typename K, int CODEC, bool FIRST>
struct RsDigit {
  int shift;
  __device__ __forceinline__ int operator()(K k) const {
    if constexpr (FIRST) k = key_enc<K, CODEC>(k);
    return (int)((k >> shift) & 0xFF);
  }
};

// Digit counts of chunk blockIdx.x: sums[c * 256 + digit], and the digit
// totals (atomically; zero on entry).  FIRST: keys are the raw input bits and
// are encoded on the fly.
template <typename K, int CODEC, bool FIRST, bool VEC>
__global__ void __launch_bounds__(kRsThreads) rs_hist_kernel(const K* __restrict__ keys, int64_t n, int shift,
                                                             int64_t num_tiles, int* __restrict__ sums,
                                                             unsigned* __restrict__ totals) {
  __shared__ int s_h[kHistCopies * kRsDigits];
#pragma unroll
  for (int k = 0; k < kHistCopies; ++k) s_h[k * kRsDigits + threadIdx.x] = 0;
  __syncthreads();
  const int64_t tpc = chunk_tiles(num_tiles, gridDim.x);
  const int64_t e_lo = blockIdx.x * tpc * kRsTile;
  int64_t e_hi = e_lo + tpc * kRsTile;
  e_hi = e_hi < n ? e_hi : n;
  smem_hist_range<K, VEC>(keys, e_lo, e_hi, s_h, RsDigit<K, CODEC, FIRST>{shift});
  __syncthreads();
  const int c = smem_hist_total(s_h);
  sums[blockIdx.x * kRsDigits + threadIdx.x] = c;
  if (c) atomicAdd(&totals[threadIdx.x], (unsigned)c);
}

// One CTA per digit d: base[c * 256 + d] = (keys with a smaller digit, from
// the totals) + (keys with digit d in chunks before c).
constexpr int kChunkScanThreads = 256;

__global__ void __launch_bounds__(kChunkScanThreads) rs_chunk_scan_kernel(const int* __restrict__ sums, int chunks,
                                                                         const unsigned* __restrict__ totals,
                                                                         int* __restrict__ base) {
  __shared__ int sw[kRsWarps];
  const int d = blockIdx.x;
  int tot;
  block_excl_scan256(threadIdx.x < d ? (int)totals[threadIdx.x] : 0, sw, &tot);
  const int below = tot;
  // chunks c = threadIdx.x * per .. + per - 1 (at most 4 per thread at 3 chunks per SM)
  const int per = (chunks + kChunkScanThreads - 1) / kChunkScanThreads;
  const int c0 = threadIdx.x * per;
  int v[8];
  int sum = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v[i] = (i < per && c0 + i < chunks) ? sums[(c0 + i) * kRsDigits + d] : 0;
    sum += v[i];
  }
  for (int c = c0 + 8; c < c0 + per && c < chunks; ++c) sum += sums[c * kRsDigits + d];  // more than 2048 chunks
  int run = below + block_excl_scan256(sum, sw, &tot);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (i < per && c0 + i < chunks) {
      base[(c0 + i) * kRsDigits + d] = run;
      run += v[i];
    }
  }
  for (int c = c0 + 8; c < c0 + per && c < chunks; ++c) {
    base[c * kRsDigits + d] = run;
    run += sums[c * kRsDigits + d];
  }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem_dst)), "l"(gsrc), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Copies `bytes` bytes from g to s with 16-byte cp.async chunks spread over
// the block (the last chunk zero-filled past `bytes`).
__device__ __forceinline__ void cp_async_block(void* s, const void* g, int bytes) {
  for (int c = threadIdx.x; c * 16 < bytes; c += kRsThreads) {
    const int sz = bytes - 16 * c < 16 ? bytes - 16 * c : 16;
    cp_async16(static_cast<uint8_t*>(s) + 16 * c, static_cast<const uint8_t*>(g) + 16 * c, sz);
  }
}

template <typename K>
struct ScatterSmem {
  static constexpr int BUF = kRsTile * ((int)sizeof(K) + 4);  // keys then indices of one tile
  static constexpr int WH = 2 * BUF;                           // per-warp digit counts
  static constexpr int START = WH + kRsWarps * kRsDigits * 4;
  static constexpr int DELTA = START + kRsDigits * 4;
  static constexpr int SW = DELTA + kRsDigits * 4;
  static constexpr int BYTES = SW + kRsWarps * 4;
};

// Stable scatter of one digit pass over chunk blockIdx.x.  FIRST: keys are
// the raw input (encoded here) and the indices are the positions; LAST: the
// keys written are decoded back to the input bits.  ASYNC (inputs 16-byte
// aligned): the next tile's keys and indices are copied into the other of
// two shared buffers with cp.async while the current tile is ranked; the
// current buffer then takes the tile sorted by digit.  Dynamic shared memory:
// ScatterSmem<K>::BYTES.
template <typename K, int CODEC, bool FIRST, bool LAST, bool ASYNC>
__global__ void __launch_bounds__(kRsThreads, 3) rs_scatter_kernel(const K* __restrict__ in_keys,
                                                                   const int* __restrict__ in_idx,
                                                                   K* __restrict__ out_keys, int* __restrict__ out_idx,
                                                                   const int* __restrict__ base, int64_t n, int shift,
                                                                   int64_t num_tiles) {
  using L = ScatterSmem<K>;
  extern __shared__ __align__(16) uint8_t sm[];
  int(*s_wh)[kRsDigits] = reinterpret_cast<int(*)[kRsDigits]>(sm + L::WH);  // per-warp counts, then bases
  int* s_start = reinterpret_cast<int*>(sm + L::START);  // first local position of each digit
  int* s_delta = reinterpret_cast<int*>(sm + L::DELTA);  // output position minus local position, per digit
  int* sw = reinterpret_cast<int*>(sm + L::SW);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t tpc = chunk_tiles(num_tiles, gridDim.x);
  int64_t t_hi = (blockIdx.x + 1) * tpc;
  t_hi = t_hi < num_tiles ? t_hi : num_tiles;
  const int64_t t_lo = blockIdx.x * tpc;
  auto tile_valid = [&](int64_t t) { return (int)(n - t * kRsTile < kRsTile ? n - t * kRsTile : kRsTile); };
  auto issue = [&](int64_t t, int b) {
    const int t0 = (int)(t * kRsTile), v = tile_valid(t);
    cp_async_block(sm + b * L::BUF, in_keys + t0, v * (int)sizeof(K));
    if constexpr (!FIRST) cp_async_block(sm + b * L::BUF + kRsTile * (int)sizeof(K), in_idx + t0, v * 4);
  };
  int goff = base[blockIdx.x * kRsDigits + threadIdx.x];  // thread d: output position of digit d's next key
  if (ASYNC && t_lo < t_hi) {
    issue(t_lo, 0);
    cp_async_commit();
  }
  int b = 0;
  for (int64_t t = t_lo; t < t_hi; ++t, b ^= (ASYNC ? 1 : 0)) {
    const int t0 = (int)(t * kRsTile);  // n < 2^31: 32-bit positions
    const int valid = tile_valid(t);
    K* bk = reinterpret_cast<K*>(sm + b * L::BUF);
    int* bi = reinterpret_cast<int*>(sm + b * L::BUF + kRsTile * (int)sizeof(K));
#pragma unroll
    for (int k = 0; k < kRsWarps; ++k) s_wh[k][threadIdx.x] = 0;
    if constexpr (ASYNC) {
      if (t + 1 < t_hi) issue(t + 1, b ^ 1);  // that buffer was released by the last barrier of tile t - 1
      cp_async_commit();
      cp_async_wait1();  // this thread's copies of tile t have landed
    }
    __syncthreads();
    K kr[kRsEpt];
    int ir[kRsEpt], rk[kRsEpt];
    // warp w ranks keys [w * 512, w * 512 + 512) of the tile in input order,
    // 32 per step; keys past the end take digit 255 and are never written
#pragma unroll
    for (int j = 0; j < kRsEpt; ++j) {
      const int e = w * (kRsEpt * 32) + j * 32 + lane;
      if (e < valid) {
        K k = ASYNC ? bk[e] : in_keys[t0 + e];
        if constexpr (FIRST) k = key_enc<K, CODEC>(k);
        kr[j] = k;
        ir[j] = FIRST ? t0 + e : (ASYNC ? bi[e] : in_idx[t0 + e]);
      } else {
        kr[j] = (K)~(K)0;
        ir[j] = 0;
      }
    }
#pragma unroll
    for (int j = 0; j < kRsEpt; ++j) {
      const int d = (kr[j] >> shift) & 0xFF;
      const unsigned peers = digit_peers(d);
      const int r = __popc(peers & lt);
      const int last = 31 - __clz(peers);
      // every lane's read has returned before any lane passes the shuffle,
      // so the last peer's update below cannot overtake a peer's read
      const int b0 = __shfl_sync(0xffffffffu, s_wh[w][d], last);
      if (lane == last) s_wh[w][d] = b0 + r + 1;  // the last peer publishes the new count
      __syncwarp();
      rk[j] = b0 + r;
    }
    __syncthreads();  // also: the input buffer is no longer read
    // thread d: per-warp bases of digit d, then the tile-local digit starts
    const int d_own = threadIdx.x;
    int c_own = 0;
#pragma unroll
    for (int k = 0; k < kRsWarps; ++k) {
      const int v = s_wh[k][d_own];
      s_wh[k][d_own] = c_own;
      c_own += v;
    }
    int tot;
    const int start = block_excl_scan256(c_own, sw, &tot);
    s_start[d_own] = start;
    s_delta[d_own] = goff - start;
    goff += c_own;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kRsEpt; ++j) {
      const int d = (kr[j] >> shift) & 0xFF;
      const int pos = s_start[d] + s_wh[w][d] + rk[j];
      bk[pos] = kr[j];
      bi[pos] = ir[j];
    }
    __syncthreads();
    for (int p = threadIdx.x; p < valid; p += kRsThreads) {
      const K k = bk[p];
      const int g = s_delta[(k >> shift) & 0xFF] + p;
      out_keys[g] = LAST ? key_dec<K, CODEC>(k) : k;
      out_idx[g] = bi[p];
    }
    __syncthreads();  // the buffer and the per-digit arrays are reused
  }
}

// ---------------------------------------------------------------------------
// Top-k over 16-bit keys.  The selection key merges -0 with +0 and maps every
// NaN to the largest key: the reference compares values (x <= pivot is false
// for NaN, so NaNs always rank above the pivot).
enum TopkCodec { kTopkInt16 = 1, kTopkFp16 = 2, kTopkBf16 = 3 };

template <int CODEC>
__device__ __forceinline__ uint32_t topk_key(uint16_t b) {
  if constexpr (CODEC == kTopkInt16) {
    return (uint32_t)(b ^ 0x8000u);
  } else {
    const uint32_t em = CODEC == kTopkFp16 ? 0x7C00u : 0x7F80u;  // exponent field
    if ((b & em) == em && (b & ~em & 0x7FFFu)) return 0xFFFFu;  // NaN
    if ((b & 0x7FFFu) == 0) return 0x8000u;                     // +-0
    return (b & 0x8000u) ? (uint32_t)(uint16_t)~b : (uint32_t)(b | 0x8000u);
  }
}

struct TopkState {
  int hi;            // high byte of the k-th largest key
  int krem;          // elements still to take inside that high byte
  int thr;           // the k-th largest key
  int ties;          // elements equal to thr to take (lowest positions first)
  long long above;   // elements above thr
  int pad[10];
};
static_assert(sizeof(TopkState) == 64, "state");

// 16 consecutive elements from e0 (16-byte vector loads when VEC and the
// run is inside the array; elements past the end read as 0).
template <bool VEC>
__device__ __forceinline__ void load16(const uint16_t* __restrict__ x, int64_t e0, int64_t n, uint16_t (&v)[16]) {
  if (VEC && e0 + 16 <= n) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(x + e0));
    const uint4 b = __ldg(reinterpret_cast<const uint4*>(x + e0) + 1);
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[2 * i] = (uint16_t)(w[i] & 0xFFFFu);
      v[2 * i + 1] = (uint16_t)(w[i] >> 16);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = e0 + i < n ? x[e0 + i] : (uint16_t)0;
  }
}

template <int CODEC, int LEVEL>
struct TopkDigit {
  int hi;
  __device__ __forceinline__ int operator()(uint16_t b) const {
    const uint32_t k = topk_key<CODEC>(b);
    if (LEVEL == 0) return (int)(k >> 8);
    return (int)(k >> 8) == hi ? (int)(k & 0xFF) : -1;
  }
};

// 256-bin histogram of the key's high byte (LEVEL 0), or of the low byte
// among keys whose high byte is st->hi (LEVEL 1), over contiguous chunks of
// tiles; bins must be zero on entry.
template <int CODEC, int LEVEL, bool VEC>
__global__ void __launch_bounds__(kRsThreads) topk_hist_kernel(const uint16_t* __restrict__ x, int64_t n,
                                                               int64_t num_tiles, const TopkState* __restrict__ st,
                                                               unsigned* __restrict__ bins) {
  __shared__ int s_h[kHistCopies * kRsDigits];
#pragma unroll
  for (int k = 0; k < kHistCopies; ++k) s_h[k * kRsDigits + threadIdx.x] = 0;
  __syncthreads();
  const int64_t tpc = chunk_tiles(num_tiles, gridDim.x);
  const int64_t e_lo = blockIdx.x * tpc * kRsTile;
  int64_t e_hi = e_lo + tpc * kRsTile;
  e_hi = e_hi < n ? e_hi : n;
  smem_hist_range<uint16_t, VEC>(x, e_lo, e_hi, s_h, TopkDigit<CODEC, LEVEL>{LEVEL ? st->hi : 0});
  __syncthreads();
  const int c = smem_hist_total(s_h);
  if (c) atomicAdd(&bins[threadIdx.x], (unsigned)c);
}

// One CTA: the bin holding the k-th largest key, from the top of the histogram.
template <int LEVEL>
__global__ void __launch_bounds__(kRsThreads) topk_pick_kernel(const unsigned* __restrict__ bins, long long k,
                                                               TopkState* st) {
  __shared__ int sw[kRsWarps];
  __shared__ int s_suffix[kRsDigits + 1];
  const int d = threadIdx.x;
  // suffix sums: s_suffix[d] = keys in bins >= d (scan of the reversed bins)
  const int c = (int)bins[kRsDigits - 1 - d];
  int tot;
  const int pre = block_excl_scan256(c, sw, &tot);
  s_suffix[kRsDigits - 1 - d] = pre + c;
  if (d == 0) s_suffix[kRsDigits] = 0;
  __syncthreads();
  const long long want = LEVEL == 0 ? k : (long long)st->krem;
  if ((long long)s_suffix[d] >= want && (long long)s_suffix[d + 1] < want) {
    const int above = s_suffix[d + 1];
    if (LEVEL == 0) {
      st->hi = d;
      st->krem = (int)(want - above);
      st->above = above;
    } else {
      st->thr = (st->hi << 8) | d;
      st->ties = (int)(want - above);
      st->above += above;
    }
  }
}

// Per tile: elements above thr and equal to thr -- one warp per tile (each
// lane 128 consecutive elements in 16-byte loads, all in flight), a warp sum,
// no block barrier.
template <int CODEC, bool VEC>
__global__ void __launch_bounds__(kRsThreads) topk_count_kernel(const uint16_t* __restrict__ x, int64_t n,
                                                                int64_t num_tiles, const TopkState* __restrict__ st,
                                                                int* __restrict__ c_above, int* __restrict__ c_tie) {
  const int lane = threadIdx.x & 31;
  const uint32_t thr = (uint32_t)st->thr;
  const int64_t warps = (int64_t)gridDim.x * kRsWarps;
  for (int64_t t = (int64_t)blockIdx.x * kRsWarps + (threadIdx.x >> 5); t < num_tiles; t += warps) {  // warp-uniform
    int aq = 0;  // above in the low half, equal in the high half
#pragma unroll
    for (int q = 0; q < kRsTile / 32 / 16; ++q) {  // 8 runs of 16 elements per lane
      const int64_t e0 = t * kRsTile + ((int64_t)q * 32 + lane) * 16;
      uint16_t v[16];
      load16<VEC>(x, e0, n, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const uint32_t k = topk_key<CODEC>(v[j]);
        const bool in = e0 + j < n;
        aq += (in && k > thr) ? 1 : ((in && k == thr) ? 0x10000 : 0);
      }
    }
    aq = warp_sum_any(aq);
    if (lane == 0) {
      c_above[t] = aq & 0xFFFF;
      c_tie[t] = aq >> 16;
    }
  }
}

// One CTA: per tile, the ties before it and the output offset (taken =
// above + the ties still wanted); off[num_tiles] = k.
__global__ void __launch_bounds__(kRsThreads) topk_offsets_kernel(const int* __restrict__ c_above,
                                                                  const int* __restrict__ c_tie, int64_t num_tiles,
                                                                  const TopkState* __restrict__ st,
                                                                  int* __restrict__ tie_before, int* __restrict__ off) {
  __shared__ int sw[kRsWarps];
  const int ties = st->ties;
  const int64_t per = (num_tiles + kRsThreads - 1) / kRsThreads;
  const int64_t b0 = (int64_t)threadIdx.x * per;
  const int64_t b1 = b0 + per < num_tiles ? b0 + per : num_tiles;
  int qs = 0;
  for (int64_t t = b0; t < b1; ++t) qs += c_tie[t];
  int tot;
  int q = block_excl_scan256(qs, sw, &tot);
  int ss = 0;
  for (int64_t t = b0; t < b1; ++t) {
    const int c = c_tie[t];
    int take = ties - q;
    take = take < 0 ? 0 : (take > c ? c : take);
    ss += c_above[t] + take;
    q += c;
  }
  int s = block_excl_scan256(ss, sw, &tot);
  q -= qs;  // back to this thread's first tile
  for (int64_t t = b0; t < b1; ++t) {
    const int c = c_tie[t];
    int take = ties - q;
    take = take < 0 ? 0 : (take > c ? c : take);
    tie_before[t] = q;
    off[t] = s;
    s += c_above[t] + take;
    q += c;
  }
  if (threadIdx.x == kRsThreads - 1) off[num_tiles] = s;
}

// Emits the selected elements of every tile in index order (values and int32
// positions).  Tiles with nothing selected are skipped without reading them.
template <int CODEC, bool VEC>
__global__ void __launch_bounds__(kRsThreads) topk_emit_kernel(const uint16_t* __restrict__ x, int64_t n,
                                                               int64_t num_tiles, const TopkState* __restrict__ st,
                                                               const int* __restrict__ tie_before,
                                                               const int* __restrict__ off, int64_t k,
                                                               uint16_t* __restrict__ out, int* __restrict__ idx_out) {
  __shared__ int sw[kRsWarps];
  const uint32_t thr = (uint32_t)st->thr;
  const int ties = st->ties;
  for (int64_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    const int o0 = off[t];
    if (off[t + 1] == o0) continue;  // block-uniform
    const int64_t e0 = t * kRsTile + (int64_t)threadIdx.x * kRsEpt;  // 16 consecutive elements per thread
    uint16_t xv[16];
    load16<VEC>(x, e0, n, xv);
    unsigned am = 0, qm = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const uint32_t kk = topk_key<CODEC>(xv[j]);
      const bool in = e0 + j < n;
      am |= (unsigned)(in && kk > thr) << j;
      qm |= (unsigned)(in && kk == thr) << j;
    }
    int tot;
    // ties of this thread that are still wanted: the first (ties - rank) of them
    const int tr = tie_before[t] + block_excl_scan256(__popc(qm), sw, &tot);
    int want = ties - tr;
    want = want < 0 ? 0 : want;
    unsigned take = qm;
    for (int c = __popc(qm); c > want; --c) take &= ~(1u << (31 - __clz(take)));  // drop the last ties
    const unsigned selm = am | take;
    int o = o0 + block_excl_scan256(__popc(selm), sw, &tot);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (((selm >> j) & 1u) && o < k) {
        out[o] = xv[j];
        idx_out[o] = (int)(e0 + j);
        ++o;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Top-k pivot estimator (kernel_topk_pivot.h:96-160).  Block b reads up to
// 8 tiles of num_samples * 32 elements from tile b * tiles_per_block on; per
// tile, each 32-element group gives its k_inner-th largest value, those
// values replace the first entries of the tile's first 32 elements, and the
// k_outer-th largest of these 32 is the tile's estimate; the block writes the
// largest estimate.  Elements past the end read as -inf.
__device__ __forceinline__ float kth_largest32(float v, int k) {
  const int lane = threadIdx.x & 31;
  int rank = 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const float o = __shfl_sync(0xffffffffu, v, j);
    rank += (o > v) || (o == v && j < lane);
  }
  const unsigned hit = __ballot_sync(0xffffffffu, rank == k - 1);
  return __shfl_sync(0xffffffffu, v, hit ? __ffs(hit) - 1 : 0);
}

__global__ void __launch_bounds__(kRsThreads) topk_pivot_kernel(const __half* __restrict__ x, int64_t n,
                                                                int num_samples, int k_inner, int k_outer,
                                                                int64_t tiles_per_block, int64_t num_tiles,
                                                                __half* __restrict__ out) {
  __shared__ float s_est[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t tile_len = (int64_t)num_samples * 32;
  const int groups = num_samples < 32 ? num_samples : 32;  // estimates that reach the outer selection
  float best = -INFINITY;
  for (int it = 0; it < 8; ++it) {
    const int64_t tile = blockIdx.x * tiles_per_block + it;
    if (tile >= num_tiles) break;  // block-uniform
    const int64_t base = tile * tile_len;
    for (int g = w; g < groups; g += kRsWarps) {
      const int64_t e = base + (int64_t)g * 32 + lane;
      const float v = e < n ? __half2float(x[e]) : -INFINITY;
      const float kth = kth_largest32(v, k_inner);
      if (lane == 0) s_est[g] = kth;
    }
    __syncthreads();
    if (w == 0) {
      const int64_t e = base + lane;
      const float v = lane < groups ? s_est[lane] : (e < n ? __half2float(x[e]) : -INFINITY);
      const float est = kth_largest32(v, k_outer);
      best = fmaxf(best, est);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = __float2half_rn(best);
}

// ---------------------------------------------------------------------------
// Host side.

static int64_t rs_tiles(int64_t n) { return (n + kRsTile - 1) / kRsTile; }

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// tmp layout: keys[n] (K) | idx[n] (int32) | sums[chunks * 256] | base[chunks * 256] | totals[256]
constexpr int kRsChunksPerSm = 3;  // the scatter kernel holds 3 CTAs per SM

static int rs_chunks(int64_t tiles) {
  int64_t c = (int64_t)sm_count() * kRsChunksPerSm;
  if (tiles < c) c = tiles;
  return (int)(c < 1 ? 1 : c);
}

static size_t rs_tmp_bytes(int key_bytes, int64_t n) {
  const int C = rs_chunks(rs_tiles(n));
  return align256((size_t)n * key_bytes) + align256((size_t)n * 4) + 2 * align256((size_t)C * kRsDigits * 4) +
         align256(kRsDigits * 4);
}

template <typename K, int CODEC, bool FIRST, bool LAST>
static cudaError_t launch_scatter(bool async_ok, int C, cudaStream_t st, const K* src_k, const int* src_i, K* dk, int* di,
                                  const int* base, int64_t n, int shift, int64_t T) {
  constexpr int smem = ScatterSmem<K>::BYTES;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(rs_scatter_kernel<K, CODEC, FIRST, LAST, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(rs_scatter_kernel<K, CODEC, FIRST, LAST, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  if (async_ok)
    rs_scatter_kernel<K, CODEC, FIRST, LAST, true><<<C, kRsThreads, smem, st>>>(src_k, src_i, dk, di, base, n, shift, T);
  else
    rs_scatter_kernel<K, CODEC, FIRST, LAST, false><<<C, kRsThreads, smem, st>>>(src_k, src_i, dk, di, base, n, shift, T);
  return cudaGetLastError();
}

template <typename K, int CODEC>
static tcu_status_t radix_sort_t(const K* x, int64_t n, K* out, int* idx_out, uint8_t* tmp, cudaStream_t st) {
  const int64_t T = rs_tiles(n);
  const int C = rs_chunks(T);
  K* tk = reinterpret_cast<K*>(tmp);
  int* ti = reinterpret_cast<int*>(tmp + align256((size_t)n * sizeof(K)));
  int* sums = reinterpret_cast<int*>(reinterpret_cast<uint8_t*>(ti) + align256((size_t)n * 4));
  int* base = reinterpret_cast<int*>(reinterpret_cast<uint8_t*>(sums) + align256((size_t)C * kRsDigits * 4));
  unsigned* totals = reinterpret_cast<unsigned*>(reinterpret_cast<uint8_t*>(base) + align256((size_t)C * kRsDigits * 4));
  constexpr int passes = (int)sizeof(K);
  // ping-pong so that the last pass lands in out / idx_out
  const K* src_k = x;
  const int* src_i = nullptr;
  for (int p = 0; p < passes; ++p) {
    const bool last = p == passes - 1;
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    K* dk = to_out ? out : tk;
    int* di = to_out ? idx_out : ti;
    const int shift = 8 * p;
    cudaError_t e1 = cudaMemsetAsync(totals, 0, kRsDigits * 4, st);
    if (e1 != cudaSuccess) return cuda_fail(e1, "cudaMemsetAsync(radix totals)");
    if (p == 0 && aligned16(src_k))
      rs_hist_kernel<K, CODEC, true, true><<<C, kRsThreads, 0, st>>>(src_k, n, shift, T, sums, totals);
    else if (p == 0)
      rs_hist_kernel<K, CODEC, true, false><<<C, kRsThreads, 0, st>>>(src_k, n, shift, T, sums, totals);
    else  // the scratch and output buffers are 16-byte aligned
      rs_hist_kernel<K, CODEC, false, true><<<C, kRsThreads, 0, st>>>(src_k, n, shift, T, sums, totals);
    rs_chunk_scan_kernel<<<kRsDigits, kChunkScanThreads, 0, st>>>(sums, C, totals, base);
    const bool async_ok = aligned16(src_k) && (p == 0 || aligned16(src_i));
    if (p == 0 && last) e1 = launch_scatter<K, CODEC, true, true>(async_ok, C, st, src_k, src_i, dk, di, base, n, shift, T);
    else if (p == 0) e1 = launch_scatter<K, CODEC, true, false>(async_ok, C, st, src_k, src_i, dk, di, base, n, shift, T);
    else if (last) e1 = launch_scatter<K, CODEC, false, true>(async_ok, C, st, src_k, src_i, dk, di, base, n, shift, T);
    else e1 = launch_scatter<K, CODEC, false, false>(async_ok, C, st, src_k, src_i, dk, di, base, n, shift, T);
    if (e1 != cudaSuccess) return cuda_fail(e1, "radix scatter launch");
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "radix sort launch");
    src_k = dk;
    src_i = di;
  }
  return TCU_OK;
}

static int rs_grid(int64_t tiles, int per_sm) {
  int64_t g = (int64_t)sm_count() * per_sm;
  if (tiles < g) g = tiles;
  return (int)(g < 1 ? 1 : g);
}

// tmp layout: bins[2][256] | state | c_above[T] | c_tie[T] | tie_before[T] | off[T + 1]
static size_t topk_tmp_bytes(int64_t n) {
  const int64_t T = rs_tiles(n);
  return 2048 + sizeof(TopkState) + 3 * align256((size_t)T * 4) + align256((size_t)(T + 1) * 4);
}

template <int CODEC>
static tcu_status_t topk_t(const uint16_t* x, int64_t n, int64_t k, uint16_t* out, int* idx_out, uint8_t* tmp,
                           cudaStream_t st) {
  const bool VEC = aligned16(x);
  const int64_t T = rs_tiles(n);
  unsigned* bins = reinterpret_cast<unsigned*>(tmp);
  TopkState* state = reinterpret_cast<TopkState*>(tmp + 2048);
  int* c_above = reinterpret_cast<int*>(tmp + 2048 + sizeof(TopkState));
  int* c_tie = reinterpret_cast<int*>(reinterpret_cast<uint8_t*>(c_above) + align256((size_t)T * 4));
  int* tie_before = reinterpret_cast<int*>(reinterpret_cast<uint8_t*>(c_tie) + align256((size_t)T * 4));
  int* off = reinterpret_cast<int*>(reinterpret_cast<uint8_t*>(tie_before) + align256((size_t)T * 4));
  cudaError_t e = cudaMemsetAsync(tmp, 0, 2048 + sizeof(TopkState), st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(topk state)");
  const int g = rs_grid(T, 8);
  const int gw = rs_grid((T + kRsWarps - 1) / kRsWarps, 8);  // a warp per tile
  const int gh = rs_grid(T, 6);  // histogram CTAs: contiguous chunks of tiles, 32 KB of counters
  if (VEC) {
    topk_hist_kernel<CODEC, 0, true><<<gh, kRsThreads, 0, st>>>(x, n, T, state, bins);
    topk_pick_kernel<0><<<1, kRsThreads, 0, st>>>(bins, k, state);
    topk_hist_kernel<CODEC, 1, true><<<gh, kRsThreads, 0, st>>>(x, n, T, state, bins + 256);
    topk_pick_kernel<1><<<1, kRsThreads, 0, st>>>(bins + 256, k, state);
    topk_count_kernel<CODEC, true><<<gw, kRsThreads, 0, st>>>(x, n, T, state, c_above, c_tie);
    topk_offsets_kernel<<<1, kRsThreads, 0, st>>>(c_above, c_tie, T, state, tie_before, off);
    topk_emit_kernel<CODEC, true><<<g, kRsThreads, 0, st>>>(x, n, T, state, tie_before, off, k, out, idx_out);
  } else {
    topk_hist_kernel<CODEC, 0, false><<<gh, kRsThreads, 0, st>>>(x, n, T, state, bins);
    topk_pick_kernel<0><<<1, kRsThreads, 0, st>>>(bins, k, state);
    topk_hist_kernel<CODEC, 1, false><<<gh, kRsThreads, 0, st>>>(x, n, T, state, bins + 256);
    topk_pick_kernel<1><<<1, kRsThreads, 0, st>>>(bins + 256, k, state);
    topk_count_kernel<CODEC, false><<<gw, kRsThreads, 0, st>>>(x, n, T, state, c_above, c_tie);
    topk_offsets_kernel<<<1, kRsThreads, 0, st>>>(c_above, c_tie, T, state, tie_before, off);
    topk_emit_kernel<CODEC, false><<<g, kRsThreads, 0, st>>>(x, n, T, state, tie_before, off, k, out, idx_out);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "topk launch");
}

static int pivot_blocks(int64_t n, int num_samples, int64_t* tiles_per_block, int64_t* num_tiles) {
  const int64_t tile_len = (int64_t)num_samples * 32;
  const int64_t T = (n + tile_len - 1) / tile_len;
  int64_t b = sm_count();
  if (T < b) b = T;
  if (b < 1) b = 1;
  if (num_tiles) *num_tiles = T;
  if (tiles_per_block) *tiles_per_block = (T + b - 1) / b;
  return (int)b;
}

}  // namespace tcu

using namespace tcu;

extern "C" {

size_t tcu_radix_sort_tmp_bytes(tcu_dtype_t dtype, int64_t n) {
  int kb = 0;
  switch (dtype) {
    case TCU_INT8: case TCU_UINT8: kb = 1; break;
    case TCU_INT16: case TCU_FLOAT16: case TCU_BFLOAT16: kb = 2; break;
    case TCU_INT32: case TCU_UINT32: case TCU_FLOAT32: kb = 4; break;
    default: return 0;
  }
  return n <= 0 ? 0 : rs_tmp_bytes(kb, n);
}

tcu_status_t tcu_radix_sort(const void* x, tcu_dtype_t dtype, int64_t n, void* out, int32_t* idx_out, void* tmp,
                            size_t tmp_bytes, void* stream) {
  if (n < 0 || n > 0x7FFFFFFFLL) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !out || !idx_out) return TCU_ERR_ARG;
  const size_t need = tcu_radix_sort_tmp_bytes(dtype, n);
  if (need == 0) return TCU_ERR_DTYPE;
  if (!tmp || tmp_bytes < need) return TCU_ERR_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(tmp) & 255u) || (reinterpret_cast<uintptr_t>(idx_out) & 3u)) return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  uint8_t* t = static_cast<uint8_t*>(tmp);
  switch (dtype) {
    case TCU_UINT8: return radix_sort_t<uint8_t, kCodecUnsigned>((const uint8_t*)x, n, (uint8_t*)out, idx_out, t, st);
    case TCU_INT8: return radix_sort_t<uint8_t, kCodecSigned>((const uint8_t*)x, n, (uint8_t*)out, idx_out, t, st);
    case TCU_INT16: return radix_sort_t<uint16_t, kCodecSigned>((const uint16_t*)x, n, (uint16_t*)out, idx_out, t, st);
    case TCU_FLOAT16:
    case TCU_BFLOAT16:
      return radix_sort_t<uint16_t, kCodecFloat>((const uint16_t*)x, n, (uint16_t*)out, idx_out, t, st);
    case TCU_UINT32: return radix_sort_t<uint32_t, kCodecUnsigned>((const uint32_t*)x, n, (uint32_t*)out, idx_out, t, st);
    case TCU_INT32: return radix_sort_t<uint32_t, kCodecSigned>((const uint32_t*)x, n, (uint32_t*)out, idx_out, t, st);
    default: return radix_sort_t<uint32_t, kCodecFloat>((const uint32_t*)x, n, (uint32_t*)out, idx_out, t, st);
  }
}

size_t tcu_topk_tmp_bytes(int64_t n) { return n <= 0 ? 0 : topk_tmp_bytes(n); }

tcu_status_t tcu_topk(const void* x, tcu_dtype_t dtype, int64_t n, int64_t k, void* out, int32_t* idx_out, void* tmp,
                      size_t tmp_bytes, void* stream) {
  if (n < 0 || n > 0x7FFFFFFFLL || k < 0 || k > n) return TCU_ERR_ARG;
  if (dtype != TCU_INT16 && dtype != TCU_FLOAT16 && dtype != TCU_BFLOAT16) return TCU_ERR_DTYPE;
  if (k == 0) return TCU_OK;
  if (!x || !out || !idx_out) return TCU_ERR_ARG;
  if (!tmp || tmp_bytes < topk_tmp_bytes(n)) return TCU_ERR_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(tmp) & 255u) || (reinterpret_cast<uintptr_t>(idx_out) & 3u) ||
      (reinterpret_cast<uintptr_t>(x) & 1u) || (reinterpret_cast<uintptr_t>(out) & 1u))
    return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  const uint16_t* xs = static_cast<const uint16_t*>(x);
  uint16_t* o = static_cast<uint16_t*>(out);
  uint8_t* t = static_cast<uint8_t*>(tmp);
  if (dtype == TCU_INT16) return topk_t<kTopkInt16>(xs, n, k, o, idx_out, t, st);
  if (dtype == TCU_FLOAT16) return topk_t<kTopkFp16>(xs, n, k, o, idx_out, t, st);
  return topk_t<kTopkBf16>(xs, n, k, o, idx_out, t, st);
}

int tcu_topk_pivot_blocks(int64_t n, int num_samples) {
  if (n <= 0 || num_samples <= 0) return 0;
  return pivot_blocks(n, num_samples, nullptr, nullptr);
}

tcu_status_t tcu_topk_pivot(const void* x, tcu_dtype_t dtype, int64_t n, int num_samples, int k_inner, int k_outer,
                            void* out, void* stream) {
  if (n <= 0 || num_samples <= 0 || k_inner < 1 || k_inner > 32 || k_outer < 1 || k_outer > 32) return TCU_ERR_ARG;
  if (dtype != TCU_FLOAT16) return TCU_ERR_DTYPE;
  if (!x || !out) return TCU_ERR_ARG;
  int64_t tpb = 0, T = 0;
  const int b = pivot_blocks(n, num_samples, &tpb, &T);
  topk_pivot_kernel<<<b, kRsThreads, 0, (cudaStream_t)stream>>>(static_cast<const __half*>(x), n, num_samples, k_inner,
                                                                k_outer, tpb, T, static_cast<__half*>(out));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "topk_pivot_kernel launch");
}

}  // extern "C"

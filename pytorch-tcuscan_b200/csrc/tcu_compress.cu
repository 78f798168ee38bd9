// tcu_compress.cu -- stream compaction on B200.
//
// Reference: run_compress / run_compress_pos / run_compress_ind /
// run_compress_ind_no_arange (src/torch/torch_compress.h:41-309) count the
// mask per block with reduce_tiles, read the total back to the host, then
// gather with the vector GatherMask instruction (kernel_compress.h:97-208).
//
// Compaction is byte/integer work bound by HBM, so it stays on the SIMT cores
// (no tensor-core reshaping).  Three launches, each a pure stream with no
// waiting between CTAs:
//   cmp_count_kernel    selected elements per tile (reads the mask once);
//   cmp_offsets_*       exclusive int64 scan of the tile counts in two
//                       parallel passes (per 1024 tiles, then the block
//                       bases) -> each tile's output offset, and the total;
//   compress_kernel     one persistent CTA per SM, tiles assigned statically.
//               warp 0 loads each tile's mask, values (and gathered indices)
//               with 2-D TMA copies into a ring of shared-memory stages.  Each
//               array is seen as rows of EPT elements, one row per worker
//               thread, with the TMA swizzle of the row width, so every worker
//               reads its own row without bank conflicts.
//               warps 1-16: four worker warpgroups taking every fourth stage:
//               selection bits from the mask row, the tile-local exclusive
//               scan of the per-thread counts, compaction of the selected
//               values from registers back into the stage (in place), then
//               coalesced stores at the tile's precomputed offset.
// run_compress needs the count on the host before it can size its output, so
// the count pass is work it has to do anyway (tcu_compress_count, then
// tcu_compress_counted); a single-pass look-back variant was measured slower
// here: with 24-KB tiles every tile waited on its predecessors' counts.
// The per-tile counts and offsets live in the workspace's descriptor region
// and are zeroed after use (the region must hold only look-back descriptors
// or zeros between launches).
#include <cuda_runtime.h>

#include <cstdio>

#include "tcu_host.h"

namespace tcu {

struct CompressParams {
  const void* x;
  const int8_t* mask;
  const void* idx_in;         // optional gathered indices (compress_ind)
  void* out;
  void* idx_out;              // optional
  int64_t n;
  int64_t capacity;           // elements the outputs can hold (compress_pos output_len)
  int64_t num_tiles;
  int64_t full_rows;          // n / EPT: rows the tensor maps cover
  int has_map;                // full_rows > 0
  const long long* offsets;   // per-tile output offsets (workspace)
  WsHeader* ws;
  uint64_t timeout_ns;
};

constexpr int kCmpWG = 4;                       // worker warpgroups
constexpr int kCmpThreads = 32 + 128 * kCmpWG;  // producer + workers
constexpr int kCmpStageBudget = 200 * 1024;
constexpr int kCmpMaxStages = 16;
constexpr uint32_t kCmpSentinel = 0xFFFFFFFFu;

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

// Elements per worker row for an element / index size: the longest row of
// 64, 32 or 16 elements with at most 128 bytes of each array per row (one
// swizzled TMA box row) and a ring of at least five 128-row stages in the
// stage budget.  An earlier rule (64 up to 2 bytes per element, 32 up to 4,
// else 16) gave fp16 values with int32 indices 16-element rows, where 32 fit.
__host__ __device__ constexpr int cmp_ept(int eb, int ib) {
  return (64 * eb <= 128 && 64 * ib <= 128 && 128 * 64 * (1 + eb + ib) * 5 <= kCmpStageBudget)   ? 64
         : (32 * eb <= 128 && 32 * ib <= 128 && 128 * 32 * (1 + eb + ib) * 5 <= kCmpStageBudget) ? 32
                                                                                                   : 16;
}
// Elements per row for an index mode: gathered indices (1) are staged like
// the values; generated positions (2) need only a 16-bit tile-local offset
// per element in the compaction scratch.  Staging 4-byte positions cut fp16
// rows to 16 elements and took 620 us at 2^28 against 205 us without them.
__host__ __device__ constexpr int cmp_ept_for(int eb, int idx_mode, int ib) {
  return cmp_ept(eb, idx_mode == 2 ? 2 : (idx_mode ? ib : 0));
}

template <int EB, int IDX, int IB>
struct CmpCfg {
  static constexpr int IBX = IDX == 1 ? IB : (IDX == 2 ? 2 : 0);  // index bytes per element in the stage
  static constexpr int RB = EB + IBX;
  static constexpr int EPT = cmp_ept_for(EB, IDX, IB);
  static constexpr int TILE = 128 * EPT;
  static constexpr int SPAN_M = EPT;           // bytes of one mask row
  static constexpr int SPAN_X = EPT * EB;      // bytes of one value row
  static constexpr int SPAN_I = EPT * (IB > 0 ? IB : 4);
  static constexpr int X_OFF = TILE;
  static constexpr int I_OFF = TILE * (1 + EB);
  static constexpr int STAGE = TILE * (1 + RB);
  static constexpr int NST_RAW = kCmpStageBudget / STAGE;
  static constexpr int NST = NST_RAW > kCmpMaxStages ? kCmpMaxStages : NST_RAW;
  static constexpr int CTRL = 1024;
  static constexpr int SMEM = CTRL + NST * STAGE + 1024;  // + alignment slack
  static_assert(NST >= kCmpWG + 1, "stage ring too short");
  static_assert(SPAN_X <= 128 && SPAN_M <= 128 && (IDX != 1 || SPAN_I <= 128), "row span");
  static_assert(STAGE % 1024 == 0, "stage alignment");
  static_assert(IDX != 2 || TILE <= 65536, "tile-local positions are 16-bit");
};

struct CmpCtrl {
  uint64_t full[kCmpMaxStages];
  uint64_t empty[kCmpMaxStages];
  uint32_t stage_tid[kCmpMaxStages];
  int wsum[kCmpWG][4];
  int vote[kCmpWG][4];
  int abort_flag;
};
static_assert(sizeof(CmpCtrl) <= 1024, "control block");

// Byte address of 16-byte chunk v of row r in a TMA-swizzled area of
// `span`-byte rows (span 16 = no swizzle).
__device__ __forceinline__ uint32_t row_chunk(int r, int v, int span) {
  const uint32_t o = (uint32_t)(r * span + 16 * v);
  return span >= 32 ? swz(o, (uint32_t)span) : o;
}

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

// Sets element j of a register vector run (constant j after unrolling).
template <int EB>
__device__ __forceinline__ void vec_set(uint4* v, int j, typename ElemT<EB>::T e) {
  constexpr int PER = 16 / EB;
  uint4& w = v[j / PER];
  const int b = (j % PER) * EB;
  uint32_t lo;
  if constexpr (EB >= 4) {
    lo = (uint32_t)e;
  } else {
    constexpr uint32_t M = EB == 1 ? 0xFFu : 0xFFFFu;
    const int sh = 8 * (b % 4);
    const uint32_t cur = (b < 4) ? w.x : (b < 8) ? w.y : (b < 12) ? w.z : w.w;
    lo = (cur & ~(M << sh)) | (((uint32_t)e & M) << sh);
  }
  if (b < 4) w.x = lo;
  else if (b < 8) w.y = lo;
  else if (b < 12) w.z = lo;
  else w.w = lo;
  if constexpr (EB == 8) {
    const uint32_t hi = (uint32_t)((unsigned long long)e >> 32);
    if (b < 4) w.y = hi;
    else w.w = hi;
  }
}

// Writes a run of `len` elements, val(0 .. len-1), to dst[g0 .. g0 + len)
// (positions below cap only), the 128 threads of a warpgroup together:
// 16-byte stores for the vectors that lie inside the run, element stores for
// the ragged ends (or for all of it when dst is not 16-byte aligned).  One
// store per element kept the store loop of split -- every element of the
// tile written -- bound by store instructions.
template <typename E, typename ValF>
__device__ __forceinline__ void store_run(ValF val, int len, E* dst, long long g0, long long cap, int t) {
  constexpr int V = 16 / (int)sizeof(E);
  const long long end = g0 + len < cap ? g0 + len : cap;
  if (end <= g0) return;
  if ((reinterpret_cast<uintptr_t>(dst) & 15u) != 0) {
    for (long long e = g0 + t; e < end; e += 128) dst[e] = val((int)(e - g0));
    return;
  }
  const long long v0 = g0 / V, v1 = (end - 1) / V;
  for (long long vb = v0 + t; vb <= v1; vb += 128) {
    const long long e0 = vb * V;
    if (e0 >= g0 && e0 + V <= end) {
      union {
        uint4 u;
        E e[V];
      } w;
#pragma unroll
      for (int i = 0; i < V; ++i) w.e[i] = val((int)(e0 - g0) + i);
      *reinterpret_cast<uint4*>(dst + e0) = w.u;
    } else {
#pragma unroll
      for (int i = 0; i < V; ++i) {
        const long long e = e0 + i;
        if (e >= g0 && e < end) dst[e] = val((int)(e - g0));
      }
    }
  }
}

// IDX: 0 none, 1 gather idx_in (IB bytes), 2 positions (int32 when IB == 4,
// int64 when IB == 8).  SPLIT: stable partition instead of compaction -- every
// element is written, the selected ones at their compaction offsets and the
// others after all selected ones (at total + the unselected elements before
// them), so a tile writes two runs.
template <int EB, int IDX, int IB, bool SPLIT>
__global__ void __launch_bounds__(kCmpThreads, 1)
    compress_kernel(const __grid_constant__ CUtensorMap mmap, const __grid_constant__ CUtensorMap xmap,
                    const __grid_constant__ CUtensorMap imap, const CompressParams p) {
  using C = CmpCfg<EB, IDX, IB>;
  using T = typename ElemT<EB>::T;
  using I = typename ElemT<(IB > 0 ? IB : 4)>::T;
  constexpr int EPT = C::EPT;
  constexpr int TILE = C::TILE;
  constexpr int NST = C::NST;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  CmpCtrl* ctl = reinterpret_cast<CmpCtrl*>(smem);
  uint8_t* stages = smem + C::CTRL;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WaitCtx wc{p.ws, &ctl->abort_flag, p.timeout_ns};

  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&ctl->full[s], 1);
      mbar_init(&ctl->empty[s], 1);
    }
    ctl->abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0 && p.has_map) {
    prefetch_tmap(&mmap);
    prefetch_tmap(&xmap);
    if constexpr (IDX == 1) prefetch_tmap(&imap);
  }
  __syncthreads();

  if (warp == 0) {
    // ================= producer: this CTA's tiles, in order =================
    if (lane == 0) {
      uint32_t issued[kCmpMaxStages];
#pragma unroll
      for (int s = 0; s < kCmpMaxStages; ++s) issued[s] = 0;
      uint32_t seq = 0;
      int sentinels = 0;  // one stop marker per worker warpgroup
      int64_t tile = blockIdx.x;
      while (sentinels < kCmpWG) {
        const int s = seq % NST;
        if (seq >= (uint32_t)NST && !mbar_wait(&ctl->empty[s], ((seq / NST) & 1u) ^ 1u, wc, 21, seq)) break;
        const bool live = sentinels == 0 && tile < p.num_tiles && !aborted(wc);
        const uint32_t tid = live ? (uint32_t)tile : kCmpSentinel;
        ctl->stage_tid[s] = tid;
        issued[s]++;
        const int64_t row0 = tile * 128;
        if (live && p.has_map && row0 < p.full_rows) {
          uint8_t* st = stages + s * C::STAGE;
          mbar_arrive_expect_tx(&ctl->full[s], (uint32_t)(TILE * (1 + EB + (IDX == 1 ? IB : 0))));
          tma_load_2d(st, &mmap, 0, (int32_t)row0, &ctl->full[s]);
          tma_load_2d(st + C::X_OFF, &xmap, 0, (int32_t)row0, &ctl->full[s]);
          if constexpr (IDX == 1) tma_load_2d(st + C::I_OFF, &imap, 0, (int32_t)row0, &ctl->full[s]);
        } else {
          mbar_arrive(&ctl->full[s]);
        }
        if (live) tile += gridDim.x;
        else ++sentinels;
        ++seq;
      }
      // every copy issued must have landed before the CTA exits
      for (int s = 0; s < NST; ++s)
        if (issued[s]) mbar_drain(&ctl->full[s], (issued[s] - 1) & 1u, p.timeout_ns);
    }
  } else {
    // ================= worker warpgroups =================
    const int w = (warp - 1) >> 2;
    const int q = (warp - 1) & 3;
    const int wg_thread = threadIdx.x - 32 - 128 * w;
    const uint32_t bar_id = 1 + w;
    for (uint32_t seq = w;; seq += kCmpWG) {
      const int s = seq % NST;
      int ok = 1;
      if (lane == 0) ok = mbar_wait(&ctl->full[s], (seq / NST) & 1u, wc, 23, seq) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (lane == 0) ctl->vote[w][q] = ok;
      named_bar_sync(bar_id, 128);
      const int all_ok = ctl->vote[w][0] & ctl->vote[w][1] & ctl->vote[w][2] & ctl->vote[w][3];
      const uint32_t tid = *(volatile uint32_t*)&ctl->stage_tid[s];
      if (!all_ok || tid == kCmpSentinel) break;
      const long long pre = p.offsets[tid];  // in flight while the stage is read
      uint8_t* st = stages + s * C::STAGE;
      const int64_t row = (int64_t)tid * 128 + wg_thread;
      const int64_t e0 = row * EPT;  // first element of this thread's row
      const bool in_smem = row < p.full_rows;
      const bool is_tail = row == p.full_rows && e0 < p.n;

      // ---- selection bits and payload registers ----
      unsigned long long sel = 0;
      uint4 xr[C::SPAN_X / 16];
      uint4 ir[IDX == 1 ? C::SPAN_I / 16 : 1];
      if (in_smem) {
#pragma unroll
        for (int v = 0; v < C::SPAN_M / 16; ++v) {
          const uint4 m = *reinterpret_cast<const uint4*>(st + row_chunk(wg_thread, v, C::SPAN_M));
          sel |= (unsigned long long)(sel4(m.x) | (sel4(m.y) << 4) | (sel4(m.z) << 8) | (sel4(m.w) << 12)) << (16 * v);
        }
        if (SPLIT || sel) {
#pragma unroll
          for (int v = 0; v < C::SPAN_X / 16; ++v)
            xr[v] = *reinterpret_cast<const uint4*>(st + C::X_OFF + row_chunk(wg_thread, v, C::SPAN_X));
          if constexpr (IDX == 1) {
#pragma unroll
            for (int v = 0; v < C::SPAN_I / 16; ++v)
              ir[v] = *reinterpret_cast<const uint4*>(st + C::I_OFF + row_chunk(wg_thread, v, C::SPAN_I));
          }
        }
      } else if (is_tail) {  // ragged end of the input: plain loads
#pragma unroll
        for (int v = 0; v < C::SPAN_X / 16; ++v) xr[v] = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int v = 0; v < (IDX == 1 ? C::SPAN_I / 16 : 1); ++v) ir[v] = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
          if (e0 + j < p.n) {
            const bool on = p.mask[e0 + j] != 0;
            if (on) sel |= 1ull << j;
            if (SPLIT || on) {
              vec_set<EB>(xr, j, static_cast<const T*>(p.x)[e0 + j]);
              if constexpr (IDX == 1) vec_set<(IB > 0 ? IB : 4)>(ir, j, static_cast<const I*>(p.idx_in)[e0 + j]);
            }
          }
        }
      }
      const int cnt = __popcll(sel);

      // ---- tile-local exclusive scan of the per-thread counts ----
      int inc = cnt;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += o;
      }
      if (lane == 31) ctl->wsum[w][q] = inc;
      named_bar_sync(bar_id, 128);  // also: every row of the stage is in registers
      int wpre = 0, total = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int v = ctl->wsum[w][k];
        if (k < q) wpre += v;
        total += v;
      }
      const int local = wpre + inc - cnt;

      // ---- compaction in place (values over the value rows, indices over the index rows) ----
      {
        T* sx = reinterpret_cast<T*>(st + C::X_OFF);
        I* si = reinterpret_cast<I*>(st + C::I_OFF);
        uint16_t* sp = reinterpret_cast<uint16_t*>(st + C::I_OFF);  // IDX 2: tile-local positions
        const int lrow = wg_thread * EPT;                           // this row's first position in the tile
        int o = local;
        if constexpr (SPLIT) {
          // unselected elements before this row: all earlier rows of the tile are full
          int u = total + wg_thread * EPT - local;
          const int nv = in_smem ? EPT : (is_tail ? (int)(p.n - e0) : 0);
#pragma unroll
          for (int j = 0; j < EPT; ++j) {
            if (j < nv) {
              const bool on = (sel >> j) & 1ull;
              const int d = on ? o : u;
              sx[d] = vec_elem<EB>(xr, j);
              if constexpr (IDX == 1) si[d] = (I)vec_elem<(IB > 0 ? IB : 4)>(ir, j);
              if constexpr (IDX == 2) sp[d] = (uint16_t)(lrow + j);
              o += on ? 1 : 0;
              u += on ? 0 : 1;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < EPT; ++j) {
            if ((sel >> j) & 1ull) {
              sx[o] = vec_elem<EB>(xr, j);
              if constexpr (IDX == 1) si[o] = (I)vec_elem<(IB > 0 ? IB : 4)>(ir, j);
              if constexpr (IDX == 2) sp[o] = (uint16_t)(lrow + j);
              ++o;
            }
          }
        }
      }
      named_bar_sync(bar_id, 128);  // compacted run complete in shared memory

      // ---- coalesced stores of the compacted run ----
      {
        const T* sx = reinterpret_cast<const T*>(st + C::X_OFF);
        const I* si = reinterpret_cast<const I*>(st + C::I_OFF);
        const uint16_t* sp = reinterpret_cast<const uint16_t*>(st + C::I_OFF);
        const int64_t t0 = (int64_t)tid * TILE;
        const int valid = SPLIT ? (int)(p.n - t0 < TILE ? p.n - t0 : TILE) : total;
        // selected run at pre, unselected run after every selected element
        const long long ubase = SPLIT ? p.offsets[p.num_tiles] + (t0 - pre) - total : 0;
        if constexpr (SPLIT) {
          // every element of the tile is written: two runs with 16-byte stores
          // (0.534 -> 0.430 ms for fp16 at 2^28); the compaction's own run
          // (~30 % of the elements) measured no faster that way, and slower
          // for 1-byte values, so it keeps element stores
          T* out = static_cast<T*>(p.out);
          I* iout = static_cast<I*>(p.idx_out);
          const int nu = valid - total;
          store_run<T>([&](int j) { return sx[j]; }, total, out, pre, p.capacity, wg_thread);
          store_run<T>([&](int j) { return sx[total + j]; }, nu, out, ubase + total, p.capacity, wg_thread);
          if constexpr (IDX == 1) {
            store_run<I>([&](int j) { return si[j]; }, total, iout, pre, p.capacity, wg_thread);
            store_run<I>([&](int j) { return si[total + j]; }, nu, iout, ubase + total, p.capacity, wg_thread);
          }
        } else {
          for (int i = wg_thread; i < valid; i += 128) {
            const long long g = pre + i;
            if (g < p.capacity) {
              static_cast<T*>(p.out)[g] = sx[i];
              if constexpr (IDX == 1) static_cast<I*>(p.idx_out)[g] = si[i];
              if constexpr (IDX == 2) static_cast<I*>(p.idx_out)[g] = (I)(t0 + sp[i]);
            }
          }
        }
      }
      named_bar_sync(bar_id, 128);  // every thread is done with the stage
      if (wg_thread == 0) mbar_arrive(&ctl->empty[s]);
    }
  }
}

// Selected elements of every tile (mask != 0): one warp per tile, every lane
// with all of its 16-byte mask vectors in flight, a warp sum and no block
// barrier; grid-stride over tiles.
template <int TILE>
__global__ void __launch_bounds__(256) cmp_count_kernel(const int8_t* __restrict__ mask, int64_t n, int64_t num_tiles,
                                                        int* __restrict__ counts) {
  constexpr int NV = TILE / 512;  // 16-byte vectors per lane: 16, 8 or 4
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * 8;
  for (int64_t t = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); t < num_tiles; t += warps) {  // warp-uniform
    const int64_t e0 = t * TILE;
    int c = 0;
    if (e0 + TILE <= n) {
      uint4 m[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) m[v] = __ldg(reinterpret_cast<const uint4*>(mask + e0) + v * 32 + lane);
#pragma unroll
      for (int v = 0; v < NV; ++v)
        c += __popc(sel4(m[v].x) | (sel4(m[v].y) << 4) | (sel4(m[v].z) << 8) | (sel4(m[v].w) << 12));
    } else {
      for (int64_t e = e0 + lane; e < n; e += 32) c += mask[e] != 0;
    }
    c = warp_sum_any(c);
    if (lane == 0) counts[t] = c;
  }
}

// Tile offsets in two parallel passes.  Pass 1, one CTA per 1024 tiles:
// exclusive scan of the counts -> offsets relative to the block, and the
// block's total in blk[b].
__device__ __forceinline__ long long block_excl_scan1024(long long v, long long* s_w, long long* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const long long o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) s_w[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    long long w = s_w[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const long long o = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += o;
    }
    s_w[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  *total = s_w[31];
  return (wid ? s_w[wid - 1] : 0) + inc - v;
}

__global__ void __launch_bounds__(1024) cmp_offsets_local_kernel(const int* __restrict__ counts, int64_t num_tiles,
                                                                 long long* __restrict__ offsets,
                                                                 long long* __restrict__ blk, long long* count_out) {
  __shared__ long long s_w[32];
  const int64_t t = (int64_t)blockIdx.x * 1024 + threadIdx.x;
  const long long v = t < num_tiles ? counts[t] : 0;
  long long tot;
  const long long ex = block_excl_scan1024(v, s_w, &tot);
  if (t < num_tiles) offsets[t] = ex;
  if (threadIdx.x == 0) {
    blk[blockIdx.x] = tot;
    if (gridDim.x == 1) {  // one block: these are the final offsets (no second pass)
      offsets[num_tiles] = tot;
      if (count_out) *count_out = tot;
    }
  }
}

// Pass 2: each block adds the totals of the blocks before it; the last block
// writes offsets[num_tiles] = total (and *count_out).
__global__ void __launch_bounds__(1024) cmp_offsets_add_kernel(long long* __restrict__ offsets, int64_t num_tiles,
                                                               const long long* __restrict__ blk, int64_t nblk,
                                                               long long* count_out) {
  __shared__ long long s_w[32];
  long long part = 0;
  for (int64_t i = threadIdx.x; i < (int64_t)blockIdx.x; i += 1024) part += blk[i];
  long long base;
  block_excl_scan1024(part, s_w, &base);  // only the total is used
  const int64_t t = (int64_t)blockIdx.x * 1024 + threadIdx.x;
  if (t < num_tiles) offsets[t] += base;
  if (blockIdx.x == nblk - 1 && threadIdx.x == 0) {
    const long long total = base + blk[blockIdx.x];
    offsets[num_tiles] = total;
    if (count_out) *count_out = total;
  }
}

// Output position of every segment start: the number of selected elements
// before it = the offset of its tile + the selected elements between the tile
// start and the segment start.  One warp per segment start.
__global__ void __launch_bounds__(256) seg_positions_kernel(const int8_t* __restrict__ mask, int64_t n,
                                                            const long long* __restrict__ starts, int64_t nseg,
                                                            const long long* __restrict__ offsets, int64_t tile,
                                                            long long* __restrict__ pos) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (i >= nseg) return;  // warp-uniform
  long long s = starts[i];
  s = s < 0 ? 0 : (s > n ? n : s);
  const int64_t t = s / tile;
  const long long base = offsets[t];
  const int64_t e0 = t * tile;
  const int64_t len = s - e0;
  const int64_t nv = len / 16;
  const uint4* mv = reinterpret_cast<const uint4*>(mask + e0);
  unsigned long long c = 0;
  for (int64_t v = lane; v < nv; v += 32) {
    const uint4 w = __ldg(mv + v);
    c += __popc(sel4(w.x) | (sel4(w.y) << 4) | (sel4(w.z) << 8) | (sel4(w.w) << 12));
  }
  for (int64_t e = nv * 16 + lane; e < len; e += 32) c += mask[e0 + e] != 0;
  c = warp_sum_any(c);
  if (lane == 0) pos[i] = base + (long long)c;
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

// ---------------------------------------------------------------------------
// Host side.  The tile is a function of the element and index sizes; the
// per-tile counts and offsets sit in the workspace's descriptor region:
// offsets[num_tiles + 1] (int64), counts[num_tiles] (int32), then one int64
// block total per 1024 tiles.
static int64_t compress_tile(int elem_bytes, int idx_mode, int idx_bytes) {
  return 128 * cmp_ept_for(elem_bytes, idx_mode, idx_bytes);
}

struct CmpScratch {
  long long* offsets;
  int* counts;
  long long* blk;  // per 1024 tiles: the block total of the offset scan
  int64_t tiles;
  int64_t nblk;
  size_t bytes;
};

static tcu_status_t cmp_scratch(void* ws, size_t ws_bytes, int64_t n, int64_t tile, CmpScratch* sc) {
  sc->tiles = (n + tile - 1) / tile;
  sc->nblk = (sc->tiles + 1023) / 1024;
  const size_t cnt_off = (size_t)(sc->tiles + 1) * 8;
  const size_t blk_off = (cnt_off + (size_t)sc->tiles * 4 + 7) & ~(size_t)7;
  sc->bytes = blk_off + (size_t)sc->nblk * 8;
  if (!ws || ws_bytes < 128 + sc->bytes || ws_capacity(ws_bytes) * 16 < (int64_t)sc->bytes) return TCU_ERR_WORKSPACE;
  uint8_t* base = reinterpret_cast<uint8_t*>(ws_descs(ws));
  sc->offsets = reinterpret_cast<long long*>(base);
  sc->counts = reinterpret_cast<int*>(base + cnt_off);
  sc->blk = reinterpret_cast<long long*>(base + blk_off);
  return TCU_OK;
}

static tcu_status_t cmp_clear(void* ws, const CmpScratch& sc, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(ws_descs(ws), 0, sc.bytes, st);
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(compress scratch)");
}

static tcu_status_t cmp_count(const int8_t* mask, int64_t n, int64_t tile, const CmpScratch& sc, long long* count_out,
                              cudaStream_t st) {
  int64_t grid = (sc.tiles + 7) / 8;  // one warp per tile
  const int64_t cap = (int64_t)sm_count() * 8;
  if (grid > cap) grid = cap;
  if (tile == 8192) cmp_count_kernel<8192><<<(int)grid, 256, 0, st>>>(mask, n, sc.tiles, sc.counts);
  else if (tile == 4096) cmp_count_kernel<4096><<<(int)grid, 256, 0, st>>>(mask, n, sc.tiles, sc.counts);
  else cmp_count_kernel<2048><<<(int)grid, 256, 0, st>>>(mask, n, sc.tiles, sc.counts);
  if (sc.nblk > 0x7FFFFFFF) return TCU_ERR_ARG;
  cmp_offsets_local_kernel<<<(unsigned)sc.nblk, 1024, 0, st>>>(sc.counts, sc.tiles, sc.offsets, sc.blk, count_out);
  if (sc.nblk > 1)
    cmp_offsets_add_kernel<<<(unsigned)sc.nblk, 1024, 0, st>>>(sc.offsets, sc.tiles, sc.blk, sc.nblk, count_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "compress count launch");
}

template <int EB, int IDX, int IB, bool SPLIT>
static tcu_status_t launch_compress(CompressParams& p, cudaStream_t st) {
  using C = CmpCfg<EB, IDX, IB>;
  p.full_rows = p.n / C::EPT;
  p.has_map = p.full_rows > 0 ? 1 : 0;
  const int64_t rows = p.full_rows + (p.n % C::EPT ? 1 : 0);
  p.num_tiles = (rows + 127) / 128;
  if (p.num_tiles > 0x7FFFFFF0LL) return TCU_ERR_ARG;
  CUtensorMap mm{}, xm{}, im{};
  if (p.has_map) {
    tcu_status_t s = make_map_2d(&mm, p.mask, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, C::SPAN_M, p.full_rows, C::SPAN_M, 128);
    if (s == TCU_OK) s = make_map_2d(&xm, p.x, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, C::SPAN_X, p.full_rows, C::SPAN_X, 128);
    if (s == TCU_OK && IDX == 1)
      s = make_map_2d(&im, p.idx_in, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, C::SPAN_I, p.full_rows, C::SPAN_I, 128);
    if (s != TCU_OK) return s;
  }
  auto kern = compress_kernel<EB, IDX, IB, SPLIT>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(compress)");
    attr_set = true;
  }
  int grid = grid_ctas();
  if (p.num_tiles < grid) grid = (int)p.num_tiles;
  kern<<<grid, kCmpThreads, C::SMEM, st>>>(mm, xm, im, p);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "compress_kernel launch");
}

static tcu_status_t cmp_check(const void* x, int elem_bytes, const int8_t* mask, const void* idx_in, int idx_bytes,
                              int idx_mode, const void* out, const void* idx_out) {
  if (!x || !mask || !out) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(mask) || !aligned16(out)) return TCU_ERR_ALIGN;
  if (idx_mode < 0 || idx_mode > 2) return TCU_ERR_ARG;
  if (idx_mode != 0 && (!idx_out || (idx_bytes != 4 && idx_bytes != 8))) return TCU_ERR_ARG;
  if (idx_mode == 1 && (!idx_in || !aligned16(idx_in))) return idx_in ? TCU_ERR_ALIGN : TCU_ERR_ARG;
  if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return TCU_ERR_DTYPE;
  return TCU_OK;
}

// The compaction pass, with the tile offsets already in the workspace.
static tcu_status_t cmp_run(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in,
                            int idx_bytes, int idx_mode, void* out, void* idx_out, int64_t capacity,
                            const CmpScratch& sc, void* ws, cudaStream_t st, bool split = false) {
  CompressParams p{};
  p.x = x;
  p.mask = mask;
  p.idx_in = idx_in;
  p.out = out;
  p.idx_out = idx_out;
  p.n = n;
  p.capacity = capacity;
  p.offsets = sc.offsets;
  p.ws = static_cast<WsHeader*>(ws);
  p.timeout_ns = timeout_ns();
  if (split) {  // stable partition: values only or with gathered indices
#define TCU_SPL(EB)                                                        \
  if (idx_mode == 0) return launch_compress<EB, 0, 0, true>(p, st);       \
  if (idx_bytes == 4) return launch_compress<EB, 1, 4, true>(p, st);      \
  return launch_compress<EB, 1, 8, true>(p, st)
    if (idx_mode == 2) return TCU_ERR_ARG;
    switch (elem_bytes) {
      case 1: TCU_SPL(1);
      case 2: TCU_SPL(2);
      case 4: TCU_SPL(4);
      default: TCU_SPL(8);
    }
#undef TCU_SPL
  }
#define TCU_CMP(EB, IDX, IB) return launch_compress<EB, IDX, IB, false>(p, st)
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
    default:
      if (idx_mode == 0) TCU_CMP(8, 0, 0);
      if (idx_mode == 1) { if (idx_bytes == 4) TCU_CMP(8, 1, 4); TCU_CMP(8, 1, 8); }
      if (idx_bytes == 4) TCU_CMP(8, 2, 4);
      TCU_CMP(8, 2, 8);
  }
#undef TCU_CMP
}

static tcu_status_t zero_count(void* count_dev, cudaStream_t st) {
  if (!count_dev) return TCU_OK;
  cudaError_t e = cudaMemsetAsync(count_dev, 0, sizeof(long long), st);
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(count)");
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

tcu_status_t tcu_compress_count(const int8_t* mask, int64_t n, int elem_bytes, int idx_mode, int idx_bytes,
                                void* count_dev, void* ws, size_t ws_bytes, void* stream) {
  if (n < 0) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) return zero_count(count_dev, st);
  if (!mask) return TCU_ERR_ARG;
  if (!aligned16(mask) || (reinterpret_cast<uintptr_t>(count_dev) & 7u)) return TCU_ERR_ALIGN;
  if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return TCU_ERR_DTYPE;
  const int64_t tile = compress_tile(elem_bytes, idx_mode, idx_bytes);
  CmpScratch sc;
  tcu_status_t s = cmp_scratch(ws, ws_bytes, n, tile, &sc);
  if (s != TCU_OK) return s;
  return cmp_count(mask, n, tile, sc, static_cast<long long*>(count_dev), st);
}

tcu_status_t tcu_compress_counted(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in,
                                  int idx_bytes, int idx_mode, void* out, void* idx_out, int64_t capacity, void* ws,
                                  size_t ws_bytes, void* stream) {
  if (n < 0 || capacity < 0) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) return TCU_OK;
  tcu_status_t s = cmp_check(x, elem_bytes, mask, idx_in, idx_bytes, idx_mode, out, idx_out);
  if (s != TCU_OK) return s;
  CmpScratch sc;
  s = cmp_scratch(ws, ws_bytes, n, compress_tile(elem_bytes, idx_mode, idx_bytes), &sc);
  if (s != TCU_OK) return s;
  s = cmp_run(x, elem_bytes, mask, n, idx_in, idx_bytes, idx_mode, out, idx_out, capacity, sc, ws, st);
  if (s != TCU_OK) return s;
  return cmp_clear(ws, sc, st);
}

tcu_status_t tcu_compress(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in,
                          int idx_bytes, int idx_mode, void* out, void* idx_out, int64_t capacity, void* count_dev,
                          void* ws, size_t ws_bytes, void* stream) {
  if (n < 0 || capacity < 0) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) return zero_count(count_dev, st);
  tcu_status_t s = cmp_check(x, elem_bytes, mask, idx_in, idx_bytes, idx_mode, out, idx_out);
  if (s != TCU_OK) return s;
  if (reinterpret_cast<uintptr_t>(count_dev) & 7u) return TCU_ERR_ALIGN;
  const int64_t tile = compress_tile(elem_bytes, idx_mode, idx_bytes);
  CmpScratch sc;
  s = cmp_scratch(ws, ws_bytes, n, tile, &sc);
  if (s == TCU_OK) s = cmp_count(mask, n, tile, sc, static_cast<long long*>(count_dev), st);
  if (s == TCU_OK) s = cmp_run(x, elem_bytes, mask, n, idx_in, idx_bytes, idx_mode, out, idx_out, capacity, sc, ws, st);
  if (s != TCU_OK) return s;
  return cmp_clear(ws, sc, st);
}

tcu_status_t tcu_compress_segments(const void* x, int elem_bytes, const int8_t* mask, int64_t n,
                                   const int64_t* seg_starts, int64_t nseg, void* out, int64_t capacity,
                                   int64_t* seg_pos, void* ws, size_t ws_bytes, void* stream) {
  if (n < 0 || nseg < 0 || capacity < 0 || !seg_pos || (nseg > 0 && !seg_starts)) return TCU_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(seg_pos) & 7u) || (reinterpret_cast<uintptr_t>(seg_starts) & 7u))
    return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) {
    cudaError_t e = cudaMemsetAsync(seg_pos, 0, (size_t)(nseg + 1) * sizeof(int64_t), st);
    return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(seg_pos)");
  }
  tcu_status_t s = cmp_check(x, elem_bytes, mask, nullptr, 0, 0, out, nullptr);
  if (s != TCU_OK) return s;
  const int64_t tile = compress_tile(elem_bytes, 0, 0);
  CmpScratch sc;
  s = cmp_scratch(ws, ws_bytes, n, tile, &sc);
  if (s == TCU_OK) s = cmp_count(mask, n, tile, sc, reinterpret_cast<long long*>(seg_pos + nseg), st);
  if (s == TCU_OK) s = cmp_run(x, elem_bytes, mask, n, nullptr, 0, 0, out, nullptr, capacity, sc, ws, st);
  if (s != TCU_OK) return s;
  if (nseg > 0) {
    const int64_t blocks = (nseg * 32 + 255) / 256;
    if (blocks > 0x7FFFFFFF) return TCU_ERR_ARG;
    seg_positions_kernel<<<(unsigned)blocks, 256, 0, st>>>(mask, n, reinterpret_cast<const long long*>(seg_starts),
                                                           nseg, sc.offsets, tile,
                                                           reinterpret_cast<long long*>(seg_pos));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "seg_positions_kernel launch");
  }
  return cmp_clear(ws, sc, st);
}

// Stable partition (the reference's run_split / run_split_ind,
// src/torch/torch_split.h:33-79 and :91-142): out[0, k) = x[mask != 0],
// out[k, n) = x[mask == 0], both in input order; with idx_mode 1 the same
// permutation is applied to idx_in.  One count pass, one offset scan, one
// streaming pass that writes both runs of every tile.
tcu_status_t tcu_split(const void* x, int elem_bytes, const int8_t* mask, int64_t n, const void* idx_in, int idx_bytes,
                       int idx_mode, void* out, void* idx_out, void* count_dev, void* ws, size_t ws_bytes,
                       void* stream) {
  if (n < 0) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) return zero_count(count_dev, st);
  if (idx_mode != 0 && idx_mode != 1) return TCU_ERR_ARG;
  tcu_status_t s = cmp_check(x, elem_bytes, mask, idx_in, idx_bytes, idx_mode, out, idx_out);
  if (s != TCU_OK) return s;
  if (reinterpret_cast<uintptr_t>(count_dev) & 7u) return TCU_ERR_ALIGN;
  const int64_t tile = compress_tile(elem_bytes, idx_mode, idx_bytes);
  CmpScratch sc;
  s = cmp_scratch(ws, ws_bytes, n, tile, &sc);
  if (s == TCU_OK) s = cmp_count(mask, n, tile, sc, static_cast<long long*>(count_dev), st);
  if (s == TCU_OK) s = cmp_run(x, elem_bytes, mask, n, idx_in, idx_bytes, idx_mode, out, idx_out, n, sc, ws, st, true);
  if (s != TCU_OK) return s;
  return cmp_clear(ws, sc, st);
}

}  // extern "C"

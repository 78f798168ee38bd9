// tcu_scan_tc.cuh -- the tensor-core scan kernel family (sm_100a).
//
// The reference computes local prefix sums on the matrix unit: the input is
// viewed as rows of S elements, each row block is multiplied by the constant
// upper-triangular all-ones matrix U (z = x . U gives every row's inclusive
// prefix), and the vector cores then propagate carries across rows and blocks
// (src/kernels/kernel_row_scan.h:19-46, kernel_complete_rows.h:99-161).
//
// B200 design, one persistent CTA per SM, warp-specialised:
//   warp 0      TMA producer: fetches chunk ids from a global counter and
//               loads each chunk (128 rows x S elements) into a 4-stage
//               swizzled SMEM ring with cp.async.bulk.tensor.
//   warp 1      MMA issuer: tcgen05.mma (kind::i8 -> s32 or kind::f16 -> f32)
//               of the chunk against U (built once in SMEM), accumulator in
//               a TMEM ring; tcgen05.commit frees the stage / fills TMEM.
//   warps 2-9   two epilogue warpgroups taking alternate chunks: tcgen05.ld
//               of the row prefixes (thread = row), warp-shuffle scan of the
//               row totals, decoupled look-back across chunks (Merrill &
//               Garland 2016) with an FP64 / int64 carry chain, carry add,
//               swizzled SMEM staging and TMA store of the output rows.
// The last partial row (n % S elements) is scanned by its owning epilogue
// thread from global memory; TMA never touches memory past the last full row.
#pragma once

#include <cuda.h>

#include "tcu_device.cuh"

namespace tcu {

enum ScanMode : int {
  kScanFull = 0,    // full inclusive scan with look-back carries (MCSCAN)
  kScanRows = 1,    // per-row (length S) scans only (row_scan)
  kScanBlocks = 2,  // scans restarting every seg_rows rows (block_scan)
};

struct ScanParams {
  const void* x;      // input base (tail row loads)
  void* z;            // output base (tail row stores)
  int64_t n;          // elements
  int64_t full_rows;  // n / W
  int32_t tail;       // n % W
  int32_t seg_rows;   // kScanBlocks: rows per segment
  int64_t num_chunks;
  double start_f;     // starting value (run_scan_single_core's starting_sum)
  long long start_i;
  WsHeader* ws;
  uint32_t* flags;
  LbValue* vals;
  uint64_t timeout_ns;
  int has_in_map;
  int has_out_map;
};

constexpr uint32_t kSentinel = 0xFFFFFFFFu;
constexpr int kThreads = 320;  // 10 warps

template <typename InT, int W>
struct ScanCfg {
  static constexpr int ELEM = (int)sizeof(InT);
  static constexpr bool IS_INT = (ELEM == 1);
  static constexpr int RB = W * ELEM;                 // row bytes
  static constexpr int SW = RB < 128 ? RB : 128;      // swizzle span
  static constexpr int KB = RB / SW;                  // K blocks of SW bytes
  static constexpr int KSTEPS = SW / 32;              // 32-byte MMA K steps per block
  static constexpr int STAGE_BYTES = 128 * RB;
  static constexpr int NSTAGE = STAGE_BYTES <= 16384 ? 4 : 3;
  static constexpr int NACC = (512 / W) < 8 ? (512 / W) : 8;
  static constexpr int TMEM_NEED = NACC * W;
  static constexpr int TMEM_COLS = TMEM_NEED <= 32 ? 32 : (TMEM_NEED <= 64 ? 64 : (TMEM_NEED <= 128 ? 128 : (TMEM_NEED <= 256 ? 256 : 512)));
  static constexpr int B_BYTES = W * RB;
  static constexpr int OBW = W < 32 ? W : 32;         // output TMA box width (elements)
  static constexpr int OSW = OBW * 4;                 // output box row bytes = swizzle span
  static constexpr int FILLW = W < 64 ? W : 64;       // columns staged per fill
  static constexpr int NFILL = W / FILLW;
  static constexpr int STG_BYTES = 128 * FILLW * 4;
  static constexpr int OFF_B = NSTAGE * STAGE_BYTES;
  static constexpr int OFF_STG = OFF_B + ((B_BYTES + 1023) / 1024) * 1024;
  static constexpr int OFF_CTRL = OFF_STG + 2 * STG_BYTES;
  static constexpr int CTRL_BYTES = 1024;
  static constexpr int SMEM_BYTES = OFF_CTRL + CTRL_BYTES + 1024;  // + alignment slack
  static_assert(W == 16 || W == 32 || W == 64 || W == 128, "S");
  static_assert(RB >= 32, "row must hold one 32-byte MMA K step");
};

struct ScanCtrl {
  uint64_t full[4];
  uint64_t empty[4];
  uint64_t tfull[8];
  uint64_t tempty[8];
  uint64_t drain;
  uint32_t stage_cid[4];
  uint32_t acc_cid[8];
  uint32_t tmem_base;
  uint32_t epoch;
  int abort_flag;
  int pad;
  double wsum_f[2][4];
  long long wsum_i[2][4];
  int wflag[2][4];
  int wait_ok[2][4];
  double prefix_f[2];
  long long prefix_i[2];
};

// Value of 1 in the MMA operand encoding.
template <typename T>
__device__ __forceinline__ uint32_t one_bits();
template <>
__device__ __forceinline__ uint32_t one_bits<int8_t>() { return 0x01u; }
template <>
__device__ __forceinline__ uint32_t one_bits<__half>() { return 0x3C00u; }
template <>
__device__ __forceinline__ uint32_t one_bits<__nv_bfloat16>() { return 0x3F80u; }

template <typename T>
__device__ __forceinline__ float load_elem(const T* p);
template <>
__device__ __forceinline__ float load_elem<__half>(const __half* p) { return __half2float(*p); }
template <>
__device__ __forceinline__ float load_elem<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// ---------------------------------------------------------------------------
// Segmented carry operator on (flag, value): (f1,v1) + (f2,v2) =
// (f1|f2, f2 ? v2 : v1+v2).  Plain scans only ever use flag = 0.
template <typename V>
__device__ __forceinline__ void seg_combine(int& f, V& v, int f_prev, V v_prev) {
  if (!f) v = v_prev + v;
  f |= f_prev;
}

template <typename V>
__device__ __forceinline__ V shfl_up_v(V v, int d) {
  return __shfl_up_sync(0xffffffffu, v, d);
}

template <typename V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// ---------------------------------------------------------------------------
// Decoupled look-back for chunk `cid`, run by one full warp.  Publishes the
// chunk aggregate, then walks predecessors 32 at a time until it meets an
// inclusive prefix (or the start of the input) and returns the exclusive
// prefix of the chunk.  V = double (floating scans) or long long (integer).
template <typename V>
__device__ __forceinline__ V lookback(uint32_t cid, V agg, V start, const ScanParams& p, uint32_t epoch,
                                      const WaitCtx& wc) {
  const int lane = threadIdx.x & 31;
  const uint32_t tag = (epoch & 0x1FFFFFFFu) << 3;
  auto put_val = [&](LbValue& lv, V v, bool inc) {
    if constexpr (__is_same(V, double)) {
      if (inc) lv.inc_f = v; else lv.agg_f = v;
    } else {
      if (inc) lv.inc_i = v; else lv.agg_i = v;
    }
  };
  if (cid == 0) {
    if (lane == 0) {
      put_val(p.vals[0], start + agg, true);
      st_release_u32(p.flags, tag | LB_INC);
    }
    return start;
  }
  if (lane == 0) {
    put_val(p.vals[cid], agg, false);
    st_release_u32(p.flags + cid, tag | LB_AGG);
  }
  V acc = V(0);
  int64_t pos = (int64_t)cid - 1;
  while (true) {
    const int64_t idx = pos - lane;
    uint32_t state;
    V val;
    if (idx < 0) {
      state = LB_INC;
      val = (idx == -1) ? start : V(0);
    } else {
      uint32_t f = ld_acquire_u32(p.flags + idx);
      if ((f & ~7u) != tag || (f & 3u) == 0u) {
        const uint64_t t0 = globaltimer();
        uint32_t it = 0;
        while (true) {
          f = ld_acquire_u32(p.flags + idx);
          if ((f & ~7u) == tag && (f & 3u) != 0u) break;
          if (aborted(wc)) { f = tag | LB_INC; break; }
          if ((++it & 31u) == 0u && globaltimer() - t0 > wc.timeout_ns) {
            raise_abort(wc, 100, cid);
            f = tag | LB_INC;
            break;
          }
        }
      }
      state = f & 3u;
      if constexpr (__is_same(V, double)) {
        val = ld_relaxed_f64(state == LB_INC ? &p.vals[idx].inc_f : &p.vals[idx].agg_f);
      } else {
        val = ld_relaxed_s64(state == LB_INC ? &p.vals[idx].inc_i : &p.vals[idx].agg_i);
      }
      if (aborted(wc)) val = V(0);
    }
    const uint32_t m = __ballot_sync(0xffffffffu, state == LB_INC);
    if (m) {
      const int j = __ffs(m) - 1;
      acc += warp_sum(lane <= j ? val : V(0));
      break;
    }
    acc += warp_sum(val);
    pos -= 32;
  }
  if (lane == 0) {
    put_val(p.vals[cid], acc + agg, true);
    st_release_u32(p.flags + cid, tag | LB_INC);
  }
  return acc;
}

// ---------------------------------------------------------------------------
template <typename InT, int W, int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    scan_tc_kernel(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap out_map,
                   const ScanParams p) {
  using C = ScanCfg<InT, W>;
  constexpr bool IS_INT = C::IS_INT;
  using V = typename std::conditional<IS_INT, long long, double>::type;

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  ScanCtrl* ctl = (ScanCtrl*)(smem + C::OFF_CTRL);
  uint8_t* bmat = smem + C::OFF_B;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  WaitCtx wc{p.ws, &ctl->abort_flag, p.timeout_ns};

  // ---- setup ----
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::NSTAGE; ++s) {
      mbar_init(&ctl->full[s], 1);
      mbar_init(&ctl->empty[s], 1);
    }
    for (int a = 0; a < C::NACC; ++a) {
      mbar_init(&ctl->tfull[a], 2);  // tcgen05.commit + releasing arrive after acc_cid
      mbar_init(&ctl->tempty[a], 4);
    }
    mbar_init(&ctl->drain, 1);
    ctl->abort_flag = 0;
    ctl->epoch = *(volatile uint32_t*)&p.ws->epoch;
    fence_mbar_init();
  }
  // Constant operand B (K-major): row n holds U[k][n] = (k <= n).
  {
    constexpr int CPR = C::RB / 16;  // 16-byte chunks per row
    const uint32_t one = one_bits<InT>();
    for (int t = threadIdx.x; t < W * CPR; t += kThreads) {
      const int nrow = t / CPR, c = t % CPR;
      const int kb = (c * 16) / C::SW, cin = c % (C::SW / 16);
      const int k0 = (kb * C::SW + cin * 16) / C::ELEM;
      uint32_t w[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t word = 0;
        if (C::ELEM == 1) {
#pragma unroll
          for (int b = 0; b < 4; ++b) word |= ((k0 + q * 4 + b) <= nrow ? one : 0u) << (8 * b);
        } else {
#pragma unroll
          for (int b = 0; b < 2; ++b) word |= ((k0 + q * 2 + b) <= nrow ? one : 0u) << (16 * b);
        }
        w[q] = word;
      }
      uint8_t* dst = bmat + kb * (W * C::SW) + swz(nrow * C::SW + cin * 16, C::SW);
      *(uint4*)dst = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
  fence_proxy_async_smem();
  if (warp == 1) {
    tmem_alloc(&ctl->tmem_base, C::TMEM_COLS);
    tmem_relinquish();
  }
  if (warp == 0 && lane == 0 && p.has_in_map) prefetch_tmap(&in_map);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = ctl->tmem_base;
  const uint32_t epoch = ctl->epoch;

  if (warp == 0) {
    // ================= TMA producer =================
    if (lane == 0) {
      uint32_t issued[4] = {0, 0, 0, 0};
      uint32_t next = atomicAdd(&p.ws->chunk_counter, 1u);
      for (uint32_t i = 0;; ++i) {
        const int s = i % C::NSTAGE;
        if (i >= (uint32_t)C::NSTAGE) {
          if (!mbar_wait(&ctl->empty[s], ((i / C::NSTAGE) & 1u) ^ 1u, wc, 1, next)) break;
        }
        const uint32_t cid = next;
        const bool live = (int64_t)cid < p.num_chunks;
        if (live) next = atomicAdd(&p.ws->chunk_counter, 1u);
        ctl->stage_cid[s] = live ? cid : kSentinel;
        issued[s]++;
        const int64_t row0 = (int64_t)cid * 128;
        if (live && p.has_in_map && row0 < p.full_rows) {
          mbar_arrive_expect_tx(&ctl->full[s], C::STAGE_BYTES);
#pragma unroll
          for (int kb = 0; kb < C::KB; ++kb) {
            tma_load_2d(smem + s * C::STAGE_BYTES + kb * (128 * C::SW), &in_map, kb * (C::SW / C::ELEM),
                        (int32_t)row0, &ctl->full[s]);
          }
        } else {
          mbar_arrive(&ctl->full[s]);
        }
        if (!live || aborted(wc)) break;
      }
      // drain: every load issued must have landed before the CTA exits
      for (int s = 0; s < C::NSTAGE; ++s)
        if (issued[s]) mbar_drain(&ctl->full[s], (issued[s] - 1) & 1u, p.timeout_ns);
    }
  } else if (warp == 1) {
    // ================= MMA issuer =================
    if (lane == 0) {
      constexpr uint32_t IDESC = IS_INT ? umma_idesc(CF_S32, AB_S8, 128, W)
                                        : umma_idesc(CF_F32, __is_same(InT, __nv_bfloat16) ? AB_BF16 : AB_F16, 128, W);
      const uint32_t b_addr = smem_u32(bmat);
      for (uint32_t i = 0;; ++i) {
        const int s = i % C::NSTAGE;
        if (!mbar_wait(&ctl->full[s], (i / C::NSTAGE) & 1u, wc, 2, i)) break;
        const uint32_t cid = *(volatile uint32_t*)&ctl->stage_cid[s];
        const int a = i % C::NACC;
        if (i >= (uint32_t)C::NACC) {
          if (!mbar_wait(&ctl->tempty[a], ((i / C::NACC) & 1u) ^ 1u, wc, 3, cid)) break;
        }
        if (cid == kSentinel) {
          ctl->acc_cid[a] = kSentinel;
          mbar_arrive(&ctl->tfull[a]);
          mbar_arrive(&ctl->tfull[a]);
          const uint32_t i2 = i + 1;
          const int a2 = i2 % C::NACC;
          if (i2 >= (uint32_t)C::NACC) {
            if (!mbar_wait(&ctl->tempty[a2], ((i2 / C::NACC) & 1u) ^ 1u, wc, 4, cid)) break;
          }
          ctl->acc_cid[a2] = kSentinel;
          mbar_arrive(&ctl->tfull[a2]);
          mbar_arrive(&ctl->tfull[a2]);
          break;
        }
        ctl->acc_cid[a] = cid;
        mbar_arrive(&ctl->tfull[a]);  // releases the acc_cid store to the epilogue
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(a * W);
        const uint32_t a_addr = smem_u32(smem + s * C::STAGE_BYTES);
#pragma unroll
        for (int kb = 0; kb < C::KB; ++kb) {
#pragma unroll
          for (int ks = 0; ks < C::KSTEPS; ++ks) {
            const uint64_t ad = umma_desc_kmajor(a_addr + kb * (128 * C::SW) + ks * 32, C::SW);
            const uint64_t bd = umma_desc_kmajor(b_addr + kb * (W * C::SW) + ks * 32, C::SW);
            if constexpr (IS_INT) {
              mma_i8(d_tmem, ad, bd, IDESC, (kb | ks) != 0);
            } else {
              mma_f16(d_tmem, ad, bd, IDESC, (kb | ks) != 0);
            }
          }
        }
        tc_commit(&ctl->empty[s]);
        tc_commit(&ctl->tfull[a]);
      }
      tc_commit(&ctl->drain);
      mbar_drain(&ctl->drain, 0, p.timeout_ns);
    }
  } else {
    // ================= epilogue warpgroups =================
    const int g = (warp - 2) >> 2;           // warpgroup 0 / 1
    const int q = warp & 3;                  // TMEM lane quarter
    const int r = q * 32 + lane;             // row within the chunk
    const int wg_thread = threadIdx.x - 64 - g * 128;
    const uint32_t bar_id = 1 + g;
    uint8_t* stg = smem + C::OFF_STG + g * C::STG_BYTES;
    const V start = IS_INT ? (V)p.start_i : (V)p.start_f;

    for (uint32_t i = g;; i += 2) {
      const int a = i % C::NACC;
      // One lane per warp waits; the four warps then vote at a named barrier
      // that all of them always reach, so an abort is warpgroup-uniform and
      // no warp is ever left waiting at a barrier the others skipped.
      int ok = 1;
      if (lane == 0) ok = mbar_wait(&ctl->tfull[a], (i / C::NACC) & 1u, wc, 5, i) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (lane == 0) ctl->wait_ok[g][q] = ok;
      named_bar_sync(bar_id, 128);
      const int all_ok = ctl->wait_ok[g][0] & ctl->wait_ok[g][1] & ctl->wait_ok[g][2] & ctl->wait_ok[g][3];
      if (!all_ok) break;
      const uint32_t cid = *(volatile uint32_t*)&ctl->acc_cid[a];
      if (cid == kSentinel) break;
      tc_fence_after();
      uint32_t v[W];
#pragma unroll
      for (int c = 0; c < W / 16; ++c) {
        tmem_ld16(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * W + c * 16),
                  *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]));
      }
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ctl->tempty[a]);

      const int64_t grow = (int64_t)cid * 128 + r;
      const bool is_full = grow < p.full_rows;
      const bool is_tail = (grow == p.full_rows) && p.tail > 0;
      if (is_tail) {
        // partial last row: scan it from global memory (< W elements)
        const int64_t base = p.full_rows * W;
        if constexpr (IS_INT) {
          int acc = 0;
          const int8_t* xs = (const int8_t*)p.x + base;
#pragma unroll
          for (int j = 0; j < W; ++j) {
            if (j < p.tail) acc += xs[j];
            v[j] = (uint32_t)acc;
          }
        } else {
          float acc = 0.f;
          const InT* xs = (const InT*)p.x + base;
#pragma unroll
          for (int j = 0; j < W; ++j) {
            if (j < p.tail) acc += load_elem<InT>(xs + j);
            v[j] = __float_as_uint(acc);
          }
        }
      } else if (!is_full) {
#pragma unroll
        for (int j = 0; j < W; ++j) v[j] = 0u;
      }

      V carry = V(0);
      if constexpr (MODE != kScanRows) {
        // row totals -> segmented warp scan -> cross-warp -> chunk look-back
        V t = IS_INT ? (V)(int)v[W - 1] : (V)__uint_as_float(v[W - 1]);
        int f = (MODE == kScanBlocks) ? (int)((grow % p.seg_rows) == 0) : 0;
        V ti = t;
        int fi = f;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const V tp = shfl_up_v(ti, d);
          const int fp = __shfl_up_sync(0xffffffffu, fi, d);
          if (lane >= d) seg_combine(fi, ti, fp, tp);
        }
        // exclusive within the warp
        V te = shfl_up_v(ti, 1);
        int fe = __shfl_up_sync(0xffffffffu, fi, 1);
        if (lane == 0) { te = V(0); fe = 0; }
        if (lane == 31) {
          if constexpr (IS_INT) ctl->wsum_i[g][q] = ti; else ctl->wsum_f[g][q] = ti;
          ctl->wflag[g][q] = fi;
        }
        if (wg_thread == 0) bulk_wait_read0();  // staging buffer free again
        named_bar_sync(bar_id, 128);
        // prefix of the warps before this one, and the chunk aggregate
        V wpre = V(0);
        int wf = 0;
        V agg = V(0);
        int af = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const V wv = IS_INT ? (V)ctl->wsum_i[g][k] : (V)ctl->wsum_f[g][k];
          const int wfl = ctl->wflag[g][k];
          if (k < q) { if (wfl) { wpre = wv; wf = 1; } else { wpre += wv; } }
          if (wfl) { agg = wv; af = 1; } else { agg += wv; }
        }
        (void)af;
        // row exclusive carry within the chunk = warp prefix (+) lane exclusive
        V rex = te;
        int rf = fe;
        if (!rf) rex = wpre + rex;
        rf |= wf;
        if constexpr (MODE == kScanFull) {
          if (q == 0) {
            const V pre = lookback<V>(cid, agg, start, p, epoch, wc);
            if (lane == 0) {
              if constexpr (IS_INT) ctl->prefix_i[g] = pre; else ctl->prefix_f[g] = pre;
            }
          }
          named_bar_sync(bar_id, 128);
          const V pre = IS_INT ? (V)ctl->prefix_i[g] : (V)ctl->prefix_f[g];
          carry = rf ? rex : pre + rex;
        } else {
          // kScanBlocks: every chunk starts a new segment; a row that starts
          // a segment takes no carry at all.
          carry = f ? V(0) : rex;
        }
      } else {
        if (wg_thread == 0) bulk_wait_read0();
        named_bar_sync(bar_id, 128);
      }

      // ---- carry add, SMEM staging, TMA store ----
#pragma unroll
      for (int h = 0; h < C::NFILL; ++h) {
        if (h > 0) {
          if (wg_thread == 0) bulk_wait_read0();
          named_bar_sync(bar_id, 128);
        }
#pragma unroll
        for (int j4 = 0; j4 < C::FILLW / 4; ++j4) {
          const int col = h * C::FILLW + j4 * 4;
          uint32_t o[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if constexpr (IS_INT) {
              o[e] = (uint32_t)((long long)(int)v[col + e] + carry);
            } else {
              o[e] = __float_as_uint(__uint_as_float(v[col + e]) + (float)carry);
            }
          }
          const int box = (j4 * 4) / C::OBW;
          const int cin = (j4 * 4) % C::OBW;
          uint8_t* dst = stg + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW);
          *(uint4*)dst = make_uint4(o[0], o[1], o[2], o[3]);
          if (is_tail) {
            uint32_t* zt = (uint32_t*)p.z + p.full_rows * W;
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (col + e < p.tail) zt[col + e] = o[e];
          }
        }
        fence_proxy_async_smem();
        named_bar_sync(bar_id, 128);
        if (wg_thread == 0 && p.has_out_map && (int64_t)cid * 128 < p.full_rows) {
#pragma unroll
          for (int b = 0; b < C::FILLW / C::OBW; ++b)
            tma_store_2d(&out_map, h * C::FILLW + b * C::OBW, (int32_t)((int64_t)cid * 128), stg + b * (128 * C::OSW));
          bulk_commit();
        }
      }
    }
    if (wg_thread == 0) bulk_wait_all0();
  }

  // ---- teardown ----
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, C::TMEM_COLS);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t prev = atomicAdd(&p.ws->done_ctas, 1u);
    if (prev == gridDim.x - 1) {
      p.ws->chunk_counter = 0;
      p.ws->done_ctas = 0;
      __threadfence();
      atomicAdd(&p.ws->epoch, 1u);
    }
  }
}

}  // namespace tcu

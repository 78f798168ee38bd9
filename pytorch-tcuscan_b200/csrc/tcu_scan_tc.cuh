// tcu_scan_tc.cuh -- the tensor-core scan kernel family (sm_100a).
//
// The reference computes local prefix sums on the matrix unit: the input is
// viewed as rows of S elements, each row block is multiplied by the constant
// upper-triangular all-ones matrix U (z = x . U gives every row's inclusive
// prefix), and the vector cores then propagate carries across rows and blocks
// (src/kernels/kernel_row_scan.h:19-46, kernel_complete_rows.h:99-161).
//
// B200 design, one persistent CTA per SM, warp-specialised:
//   warp 0      TMA producer: fetches tile ids from a global counter; a tile
//               is 256/S blocks of 128 rows x S elements (32768 elements),
//               loaded block by block into a swizzled SMEM ring with
//               cp.async.bulk.tensor.
//   warp 1      MMA issuer: tcgen05.mma (kind::i8 -> s32, kind::f16 -> f32) of
//               every block against U (built once in SMEM); a tile's blocks
//               fill one 256-column half of TMEM (one half per warpgroup).
//   warps 2-9   two epilogue warpgroups taking alternate tiles.  Per tile:
//               (A) tcgen05.ld of each block's last column = row totals,
//               warp-shuffle scans -> row offsets and the tile aggregate;
//               (B) decoupled look-back over a 512-tile window (FP64 / int64
//               carry chain); (C) drain: tcgen05.ld of every row, carry add,
//               swizzled SMEM staging (double buffered), TMA store; each
//               block's TMEM columns are released as soon as they are read.
// The last partial row (n % S elements) is scanned by its owning epilogue
// thread from global memory; TMA never touches memory past the last full row.
#pragma once

#include <cuda.h>

#include "tcu_lookback.cuh"

namespace tcu {

// fp32 input already split into bf16 operands: every 64-element row is
// stored as 64 bf16 hi = RN(x) then 64 bf16 lo = RN(x - hi) (256 bytes, the
// size of the fp32 row), so the two TMA boxes of a row land as the hi and lo
// MMA operand rows and no conversion pass is needed.  Written by the SpMV
// products kernel.
struct SplitF32 {
  uint32_t bits;
};

enum ScanMode : int {
  kScanFull = 0,     // full inclusive scan with look-back carries (MCSCAN)
  kScanRows = 1,     // per-row (length S) scans only (row_scan)
  kScanBlocks = 2,   // scans restarting every seg_rows rows (block_scan)
  kSegFlags = 3,     // segmented scan, int8 flags mark segment starts (seg_scan)
  kSegEnds = 4,      // segmented scan, int8 flags mark segment ends (seg_sum)
  kSegBounds = 5,    // segments from a sorted start array (indptr / offsets)
  kSegPeriodic = 6,  // segments of a fixed length (scan_batch)
  kScanFullSmall = 7,  // kScanFull with one 128 x W block per tile (small inputs: every SM gets a tile)
};
constexpr bool is_seg(int mode) { return mode >= kSegFlags && mode <= kSegPeriodic; }
constexpr bool is_full(int mode) { return mode == kScanFull || mode == kScanFullSmall; }

struct ScanParams {
  const void* x;      // input base (tail row loads)
  void* z;            // output base (tail row stores)
  int64_t n;          // elements
  int64_t full_rows;  // n / W
  int32_t tail;       // n % W
  int32_t seg_rows;   // kScanBlocks: rows per segment
  int64_t num_tiles;
  double start_f;     // starting value (run_scan_single_core's starting_sum)
  long long start_i;
  const void* start_dev;  // optional: one value added to the start, read when the kernel runs (chained chunks)
  int start_dev_kind;     // its type: 0 int32, 1 fp32, 2 int64, 3 fp64
  WsHeader* ws;
  TileDesc* descs;
  uint64_t timeout_ns;
  int has_map;        // full_rows > 0: TMA maps are valid
  unsigned long long* phase_ns;  // optional per-phase time counters (nullptr = off)
  // segmented modes
  const int8_t* flags;   // kSegFlags / kSegEnds
  const void* bounds;    // kSegBounds: non-decreasing segment starts
  int64_t nbounds;
  int bounds64;          // bounds are int64 (else int32)
  int out_sums;          // kSegBounds: write one sum per segment instead of the scan
  int64_t period;        // kSegPeriodic
  void* seg_out;         // kSegBounds sums: nbounds - 1 entries (fp32 / int32)
  const long long* tile_first;  // kSegBounds: first bound index of every tile (precomputed)
};

// Phase counters (nanoseconds summed over warpgroups / roles):
// 0 epilogue wait for the MMA, 1 row totals, 2 look-back, 3 drain,
// 4 producer waits for free stages, 5 summer (including its waits for data),
// 6 summer waits for landed data (part of 5), 7 tiles processed.
__device__ __forceinline__ void phase_add(const ScanParams& p, int k, uint64_t dt) {
  if (p.phase_ns) atomicAdd(p.phase_ns + k, (unsigned long long)dt);
}

constexpr uint32_t kSentinel = 0xFFFFFFFFu;
constexpr int kThreads = 384;  // 12 warps: producer, MMA, 2 epilogue warpgroups, summer, second summer / converter
constexpr int kMaxSmem = 232448;

template <typename InT, int W, bool SEG = false, bool SMALL = false>
struct ScanCfg {
  static constexpr int IN_BYTES = (int)sizeof(InT);   // input element bytes
  static constexpr bool IS_F32 = (IN_BYTES == 4);     // fp32: split into two 16-bit operands
  static constexpr bool PRESPLIT = __is_same(InT, SplitF32);  // ... already split in memory (bf16 hi + lo)
  // fp32 input split in SMEM into scaled fp16 hi + lo operands, with every
  // row's exact total computed from the fp32 values (convert_f32_rows)
  static constexpr bool F16SPLIT = IS_F32 && !PRESPLIT;
  static constexpr int ELEM = IS_F32 ? 2 : IN_BYTES;  // MMA operand element bytes
  static constexpr bool IS_INT = (IN_BYTES == 1);
  static constexpr int RB = W * ELEM;                 // operand row bytes
  static constexpr int SW = RB < 128 ? RB : 128;      // operand swizzle span
  static constexpr int KB = RB / SW;                  // K blocks of SW bytes
  static constexpr int KSTEPS = SW / 32;              // 32-byte MMA K steps per block
  static constexpr int IN_RB = W * IN_BYTES;          // input row bytes (TMA geometry)
  static constexpr int IN_SW = IN_RB < 128 ? IN_RB : 128;
  static constexpr int IN_KB = IN_RB / IN_SW;
  static constexpr int STAGE_BYTES = 128 * IN_RB;
  static constexpr int TERM_BYTES = 128 * RB;         // fp32: hi operand at 0, lo at TERM_BYTES
  static constexpr int BPT = SMALL ? 1 : 256 / W;     // blocks per tile
  static constexpr int TILE_ELEMS = 128 * W * BPT;
  static constexpr int B_BYTES = W * RB;
  // columns staged per fill: whole rows up to 64 columns.  Narrower,
  // double-buffered fills (32 columns at W = 64, 16 for fp32) were measured
  // slower for fp16 and fp32 alike: each fill costs two warpgroup barriers.
  static constexpr int FILLW = W < 64 ? W : 64;
  // output TMA box width (elements): at most 32 columns, within one fill
  static constexpr int OBW = FILLW < 32 ? FILLW : 32;
  static constexpr int OSW = OBW * 4;                 // output box row bytes = swizzle span
  static constexpr int NFILL = W / FILLW;
  static constexpr int STG_BYTES = 128 * FILLW * 4;
  // Shared memory: input stage ring | U | output staging | control.  The ring
  // holds as many blocks as fit (at least one tile, at most four); output
  // staging is double buffered unless that would leave under two tiles of
  // input stages.
  static constexpr int CTRL_BYTES = 3840;
  static constexpr int B_ALLOC = ((B_BYTES + 1023) / 1024) * 1024;
  // segmented modes keep one 64-bit start mask per row of a tile per warpgroup
  static constexpr int MASK_BYTES = SEG ? 2 * BPT * 128 * 8 : 0;
  // F16SPLIT: per row of a tile per warpgroup, the power-of-two factor that
  // undoes the row's operand scale (float) and the row's exact total (double)
  static constexpr int RS_BYTES = F16SPLIT ? 2 * BPT * 128 * 4 : 0;
  static constexpr int RT_BYTES = F16SPLIT ? 2 * BPT * 128 * 8 : 0;
  static constexpr int FIXED = 1024 + CTRL_BYTES + B_ALLOC + MASK_BYTES + RS_BYTES + RT_BYTES;
  // threads per CTA: 12 warps, or 14 for the fp32 split (four converter
  // warps, warps 10-13, 32 rows of every stage each: the conversion is the
  // most instruction-heavy stage of the pipeline)
  static constexpr int THREADS = F16SPLIT ? 448 : kThreads;
  static constexpr int NCONV = F16SPLIT ? 4 : 2;  // warps arriving on conv[s] (fp32 converters / fp16 summers)
  static constexpr int NST_DOUBLE = (kMaxSmem - FIXED - 4 * STG_BYTES) / STAGE_BYTES;
  static constexpr int STG_BUFS = NST_DOUBLE >= 2 * BPT ? 2 : 1;
  static constexpr int NST_FIT = (kMaxSmem - FIXED - 2 * STG_BUFS * STG_BYTES) / STAGE_BYTES;
  static constexpr int NST_CAP = 4 * BPT < 32 ? 4 * BPT : 32;
  static constexpr int NSTAGE = NST_FIT < NST_CAP ? NST_FIT : NST_CAP;
  static constexpr int OFF_B = NSTAGE * STAGE_BYTES;
  static constexpr int OFF_STG = OFF_B + B_ALLOC;
  static constexpr int OFF_MASK = OFF_STG + 2 * STG_BUFS * STG_BYTES;
  static constexpr int OFF_RT = OFF_MASK + MASK_BYTES;  // double[2][BPT][128] (8-byte aligned)
  static constexpr int OFF_RS = OFF_RT + RT_BYTES;      // float[2][BPT][128]
  static constexpr int OFF_CTRL = OFF_RS + RS_BYTES;
  static constexpr int SMEM_BYTES = OFF_CTRL + CTRL_BYTES + 1024;  // + alignment slack
  static_assert(NSTAGE >= BPT, "stage ring must hold a whole tile");
  static_assert(!SEG || W == 32 || W == 64, "segmented modes use S = 32 or 64");
  static_assert(!IS_F32 || W == 64, "fp32 inputs use 64-column rows");
  static_assert(W == 16 || W == 32 || W == 64 || W == 128, "S");
  static_assert(RB >= 32, "row must hold one 32-byte MMA K step");
  static_assert(SMEM_BYTES <= kMaxSmem, "shared memory budget");
};

struct ScanCtrl {
  uint64_t full[32];
  uint64_t empty[32];
  uint64_t conv[32];                // fp32: stage converted to bf16 hi/lo operands (two converter warps)
  double cv_sum[32][3];             // partial stage sums of the converters / second summer after warp 10
  uint64_t tile_full[2];
  uint64_t slot_empty[2][16];
  uint64_t drain;
  uint64_t agg_full[8];             // summer -> epilogue: tile aggregate published / bound index ready
  uint64_t agg_empty[8];            // epilogue -> summer: ring slot free
  uint64_t rt_free[2];              // F16SPLIT: warpgroup g has read its row scales / totals (converters may refill)
  long long tile_i0[8];             // kSegBounds: first bound index >= tile start
  int wg_vote[2][4];
  uint32_t stage_cid[32];
  uint32_t tile_cid[2];
  uint32_t tmem_base;
  uint32_t epoch;
  int abort_flag;
  int wait_ok[2][4];
  unsigned long long wt[2][16][4];  // warp totals per block (value bits)
  uint8_t wt_flag[2][16][4];        // warp segment flags per block
  LbScratch lb[2];
};
static_assert(sizeof(ScanCtrl) <= 3840, "control block");

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
template <>
__device__ __forceinline__ float load_elem<float>(const float* p) { return *p; }

// Element e of a 1-D input as float (fp16, fp32 or pre-split fp32 rows).
template <typename InT>
__device__ __forceinline__ float load_at(const void* x, int64_t e) {
  if constexpr (__is_same(InT, SplitF32)) {
    const __nv_bfloat16* row = static_cast<const __nv_bfloat16*>(x) + (e >> 6) * 128;
    return __bfloat162float(row[e & 63]) + __bfloat162float(row[64 + (e & 63)]);
  } else {
    return load_elem<InT>(static_cast<const InT*>(x) + e);
  }
}

// Starting value of a full scan: the host-given start plus, for chained
// chunks, the previous chunk's last output read from device memory.
template <typename V, bool IS_INT, typename P>
__device__ __forceinline__ V scan_start(const P& p) {
  V s = IS_INT ? (V)p.start_i : (V)p.start_f;
  if (p.start_dev) {
    switch (p.start_dev_kind) {
      case 0: s += (V)*static_cast<const int*>(p.start_dev); break;
      case 1: s += (V)*static_cast<const float*>(p.start_dev); break;
      case 2: s += (V)*static_cast<const long long*>(p.start_dev); break;
      default: s += (V)*static_cast<const double*>(p.start_dev); break;
    }
  }
  return s;
}

// Segmented carry operator on (flag, value): (f1,v1) + (f2,v2) =
// (f1|f2, f2 ? v2 : v1+v2).  Plain scans only ever use flag = 0.
template <typename V>
__device__ __forceinline__ void seg_combine(int& f, V& v, int f_prev, V v_prev) {
  if (!f) v = v_prev + v;
  f |= f_prev;
}

// Pairs of fp32 values in one 64-bit register pair (Blackwell f32x2
// arithmetic: both lanes rounded to nearest, as the scalar instructions).
typedef unsigned long long f32x2_t;
__device__ __forceinline__ f32x2_t f2_make(float a, float b) {
  return (f32x2_t)__float_as_uint(a) | ((f32x2_t)__float_as_uint(b) << 32);
}
__device__ __forceinline__ float f2_lo(f32x2_t p) { return __uint_as_float((uint32_t)p); }
__device__ __forceinline__ float f2_hi(f32x2_t p) { return __uint_as_float((uint32_t)(p >> 32)); }
__device__ __forceinline__ f32x2_t f2_add(f32x2_t a, f32x2_t b) {
  f32x2_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2_t f2_sub(f32x2_t a, f32x2_t b) {
  f32x2_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2_t f2_mul(f32x2_t a, f32x2_t b) {
  f32x2_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2_t f2_fma(f32x2_t a, f32x2_t b, f32x2_t c) {
  f32x2_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f32x2_t f2_bits(uint32_t a, uint32_t b) {
  return (f32x2_t)a | ((f32x2_t)b << 32);
}

// In-place split of rows [row0, row1) of an fp32 block into the two fp16
// MMA operand tiles, with every row's exact total; one lane per row (32 rows
// per pass, no cross-lane work).  Each 64-column row arrives as two 128-byte
// halves (TMA boxes at +0 and +term_bytes, same swizzle) and is rewritten as
// 64 fp16 hi in the first slot and 64 fp16 lo in the second.  For a row whose
// largest |x| lies in [2^e, 2^(e+1)):
//   y  = x * 2^k, k = 14 - e            (exact; |y| < 2^15)
//   hi = y rounded to a multiple of 16  (|hi| / 16 <= 2048: exact in fp16)
//   r  = y - hi                         (exact in fp32; |r| <= 8)
//   lo = RN_fp16(r)                     (|r - lo| <= 2^-8 = 2^-22 of 2^14)
// so hi + lo carries 22 significant bits of the row's scale, and the
// epilogue multiplies the MMA result by 2^-k (exact).  The row total is
// 2^-k * (sum hi + sum r): the hi sum is exact in fp32 (multiples of 16
// below 2^21) and the r sum is within 2^-16 of 512 in fp32, combined in FP64
// -- the total of the fp32 inputs themselves, not of their split, so the
// carries between rows and tiles carry no split error.  rs_out[row] = 2^-k,
// rt_out[row] = the total.  Rows in [r_lo, vrows) are also added to acc.
// The lane loads its whole row before writing it.  Non-finite rows keep k = 0.
__device__ __forceinline__ void convert_f32_rows(uint8_t* X0, int term_bytes, int row0, int row1, int r_lo,
                                                 int vrows, bool sums, double& acc, float* rs_out,
                                                 double* rt_out) {
  uint8_t* X1 = X0 + term_bytes;
  const int lane = threadIdx.x & 31;
  const float kRound16 = 201326592.0f;  // 1.5 * 2^27: (y + c) - c rounds y to a multiple of 16
  const f32x2_t c2 = f2_make(kRound16, kRound16);
#pragma unroll 1
  for (int row = row0 + lane; row < row1; row += 32) {
    f32x2_t v[32];  // the row's 64 values as pairs (columns 2i, 2i + 1)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const uint32_t off = swz(row * 128 + c * 16, 128);
      const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(X0 + off);
      const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(X1 + off);
      v[2 * c] = a.x; v[2 * c + 1] = a.y;
      v[16 + 2 * c] = b.x; v[17 + 2 * c] = b.y;
    }
    float mx[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
      mx[q] = fmaxf(fmaxf(fmaxf(fabsf(f2_lo(v[4 * q])), fabsf(f2_hi(v[4 * q]))),
                          fmaxf(fabsf(f2_lo(v[4 * q + 1])), fabsf(f2_hi(v[4 * q + 1])))),
                    fmaxf(fmaxf(fabsf(f2_lo(v[4 * q + 2])), fabsf(f2_hi(v[4 * q + 2]))),
                          fmaxf(fabsf(f2_lo(v[4 * q + 3])), fabsf(f2_hi(v[4 * q + 3])))));
    const float m = fmaxf(fmaxf(fmaxf(mx[0], mx[1]), fmaxf(mx[2], mx[3])),
                          fmaxf(fmaxf(mx[4], mx[5]), fmaxf(mx[6], mx[7])));
    const int eb = (int)((__float_as_uint(m) >> 23) & 0xFFu);  // biased exponent of the row's max
    int k = eb == 0xFF ? 0 : 141 - eb;                          // 14 - (eb - 127)
    k = k > 126 ? 126 : k;                                      // k >= -113 always
    const float sc = __uint_as_float((uint32_t)(k + 127) << 23);
    const f32x2_t sc2 = f2_make(sc, sc);
    f32x2_t shi[2] = {0ull, 0ull}, sr[2] = {0ull, 0ull};
#pragma unroll
    for (int c = 0; c < 8; ++c) {  // output chunk c: columns 8c .. 8c + 7 of the hi and lo rows
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const f32x2_t y = f2_mul(v[4 * c + e], sc2);
        const f32x2_t h = f2_sub(f2_add(y, c2), c2);
        const f32x2_t r = f2_sub(y, h);
        shi[e & 1] = f2_add(shi[e & 1], h);
        sr[e & 1] = f2_add(sr[e & 1], r);
        const __half2 hh = __floats2half2_rn(f2_lo(h), f2_hi(h)), ll = __floats2half2_rn(f2_lo(r), f2_hi(r));
        hw[e] = *reinterpret_cast<const uint32_t*>(&hh);
        lw[e] = *reinterpret_cast<const uint32_t*>(&ll);
      }
      const uint32_t off = swz(row * 128 + c * 16, 128);
      *reinterpret_cast<uint4*>(X0 + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(X1 + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    const f32x2_t sh = f2_add(shi[0], shi[1]), sl = f2_add(sr[0], sr[1]);
    const float th = __fadd_rn(f2_lo(sh), f2_hi(sh));  // exact
    const float tr = __fadd_rn(f2_lo(sl), f2_hi(sl));
    const float rsc = __uint_as_float((uint32_t)(127 - k) << 23);  // 2^-k
    const double tot = ((double)th + (double)tr) * (double)rsc;
    rs_out[row] = rsc;
    rt_out[row] = tot;
    if (sums && row < vrows && row >= r_lo) acc += tot;
  }
  fence_proxy_async_smem();  // generic-proxy writes -> tcgen05 operand reads
  __syncwarp();
}

// Sum of rows [r_lo, vrows) among rows [4 * it_lo, 4 * it_hi) of a
// pre-split stage (hi rows at X0, lo rows at X0 + term_bytes; the swizzle
// only permutes 16-byte chunks inside a row, so rows are read as stored).
__device__ __forceinline__ void sum_split_rows(const uint8_t* X0, int term_bytes, int it_lo, int it_hi, int r_lo,
                                               int vrows, float& acc) {
  const int lane = threadIdx.x & 31;
  const int rr = lane >> 3, cidx = lane & 7;
#pragma unroll 4
  for (int it = it_lo; it < it_hi; ++it) {
    const int row = it * 4 + rr;
    if (row < vrows && row >= r_lo) {
      const uint4 h = *reinterpret_cast<const uint4*>(X0 + row * 128 + cidx * 16);
      const uint4 l = *reinterpret_cast<const uint4*>(X0 + term_bytes + row * 128 + cidx * 16);
      const __nv_bfloat162* hb = reinterpret_cast<const __nv_bfloat162*>(&h);
      const __nv_bfloat162* lb = reinterpret_cast<const __nv_bfloat162*>(&l);
      float t8 = 0.f;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const float2 a = __bfloat1622float2(hb[t]), b = __bfloat1622float2(lb[t]);
        t8 += (a.x + b.x) + (a.y + b.y);
      }
      acc += t8;
    }
  }
}

// Sum of rows [row_lo, row_hi) of an int8 / fp16 stage (K blocks of SW-byte
// rows, 128 rows each) by one warp: int8 exactly with dp4a, fp16 in FP32
// chains of at most 64 values per lane (the caller adds each stage's partial
// to an FP64 aggregate).  Four 16-byte loads in flight per lane.
template <typename InT, int W>
__device__ __forceinline__ void sum_stage_rows(const uint8_t* stage, int row_lo, int row_hi, int& acci,
                                               float& accf) {
  using C = ScanCfg<InT, W>;
  constexpr int CPR = C::SW / 16;  // 16-byte chunks per row of one K block
  const int lane = threadIdx.x & 31;
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
  auto add = [&](const uint4 w, float& sa, float& sb) {
    if constexpr (C::IS_INT) {
      acci = __dp4a((int)w.x, 0x01010101, acci);
      acci = __dp4a((int)w.y, 0x01010101, acci);
      acci = __dp4a((int)w.z, 0x01010101, acci);
      acci = __dp4a((int)w.w, 0x01010101, acci);
    } else {
      const __half2* h = reinterpret_cast<const __half2*>(&w);
      const float2 f0 = __half22float2(h[0]), f1 = __half22float2(h[1]);
      const float2 f2 = __half22float2(h[2]), f3 = __half22float2(h[3]);
      sa += (f0.x + f0.y) + (f1.x + f1.y);
      sb += (f2.x + f2.y) + (f3.x + f3.y);
    }
  };
  const int v1 = row_hi * CPR;
#pragma unroll
  for (int kb = 0; kb < C::KB; ++kb) {
    const uint4* src = reinterpret_cast<const uint4*>(stage + kb * (128 * C::SW));
    int v = row_lo * CPR + lane;
    for (; v + 96 < v1; v += 128) {
      const uint4 w0 = src[v], w1 = src[v + 32], w2 = src[v + 64], w3 = src[v + 96];
      add(w0, s0, s1);
      add(w1, s2, s3);
      add(w2, s0, s1);
      add(w3, s2, s3);
    }
    for (; v < v1; v += 32) add(src[v], s0, s1);
  }
  if constexpr (!C::IS_INT) accf += (s0 + s1) + (s2 + s3);
}

template <typename InT>
struct OperandT { using T = InT; };
template <>
struct OperandT<float> { using T = __half; };
template <>
struct OperandT<SplitF32> { using T = __nv_bfloat16; };

// Build the constant operand B (K-major): row n holds U[k][n] = (k <= n).
template <typename InT, int W>
__device__ __forceinline__ void build_upper(uint8_t* bmat) {
  using C = ScanCfg<InT, W>;
  constexpr int CPR = C::RB / 16;  // 16-byte chunks per row
  const uint32_t one = one_bits<typename OperandT<InT>::T>();
  for (int t = threadIdx.x; t < W * CPR; t += blockDim.x) {
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

// Inclusive prefix of the partial last row, 16 columns at a time (the
// accumulator carries across calls).  Only the thread owning that row calls
// it; it never reads past element n-1.
template <typename InT, int W>
__device__ __forceinline__ void tail_chunk(const ScanParams& p, int col0, uint32_t (&v)[16], float& accf,
                                           int& acci) {
  const int64_t base = p.full_rows * (int64_t)W + col0;
  if constexpr (sizeof(InT) == 1) {
    const int8_t* xs = (const int8_t*)p.x + base;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (col0 + j < p.tail) acci += xs[j];
      v[j] = (uint32_t)acci;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (col0 + j < p.tail) accf += load_at<InT>(p.x, base + j);
      v[j] = __float_as_uint(accf);
    }
  }
}

// Epilogue of one warpgroup (128 threads; thread = row of every block).
template <typename InT, int W, int MODE>
__device__ __forceinline__ void scan_epilogue(const ScanParams& p, const CUtensorMap& out_map, uint8_t* smem,
                                              ScanCtrl* ctl, uint32_t tmem_base, uint32_t epoch,
                                              const WaitCtx& wc) {
  using C = ScanCfg<InT, W, false, MODE == kScanFullSmall>;
  constexpr bool IS_INT = C::IS_INT;
  constexpr int BPT = C::BPT;
  using V = typename std::conditional<IS_INT, long long, double>::type;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int g = (warp - 2) >> 2;  // warpgroup 0 / 1
  const int q = warp & 3;         // TMEM lane quarter
  const int r = q * 32 + lane;    // row within a block
  const int wg_thread = threadIdx.x - 64 - g * 128;
  const uint32_t bar_id = 1 + g;
  uint8_t* stg_base = smem + C::OFF_STG + g * C::STG_BUFS * C::STG_BYTES;
  const V start = scan_start<V, IS_INT>(p);
  uint32_t nfill = 0;
  // F16SPLIT: this warpgroup's row totals and row scale factors
  const double* rtg = reinterpret_cast<const double*>(smem + C::OFF_RT) + g * BPT * 128;
  const float* rsg = reinterpret_cast<const float*>(smem + C::OFF_RS) + g * BPT * 128;

  const bool prof = p.phase_ns != nullptr && wg_thread == 0;
  uint64_t t_mark = prof ? globaltimer() : 0;
  for (uint32_t i = g;; i += 2) {
    const uint32_t u = i >> 1;
    // One lane per warp waits; the four warps then vote at a named barrier
    // that all of them always reach, so an abort is warpgroup-uniform.
    int ok = 1;
    if (lane == 0) ok = mbar_wait(&ctl->tile_full[g], u & 1u, wc, 5, i) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (lane == 0) ctl->wait_ok[g][q] = ok;
    named_bar_sync(bar_id, 128);
    const int all_ok = ctl->wait_ok[g][0] & ctl->wait_ok[g][1] & ctl->wait_ok[g][2] & ctl->wait_ok[g][3];
    const uint32_t tid = *(volatile uint32_t*)&ctl->tile_cid[g];
    if (!all_ok || tid == kSentinel) break;
    if (prof) { const uint64_t t = globaltimer(); phase_add(p, 0, t - t_mark); phase_add(p, 7, 1); t_mark = t; }
    tc_fence_after();
    const uint32_t tm = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(g * 256);
    const int64_t row_tile0 = (int64_t)tid * BPT * 128;

    // ---- (A) row totals -> row offsets within the tile, tile aggregate ----
    V rowex[BPT];
#pragma unroll
    for (int j = 0; j < BPT; ++j) rowex[j] = V(0);
    // F16SPLIT: the row scale factors of the tile, read here with the row
    // totals so both arrays are free for the converters after phase A
    float rsv[BPT];
#pragma unroll
    for (int j = 0; j < BPT; ++j) rsv[j] = C::F16SPLIT ? rsg[j * 128 + r] : 1.f;
    if constexpr (MODE != kScanRows) {
      uint32_t tb[BPT];
      if constexpr (!C::F16SPLIT) {
#pragma unroll
        for (int j = 0; j < BPT; ++j) tb[j] = tmem_ld1(tm + (uint32_t)(j * W + W - 1));
        tmem_wait_ld();
      }
      int fl[BPT];
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        const int64_t grow = row_tile0 + j * 128 + r;
        if (grow >= p.full_rows) {
          tb[j] = 0u;
          if (grow == p.full_rows && p.tail > 0) {
            float af = 0.f;
            int ai = 0;
            uint32_t tmp[16];
#pragma unroll
            for (int c = 0; c < W / 16; ++c) tail_chunk<InT, W>(p, c * 16, tmp, af, ai);
            tb[j] = IS_INT ? (uint32_t)ai : __float_as_uint(af);
          }
        }
        fl[j] = (MODE == kScanBlocks) ? (int)((grow % p.seg_rows) == 0) : 0;
      }
      int rowf[BPT];
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        V ti = IS_INT ? (V)(int)tb[j] : (V)__uint_as_float(tb[j]);
        if constexpr (C::F16SPLIT) {  // the exact row totals of the converters
          if (row_tile0 + j * 128 + r < p.full_rows) ti = (V)rtg[j * 128 + r];
        }
        int fi = fl[j];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const V tp = __shfl_up_sync(0xffffffffu, ti, d);
          const int fp = __shfl_up_sync(0xffffffffu, fi, d);
          if (lane >= d) seg_combine(fi, ti, fp, tp);
        }
        V te = __shfl_up_sync(0xffffffffu, ti, 1);
        int fe = __shfl_up_sync(0xffffffffu, fi, 1);
        if (lane == 0) { te = V(0); fe = 0; }
        rowex[j] = te;
        rowf[j] = fe;
        if (lane == 31) {
          ctl->wt[g][j][q] = v_bits<V>(ti);
          ctl->wt_flag[g][j][q] = (uint8_t)fi;
        }
      }
      named_bar_sync(bar_id, 128);
      if (C::F16SPLIT && wg_thread == 0) mbar_arrive(&ctl->rt_free[g]);  // every thread has read rs / rt
      V run = V(0);
      int runf = 0;
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        V wpre = V(0), bsum = V(0);
        int wf = 0, bf = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const V wv = v_from_bits<V>(ctl->wt[g][j][k]);
          const int wfl = ctl->wt_flag[g][j][k];
          if (k < q) { if (wfl) { wpre = wv; wf = 1; } else { wpre += wv; } }
          if (wfl) { bsum = wv; bf = 1; } else { bsum += wv; }
        }
        V ex = rowex[j];
        int exf = rowf[j];
        if (!exf) { ex = wpre + ex; exf = wf; }
        if (!exf) { ex = run + ex; exf = runf; }
        rowex[j] = (MODE == kScanBlocks && fl[j]) ? V(0) : ex;
        if (bf) { run = bsum; runf = 1; } else { run += bsum; }
      }
      if (prof) { const uint64_t t = globaltimer(); phase_add(p, 1, t - t_mark); t_mark = t; }
      if constexpr (is_full(MODE)) {
        // The summer warp published this tile's aggregate as soon as its data
        // landed; wait for that (ordering: the inclusive prefix must not be
        // overwritten by a late aggregate), then look back.
        const int m = i & 7;
        if (wg_thread == 0) mbar_wait(&ctl->agg_full[m], (i >> 3) & 1u, wc, 6, i);
        const V pre = wg_lookback<V>((int64_t)tid, run, start, p.descs, epoch, wc, &ctl->lb[g], wg_thread, bar_id);
        if (wg_thread == 0) mbar_arrive(&ctl->agg_empty[m]);
#pragma unroll
        for (int j = 0; j < BPT; ++j) rowex[j] = pre + rowex[j];
        if (prof) { const uint64_t t = globaltimer(); phase_add(p, 2, t - t_mark); t_mark = t; }
      }
    }

    // ---- (C) drain: carry add, staging, TMA store ----
#pragma unroll 1
    for (int j = 0; j < BPT; ++j) {
      const int64_t brow0 = row_tile0 + j * 128;
      const bool is_tail = (brow0 + r == p.full_rows) && p.tail > 0;
      float accf = 0.f;
      int acci = 0;
      const float cf = IS_INT ? 0.f : (float)rowex[j];
      const uint32_t ci = IS_INT ? (uint32_t)(long long)rowex[j] : 0u;
#pragma unroll
      for (int h = 0; h < C::NFILL; ++h) {
        uint8_t* stg = stg_base + (nfill % C::STG_BUFS) * C::STG_BYTES;
        if (wg_thread == 0) {  // the store that last used this buffer has read it
          if (C::STG_BUFS == 2) bulk_wait_read1(); else bulk_wait_read0();
        }
        named_bar_sync(bar_id, 128);
        uint32_t v[C::FILLW];
#pragma unroll
        for (int c = 0; c < C::FILLW / 16; ++c)
          tmem_ld16(tm + (uint32_t)(j * W + h * C::FILLW + c * 16), *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]));
        tmem_wait_ld();
        if (h == C::NFILL - 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&ctl->slot_empty[g][j]);  // block j's TMEM columns are free
        }
        if (!is_tail) {
          // y = z + carry (fp32 split: z * 2^-k + carry, the scale a power of
          // two so the product is exact and the fused form rounds once, as
          // the separate multiply and add do), two columns per instruction
#pragma unroll
          for (int e4 = 0; e4 < C::FILLW / 4; ++e4) {
            uint4 o;
            const uint32_t* ve = &v[e4 * 4];
            if constexpr (IS_INT) {
              o = make_uint4(ve[0] + ci, ve[1] + ci, ve[2] + ci, ve[3] + ci);
            } else {
              const f32x2_t c2 = f2_make(cf, cf);
              f32x2_t a = f2_bits(ve[0], ve[1]), b = f2_bits(ve[2], ve[3]);
              if constexpr (C::F16SPLIT) {
                const f32x2_t s2 = f2_make(rsv[j], rsv[j]);
                a = f2_fma(a, s2, c2);
                b = f2_fma(b, s2, c2);
              } else {
                a = f2_add(a, c2);
                b = f2_add(b, c2);
              }
              o = make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
            }
            const int cc = e4 * 4;
            const int box = cc / C::OBW, cin = cc % C::OBW;
            *(uint4*)(stg + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW)) = o;
          }
        } else {
          // the ragged last row: prefixes from global memory, written to z
          // directly as well as staged
#pragma unroll
          for (int c = 0; c < C::FILLW / 16; ++c)
            tail_chunk<InT, W>(p, h * C::FILLW + c * 16, *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]), accf, acci);
#pragma unroll
          for (int e4 = 0; e4 < C::FILLW / 4; ++e4) {
            uint32_t o[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              if constexpr (IS_INT) o[e] = v[e4 * 4 + e] + ci;
              else o[e] = __float_as_uint(__uint_as_float(v[e4 * 4 + e]) + cf);
            }
            const int cc = e4 * 4;
            const int box = cc / C::OBW, cin = cc % C::OBW;
            uint8_t* dst = stg + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW);
            *(uint4*)dst = make_uint4(o[0], o[1], o[2], o[3]);
            uint32_t* zt = (uint32_t*)p.z + p.full_rows * (int64_t)W + h * C::FILLW + cc;
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (h * C::FILLW + cc + e < p.tail) zt[e] = o[e];
          }
        }
        fence_proxy_async_smem();
        named_bar_sync(bar_id, 128);
        if (wg_thread == 0) {
          if (p.has_map && brow0 < p.full_rows) {
#pragma unroll
            for (int b = 0; b < C::FILLW / C::OBW; ++b)
              tma_store_2d(&out_map, h * C::FILLW + b * C::OBW, (int32_t)brow0, stg + b * (128 * C::OSW));
          }
          bulk_commit();
        }
        ++nfill;
      }
    }
    if (prof) { const uint64_t t = globaltimer(); phase_add(p, 3, t - t_mark); t_mark = t; }
  }
  if (wg_thread == 0) bulk_wait_all0();
}

// Segment-start array element (int32 or int64).
__device__ __forceinline__ long long bound_at(const ScanParams& p, int64_t i) {
  return p.bounds64 ? __ldg(static_cast<const long long*>(p.bounds) + i)
                    : (long long)__ldg(static_cast<const int*>(p.bounds) + i);
}

// First index i in [0, nbounds] with bounds[i] >= target (warp-cooperative,
// 32-way search: four rounds for a million entries).  Run by one full warp.
__device__ __forceinline__ long long warp_lower_bound(const ScanParams& p, long long target) {
  const int lane = threadIdx.x & 31;
  long long lo = 0, hi = p.nbounds;
  while (hi - lo > 32) {
    const long long step = (hi - lo + 31) / 32;
    const long long pos = lo + lane * step;
    const bool below = pos < hi && bound_at(p, pos) < target;
    const int c = __popc(__ballot_sync(0xffffffffu, below));
    const long long nlo = c == 0 ? lo : lo + (c - 1) * step + 1;
    const long long nhi = (c == 32) ? hi : min(hi, lo + (long long)c * step);
    lo = nlo;
    hi = nhi;
  }
  const long long pos = lo + lane;
  const bool below = pos < hi && bound_at(p, pos) < target;
  return lo + __popc(__ballot_sync(0xffffffffu, below));
}

// tile_first[t] = first index i with bounds[i] >= t * tile_elems, for every
// tile, in one pass over the (non-decreasing) bounds: bound k owns the tiles
// after its predecessor's tile up to its own.  No search, O(nbounds + tiles).
__global__ void __launch_bounds__(256) bounds_tiles_kernel(const void* bounds, int bounds64, int64_t nbounds,
                                                           int64_t tile_elems, int64_t num_tiles,
                                                           long long* __restrict__ tile_first) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= nbounds; k += stride) {
    int64_t t_prev = -1, t_cur = num_tiles - 1;
    if (k > 0) {
      long long b = bounds64 ? __ldg(static_cast<const long long*>(bounds) + k - 1)
                             : (long long)__ldg(static_cast<const int*>(bounds) + k - 1);
      b = b < 0 ? 0 : b;
      t_prev = b / tile_elems;
    }
    if (k < nbounds) {
      long long b = bounds64 ? __ldg(static_cast<const long long*>(bounds) + k)
                             : (long long)__ldg(static_cast<const int*>(bounds) + k);
      b = b < 0 ? 0 : b;
      const int64_t t = b / tile_elems;
      t_cur = t < num_tiles - 1 ? t : num_tiles - 1;
    }
    for (int64_t t = t_prev + 1; t <= t_cur; ++t) tile_first[t] = k;
  }
}

// Last segment start inside tile `tid` (elements [tid * tile, min(.., n))),
// or -1: the largest bound in the tile for sorted bounds (the bounds of the
// tile are [tile_first[tid], tile_first[tid + 1]); the last tile also skips
// bounds at or past n), the largest multiple of the period for periodic
// segments.  Warp-uniform result.
template <int MODE>
__device__ __forceinline__ long long tile_last_start(const ScanParams& p, uint32_t tid, int64_t tile) {
  const int64_t e0 = (int64_t)tid * tile;
  const int64_t e1 = e0 + tile < p.n ? e0 + tile : p.n;
  if constexpr (MODE == kSegPeriodic) {
    const int64_t m = ((e1 - 1) / p.period) * p.period;
    return m >= e0 ? m : -1;
  } else {
    if (!p.tile_first || p.nbounds == 0) return -1;
    const int lane = threadIdx.x & 31;
    auto clampi = [&](long long v) { return v < 0 ? 0 : (v > p.nbounds ? p.nbounds : v); };
    const long long i0 = clampi(__ldg(p.tile_first + tid));
    const long long i1 = (int64_t)tid + 1 < p.num_tiles ? clampi(__ldg(p.tile_first + tid + 1)) : p.nbounds;
    for (long long hi = i1 - 1; hi >= i0; hi -= 32) {
      const long long kk = hi - lane;
      const long long b = kk >= i0 ? bound_at(p, kk) : -1;
      const unsigned ok = __ballot_sync(0xffffffffu, kk >= i0 && b >= e0 && b < e1);
      if (ok) return __shfl_sync(0xffffffffu, b, __ffs(ok) - 1);
      if (__shfl_sync(0xffffffffu, b, 31) >= 0 && __shfl_sync(0xffffffffu, b, 31) < e0) break;
    }
    return -1;
  }
}

// Publishes the segmented aggregate of a tile from the summer's per-lane
// sums: the ragged last row of the input is added from global memory (from
// the last segment start on, when it lies in that row), then the warp total
// goes out flagged as a segment start when the tile holds one.
template <typename InT, int W, int MODE>
__device__ __forceinline__ void ctl_publish_seg(const ScanParams& p, uint32_t tid, long long ls, int acci, float accf,
                                                double accd, uint32_t epoch, int lane) {
  using C = ScanCfg<InT, W, true>;
  using V = typename std::conditional<C::IS_INT, long long, double>::type;
  const int64_t e0 = (int64_t)tid * C::TILE_ELEMS;
  const int64_t tail0 = p.full_rows * (int64_t)W;
  if (p.tail > 0 && tail0 >= e0 && tail0 < e0 + C::TILE_ELEMS) {
    const int64_t from = ls > tail0 ? ls : tail0;
    for (int64_t e = from + lane; e < p.n; e += 32) {
      if constexpr (C::IS_INT) acci += (int)static_cast<const int8_t*>(p.x)[e];
      else if constexpr (C::IS_F32) accd += (double)load_at<InT>(p.x, e);
      else accf += load_at<InT>(p.x, e);
    }
  }
  V agg;
  if constexpr (C::IS_INT) agg = (V)warp_sum_any(acci);
  else agg = warp_sum_any((double)accf + accd);
  if (lane == 0) publish_aggregate<V>((int64_t)tid, agg, ls >= 0 ? 1 : 0, V(0), p.descs, epoch);
}

// Summer warp: sums every tile straight from the TMA-filled SMEM stages (rows
// past the input are skipped, the partial last row is read from global) and
// publishes the tile aggregate at once, then hands (tile, aggregate) to the
// look-back warp.  It never waits on another CTA, so a tile's aggregate is
// visible about one TMA latency after the tile id was taken -- successors'
// look-backs never queue behind this CTA's backlog.  For the row/block modes
// it only releases the stages.
template <typename InT, int W, int MODE>
__device__ __forceinline__ void scan_summer(const ScanParams& p, uint8_t* smem, ScanCtrl* ctl, uint32_t epoch,
                                                const WaitCtx& wc) {
  using C = ScanCfg<InT, W, is_seg(MODE), MODE == kScanFullSmall>;
  constexpr bool IS_INT = C::IS_INT;
  constexpr int BPT = C::BPT;
  using V = typename std::conditional<IS_INT, long long, double>::type;
  const int lane = threadIdx.x & 31;
  const V start = scan_start<V, IS_INT>(p);
  const bool prof = p.phase_ns != nullptr && lane == 0;
  // Modes whose tile aggregate this warp publishes as soon as the data lands:
  // the full scan, and the segmented modes whose last segment start in a tile
  // is known without reading the tile (sorted bounds, fixed period).  For the
  // latter the aggregate is the sum after that start, flagged as a segment
  // start, which ends every look-back that reaches the tile.
  constexpr bool SEG_EARLY = (MODE == kSegBounds || MODE == kSegPeriodic);
  constexpr bool SUMS = (is_full(MODE) || SEG_EARLY);
  uint32_t k = 0;
  uint32_t i = 0;
  for (;; ++i) {
    const uint64_t t0 = prof ? globaltimer() : 0;
    bool stop = false;
    uint32_t tid = 0;
    float accf = 0.f;
    double accd = 0.0;
    int acci = 0;
    long long ls = -1;  // last segment start of the tile (SEG_EARLY), -1 = none
    for (int j = 0; j < BPT; ++j, ++k) {
      const int s = k % C::NSTAGE;
      // every lane observes the TMA barrier before reading the stage
      const uint64_t tw = prof ? globaltimer() : 0;
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&ctl->full[s], (k / C::NSTAGE) & 1u, wc, 7, i));
      if (prof) phase_add(p, 6, globaltimer() - tw);
      if (!ok) { stop = true; break; }
      const uint32_t cid = *(volatile uint32_t*)&ctl->stage_cid[s];
      if (cid == kSentinel) {
        // the MMA warp of an fp32 launch waits on conv[]: pass the stop on
        if (C::IS_F32 && lane == 0) mbar_arrive(&ctl->conv[s]);
        stop = true;
        break;
      }
      tid = cid;
      if (SEG_EARLY && j == 0) ls = tile_last_start<MODE>(p, tid, C::TILE_ELEMS);
      // rows of this block summed from shared memory: all valid rows, or
      // (SEG_EARLY) those after the tile's last segment start; the start's
      // own row is summed from its start column, from global memory
      int r_lo = 0;
      if (SEG_EARLY && ls >= 0) {
        const int64_t be0 = (int64_t)tid * C::TILE_ELEMS + (int64_t)j * 128 * W;
        if (ls >= be0 + 128 * (int64_t)W) {
          r_lo = 128;
        } else if (ls >= be0) {
          const int lsr = (int)((ls - be0) / W);
          r_lo = lsr + 1;
          if (be0 / W + lsr < p.full_rows) {
            const int64_t rend = be0 + (int64_t)(lsr + 1) * W;
            for (int64_t e = ls + lane; e < rend; e += 32) {
              if constexpr (IS_INT) acci += (int)static_cast<const int8_t*>(p.x)[e];
              else if constexpr (C::IS_F32) accd += (double)load_at<InT>(p.x, e);
              else accf += load_at<InT>(p.x, e);
            }
          }
        }
      }
      if constexpr (C::IS_F32) {
        // rows 0-63 here, rows 64-127 by the second converter warp; the MMA
        // waits for both (conv[s] counts two arrivals)
        uint8_t* X0 = smem + s * C::STAGE_BYTES;
        const int64_t row0 = ((int64_t)tid * BPT + j) * 128;
        const int64_t vr = p.full_rows - row0;
        const int vrows = vr <= 0 ? 0 : (vr >= 128 ? 128 : (int)vr);
        if constexpr (C::PRESPLIT) {
          float acc = 0.f;  // this stage's partial (FP32), then the FP64 tile aggregate
          if (SUMS) sum_split_rows(X0, C::TERM_BYTES, 0, 16, r_lo, vrows, acc);
          accd += (double)acc;
        } else {
          // the row scales / totals of this TMEM half are free once its
          // warpgroup has read them for the tile two before this one
          const int g = i & 1;
          const uint32_t u = i >> 1;
          if (u >= 1 && !__all_sync(0xffffffffu, mbar_wait(&ctl->rt_free[g], (u - 1) & 1u, wc, 11, i))) {
            stop = true;
            break;
          }
          const int rix = (g * BPT + j) * 128;
          convert_f32_rows(X0, C::TERM_BYTES, 0, 128 / C::NCONV, r_lo, vrows, SUMS, accd,
                           reinterpret_cast<float*>(smem + C::OFF_RS) + rix,
                           reinterpret_cast<double*>(smem + C::OFF_RT) + rix);
        }
        if (lane == 0) mbar_arrive(&ctl->conv[s]);
        if constexpr (SUMS) {  // the other converters' sums, stored before their conv arrivals
          const bool okc = __all_sync(0xffffffffu, mbar_wait(&ctl->conv[s], (k / C::NSTAGE) & 1u, wc, 9, i));
          if (!okc) { stop = true; break; }
          if (lane == 0)
            for (int c = 0; c < C::NCONV - 1; ++c) accd += ctl->cv_sum[s][c];
        }
      }
      if constexpr (SUMS && !C::IS_F32) {
        // int8: the whole stage here (dp4a is cheap); fp16: rows [r_lo, 64)
        // here and rows [64, 128) by warp 11, which leaves its partial in
        // cv_sum[s] before its conv arrival -- the stage is released only
        // after both halves have been read
        const int64_t row0 = ((int64_t)tid * BPT + j) * 128;
        int64_t vr = p.full_rows - row0;
        const int vrows = vr <= 0 ? 0 : (vr >= 128 ? 128 : (int)vr);
        float sf = 0.f;
        if constexpr (IS_INT) {
          sum_stage_rows<InT, W>(smem + s * C::STAGE_BYTES, r_lo, vrows, acci, sf);
        } else {
          sum_stage_rows<InT, W>(smem + s * C::STAGE_BYTES, r_lo, vrows < 64 ? vrows : 64, acci, sf);
          accd += (double)sf;
          __syncwarp();
          if (lane == 0) mbar_arrive(&ctl->conv[s]);
          const bool okc = __all_sync(0xffffffffu, mbar_wait(&ctl->conv[s], (k / C::NSTAGE) & 1u, wc, 13, i));
          if (!okc) { stop = true; break; }
          if (lane == 0) accd += ctl->cv_sum[s][0];
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&ctl->empty[s]);  // this consumer is done with the stage
    }
    if (stop) break;
    if constexpr (MODE == kSegBounds) {
      // first bound index of the tile (precomputed for every tile in one
      // parallel pass over the bounds; clamped so a stale entry can never
      // index outside them)
      long long i0;
      if (p.tile_first) {
        i0 = __ldg(p.tile_first + tid);
        i0 = i0 < 0 ? 0 : (i0 > p.nbounds ? p.nbounds : i0);
      } else {
        i0 = warp_lower_bound(p, (long long)tid * C::TILE_ELEMS);
      }
      ctl_publish_seg<InT, W, MODE>(p, tid, ls, acci, accf, accd, epoch, lane);
      int ok = 1;
      if (lane == 0) {
        const int m = i & 7;
        if (i >= 8) ok = mbar_wait(&ctl->agg_empty[m], ((i >> 3) & 1u) ^ 1u, wc, 8, i) ? 1 : 0;
        if (ok) {
          ctl->tile_i0[m] = i0;
          mbar_arrive(&ctl->agg_full[m]);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (prof) phase_add(p, 5, globaltimer() - t0);
      if (!ok) break;
    }
    if constexpr (MODE == kSegPeriodic) {
      ctl_publish_seg<InT, W, MODE>(p, tid, ls, acci, accf, accd, epoch, lane);
      int ok = 1;
      if (lane == 0) {
        const int m = i & 7;
        if (i >= 8) ok = mbar_wait(&ctl->agg_empty[m], ((i >> 3) & 1u) ^ 1u, wc, 8, i) ? 1 : 0;
        if (ok) mbar_arrive(&ctl->agg_full[m]);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (prof) phase_add(p, 5, globaltimer() - t0);
      if (!ok) break;
    }
    if constexpr (is_full(MODE)) {
      const int64_t tile_row0 = (int64_t)tid * BPT * 128;
      if (lane == 0 && p.tail > 0 && p.full_rows >= tile_row0 && p.full_rows < tile_row0 + BPT * 128) {
        float af = 0.f;
        int ai = 0;
        uint32_t tmp[16];
#pragma unroll
        for (int c = 0; c < W / 16; ++c) tail_chunk<InT, W>(p, c * 16, tmp, af, ai);
        accf += af;
        acci += ai;
      }
      V agg;
      if constexpr (IS_INT) agg = (V)warp_sum_any(acci);
      else agg = warp_sum_any((double)accf + accd);
      int ok = 1;
      if (lane == 0) {
        publish_aggregate<V>((int64_t)tid, agg, 0, start, p.descs, epoch);
        const int m = i & 7;
        if (i >= 8) ok = mbar_wait(&ctl->agg_empty[m], ((i >> 3) & 1u) ^ 1u, wc, 8, i) ? 1 : 0;
        if (ok) mbar_arrive(&ctl->agg_full[m]);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (prof) phase_add(p, 5, globaltimer() - t0);
      if (!ok) break;
    }
  }
}

// Second converter warp: for fp32 launches it splits rows 64-127 of every
// stage; for fp16 launches whose tile aggregate the summer publishes it sums
// rows 64-127.  Either way it leaves the sum of its rows (those after the
// tile's last segment start, for the modes whose aggregate the summer
// publishes) in cv_sum[s] before its conv arrival.  Idle otherwise.
template <typename InT, int W, int MODE>
__device__ __forceinline__ void scan_converter2(const ScanParams& p, uint8_t* smem, ScanCtrl* ctl,
                                                const WaitCtx& wc, int cidx) {
  using C = ScanCfg<InT, W, is_seg(MODE), MODE == kScanFullSmall>;
  constexpr bool SUMS_ANY = (is_full(MODE) || MODE == kSegBounds || MODE == kSegPeriodic);
  if constexpr (!C::IS_F32 && !C::IS_INT && SUMS_ANY) {
    constexpr int BPT = C::BPT;
    constexpr bool SEG_EARLY = (MODE == kSegBounds || MODE == kSegPeriodic);
    const int lane = threadIdx.x & 31;
    uint32_t k = 0;
    for (uint32_t i = 0;; ++i) {
      long long ls = -1;
      bool stop = false;
      for (int j = 0; j < BPT; ++j, ++k) {
        const int s = k % C::NSTAGE;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&ctl->full[s], (k / C::NSTAGE) & 1u, wc, 14, i));
        if (!ok) { stop = true; break; }
        const uint32_t tid = *(volatile uint32_t*)&ctl->stage_cid[s];
        if (tid == kSentinel) { stop = true; break; }
        if (SEG_EARLY && j == 0) ls = tile_last_start<MODE>(p, tid, C::TILE_ELEMS);
        int r_lo = 0;
        if (SEG_EARLY && ls >= 0) {
          const int64_t be0 = (int64_t)tid * C::TILE_ELEMS + (int64_t)j * 128 * W;
          if (ls >= be0 + 128 * (int64_t)W) r_lo = 128;
          else if (ls >= be0) r_lo = (int)((ls - be0) / W) + 1;
        }
        const int64_t row0 = ((int64_t)tid * BPT + j) * 128;
        const int64_t vr = p.full_rows - row0;
        const int vrows = vr <= 0 ? 0 : (vr >= 128 ? 128 : (int)vr);
        int acci = 0;
        float accf = 0.f;
        sum_stage_rows<InT, W>(smem + s * C::STAGE_BYTES, r_lo > 64 ? r_lo : 64, vrows, acci, accf);
        const double t = warp_sum_any((double)accf);
        if (lane == 0) ctl->cv_sum[s][0] = t;
        __syncwarp();
        if (lane == 0) mbar_arrive(&ctl->conv[s]);
      }
      if (stop) break;
    }
  }
  if constexpr (C::IS_F32) {
    constexpr int BPT = C::BPT;
    constexpr bool SUMS = (is_full(MODE) || MODE == kSegBounds || MODE == kSegPeriodic);
    const int lane = threadIdx.x & 31;
    uint32_t k = 0;
    for (uint32_t i = 0;; ++i) {
      long long ls = -1;
      bool stop = false;
      for (int j = 0; j < BPT; ++j, ++k) {
        const int s = k % C::NSTAGE;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&ctl->full[s], (k / C::NSTAGE) & 1u, wc, 10, i));
        if (!ok) { stop = true; break; }
        const uint32_t tid = *(volatile uint32_t*)&ctl->stage_cid[s];
        if (tid == kSentinel) {
          if (lane == 0) mbar_arrive(&ctl->conv[s]);
          stop = true;
          break;
        }
        if ((MODE == kSegBounds || MODE == kSegPeriodic) && j == 0) ls = tile_last_start<MODE>(p, tid, C::TILE_ELEMS);
        int r_lo = 0;
        if ((MODE == kSegBounds || MODE == kSegPeriodic) && ls >= 0) {
          const int64_t be0 = (int64_t)tid * C::TILE_ELEMS + (int64_t)j * 128 * W;
          if (ls >= be0 + 128 * (int64_t)W) r_lo = 128;
          else if (ls >= be0) r_lo = (int)((ls - be0) / W) + 1;
        }
        const int64_t row0 = ((int64_t)tid * BPT + j) * 128;
        const int64_t vr = p.full_rows - row0;
        const int vrows = vr <= 0 ? 0 : (vr >= 128 ? 128 : (int)vr);
        double acc = 0.0;
        if constexpr (C::PRESPLIT) {
          float accf = 0.f;
          if (SUMS) sum_split_rows(smem + s * C::STAGE_BYTES, C::TERM_BYTES, 16, 32, r_lo, vrows, accf);
          acc = (double)accf;
        } else {
          const int g = i & 1;
          const uint32_t u = i >> 1;
          if (u >= 1 && !__all_sync(0xffffffffu, mbar_wait(&ctl->rt_free[g], (u - 1) & 1u, wc, 12, i))) {
            if (lane == 0) mbar_arrive(&ctl->conv[s]);
            stop = true;
            break;
          }
          const int rix = (g * BPT + j) * 128;
          constexpr int RPC = 128 / C::NCONV;  // rows per converter
          convert_f32_rows(smem + s * C::STAGE_BYTES, C::TERM_BYTES, cidx * RPC, (cidx + 1) * RPC, r_lo, vrows, SUMS, acc,
                           reinterpret_cast<float*>(smem + C::OFF_RS) + rix,
                           reinterpret_cast<double*>(smem + C::OFF_RT) + rix);
        }
        if constexpr (SUMS) {
          const double t = warp_sum_any(acc);
          if (lane == 0) ctl->cv_sum[s][cidx - 1] = t;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&ctl->conv[s]);
      }
      if (stop) break;
    }
  }
}

// ---------------------------------------------------------------------------
// Segmented modes.

// Warpgroup-wide count of `pred` (two named barriers).
__device__ __forceinline__ int wg_count(bool pred, int* votes, int lane, int q, uint32_t bar_id) {
  const int c = __popc(__ballot_sync(0xffffffffu, pred));
  if (lane == 0) votes[q] = c;
  named_bar_sync(bar_id, 128);
  const int t = votes[0] + votes[1] + votes[2] + votes[3];
  named_bar_sync(bar_id, 128);
  return t;
}

// Start mask of the row beginning at element a (bit j: a segment starts at
// a + j) for the flag and periodic modes.  Rows past the input have none.
template <int W, int MODE>
__device__ __forceinline__ unsigned long long row_start_mask(const ScanParams& p, int64_t a) {
  if (a >= p.n) return 0ull;
  unsigned long long m = 0;
  if constexpr (MODE == kSegPeriodic) {
    const int64_t L = p.period;
    for (int64_t pp = ((a + L - 1) / L) * L; pp < a + W; pp += L) m |= 1ull << (pp - a);
    return m;
  } else {
    const int8_t* f = p.flags + a;
    if (a + W <= p.n) {
      const uint4* fv = reinterpret_cast<const uint4*>(f);
#pragma unroll
      for (int v = 0; v < W / 16; ++v) {
        const uint4 w = __ldg(fv + v);
        const unsigned long long bits = (unsigned long long)(sel4(w.x) | (sel4(w.y) << 4) | (sel4(w.z) << 8) |
                                                             (sel4(w.w) << 12));
        m |= bits << (16 * v);
      }
    } else {
      for (int j = 0; j < W && a + j < p.n; ++j)
        if (f[j] != 0) m |= 1ull << j;
    }
    if constexpr (MODE == kSegEnds) {
      // a segment starts right after every end flag
      m = (m << 1) | ((a > 0 && p.flags[a - 1] != 0) ? 1ull : 0ull);
      if constexpr (W < 64) m &= (1ull << W) - 1ull;
    }
    return m;
  }
}

__device__ __forceinline__ uint32_t stage_lookup(const uint8_t* stg, int64_t pos_local, int W, int OBW, int OSW) {
  const int row = (int)(pos_local / W), col = (int)(pos_local % W);
  const int box = col / OBW, cin = col % OBW;
  return *reinterpret_cast<const uint32_t*>(stg + box * (128 * OSW) + swz(row * OSW + cin * 4, OSW));
}

template <typename InT, int W, int MODE>
__device__ __forceinline__ void seg_epilogue(const ScanParams& p, const CUtensorMap& out_map, uint8_t* smem,
                                             ScanCtrl* ctl, uint32_t tmem_base, uint32_t epoch,
                                             const WaitCtx& wc) {
  using C = ScanCfg<InT, W, true>;
  constexpr bool IS_INT = C::IS_INT;
  constexpr int BPT = C::BPT;
  using V = typename std::conditional<IS_INT, long long, double>::type;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int g = (warp - 2) >> 2;
  const int q = warp & 3;
  const int r = q * 32 + lane;
  const int wg_thread = threadIdx.x - 64 - g * 128;
  const uint32_t bar_id = 1 + g;
  uint8_t* stg_base = smem + C::OFF_STG + g * C::STG_BUFS * C::STG_BYTES;
  unsigned long long* smask = reinterpret_cast<unsigned long long*>(smem + C::OFF_MASK) + g * BPT * 128;
  int* votes = ctl->wg_vote[g];
  const bool sums_out = (MODE == kSegBounds) && p.out_sums;
  // F16SPLIT: this warpgroup's row totals and row scale factors
  const double* rtg = reinterpret_cast<const double*>(smem + C::OFF_RT) + g * BPT * 128;
  const float* rsg = reinterpret_cast<const float*>(smem + C::OFF_RS) + g * BPT * 128;
  const bool prof = p.phase_ns != nullptr && wg_thread == 0;
  uint64_t t_mark = prof ? globaltimer() : 0;
  uint32_t nfill = 0;

  for (uint32_t i = g;; i += 2) {
    const uint32_t u = i >> 1;
    int ok = 1;
    if (lane == 0) ok = mbar_wait(&ctl->tile_full[g], u & 1u, wc, 5, i) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (lane == 0) ctl->wait_ok[g][q] = ok;
    named_bar_sync(bar_id, 128);
    const int all_ok = ctl->wait_ok[g][0] & ctl->wait_ok[g][1] & ctl->wait_ok[g][2] & ctl->wait_ok[g][3];
    const uint32_t tid = *(volatile uint32_t*)&ctl->tile_cid[g];
    if (!all_ok || tid == kSentinel) break;
    if (prof) { const uint64_t t = globaltimer(); phase_add(p, 0, t - t_mark); phase_add(p, 7, 1); t_mark = t; }
    tc_fence_after();
    const uint32_t tm = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(g * 256);
    const int64_t row_tile0 = (int64_t)tid * BPT * 128;
    const int64_t tile_e0 = row_tile0 * W;
    const int64_t tile_e1 = min(tile_e0 + (int64_t)C::TILE_ELEMS, p.n);

    // ---- start masks of every row of the tile ----
    long long cur = 0;  // bound cursor (kSegBounds)
    if constexpr (MODE == kSegBounds) {
      const int m = i & 7;
      if (wg_thread == 0) mbar_wait(&ctl->agg_full[m], (i >> 3) & 1u, wc, 6, i);
#pragma unroll
      for (int j = 0; j < BPT; ++j) smask[j * 128 + r] = 0ull;
      named_bar_sync(bar_id, 128);
      cur = *(volatile long long*)&ctl->tile_i0[m];
      // 512 bounds per round: four independent loads per thread in flight
      for (long long base = cur;; base += 512) {
        long long bb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const long long idx = base + wg_thread + 128 * u;
          bb[u] = idx < p.nbounds ? bound_at(p, idx) : LLONG_MAX;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (bb[u] < tile_e1 && bb[u] >= tile_e0) {
            const long long off = bb[u] - tile_e0;
            atomicOr(&smask[(int)(off / W)], 1ull << (off % W));
          }
        }
        if (wg_count(bb[3] < tile_e1, votes, lane, q, bar_id) < 128) break;
      }
      if (wg_thread == 0) mbar_arrive(&ctl->agg_empty[m]);  // every thread has read tile_i0
    } else {
      if constexpr (MODE == kSegPeriodic) {  // the summer has published this tile's aggregate
        const int m = i & 7;
        if (wg_thread == 0) {
          mbar_wait(&ctl->agg_full[m], (i >> 3) & 1u, wc, 6, i);
          mbar_arrive(&ctl->agg_empty[m]);
        }
      }
#pragma unroll
      for (int j = 0; j < BPT; ++j) smask[j * 128 + r] = row_start_mask<W, MODE>(p, (row_tile0 + j * 128 + r) * W);
    }

    // ---- (A) segmented row aggregates -> row offsets, tile aggregate ----
    V rowex[BPT];
    int exf[BPT];
    // F16SPLIT: the row scale factors of the tile, read here with the row
    // totals so both arrays are free for the converters after phase A
    float rsv[BPT];
#pragma unroll
    for (int j = 0; j < BPT; ++j) rsv[j] = C::F16SPLIT ? rsg[j * 128 + r] : 1.f;
    {
      uint32_t tb[BPT];
      double tbd[BPT];  // F16SPLIT: row aggregates in FP64 (exact totals for rows without a start)
      int fl[BPT];
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        const int64_t grow = row_tile0 + j * 128 + r;
        const bool is_tail = grow == p.full_rows && p.tail > 0;
        const bool live = grow < p.full_rows || is_tail;
        const unsigned long long mk = smask[j * 128 + r];
        // row aggregate after the row's last segment start: z[W-1] - z[ls-1]
        // (z[W-1] alone when the row holds no start).  Rows of a warp with
        // no start and no ragged tail need only their last column.
        uint32_t last = 0u, base = 0u;
        if (!__any_sync(0xffffffffu, mk != 0ull || is_tail)) {
          if constexpr (!C::F16SPLIT) {
            last = tmem_ld1(tm + (uint32_t)(j * W + W - 1));
            tmem_wait_ld();
          }
        } else {
          uint32_t v[W];
#pragma unroll
          for (int c = 0; c < W / 16; ++c)
            tmem_ld16(tm + (uint32_t)(j * W + c * 16), *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]));
          tmem_wait_ld();
          if constexpr (C::F16SPLIT) {
#pragma unroll
            for (int c = 0; c < W; ++c) v[c] = __float_as_uint(__uint_as_float(v[c]) * rsv[j]);
          }
          if (is_tail) {
            float accf = 0.f;
            int acci = 0;
#pragma unroll
            for (int c = 0; c < W / 16; ++c)
              tail_chunk<InT, W>(p, c * 16, *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]), accf, acci);
          }
          if (mk != 0ull && sums_out) {
            // per-segment sums issue no TMA stores, so the staging buffer is
            // free here: the row goes through it and z[ls - 1] is read back
            const int t = 62 - __clzll((long long)mk);  // ls - 1 (-1: start at column 0)
#pragma unroll
            for (int e4 = 0; e4 < W / 4; ++e4) {
              const int box = (e4 * 4) / C::OBW, cin = (e4 * 4) % C::OBW;
              *(uint4*)(stg_base + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW)) =
                  make_uint4(v[e4 * 4], v[e4 * 4 + 1], v[e4 * 4 + 2], v[e4 * 4 + 3]);
            }
            base = t < 0 ? 0u : stage_lookup(stg_base, (int64_t)r * W + t, W, C::OBW, C::OSW);
          } else if (mk != 0ull) {
            // base = z[ls - 1], the value before the row's last start ls
            // (four independent select chains, then one pick)
            const int t = 62 - __clzll((long long)mk);  // ls - 1 (-1: start at column 0)
            uint32_t part[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4)
#pragma unroll
              for (int c = 0; c < W / 4; ++c) {
                const int col = q4 * (W / 4) + c;
                part[q4] = (col == t) ? v[col] : part[q4];
              }
            const int qsel = t < 0 ? 0 : t / (W / 4);
            base = t < 0 ? 0u : (qsel == 0 ? part[0] : qsel == 1 ? part[1] : qsel == 2 ? part[2] : part[3]);
          }
          last = v[W - 1];
        }
        const bool seen = mk != 0ull;
        if constexpr (IS_INT) tb[j] = live ? (uint32_t)((int)last - (seen ? (int)base : 0)) : 0u;
        else tb[j] = live ? __float_as_uint(__uint_as_float(last) - (seen ? __uint_as_float(base) : 0.f)) : 0u;
        if constexpr (C::F16SPLIT)  // the exact row total when the aggregate is the whole row (no start after column 0)
          tbd[j] = (live && mk <= 1ull && !is_tail) ? rtg[j * 128 + r] : (double)__uint_as_float(tb[j]);
        fl[j] = (live && mk != 0ull) ? 1 : 0;
      }
      int rowf[BPT];
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        V ti = IS_INT ? (V)(int)tb[j] : (V)__uint_as_float(tb[j]);
        if constexpr (C::F16SPLIT) ti = (V)tbd[j];
        int fi = fl[j];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const V tp = __shfl_up_sync(0xffffffffu, ti, d);
          const int fp = __shfl_up_sync(0xffffffffu, fi, d);
          if (lane >= d) seg_combine(fi, ti, fp, tp);
        }
        V te = __shfl_up_sync(0xffffffffu, ti, 1);
        int fe = __shfl_up_sync(0xffffffffu, fi, 1);
        if (lane == 0) { te = V(0); fe = 0; }
        rowex[j] = te;
        rowf[j] = fe;
        if (lane == 31) {
          ctl->wt[g][j][q] = v_bits<V>(ti);
          ctl->wt_flag[g][j][q] = (uint8_t)fi;
        }
      }
      named_bar_sync(bar_id, 128);
      if (C::F16SPLIT && wg_thread == 0) mbar_arrive(&ctl->rt_free[g]);  // every thread has read rs / rt
      V run = V(0);
      int runf = 0;
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        V wpre = V(0), bsum = V(0);
        int wf = 0, bf = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const V wv = v_from_bits<V>(ctl->wt[g][j][k]);
          const int wfl = ctl->wt_flag[g][j][k];
          if (k < q) { if (wfl) { wpre = wv; wf = 1; } else { wpre += wv; } }
          if (wfl) { bsum = wv; bf = 1; } else { bsum += wv; }
        }
        V ex = rowex[j];
        int f = rowf[j];
        if (!f) { ex = wpre + ex; f = wf; }
        if (!f) { ex = run + ex; f = runf; }
        rowex[j] = ex;
        exf[j] = f;
        if (bf) { run = bsum; runf = 1; } else { run += bsum; }
      }
      if (prof) { const uint64_t t = globaltimer(); phase_add(p, 1, t - t_mark); t_mark = t; }
      // publish the (segmented) tile aggregate, then look back; a tile that
      // holds a segment start ends every look-back that reaches it
      // (sorted bounds and periodic segments: the summer warp published it
      // as soon as the tile's data landed)
      if (MODE != kSegBounds && MODE != kSegPeriodic && wg_thread == 0)
        publish_aggregate<V>((int64_t)tid, run, runf, V(0), p.descs, epoch);
      const V pre = wg_lookback<V>((int64_t)tid, run, V(0), p.descs, epoch, wc, &ctl->lb[g], wg_thread, bar_id,
                                   runf);
#pragma unroll
      for (int j = 0; j < BPT; ++j)
        if (!exf[j]) rowex[j] = pre + rowex[j];
      if (prof) { const uint64_t t = globaltimer(); phase_add(p, 2, t - t_mark); t_mark = t; }
    }

    // ---- (C) drain: in-row segment fix-ups, carry, staging, output ----
#pragma unroll 1
    for (int j = 0; j < BPT; ++j) {
      const int64_t brow0 = row_tile0 + j * 128;
      const int64_t grow = brow0 + r;
      const bool is_tail = (grow == p.full_rows) && p.tail > 0;
      const unsigned long long mk = smask[j * 128 + r];
      float accf = 0.f;
      int acci = 0;
      const float cf = IS_INT ? 0.f : (float)rowex[j];
      const uint32_t ci = IS_INT ? (uint32_t)(long long)rowex[j] : 0u;
      uint8_t* stg = stg_base + (nfill % C::STG_BUFS) * C::STG_BYTES;
      // per-segment sums: the first chunk of this block's bounds is loaded
      // now, its latency hidden behind the row work below
      long long pf_b = LLONG_MAX, pf_bp = 0;
      if (sums_out) {
        const long long idx = cur + wg_thread;
        if (idx < p.nbounds) pf_b = bound_at(p, idx);
        if (idx >= 1 && idx - 1 < p.nbounds) pf_bp = bound_at(p, idx - 1);
      }
      if (wg_thread == 0) {
        if (C::STG_BUFS == 2) bulk_wait_read1(); else bulk_wait_read0();
      }
      named_bar_sync(bar_id, 128);
      uint32_t v[W];
#pragma unroll
      for (int c = 0; c < W / 16; ++c)
        tmem_ld16(tm + (uint32_t)(j * W + c * 16), *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]));
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ctl->slot_empty[g][j]);
      // warps whose rows hold no segment start and no ragged tail: y = z +
      // carry (fp32 split: z * 2^-k + carry, fused), two columns per instruction
      const bool plain = !sums_out && !__any_sync(0xffffffffu, mk != 0ull || is_tail);
      if (plain) {
#pragma unroll
        for (int e4 = 0; e4 < W / 4; ++e4) {
          uint4 o;
          const uint32_t* ve = &v[e4 * 4];
          if constexpr (IS_INT) {
            o = make_uint4(ve[0] + ci, ve[1] + ci, ve[2] + ci, ve[3] + ci);
          } else {
            const f32x2_t c2 = f2_make(cf, cf);
            f32x2_t a = f2_bits(ve[0], ve[1]), b = f2_bits(ve[2], ve[3]);
            if constexpr (C::F16SPLIT) {
              const f32x2_t s2 = f2_make(rsv[j], rsv[j]);
              a = f2_fma(a, s2, c2);
              b = f2_fma(b, s2, c2);
            } else {
              a = f2_add(a, c2);
              b = f2_add(b, c2);
            }
            o = make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
          }
          const int cc = e4 * 4;
          const int box = cc / C::OBW, cin = cc % C::OBW;
          *(uint4*)(stg + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW)) = o;
        }
      } else {
      if constexpr (C::F16SPLIT) {  // undo the row's operand scale (a power of two: exact)
#pragma unroll
        for (int c = 0; c < W; ++c) v[c] = __float_as_uint(__uint_as_float(v[c]) * rsv[j]);
      }
      if (is_tail) {
#pragma unroll
        for (int c = 0; c < W / 16; ++c)
          tail_chunk<InT, W>(p, c * 16, *reinterpret_cast<uint32_t(*)[16]>(&v[c * 16]), accf, acci);
      }
      if (sums_out) {
        // per-segment sums need y only at segment ends: stage the raw row
        // prefixes z and keep the row's carry (in place of its start mask,
        // which this path no longer reads); the sums loop below forms
        // y[e] = z[e] - z[s - 1] or z[e] + carry with the same arithmetic
#pragma unroll
        for (int e4 = 0; e4 < W / 4; ++e4) {
          const int box = (e4 * 4) / C::OBW, cin = (e4 * 4) % C::OBW;
          *(uint4*)(stg + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW)) =
              make_uint4(v[e4 * 4], v[e4 * 4 + 1], v[e4 * 4 + 2], v[e4 * 4 + 3]);
        }
        smask[j * 128 + r] = IS_INT ? (unsigned long long)ci : (unsigned long long)__float_as_uint(cf);
      }
      // y[col] = z[col] - sub, with sub = -carry before the row's first
      // segment start and z[s - 1] (0 for s = 0) from a start s on; z + c and
      // z - (-c) round identically, so this matches the carry-add form
      const uint32_t mlo = (uint32_t)mk, mhi = (uint32_t)(mk >> 32);
      uint32_t subi = 0u - ci;
      float subf = -cf;
      if (!sums_out) {
#pragma unroll
        for (int e4 = 0; e4 < W / 4; ++e4) {
          uint32_t o[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int col = e4 * 4 + e;
            const bool st = ((col < 32 ? mlo : mhi) >> (col & 31)) & 1u;
            if (st) {
              subi = col ? v[col - 1] : 0u;
              subf = col ? __uint_as_float(v[col - 1]) : 0.f;
            }
            if constexpr (IS_INT) o[e] = v[col] - subi;
            else o[e] = __float_as_uint(__uint_as_float(v[col]) - subf);
          }
          const int cc = e4 * 4;
          const int box = cc / C::OBW, cin = cc % C::OBW;
          *(uint4*)(stg + box * (128 * C::OSW) + swz(r * C::OSW + cin * 4, C::OSW)) =
              make_uint4(o[0], o[1], o[2], o[3]);
          if (is_tail) {
            uint32_t* zt = (uint32_t*)p.z + p.full_rows * (int64_t)W + cc;
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (cc + e < p.tail) zt[e] = o[e];
          }
        }
      }
      }
      fence_proxy_async_smem();
      named_bar_sync(bar_id, 128);
      if (!sums_out) {
        if (wg_thread == 0) {
          if (p.has_map && brow0 < p.full_rows) {
#pragma unroll
            for (int b = 0; b < W / C::OBW; ++b)
              tma_store_2d(&out_map, b * C::OBW, (int32_t)brow0, stg + b * (128 * C::OSW));
          }
          bulk_commit();
        }
      } else {
        // one output per segment whose last element lies in this block:
        // out[k] = y[bounds[k+1] - 1] (0 for an empty segment)
        const int64_t be0 = brow0 * W;
        const int64_t be1 = min(be0 + 128 * (int64_t)W, p.n);
        for (long long base = cur;; base += 128) {
          const long long idx = base + wg_thread;
          const bool first = base == cur;
          const long long b = first ? pf_b : (idx < p.nbounds ? bound_at(p, idx) : LLONG_MAX);
          const bool in = b <= be1;
          if (in && idx >= 1 && (b > be0 || (be0 == 0 && b == 0))) {
            const long long bp = first ? pf_bp : bound_at(p, idx - 1);
            uint32_t val = 0u;
            if (b > bp && b > be0) {
              const int64_t e = b - 1 - be0;  // the segment's last element, local
              const int er = (int)(e / W);
              const int64_t rs = be0 + (int64_t)er * W;
              const uint32_t ze = stage_lookup(stg, e, W, C::OBW, C::OSW);
              if (bp >= rs) {  // the segment starts in this row
                const uint32_t zs = bp > rs ? stage_lookup(stg, bp - 1 - be0, W, C::OBW, C::OSW) : 0u;
                val = IS_INT ? ze - zs : __float_as_uint(__uint_as_float(ze) - __uint_as_float(zs));
              } else {  // it entered the row from above: add the row's carry
                const uint32_t c = (uint32_t)smask[j * 128 + er];
                val = IS_INT ? ze + c : __float_as_uint(__uint_as_float(ze) + __uint_as_float(c));
              }
            }
            static_cast<uint32_t*>(p.seg_out)[idx - 1] = val;
          }
          const int nin = wg_count(in, votes, lane, q, bar_id);
          if (nin < 128) {
            cur = base + nin;
            break;
          }
        }
        if (wg_thread == 0) bulk_commit();  // keeps the staging double-buffer accounting uniform
      }
      ++nfill;
    }
    if (prof) { const uint64_t t = globaltimer(); phase_add(p, 3, t - t_mark); t_mark = t; }
  }
  if (wg_thread == 0) bulk_wait_all0();
}

template <typename InT, int W, int MODE>
__global__ void __launch_bounds__(ScanCfg<InT, W, is_seg(MODE), MODE == kScanFullSmall>::THREADS, 1)
    scan_tc_kernel(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap out_map,
                   const ScanParams p) {
  using C = ScanCfg<InT, W, is_seg(MODE), MODE == kScanFullSmall>;
  constexpr bool IS_INT = C::IS_INT;
  constexpr int BPT = C::BPT;
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
      mbar_init(&ctl->empty[s], 2);  // MMA commit + summer/converter arrive
      mbar_init(&ctl->conv[s], C::NCONV);
    }
    for (int m = 0; m < 8; ++m) {
      mbar_init(&ctl->agg_full[m], 1);
      mbar_init(&ctl->agg_empty[m], 1);
    }
    mbar_init(&ctl->rt_free[0], 1);
    mbar_init(&ctl->rt_free[1], 1);
    for (int g = 0; g < 2; ++g) {
      mbar_init(&ctl->tile_full[g], 2);  // tcgen05.commit + releasing arrive after tile_cid
      for (int j = 0; j < BPT; ++j) mbar_init(&ctl->slot_empty[g][j], 4);  // one arrive per epilogue warp
    }
    mbar_init(&ctl->drain, 1);
    ctl->abort_flag = 0;
    ctl->epoch = *(volatile uint32_t*)&p.ws->epoch;
    fence_mbar_init();
  }
  build_upper<InT, W>(bmat);
  fence_proxy_async_smem();
  if (warp == 1) {
    tmem_alloc(&ctl->tmem_base, 512);
    tmem_relinquish();
  }
  if (warp == 0 && lane == 0 && p.has_map) {
    prefetch_tmap(&in_map);
    prefetch_tmap(&out_map);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = ctl->tmem_base;
  const uint32_t epoch = ctl->epoch;

  if (warp == 0) {
    // ================= TMA producer =================
    // A tile id is taken only once every stage of that tile is free, and all
    // of its blocks are then issued at once: the time from taking an id to
    // its aggregate being published is one TMA round trip, never this CTA's
    // backlog.  fp32 launches, whose ring holds one tile (4 stages of 32 KB),
    // take the id when the tile's first stage is free and issue each later
    // block as its stage frees, so the next tile's loads overlap the current
    // tile's conversion instead of following it.
    constexpr int kWaitFirst = (C::F16SPLIT && C::NSTAGE < 2 * BPT) ? 1 : BPT;
    if (lane == 0) {
      uint32_t issued[32];
#pragma unroll
      for (int s = 0; s < 32; ++s) issued[s] = 0;
      uint32_t k = 0;  // block sequence number
      bool stop = false;
      while (!stop) {
        const uint64_t tw = p.phase_ns ? globaltimer() : 0;
        for (int j = 0; j < kWaitFirst && !stop; ++j) {
          const uint32_t kj = k + j;
          const int s = kj % C::NSTAGE;
          if (kj >= (uint32_t)C::NSTAGE && !mbar_wait(&ctl->empty[s], ((kj / C::NSTAGE) & 1u) ^ 1u, wc, 1, kj))
            stop = true;
        }
        if (stop) break;
        if (p.phase_ns) phase_add(p, 4, globaltimer() - tw);
        const uint32_t tid = atomicAdd(&p.ws->tile_counter, 1u);
        const bool live = (int64_t)tid < p.num_tiles;
        const int nblk = live ? BPT : 1;
        for (int j = 0; j < nblk; ++j, ++k) {
          const int s = k % C::NSTAGE;
          if (j >= kWaitFirst && k >= (uint32_t)C::NSTAGE &&
              !mbar_wait(&ctl->empty[s], ((k / C::NSTAGE) & 1u) ^ 1u, wc, 1, k)) {
            stop = true;
            break;
          }
          ctl->stage_cid[s] = live ? tid : kSentinel;
          issued[s]++;
          const int64_t row0 = ((int64_t)tid * BPT + j) * 128;
          if (live && p.has_map && row0 < p.full_rows) {
            mbar_arrive_expect_tx(&ctl->full[s], C::STAGE_BYTES);
#pragma unroll
            for (int kb = 0; kb < C::IN_KB; ++kb)
              tma_load_2d(smem + s * C::STAGE_BYTES + kb * (128 * C::IN_SW), &in_map,
                          kb * (C::IN_SW / C::IN_BYTES), (int32_t)row0, &ctl->full[s]);
          } else {
            mbar_arrive(&ctl->full[s]);
          }
        }
        if (!live || aborted(wc)) stop = true;
      }
      // every load issued must have landed before the CTA exits
      for (int s = 0; s < C::NSTAGE; ++s)
        if (issued[s]) mbar_drain(&ctl->full[s], (issued[s] - 1) & 1u, p.timeout_ns);
    }
  } else if (warp == 1) {
    // ================= MMA issuer =================
    if (lane == 0) {
      constexpr uint32_t IDESC =
          IS_INT ? umma_idesc(CF_S32, AB_S8, 128, W)
                 : umma_idesc(CF_F32, (__is_same(InT, __nv_bfloat16) || C::PRESPLIT) ? AB_BF16 : AB_F16, 128, W);
      const uint32_t b_addr = smem_u32(bmat);
      uint32_t k = 0;
      for (uint32_t i = 0;; ++i) {  // tile sequence of this CTA
        const int g = i & 1;
        const uint32_t u = i >> 1;
        bool fail = false, sentinel = false;
        for (int j = 0; j < BPT; ++j, ++k) {
          const int s = k % C::NSTAGE;
          // fp32 inputs: wait until the converter has rewritten the stage as
          // bf16 hi/lo operands (it signals the stop-marker stage too)
          if (!mbar_wait(C::IS_F32 ? &ctl->conv[s] : &ctl->full[s], (k / C::NSTAGE) & 1u, wc, 2, i)) {
            fail = true;
            break;
          }
          const uint32_t tid = *(volatile uint32_t*)&ctl->stage_cid[s];
          if (tid == kSentinel) { sentinel = true; break; }
          if (u >= 1 && !mbar_wait(&ctl->slot_empty[g][j], (u & 1u) ^ 1u, wc, 3, tid)) { fail = true; break; }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + (uint32_t)(g * 256 + j * W);
          const uint32_t a_addr = smem_u32(smem + s * C::STAGE_BYTES);
#pragma unroll
          for (int kb = 0; kb < C::KB; ++kb) {
#pragma unroll
            for (int ks = 0; ks < C::KSTEPS; ++ks) {
              const uint64_t ad = umma_desc_kmajor(a_addr + kb * (128 * C::SW) + ks * 32, C::SW);
              const uint64_t bd = umma_desc_kmajor(b_addr + kb * (W * C::SW) + ks * 32, C::SW);
              if constexpr (IS_INT) {
                mma_i8(d_tmem, ad, bd, IDESC, (kb | ks) != 0);
              } else if constexpr (C::IS_F32) {
                // split precision: D += hi . U, then D += lo . U (FP32 accumulate)
                mma_f16(d_tmem, ad, bd, IDESC, (kb | ks) != 0);
                const uint64_t adl = umma_desc_kmajor(a_addr + C::TERM_BYTES + kb * (128 * C::SW) + ks * 32, C::SW);
                mma_f16(d_tmem, adl, bd, IDESC, 1u);
              } else {
                mma_f16(d_tmem, ad, bd, IDESC, (kb | ks) != 0);
              }
            }
          }
          tc_commit(&ctl->empty[s]);
          if (j == BPT - 1) {
            ctl->tile_cid[g] = tid;
            mbar_arrive(&ctl->tile_full[g]);  // releases the tile_cid store
            tc_commit(&ctl->tile_full[g]);
          }
        }
        if (fail) break;
        if (sentinel) {
          // stop marker for both warpgroups: tile i -> g, tile i+1 -> g^1
          for (int e = 0; e < 2; ++e) {
            const uint32_t ie = i + e;
            const int ge = ie & 1;
            const uint32_t ue = ie >> 1;
            if (ue >= 1 && !mbar_wait(&ctl->slot_empty[ge][BPT - 1], (ue & 1u) ^ 1u, wc, 4, 0)) break;
            ctl->tile_cid[ge] = kSentinel;
            mbar_arrive(&ctl->tile_full[ge]);
            mbar_arrive(&ctl->tile_full[ge]);
          }
          break;
        }
      }
      tc_commit(&ctl->drain);
      mbar_drain(&ctl->drain, 0, p.timeout_ns);
    }
  } else if (warp < 10) {
    if constexpr (is_seg(MODE)) seg_epilogue<InT, W, MODE>(p, out_map, smem, ctl, tmem_base, epoch, wc);
    else scan_epilogue<InT, W, MODE>(p, out_map, smem, ctl, tmem_base, epoch, wc);
  } else if (warp == 10) {
    scan_summer<InT, W, MODE>(p, smem, ctl, epoch, wc);
  } else {
    scan_converter2<InT, W, MODE>(p, smem, ctl, wc, warp - 10);
  }

  // ---- teardown ----
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
  if (threadIdx.x == 0) {
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

}  // namespace tcu

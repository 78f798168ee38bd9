// tcu_capi.cu -- extern "C" entry points of libtcuscan.so: argument checks,
// TMA tensor-map construction, kernel selection and launch.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "tcu_host.h"
#include "tcu_scan_tc.cuh"

namespace tcu {

static thread_local char g_errmsg[512] = "";
static uint64_t g_timeout_ns = 4000000000ull;
static int g_phase_profile = 0;
static int g_max_ctas = 0;  // 0: one CTA per SM

tcu_status_t cuda_fail(cudaError_t e, const char* what) {
  snprintf(g_errmsg, sizeof(g_errmsg), "%s: %s", what, cudaGetErrorString(e));
  return TCU_ERR_LAUNCH;
}

uint64_t timeout_ns() { return g_timeout_ns; }

// Self-test of the bounded waits: one warp waits, with the library's own
// wait code, on something that nothing will ever complete -- an mbarrier
// phase (which = 0) or the look-back descriptor of tile 0 (which = 1), read
// as the look-back of tile 1 does.  The wait gives up after timeout_ns,
// records TCU_ERR_TIMEOUT with its site in the workspace and the kernel
// returns; no fault, no trap, and the context stays usable.
__global__ void selftest_wait_kernel(WsHeader* ws, TileDesc* descs, int which, uint64_t timeout_ns) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncwarp();
  WaitCtx wc{ws, &abort_flag, timeout_ns};
  if (which == 0) {
    if (threadIdx.x == 0) mbar_wait(&bar, 0u, wc, 900, 0);
  } else {
    const uint32_t epoch = *(volatile uint32_t*)&ws->epoch;
    warp_lookback<long long>(1, 0ll, 0, 0ll, descs, epoch, wc, false);
  }
  // the look-back published tile 1 under the current epoch: retire the epoch,
  // as every launch's last CTA does, so the next launch cannot read it
  __syncwarp();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&ws->epoch, 1u);
  }
}

// CTAs of a persistent launch: one per SM, capped by tcu_set_max_ctas.
int grid_ctas() {
  const int sms = sm_count();
  return (g_max_ctas > 0 && g_max_ctas < sms) ? g_max_ctas : sms;
}

int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  static int cached[64] = {0};
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = v > 0 ? v : 148;
  }
  return cached[dev];
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D row-major tensor [rows, cols] of `elem`-byte elements, box [box_rows,
// box_cols], swizzle span = box_cols * elem bytes (32/64/128; 16 = unswizzled).
// The last few encoded maps of this thread, by their arguments: a repeated
// call on the same buffers (the small scans of a serving loop or a chained
// host scan) copies the map instead of encoding it again (~1 us each).
namespace {
struct MapKey {
  const void* base;
  uint64_t cols, rows;
  int dt, elem;
  uint32_t box_cols, box_rows;
  bool operator==(const MapKey& o) const {
    return base == o.base && cols == o.cols && rows == o.rows && dt == o.dt && elem == o.elem &&
           box_cols == o.box_cols && box_rows == o.box_rows;
  }
};
struct MapCache {
  static constexpr int N = 8;
  MapKey key[N];
  CUtensorMap map[N];
  bool used[N] = {};
  int next = 0;
};
thread_local MapCache t_maps;
}  // namespace

tcu_status_t make_map_2d(CUtensorMap* m, const void* base, CUtensorMapDataType dt, int elem, uint64_t cols,
                         uint64_t rows, uint32_t box_cols, uint32_t box_rows) {
  const MapKey k{base, cols, rows, (int)dt, elem, box_cols, box_rows};
  for (int i = 0; i < MapCache::N; ++i) {
    if (t_maps.used[i] && t_maps.key[i] == k) {
      *m = t_maps.map[i];
      return TCU_OK;
    }
  }
  auto fn = encode_fn();
  if (!fn) {
    snprintf(g_errmsg, sizeof(g_errmsg), "cuTensorMapEncodeTiled entry point unavailable");
    return TCU_ERR_DEVICE;
  }
  const uint32_t span = box_cols * elem;
  CUtensorMapSwizzle sw = span == 128  ? CU_TENSOR_MAP_SWIZZLE_128B
                          : span == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                          : span == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                                       : CU_TENSOR_MAP_SWIZZLE_NONE;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * (uint64_t)elem};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    snprintf(g_errmsg, sizeof(g_errmsg), "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TCU_ERR_LAUNCH;
  }
  const int slot = t_maps.next;
  t_maps.next = (slot + 1) % MapCache::N;
  t_maps.key[slot] = k;
  t_maps.map[slot] = *m;
  t_maps.used[slot] = true;
  return TCU_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Workspace layout: 64-byte header | 64 bytes pad | TileDesc[cap].
int64_t ws_capacity(size_t bytes) {
  if (bytes < 256) return 0;
  return (int64_t)((bytes - 128) / sizeof(TileDesc));
}
TileDesc* ws_descs(void* ws) { return reinterpret_cast<TileDesc*>(static_cast<uint8_t*>(ws) + 128); }
// Eight 64-bit phase counters live in the 64 bytes between header and descriptors.
unsigned long long* ws_phase_counters(void* ws) {
  return reinterpret_cast<unsigned long long*>(static_cast<uint8_t*>(ws) + 64);
}

// ---------------------------------------------------------------------------
// Tensor-core scan launcher.
// Segment description of the segmented modes (unused fields stay zero).
struct SegArgs {
  const int8_t* flags = nullptr;
  const void* bounds = nullptr;
  int64_t nbounds = 0;
  int bounds64 = 0;
  int out_sums = 0;
  int64_t period = 0;
  void* seg_out = nullptr;
};

// Internal input type code (not part of tcu_dtype_t): pre-split fp32 rows.
constexpr tcu_dtype_t kDtypeSplitF32 = (tcu_dtype_t)100;

template <typename InT, int W, int MODE>
static tcu_status_t launch_scan_tc(const void* x, int64_t n, void* z, double start_f, long long start_i,
                                   int seg_rows, void* ws, size_t ws_bytes, cudaStream_t st,
                                   const SegArgs& sa = SegArgs(), const void* start_dev = nullptr,
                                   int start_dev_kind = 0) {
  using C = ScanCfg<InT, W, is_seg(MODE), MODE == kScanFullSmall>;
  ScanParams p{};
  p.x = x;
  p.z = z;
  p.n = n;
  p.full_rows = n / W;
  p.tail = (int32_t)(n % W);
  p.seg_rows = seg_rows;
  const int64_t total_rows = p.full_rows + (p.tail ? 1 : 0);
  const int64_t tile_rows = 128 * C::BPT;
  p.num_tiles = (total_rows + tile_rows - 1) / tile_rows;
  p.start_f = start_f;
  p.start_i = start_i;
  p.start_dev = start_dev;
  p.start_dev_kind = start_dev_kind;
  p.timeout_ns = g_timeout_ns;
  if (ws == nullptr || ws_capacity(ws_bytes) < p.num_tiles) {
    snprintf(g_errmsg, sizeof(g_errmsg), "workspace too small: %lld tiles need %zu bytes", (long long)p.num_tiles,
             tcu_workspace_bytes(n, W));
    return TCU_ERR_WORKSPACE;
  }
  if (p.num_tiles > 0xFFFFFFF0ll) return TCU_ERR_ARG;
  p.ws = static_cast<WsHeader*>(ws);
  p.descs = ws_descs(ws);
  p.phase_ns = g_phase_profile ? ws_phase_counters(ws) : nullptr;
  p.flags = sa.flags;
  p.bounds = sa.bounds;
  p.nbounds = sa.nbounds;
  p.bounds64 = sa.bounds64;
  p.out_sums = sa.out_sums;
  p.period = sa.period;
  p.seg_out = sa.seg_out;
  // kSegBounds: every tile's first bound index, precomputed into the
  // workspace after the tile descriptors (zeroed again after the scan, so the
  // descriptor region never holds stale non-descriptor data)
  long long* tile_first = nullptr;
  if (MODE == kSegBounds && sa.nbounds > 0) {
    if (ws_capacity(ws_bytes) < p.num_tiles + (p.num_tiles + 1) / 2 + 1) return TCU_ERR_WORKSPACE;
    tile_first = reinterpret_cast<long long*>(p.descs + p.num_tiles);
    int64_t grid = (sa.nbounds + 1 + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 8;
    if (grid > cap) grid = cap;
    bounds_tiles_kernel<<<(int)grid, 256, 0, st>>>(sa.bounds, sa.bounds64, sa.nbounds, (int64_t)C::TILE_ELEMS,
                                                    p.num_tiles, tile_first);
    p.tile_first = tile_first;
  }

  CUtensorMap in_map, out_map;
  std::memset(&in_map, 0, sizeof(in_map));
  std::memset(&out_map, 0, sizeof(out_map));
  p.has_map = p.full_rows > 0;
  if (p.full_rows > 0) {
    const CUtensorMapDataType idt = C::IN_BYTES == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                    : (C::IN_BYTES == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT32);
    tcu_status_t s =
        make_map_2d(&in_map, x, idt, C::IN_BYTES, W, (uint64_t)p.full_rows, C::IN_SW / C::IN_BYTES, 128);
    if (s != TCU_OK) return s;
    if (z != nullptr) {
      s = make_map_2d(&out_map, z, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, W, (uint64_t)p.full_rows, C::OBW, 128);
      if (s != TCU_OK) return s;
    }
  }
  const int smem = C::SMEM_BYTES < 120 * 1024 ? 120 * 1024 : C::SMEM_BYTES;
  auto kern = scan_tc_kernel<InT, W, MODE>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    attr_set = true;
  }
  int grid = grid_ctas();
  if (p.num_tiles < grid) grid = (int)p.num_tiles;
  kern<<<grid, C::THREADS, smem, st>>>(in_map, out_map, p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "scan_tc_kernel launch");
  if (tile_first) {
    e = cudaMemsetAsync(tile_first, 0, (size_t)p.num_tiles * sizeof(long long), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(tile_first)");
  }
  return TCU_OK;
}

// Full scans whose 32768-element tiles would leave SMs idle run with one
// 128 x S block per tile instead (kScanFullSmall).  The limit is in default
// tiles; tcu_set_small_tile_limit changes it (0 = never).
static int g_small_tile_limit = -1;  // -1: the SM count
static bool use_small_tiles(int64_t n) {
  const int64_t lim = g_small_tile_limit < 0 ? (int64_t)sm_count() : (int64_t)g_small_tile_limit;
  return (n + 32767) / 32768 < lim;
}

// Full scans of at most this many elements run on the SIMT cores
// (scan_small, tcu_scan_small.cu): below it the tensor-core tile chain, not
// HBM, bounds the launch.  Measured on B200 (CUDA-graph replays): SIMT
// ahead up to 2^18 fp16 / fp32 elements (6.3 vs 8.3 us at 2^14) and 2^20
// int8 (8.3 vs 10.3 us), the tensor cores ahead from there (fp16 2^20: 10.3
// vs 11.7 us).  tcu_set_simt_scan_limit sets one limit for every dtype
// (0 = never, negative = these defaults).
static int64_t g_simt_scan_limit = -1;
static int64_t simt_limit(tcu_dtype_t dt) {
  if (g_simt_scan_limit >= 0) return g_simt_scan_limit;
  return dt == TCU_INT8 ? (int64_t(1) << 20) : (int64_t(1) << 18);
}

static bool valid_scan_S(tcu_dtype_t dt, int S) {
  if (dt == TCU_INT8) return S == 32 || S == 64 || S == 128;
  if (dt == TCU_FLOAT16) return S == 16 || S == 32 || S == 64 || S == 128;
  return dt == TCU_FLOAT32;
}

template <int MODE>
static tcu_status_t dispatch_scan(const void* x, tcu_dtype_t dt, int64_t n, int S, void* z, double start, int seg_rows,
                                  void* ws, size_t ws_bytes, cudaStream_t st, const void* start_dev = nullptr,
                                  int sk = -1) {
  if (sk < 0) sk = dt == TCU_INT8 ? 0 : 1;  // default device start: an output element (int32 / fp32)
  if constexpr (MODE == kScanFull) {
    if (n <= simt_limit(dt) && valid_scan_S(dt, S))
      return scan_small(x, dt, n, z, start, ws, ws_bytes, st, start_dev, sk);
    if (use_small_tiles(n))
      return dispatch_scan<kScanFullSmall>(x, dt, n, S, z, start, seg_rows, ws, ws_bytes, st, start_dev, sk);
  }
  const long long si = (long long)start;
  if (dt == TCU_INT8) {
    switch (S) {
      case 32: return launch_scan_tc<int8_t, 32, MODE>(x, n, z, 0.0, si, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      case 64: return launch_scan_tc<int8_t, 64, MODE>(x, n, z, 0.0, si, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      case 128: return launch_scan_tc<int8_t, 128, MODE>(x, n, z, 0.0, si, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      default: return TCU_ERR_ARG;
    }
  }
  if (dt == TCU_FLOAT32) {  // split-precision fp16 hi + lo operands, 64-column rows
    if constexpr (is_full(MODE))
      return launch_scan_tc<float, 64, MODE>(x, n, z, start, 0, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
    return TCU_ERR_DTYPE;
  }
  if (dt == TCU_FLOAT16) {
    switch (S) {
      case 16: return launch_scan_tc<__half, 16, MODE>(x, n, z, start, 0, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      case 32: return launch_scan_tc<__half, 32, MODE>(x, n, z, start, 0, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      case 64: return launch_scan_tc<__half, 64, MODE>(x, n, z, start, 0, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      case 128: return launch_scan_tc<__half, 128, MODE>(x, n, z, start, 0, seg_rows, ws, ws_bytes, st, SegArgs(), start_dev, sk);
      default: return TCU_ERR_ARG;
    }
  }
  return TCU_ERR_DTYPE;
}

template <int MODE>
static tcu_status_t dispatch_seg(const void* x, tcu_dtype_t dt, int64_t n, int S, void* z, const SegArgs& sa, void* ws,
                                 size_t ws_bytes, cudaStream_t st) {
  const int W = S <= 32 ? 32 : 64;  // segmented results do not depend on the tile width
  if (dt == TCU_INT8) {
    if (W == 32) return launch_scan_tc<int8_t, 32, MODE>(x, n, z, 0.0, 0, 0, ws, ws_bytes, st, sa);
    return launch_scan_tc<int8_t, 64, MODE>(x, n, z, 0.0, 0, 0, ws, ws_bytes, st, sa);
  }
  if (dt == TCU_FLOAT16) {
    if (W == 32) return launch_scan_tc<__half, 32, MODE>(x, n, z, 0.0, 0, 0, ws, ws_bytes, st, sa);
    return launch_scan_tc<__half, 64, MODE>(x, n, z, 0.0, 0, 0, ws, ws_bytes, st, sa);
  }
  if (dt == TCU_FLOAT32) return launch_scan_tc<float, 64, MODE>(x, n, z, 0.0, 0, 0, ws, ws_bytes, st, sa);
  if constexpr (MODE == kSegBounds) {  // internal: fp32 rows already split into bf16 hi / lo (SpMV products)
    if (dt == kDtypeSplitF32) return launch_scan_tc<SplitF32, 64, MODE>(x, n, z, 0.0, 0, 0, ws, ws_bytes, st, sa);
  }
  return TCU_ERR_DTYPE;
}

}  // namespace tcu

using namespace tcu;

extern "C" {

int tcu_version(void) { return 100; }

const char* tcu_status_string(int s) {
  switch (s) {
    case TCU_OK: return "ok";
    case TCU_ERR_ARG: return "invalid argument";
    case TCU_ERR_DTYPE: return "unsupported dtype";
    case TCU_ERR_LAUNCH: return "CUDA launch error";
    case TCU_ERR_TIMEOUT: return "device wait timed out";
    case TCU_ERR_OOM: return "out of memory";
    case TCU_ERR_ALIGN: return "pointer not 16-byte aligned";
    case TCU_ERR_DEVICE: return "device unsupported";
    case TCU_ERR_WORKSPACE: return "workspace missing or too small";
    default: return "unknown status";
  }
}

const char* tcu_last_error_message(void) { return g_errmsg; }

void tcu_set_phase_profile(int enable) { g_phase_profile = enable ? 1 : 0; }
void tcu_set_max_ctas(int n) { g_max_ctas = n > 0 ? n : 0; }
void tcu_set_small_tile_limit(int tiles) { g_small_tile_limit = tiles < 0 ? -1 : tiles; }
void tcu_set_simt_scan_limit(int64_t n) { g_simt_scan_limit = n < 0 ? -1 : n; }
int64_t tcu_get_simt_scan_limit(void) { return g_simt_scan_limit; }
int tcu_get_small_tile_limit(void) { return g_small_tile_limit < 0 ? sm_count() : g_small_tile_limit; }
int tcu_get_max_ctas(void) { return g_max_ctas; }

tcu_status_t tcu_workspace_phase_ns(void* ws, uint64_t out[8], int clear, void* stream) {
  if (!ws) return TCU_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(out, ws_phase_counters(ws), 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && clear) {
    e = cudaMemsetAsync(ws_phase_counters(ws), 0, 8 * sizeof(uint64_t), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "phase counters");
}

void tcu_set_timeout_ns(uint64_t ns) { g_timeout_ns = ns ? ns : 4000000000ull; }
uint64_t tcu_get_timeout_ns(void) { return g_timeout_ns; }

size_t tcu_workspace_bytes(int64_t n, int S) {
  (void)S;  // the smallest look-back tile of any kernel is 2048 elements
  if (n < 0) n = 0;
  const int64_t tiles = (n + 2047) / 2048 + 2;
  return 128 + (size_t)tiles * sizeof(TileDesc);
}

tcu_status_t tcu_workspace_init(void* ws, size_t ws_bytes, void* stream) {
  if (!ws || ws_bytes < 256) return TCU_ERR_WORKSPACE;
  cudaError_t e = cudaMemsetAsync(ws, 0, ws_bytes, (cudaStream_t)stream);
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(workspace)");
}

tcu_status_t tcu_workspace_error(void* ws, uint32_t info[3], int clear, void* stream) {
  if (!ws) return TCU_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  WsHeader h;
  cudaError_t e = cudaMemcpyAsync(&h, ws, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "read workspace error");
  info[0] = h.error;
  info[1] = h.err_site;
  info[2] = h.err_chunk;
  if (clear && h.error) {
    e = cudaMemsetAsync(&static_cast<WsHeader*>(ws)->error, 0, 3 * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "clear workspace error");
  }
  return (tcu_status_t)h.error;
}

tcu_status_t tcu_selftest_wait_timeout(int which, uint64_t timeout_ns, void* ws, size_t ws_bytes, void* stream) {
  if (!ws || ws_capacity(ws_bytes) < 2) return TCU_ERR_WORKSPACE;
  if (which != 0 && which != 1) return TCU_ERR_ARG;
  if (timeout_ns == 0 || timeout_ns > 2000000000ull) return TCU_ERR_ARG;  // at most 2 s
  selftest_wait_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(static_cast<WsHeader*>(ws), ws_descs(ws), which,
                                                           timeout_ns);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "selftest_wait_kernel launch");
}

tcu_status_t tcu_scan_chained(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start,
                              const void* start_dev, void* z, void* ws, size_t ws_bytes, void* stream) {
  return tcu_scan_chained_typed(x, x_dtype, n, S, start, start_dev, x_dtype == TCU_INT8 ? TCU_INT32 : TCU_FLOAT32, z,
                                ws, ws_bytes, stream);
}

tcu_status_t tcu_scan_chained_typed(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start,
                                    const void* start_dev, tcu_dtype_t start_dtype, void* z, void* ws,
                                    size_t ws_bytes, void* stream) {
  if (n < 0) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  int sk;
  switch (start_dtype) {
    case TCU_INT32: sk = 0; break;
    case TCU_FLOAT32: sk = 1; break;
    case TCU_INT64: sk = 2; break;
    case TCU_FLOAT64: sk = 3; break;
    default: return TCU_ERR_DTYPE;
  }
  const uintptr_t amask = sk >= 2 ? 7u : 3u;
  if (!aligned16(x) || !aligned16(z) || (reinterpret_cast<uintptr_t>(start_dev) & amask)) return TCU_ERR_ALIGN;
  if (x_dtype == TCU_INT8 && S == 16) S = 32;
  return dispatch_scan<kScanFull>(x, x_dtype, n, S, z, start, 0, ws, ws_bytes, (cudaStream_t)stream, start_dev, sk);
}

tcu_status_t tcu_scan(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start, void* z, void* ws,
                      size_t ws_bytes, void* stream) {
  if (n < 0) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(z)) return TCU_ERR_ALIGN;
  if (x_dtype == TCU_INT8 && S == 16) S = 32;  // full scans are independent of S; 8-bit K step is 32
  return dispatch_scan<kScanFull>(x, x_dtype, n, S, z, start, 0, ws, ws_bytes, (cudaStream_t)stream);
}

tcu_status_t tcu_row_scan(const void* x, tcu_dtype_t x_dtype, int64_t n_rows, int S, void* z, void* ws,
                          size_t ws_bytes, void* stream) {
  if (n_rows < 0) return TCU_ERR_ARG;
  if (n_rows == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(z)) return TCU_ERR_ALIGN;
  return dispatch_scan<kScanRows>(x, x_dtype, n_rows * S, S, z, 0.0, 0, ws, ws_bytes, (cudaStream_t)stream);
}

tcu_status_t tcu_seg_scan(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, const int8_t* flags, int flags_are_ends,
                          void* z, void* ws, size_t ws_bytes, void* stream) {
  if (n < 0) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !z || !flags) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(z) || !aligned16(flags)) return TCU_ERR_ALIGN;
  SegArgs sa;
  sa.flags = flags;
  if (flags_are_ends)
    return dispatch_seg<kSegEnds>(x, x_dtype, n, S, z, sa, ws, ws_bytes, (cudaStream_t)stream);
  return dispatch_seg<kSegFlags>(x, x_dtype, n, S, z, sa, ws, ws_bytes, (cudaStream_t)stream);
}

tcu_status_t tcu_seg_bounds(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, const void* bounds,
                            tcu_dtype_t bounds_dtype, int64_t nbounds, int out_sums, void* out, void* ws,
                            size_t ws_bytes, void* stream) {
  if (n < 0 || nbounds < 0) return TCU_ERR_ARG;
  if (bounds_dtype != TCU_INT32 && bounds_dtype != TCU_INT64) return TCU_ERR_DTYPE;
  cudaStream_t st = (cudaStream_t)stream;
  if (out_sums && nbounds >= 2 && n == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)(nbounds - 1) * 4, st);
    return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(empty seg sums)");
  }
  if (n == 0 || (out_sums && nbounds < 2)) return TCU_OK;
  if (!x || !out || !bounds || nbounds < 1) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(out)) return TCU_ERR_ALIGN;
  if ((reinterpret_cast<uintptr_t>(bounds) & (bounds_dtype == TCU_INT64 ? 7u : 3u)) != 0) return TCU_ERR_ALIGN;
  SegArgs sa;
  sa.bounds = bounds;
  sa.nbounds = nbounds;
  sa.bounds64 = bounds_dtype == TCU_INT64;
  sa.out_sums = out_sums ? 1 : 0;
  sa.seg_out = out_sums ? out : nullptr;
  return dispatch_seg<kSegBounds>(x, x_dtype, n, S, out_sums ? nullptr : out, sa, ws, ws_bytes, st);
}

tcu_status_t tcu_spmv_csr(const void* vals, tcu_dtype_t dtype, const void* indptr, tcu_dtype_t indptr_dtype,
                          int64_t rows, const int32_t* cols, int64_t nnz, const void* x, int64_t x_len, int S, float* y,
                          float* prod_tmp, void* ws, size_t ws_bytes, void* stream) {
  if (rows < 0 || nnz < 0) return TCU_ERR_ARG;
  if (rows == 0) return TCU_OK;
  if (!y || !indptr || (nnz > 0 && (!prod_tmp || !vals || !cols || !x))) return TCU_ERR_ARG;
  if (nnz > 0 && !aligned16(prod_tmp)) return TCU_ERR_ALIGN;
  // products are written already split into the bf16 hi / lo operand rows
  // of the tensor-core sum, which then needs no conversion pass
  tcu_status_t s = spmv_products_split(vals, dtype, cols, nnz, x, x_len, prod_tmp, ws, stream);
  if (s != TCU_OK) return s;
  if (nnz == 0) {
    cudaError_t e = cudaMemsetAsync(y, 0, (size_t)rows * sizeof(float), (cudaStream_t)stream);
    return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(y)");
  }
  if (indptr_dtype != TCU_INT32 && indptr_dtype != TCU_INT64) return TCU_ERR_DTYPE;
  if ((reinterpret_cast<uintptr_t>(indptr) & (indptr_dtype == TCU_INT64 ? 7u : 3u)) != 0) return TCU_ERR_ALIGN;
  SegArgs sa;
  sa.bounds = indptr;
  sa.nbounds = rows + 1;
  sa.bounds64 = indptr_dtype == TCU_INT64;
  sa.out_sums = 1;
  sa.seg_out = y;
  return dispatch_seg<kSegBounds>(prod_tmp, kDtypeSplitF32, nnz, S, nullptr, sa, ws, ws_bytes, (cudaStream_t)stream);
}

tcu_status_t tcu_scan_batch(const void* x, tcu_dtype_t x_dtype, int64_t batch, int64_t len, int S, void* z, void* ws,
                            size_t ws_bytes, void* stream) {
  if (batch < 0 || len < 0) return TCU_ERR_ARG;
  if (batch == 0 || len == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(z)) return TCU_ERR_ALIGN;
  SegArgs sa;
  sa.period = len;
  return dispatch_seg<kSegPeriodic>(x, x_dtype, batch * len, S, z, sa, ws, ws_bytes, (cudaStream_t)stream);
}

tcu_status_t tcu_block_scan(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, void* z, void* ws,
                            size_t ws_bytes, void* stream) {
  if (n < 0 || S <= 0 || n % ((int64_t)S * S) != 0) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(z)) return TCU_ERR_ALIGN;
  return dispatch_scan<kScanBlocks>(x, x_dtype, n, S, z, 0.0, S, ws, ws_bytes, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Inclusive scan that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they need a
// scan: code that runs inside a custom allocator or memory-pool callback
// (allocating there would re-enter the allocator), hosts that hand a plugin a
// fixed device budget and forbid further allocations, and latency-critical
// paths that must never reach cudaMalloc's implicit synchronisation.
// tcu_scan asks its caller for a look-back workspace; this variant takes it
// from a fixed array compiled into the library instead.
namespace tcu {

constexpr size_t kNoAllocScratchBytes = 1u << 20;  // 1 MiB per GPU that loads the library
// The scratch holds a 128-byte header and one 16-byte look-back descriptor
// per 32768-element tile: (1 MiB - 128) / 16 = 65528 tiles.
constexpr int64_t kNoAllocMaxN = (int64_t)((kNoAllocScratchBytes - 128) / sizeof(TileDesc)) * 32768;

// Device scratch of tcu_scan_noalloc.  In host code this name is only a
// host-side stand-in: kernels get the device address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch on the current device.  The first call on a
// device looks the address up and zeroes the array on `st`; the address is
// cached for the life of the process (a cudaDeviceReset would make it stale).
static tcu_status_t noalloc_scratch(cudaStream_t st, void** out) {
  static std::mutex mu;
  static void* ptrs[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "tcu_scan_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 64) return TCU_ERR_DEVICE;
  std::lock_guard<std::mutex> lock(mu);
  if (ptrs[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return cuda_fail(e, "tcu_scan_noalloc: cudaGetSymbolAddress");
    e = cudaMemsetAsync(p, 0, kNoAllocScratchBytes, st);
    if (e != cudaSuccess) return cuda_fail(e, "tcu_scan_noalloc: zeroing the scratch");
    ptrs[dev] = p;
  }
  *out = ptrs[dev];
  return TCU_OK;
}

}  // namespace tcu

extern "C" tcu_status_t tcu_scan_noalloc(const void* x, tcu_dtype_t x_dtype, int64_t n, int S, double start, void* z,
                                         void* stream) {
  if (n < 0) return TCU_ERR_ARG;
  if (n > kNoAllocMaxN) {
    snprintf(g_errmsg, sizeof(g_errmsg),
             "tcu_scan_noalloc: n = %lld exceeds the %lld-element limit of its fixed scratch; "
             "use tcu_scan with a workspace",
             (long long)n, (long long)kNoAllocMaxN);
    return TCU_ERR_ARG;
  }
  if (n == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  if (!aligned16(x) || !aligned16(z)) return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = nullptr;
  tcu_status_t s = noalloc_scratch(st, &ws);
  if (s != TCU_OK) return s;
  // The tile counter, done counter and error words must start at zero (a
  // launch resets its counters when it finishes; clearing them again costs
  // nothing).  The epoch word is kept: it marks the look-back descriptors
  // left by the previous call as stale.
  uint8_t* h = static_cast<uint8_t*>(ws);
  cudaError_t e = cudaMemsetAsync(h, 0, 2 * sizeof(uint32_t), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h + 3 * sizeof(uint32_t), 0, 3 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return cuda_fail(e, "tcu_scan_noalloc: clearing the scratch header");
  if (x_dtype == TCU_INT8 && S == 16) S = 32;
  return dispatch_scan<kScanFull>(x, x_dtype, n, S, z, start, 0, ws, kNoAllocScratchBytes, st);
}

// The device-side error words of the last tcu_scan_noalloc call on the
// current device (a bounded wait that ran out): synchronises `stream`, copies
// the words out with one cudaMemcpyAsync into the caller's array (no
// allocation) and optionally clears them.  A device that has not run the
// scan yet reports TCU_OK.
extern "C" tcu_status_t tcu_scan_noalloc_error(uint32_t info[3], int clear, void* stream) {
  if (!info) return TCU_ERR_ARG;
  info[0] = info[1] = info[2] = 0;
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = nullptr;
  tcu_status_t s = noalloc_scratch(st, &ws);
  if (s != TCU_OK) return s;
  uint32_t h[3];
  cudaError_t e = cudaMemcpyAsync(h, &static_cast<WsHeader*>(ws)->error, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "tcu_scan_noalloc_error: reading the scratch header");
  info[0] = h[0];
  info[1] = h[1];
  info[2] = h[2];
  if (clear && h[0]) {
    e = cudaMemsetAsync(&static_cast<WsHeader*>(ws)->error, 0, sizeof(h), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "tcu_scan_noalloc_error: clearing");
  }
  return (tcu_status_t)h[0];
}

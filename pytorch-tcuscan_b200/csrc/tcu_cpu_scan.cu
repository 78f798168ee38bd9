// tcu_cpu_scan.cu -- the host-side inclusive scan of the reference's
// run_scan_cpu (src/torch/torch_scan_cpu.h:24-107), host code only.
//
// Semantics kept from the reference, so that results are bit-identical for
// the same block count: the input is cut into `blocks` = min(threads, n)
// contiguous blocks of ceil(n / blocks) elements; each block is scanned
// sequentially in the output type (fp32 for fp16 / fp32 input, int32 for
// int8), the block totals are scanned serially, and every element of block b
// becomes local_prefix + offset[b] (skipped where offset[b] == 0, as the
// reference does).
//
// Work order differs: the reference converts the whole input into z, scans
// z in place, then re-reads z to add the offsets (three passes over the
// output).  Here pass 1 only sums each block (reads x), and pass 2 redoes
// each block's sequential scan from x and writes local_prefix + offset once.
// The sequential sums are the same floating-point additions in the same
// order, so every rounding matches; the output is written once instead of
// three times.  Blocks run on std::thread workers (no OpenMP dependency);
// which thread runs a block does not change its result.
#include <cuda_fp16.h>

#include <cstdint>
#include <thread>
#include <vector>

#include "tcuscan.h"

namespace {

template <typename In, typename T>
inline T cvt(In v) {
  return static_cast<T>(v);
}
template <>
inline float cvt<__half, float>(__half v) {
  return __half2float(v);
}

// int32 sums wrap (two's complement) like the reference's int32 scan; the
// arithmetic is done on uint32 so the wrap is defined behaviour.
template <typename T>
struct Acc {
  using type = T;
  static inline T add(T a, T b) { return a + b; }
};
template <>
struct Acc<int32_t> {
  static inline int32_t add(int32_t a, int32_t b) {
    return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b));
  }
};

template <typename In, typename T>
T block_total(const In* x, int64_t s, int64_t e) {
  T sum = cvt<In, T>(x[s]);
  for (int64_t i = s + 1; i < e; ++i) sum = Acc<T>::add(sum, cvt<In, T>(x[i]));
  return sum;
}

template <typename In, typename T>
void block_scan_out(const In* x, T* z, int64_t s, int64_t e, T off) {
  T sum = cvt<In, T>(x[s]);
  if (off == T(0)) {  // the reference skips a zero offset (either sign of zero)
    z[s] = sum;
    for (int64_t i = s + 1; i < e; ++i) {
      sum = Acc<T>::add(sum, cvt<In, T>(x[i]));
      z[i] = sum;
    }
  } else {
    z[s] = Acc<T>::add(sum, off);
    for (int64_t i = s + 1; i < e; ++i) {
      sum = Acc<T>::add(sum, cvt<In, T>(x[i]));
      z[i] = Acc<T>::add(sum, off);
    }
  }
}

// Runs fn(b) for b in [0, blocks) on up to `workers` threads (static
// contiguous assignment; small inputs run on the calling thread).
template <typename F>
void for_blocks(int64_t blocks, int64_t workers, F&& fn) {
  if (workers <= 1 || blocks <= 1) {
    for (int64_t b = 0; b < blocks; ++b) fn(b);
    return;
  }
  if (workers > blocks) workers = blocks;
  std::vector<std::thread> pool;
  pool.reserve((size_t)workers - 1);
  const int64_t per = (blocks + workers - 1) / workers;
  for (int64_t w = 1; w < workers; ++w) {
    const int64_t b0 = w * per, b1 = b0 + per < blocks ? b0 + per : blocks;
    if (b0 >= b1) break;
    pool.emplace_back([&fn, b0, b1] {
      for (int64_t b = b0; b < b1; ++b) fn(b);
    });
  }
  for (int64_t b = 0; b < per && b < blocks; ++b) fn(b);
  for (auto& t : pool) t.join();
}

template <typename In, typename T>
void blocked_scan(const In* x, T* z, int64_t n, int64_t threads) {
  int64_t blocks = threads < 1 ? 1 : threads;
  if (blocks > n) blocks = n;
  const int64_t bs = (n + blocks - 1) / blocks;
  // below this many elements per call, worker start-up costs more than the scan
  const int64_t workers = n >= (int64_t)1 << 16 ? blocks : 1;
  std::vector<T> tot((size_t)blocks, T(0));
  for_blocks(blocks, workers, [&](int64_t b) {
    const int64_t s = b * bs, e = s + bs < n ? s + bs : n;
    if (s < e) tot[(size_t)b] = block_total<In, T>(x, s, e);
  });
  std::vector<T> off((size_t)blocks);
  T running = T(0);
  for (int64_t b = 0; b < blocks; ++b) {
    off[(size_t)b] = running;
    running = Acc<T>::add(running, tot[(size_t)b]);
  }
  for_blocks(blocks, workers, [&](int64_t b) {
    const int64_t s = b * bs, e = s + bs < n ? s + bs : n;
    if (s < e) block_scan_out<In, T>(x, z, s, e, off[(size_t)b]);
  });
}

}  // namespace

extern "C" tcu_status_t tcu_scan_cpu(const void* x, tcu_dtype_t x_dtype, int64_t n, void* z, int threads) {
  if (n < 0) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !z) return TCU_ERR_ARG;
  if (n > 0xFFFFFFFFll) return TCU_ERR_ARG;  // the reference's length is a uint32
  switch (x_dtype) {
    case TCU_INT8:
      blocked_scan<int8_t, int32_t>(static_cast<const int8_t*>(x), static_cast<int32_t*>(z), n, threads);
      return TCU_OK;
    case TCU_FLOAT16:
      blocked_scan<__half, float>(static_cast<const __half*>(x), static_cast<float*>(z), n, threads);
      return TCU_OK;
    case TCU_FLOAT32:
      blocked_scan<float, float>(static_cast<const float*>(x), static_cast<float*>(z), n, threads);
      return TCU_OK;
    default:
      return TCU_ERR_DTYPE;
  }
}

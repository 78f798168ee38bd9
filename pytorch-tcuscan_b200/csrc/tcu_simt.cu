// tcu_simt.cu -- the byte/integer utility operators of the scan family on the
// SIMT cores (HBM-bound element-wise and reduction work; none of it is
// reshaped into matrix products).
//
//   csr_gather      z[i] = values[i] * x[cols[i]]       (torch_gather.h:92-172)
//   reduce_tiles    per-block sums                       (torch_reduce.h:42-75)
//   complete_rows   MCSCAN down-sweep over rows          (torch_reduce.h:143-182)
//   complete_blocks block-prefix broadcast add           (torch_reduce.h:197-231)
//   gen_lower       tril(ones(s, s))                     (torch_gen_lower.h:31-59)
#include <cuda_runtime.h>

#include "tcu_host.h"

namespace tcu {

template <typename T>
__device__ __forceinline__ float load_elem(const T* p);
template <>
__device__ __forceinline__ float load_elem<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <>
__device__ __forceinline__ float load_elem<float>(const float* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// csr_gather.  Products are formed in the values dtype exactly as torch
// does: fp16 and fp32 products are correctly rounded once (an fp16 x fp16
// product is exact in fp32, so rounding that to fp16 equals __hmul), int16
// products wrap to 16 bits.  Column indices outside [0, x_len) read as 0 and
// record TCU_ERR_ARG in the workspace (no out-of-bounds access).
template <int DT>
__device__ __forceinline__ uint16_t mul16(uint16_t a, uint16_t b);
template <>
__device__ __forceinline__ uint16_t mul16<TCU_FLOAT16>(uint16_t a, uint16_t b) {
  return __half_as_ushort(__hmul(__ushort_as_half(a), __ushort_as_half(b)));
}
template <>
__device__ __forceinline__ uint16_t mul16<TCU_INT16>(uint16_t a, uint16_t b) {
  return (uint16_t)((int)(int16_t)a * (int)(int16_t)b);
}

template <int DT>
__global__ void __launch_bounds__(256) csr_gather16_kernel(const uint16_t* __restrict__ vals,
                                                           const int* __restrict__ cols,
                                                           const uint16_t* __restrict__ x, int64_t nnz, int64_t x_len,
                                                           uint16_t* __restrict__ z, WsHeader* ws) {
  const int64_t nv = nnz / 8;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(vals) + v);
    const int4 c0 = __ldg(reinterpret_cast<const int4*>(cols) + 2 * v);
    const int4 c1 = __ldg(reinterpret_cast<const int4*>(cols) + 2 * v + 1);
    const int cc[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    const uint32_t aw[4] = {a.x, a.y, a.z, a.w};
    uint32_t ow[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint16_t r[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = cc[2 * q + h];
        uint16_t xv = 0;
        if ((unsigned)c < (unsigned long long)x_len) xv = __ldg(x + c);
        else if (ws) record_error(ws, TCU_ERR_ARG, 200, (uint32_t)(8 * v + 2 * q + h));
        r[h] = mul16<DT>((uint16_t)(aw[q] >> (16 * h)), xv);
      }
      ow[q] = (uint32_t)r[0] | ((uint32_t)r[1] << 16);
    }
    reinterpret_cast<uint4*>(z)[v] = make_uint4(ow[0], ow[1], ow[2], ow[3]);
  }
  // ragged end
  for (int64_t i = nv * 8 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = cols[i];
    uint16_t xv = 0;
    if ((unsigned)c < (unsigned long long)x_len) xv = x[c];
    else if (ws) record_error(ws, TCU_ERR_ARG, 200, (uint32_t)i);
    z[i] = mul16<DT>(vals[i], xv);
  }
}

__global__ void __launch_bounds__(256) csr_gather32_kernel(const float* __restrict__ vals, const int* __restrict__ cols,
                                                           const float* __restrict__ x, int64_t nnz, int64_t x_len,
                                                           float* __restrict__ z, WsHeader* ws) {
  const int64_t nv = nnz / 4;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(vals) + v);
    const int4 c = __ldg(reinterpret_cast<const int4*>(cols) + v);
    const int cc[4] = {c.x, c.y, c.z, c.w};
    float xv[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      xv[h] = 0.f;
      if ((unsigned)cc[h] < (unsigned long long)x_len) xv[h] = __ldg(x + cc[h]);
      else if (ws) record_error(ws, TCU_ERR_ARG, 200, (uint32_t)(4 * v + h));
    }
    reinterpret_cast<float4*>(z)[v] =
        make_float4(__fmul_rn(a.x, xv[0]), __fmul_rn(a.y, xv[1]), __fmul_rn(a.z, xv[2]), __fmul_rn(a.w, xv[3]));
  }
  for (int64_t i = nv * 4 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = cols[i];
    float xv = 0.f;
    if ((unsigned)c < (unsigned long long)x_len) xv = x[c];
    else if (ws) record_error(ws, TCU_ERR_ARG, 200, (uint32_t)i);
    z[i] = __fmul_rn(vals[i], xv);
  }
}

// SpMV products in fp32: p[i] = float(values[i]) * float(x[cols[i]]) (an
// fp16 x fp16 product is exact in fp32; fp32 products are rounded once).
template <typename T>
__global__ void __launch_bounds__(256) spmv_products_kernel(const T* __restrict__ vals, const int* __restrict__ cols,
                                                            const T* __restrict__ x, int64_t nnz, int64_t x_len,
                                                            float* __restrict__ prod, WsHeader* ws) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = __ldg(cols + i);
    float xv = 0.f;
    if ((unsigned)c < (unsigned long long)x_len) xv = load_elem<T>(x + c);
    else if (ws) record_error(ws, TCU_ERR_ARG, 201, (uint32_t)i);
    prod[i] = __fmul_rn(load_elem<T>(vals + i), xv);
  }
}

// The same products, written pre-split for the tensor-core segmented sum:
// product i goes to row i / 64 of 256 bytes as bf16 hi = RN(p) at column
// i % 64 and bf16 lo = RN(p - hi) at column 64 + i % 64.  Each thread forms
// eight consecutive products (one 16-byte store of each half); products past
// nnz in the last group are written as zero.
template <typename T>
__global__ void __launch_bounds__(256) spmv_products_split_kernel(const T* __restrict__ vals,
                                                                  const int* __restrict__ cols,
                                                                  const T* __restrict__ x, int64_t nnz, int64_t x_len,
                                                                  uint8_t* __restrict__ prod, WsHeader* ws) {
  const int64_t groups = (nnz + 7) / 8;
  for (int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gi < groups; gi += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e0 = gi * 8;
    float pv[8];
    if (e0 + 8 <= nnz) {
      const int4 c0 = __ldg(reinterpret_cast<const int4*>(cols + e0));
      const int4 c1 = __ldg(reinterpret_cast<const int4*>(cols + e0) + 1);
      const int cc[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
      float vv[8];
      if constexpr (sizeof(T) == 4) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(vals + e0));
        const float4 b = __ldg(reinterpret_cast<const float4*>(vals + e0) + 1);
        vv[0] = a.x; vv[1] = a.y; vv[2] = a.z; vv[3] = a.w; vv[4] = b.x; vv[5] = b.y; vv[6] = b.z; vv[7] = b.w;
      } else {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(vals + e0));
        const __half2* h = reinterpret_cast<const __half2*>(&a);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const float2 f = __half22float2(h[t]);
          vv[2 * t] = f.x;
          vv[2 * t + 1] = f.y;
        }
      }
      // all eight gathers are issued before any is used (an out-of-range
      // column reads x[0] and is replaced by zero and reported afterwards)
      float xg[8];
      bool okc[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        okc[t] = (unsigned long long)(unsigned)cc[t] < (unsigned long long)x_len;
        xg[t] = load_elem<T>(x + (okc[t] ? cc[t] : 0));
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) pv[t] = __fmul_rn(vv[t], okc[t] ? xg[t] : 0.f);
      if (ws) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (!okc[t]) record_error(ws, TCU_ERR_ARG, 201, (uint32_t)(e0 + t));
      }
    } else {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        pv[t] = 0.f;
        if (e0 + t < nnz) {
          const int c = __ldg(cols + e0 + t);
          float xv = 0.f;
          if ((unsigned)c < (unsigned long long)x_len) xv = load_elem<T>(x + c);
          else if (ws) record_error(ws, TCU_ERR_ARG, 201, (uint32_t)(e0 + t));
          pv[t] = __fmul_rn(load_elem<T>(vals + e0 + t), xv);
        }
      }
    }
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(pv[2 * t], pv[2 * t + 1]);
      const float2 hf = __bfloat1622float2(h);
      const __nv_bfloat162 l = __floats2bfloat162_rn(pv[2 * t] - hf.x, pv[2 * t + 1] - hf.y);
      hi[t] = *reinterpret_cast<const uint32_t*>(&h);
      lo[t] = *reinterpret_cast<const uint32_t*>(&l);
    }
    uint8_t* row = prod + (e0 >> 6) * 256 + (e0 & 63) * 2;
    *reinterpret_cast<uint4*>(row) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(row + 128) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

// gather_spmv (tests/test_gather_spmv.py): z[i] = values[idxs[i] - 1], and 0
// where idxs[i] == 0 -- the scanned products read back at the row pointers
// (the first step of the reference's v1 SpMV, src/torch/torch_spmv.h:79-93).
// Indices past the values are reported (site 202) and read as 0.
template <int EB, typename I>
__global__ void __launch_bounds__(256) gather_spmv_kernel(const uint8_t* __restrict__ values, int64_t n_values,
                                                          const I* __restrict__ idxs, int64_t n_idx,
                                                          uint8_t* __restrict__ z, WsHeader* ws) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_idx; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = (unsigned long long)__ldg(idxs + i);
    uint32_t lo = 0, hi = 0;
    if (k >= 1 && k - 1 < (unsigned long long)n_values) {
      const uint8_t* src = values + (k - 1) * EB;
      if constexpr (EB == 2) lo = __ldg(reinterpret_cast<const uint16_t*>(src));
      if constexpr (EB == 4) lo = __ldg(reinterpret_cast<const uint32_t*>(src));
      if constexpr (EB == 8) {
        const unsigned long long v = __ldg(reinterpret_cast<const unsigned long long*>(src));
        lo = (uint32_t)v;
        hi = (uint32_t)(v >> 32);
      }
    } else if (k != 0 && ws) {
      record_error(ws, TCU_ERR_ARG, 202, (uint32_t)i);
    }
    if constexpr (EB == 2) reinterpret_cast<uint16_t*>(z)[i] = (uint16_t)lo;
    if constexpr (EB == 4) reinterpret_cast<uint32_t*>(z)[i] = lo;
    if constexpr (EB == 8) reinterpret_cast<unsigned long long*>(z)[i] = ((unsigned long long)hi << 32) | lo;
  }
}

// ---------------------------------------------------------------------------
// reduce_tiles: block b sums x[b*bl : min((b+1)*bl, n)] with
// bl = tile_len * ceil(ceil(n / tile_len) / num_blocks)
// (tests/test_reduce_tiles.py ref_reduce_tiles).  Each block is split over
// `splits` CTAs whose partials (FP64 / int64) are summed in a fixed order by a
// second kernel, so results are deterministic.
template <typename InT>
__device__ __forceinline__ void acc_add(double& a, long long& ai, InT v);
template <>
__device__ __forceinline__ void acc_add<__half>(double& a, long long&, __half v) { a += (double)__half2float(v); }
template <>
__device__ __forceinline__ void acc_add<int8_t>(double&, long long& ai, int8_t v) { ai += v; }
template <>
__device__ __forceinline__ void acc_add<float>(double& a, long long&, float v) { a += (double)v; }
template <>
__device__ __forceinline__ void acc_add<int>(double&, long long& ai, int v) { ai += v; }

template <typename InT>
__global__ void __launch_bounds__(256) reduce_tiles_partial_kernel(const InT* __restrict__ x, int64_t n, int64_t bl,
                                                                   int num_blocks, int splits,
                                                                   unsigned long long* part) {
  const int b = blockIdx.x / splits, sp = blockIdx.x % splits;
  const int64_t b0 = (int64_t)b * bl;
  const int64_t b1 = min(b0 + bl, n);
  const int64_t len = b1 > b0 ? b1 - b0 : 0;
  const int64_t chunk = (len + splits - 1) / splits;
  const int64_t s0 = b0 + sp * chunk, s1 = min(s0 + chunk, b1);
  double a = 0.0;
  long long ai = 0;
  for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) acc_add<InT>(a, ai, x[i]);
  a = warp_sum_any(a);
  ai = warp_sum_any(ai);
  __shared__ double sa[8];
  __shared__ long long si[8];
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    si[threadIdx.x >> 5] = ai;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    long long ti = 0;
    for (int k = 0; k < 8; ++k) {
      t += sa[k];
      ti += si[k];
    }
    if constexpr (__is_same(InT, int8_t) || __is_same(InT, int)) part[blockIdx.x] = (unsigned long long)ti;
    else part[blockIdx.x] = (unsigned long long)__double_as_longlong(t);
  }
}

template <typename OutT>
__global__ void reduce_tiles_final_kernel(const unsigned long long* part, int num_blocks, int splits, OutT* out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= num_blocks) return;
  if constexpr (__is_same(OutT, int)) {
    long long t = 0;
    for (int s = 0; s < splits; ++s) t += (long long)part[(int64_t)b * splits + s];
    out[b] = (int)t;
  } else {
    double t = 0.0;
    for (int s = 0; s < splits; ++s) t += __longlong_as_double((long long)part[(int64_t)b * splits + s]);
    out[b] = (float)t;
  }
}

// ---------------------------------------------------------------------------
// complete_rows (tests/test_complete_rows.py ref_complete_rows): block b of
// x (block = n / num_blocks) starts from sum(sums[:b]); each width-long row
// gets the running carry added and the carry becomes the updated row's last
// element.  Pass 1 (one CTA per block): carry[row] = prefix_b + exclusive
// scan of the row-last inputs of the block (FP64 / int64).  Pass 2 adds it.
template <typename T>
__global__ void __launch_bounds__(1024) complete_rows_carry_kernel(const T* __restrict__ x, const T* __restrict__ sums,
                                                                   int64_t block_len, int64_t width, int num_blocks,
                                                                   unsigned long long* carry) {
  const int b = blockIdx.x;
  using A = typename std::conditional<__is_same(T, float), double, long long>::type;
  __shared__ A s_pre;
  __shared__ A s_w[32];
  if (threadIdx.x < 32) {
    A v = 0;
    for (int k = threadIdx.x; k < b; k += 32) v += (A)sums[k];
    v = warp_sum_any(v);
    if (threadIdx.x == 0) s_pre = v;
  }
  __syncthreads();
  A running = s_pre;
  const int64_t rows = (block_len + width - 1) / width;
  const int64_t base = (int64_t)b * block_len;
  for (int64_t r0 = 0; r0 < rows; r0 += blockDim.x) {
    const int64_t r = r0 + threadIdx.x;
    A v = 0;
    if (r < rows) {
      const int64_t last = min((r + 1) * width, block_len) - 1;
      v = (A)x[base + last];
    }
    // block-wide exclusive scan of v
    A inc = v;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const A o = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += o;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    A wpre = 0, tot = 0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) {
      if (k < warp) wpre += s_w[k];
      tot += s_w[k];
    }
    if (r < rows) {
      const A c = running + wpre + inc - v;
      if constexpr (__is_same(A, double)) carry[(int64_t)b * rows + r] = (unsigned long long)__double_as_longlong(c);
      else carry[(int64_t)b * rows + r] = (unsigned long long)c;
    }
    running += tot;
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(256) complete_rows_add_kernel(const T* __restrict__ x, int64_t n, int64_t block_len,
                                                                int64_t width, const unsigned long long* carry,
                                                                T* __restrict__ z) {
  const int64_t rows = (block_len + width - 1) / width;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / block_len, off = i % block_len;
    const unsigned long long cb = carry[b * rows + off / width];
    if constexpr (__is_same(T, float)) z[i] = (float)((double)x[i] + __longlong_as_double((long long)cb));
    else z[i] = (T)((long long)x[i] + (long long)cb);
  }
}

// complete_blocks (tests/test_complete_blocks.py ref_complete_blocks).
template <typename T>
__global__ void __launch_bounds__(256) complete_blocks_kernel(const T* __restrict__ x, const T* __restrict__ sums,
                                                              int64_t n, int64_t block_len, int num_blocks,
                                                              T* __restrict__ z) {
  using A = typename std::conditional<__is_same(T, float), double, long long>::type;
  extern __shared__ unsigned long long s_pre[];  // exclusive prefix of sums
  if (threadIdx.x == 0) {
    A run = 0;
    for (int k = 0; k < num_blocks; ++k) {
      if constexpr (__is_same(A, double)) s_pre[k] = (unsigned long long)__double_as_longlong(run);
      else s_pre[k] = (unsigned long long)run;
      run += (A)sums[k];
    }
  }
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / block_len;
    if constexpr (__is_same(T, float)) z[i] = (float)((double)x[i] + __longlong_as_double((long long)s_pre[b]));
    else z[i] = (T)((long long)x[i] + (long long)s_pre[b]);
  }
}

template <typename T>
__global__ void gen_lower_kernel(T* z, int64_t s, T one) {
  const int64_t n = s * s;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = (i % s) <= (i / s) ? one : T(0);
}

static int grid_for(int64_t work, int per_block = 256) {
  int64_t g = (work + per_block - 1) / per_block;
  const int64_t cap = (int64_t)sm_count() * 8;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

static tcu_status_t launched(const char* what) {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, what);
}

// ---------------------------------------------------------------------------
// total: the sum of all n elements in a wide type -- int8 -> int64 (exact),
// fp16 / fp32 -> FP64 -- in a fixed order, so every call gives the same bits:
// block b sums 16-byte chunks b*256 + t, b*256 + t + grid*256, ... per thread
// (int8 chunks exactly with dp4a, fp16 / fp32 chunks in FP64), then a fixed
// warp / block tree; one block adds the block partials in a fixed tree and
// zeroes them (workspace scratch).  The exchange step of the sharded scan.
template <typename InT>
struct TotalAcc { using T = double; };
template <>
struct TotalAcc<int8_t> { using T = long long; };

template <typename InT>
__device__ __forceinline__ typename TotalAcc<InT>::T chunk_total(const uint4 w) {
  if constexpr (__is_same(InT, int8_t)) {
    int s = __dp4a((int)w.x, 0x01010101, 0);
    s = __dp4a((int)w.y, 0x01010101, s);
    s = __dp4a((int)w.z, 0x01010101, s);
    s = __dp4a((int)w.w, 0x01010101, s);
    return (long long)s;
  } else if constexpr (__is_same(InT, __half)) {
    const __half2* h = reinterpret_cast<const __half2*>(&w);
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 f = __half22float2(h[k]);
      t += (double)f.x + (double)f.y;
    }
    return t;
  } else {
    return ((double)__uint_as_float(w.x) + (double)__uint_as_float(w.y)) +
           ((double)__uint_as_float(w.z) + (double)__uint_as_float(w.w));
  }
}

template <typename InT>
__global__ void __launch_bounds__(256) total_partial_kernel(const InT* __restrict__ x, int64_t n,
                                                            typename TotalAcc<InT>::T* __restrict__ part) {
  using A = typename TotalAcc<InT>::T;
  constexpr int VPC = 16 / (int)sizeof(InT);  // elements per 16-byte chunk
  const int64_t nchunks = n / VPC;
  const uint4* xv = reinterpret_cast<const uint4*>(x);
  A acc = 0;
  for (int64_t c = (int64_t)blockIdx.x * 256 + threadIdx.x; c < nchunks; c += (int64_t)gridDim.x * 256)
    acc += chunk_total<InT>(__ldg(xv + c));
  if (blockIdx.x == 0) {  // the elements after the last whole chunk
    for (int64_t i = nchunks * VPC + threadIdx.x; i < n; i += 256) {
      if constexpr (__is_same(InT, int8_t)) acc += (long long)x[i];
      else if constexpr (__is_same(InT, __half)) acc += (double)__half2float(x[i]);
      else acc += (double)x[i];
    }
  }
  acc = warp_sum_any(acc);
  __shared__ A sw[8];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    A t = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += sw[k];
    part[blockIdx.x] = t;
  }
}

template <typename A>
__global__ void __launch_bounds__(256) total_final_kernel(A* __restrict__ part, int nparts, A* __restrict__ out) {
  A acc = 0;
  for (int k = threadIdx.x; k < nparts; k += 256) acc += part[k];
  acc = warp_sum_any(acc);
  __shared__ A sw[8];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
  __syncthreads();  // every partial has been read
  for (int k = threadIdx.x; k < nparts; k += 256) part[k] = 0;
  if (threadIdx.x == 0) {
    A t = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += sw[k];
    *out = t;
  }
}

template <typename InT>
static tcu_status_t run_total(const void* x, int64_t n, void* out, void* ws, size_t ws_bytes, cudaStream_t st) {
  using A = typename TotalAcc<InT>::T;
  constexpr int VPC = 16 / (int)sizeof(InT);
  int64_t grid = (n / VPC + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 4;
  grid = grid < 1 ? 1 : (grid > cap ? cap : grid);
  if (!ws || ws_capacity(ws_bytes) * (int64_t)sizeof(TileDesc) < grid * (int64_t)sizeof(A)) return TCU_ERR_WORKSPACE;
  A* part = reinterpret_cast<A*>(ws_descs(ws));  // zeroed again by the final kernel
  total_partial_kernel<InT><<<(unsigned)grid, 256, 0, st>>>(static_cast<const InT*>(x), n, part);
  total_final_kernel<A><<<1, 256, 0, st>>>(part, (int)grid, static_cast<A*>(out));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TCU_OK : cuda_fail(e, "total launch");
}

// Scratch written into a workspace's look-back descriptor region is zeroed
// after use, so that the region only ever holds descriptors or zeros: stale
// partial sums could otherwise read as a valid descriptor of a later launch
// whose epoch happens to match their bits.
static tcu_status_t clear_scratch(void* ws, size_t bytes, cudaStream_t st, const char* what) {
  cudaError_t e = cudaMemsetAsync(static_cast<uint8_t*>(ws) + 128, 0, bytes, st);
  return e == cudaSuccess ? launched(what) : cuda_fail(e, what);
}

}  // namespace tcu

using namespace tcu;

extern "C" {

tcu_status_t tcu_csr_gather(const void* values, tcu_dtype_t dtype, const int32_t* cols, int64_t nnz, const void* x,
                            int64_t x_len, void* z, void* ws, void* stream) {
  if (nnz < 0 || x_len < 0) return TCU_ERR_ARG;
  if (nnz == 0) return TCU_OK;
  if (!values || !cols || !x || !z) return TCU_ERR_ARG;
  if (!aligned16(values) || !aligned16(cols) || !aligned16(z)) return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  WsHeader* h = static_cast<WsHeader*>(ws);
  if (dtype == TCU_FLOAT16) {
    csr_gather16_kernel<TCU_FLOAT16><<<grid_for(nnz / 8 + 1), 256, 0, st>>>(
        (const uint16_t*)values, cols, (const uint16_t*)x, nnz, x_len, (uint16_t*)z, h);
  } else if (dtype == TCU_INT16) {
    csr_gather16_kernel<TCU_INT16><<<grid_for(nnz / 8 + 1), 256, 0, st>>>(
        (const uint16_t*)values, cols, (const uint16_t*)x, nnz, x_len, (uint16_t*)z, h);
  } else if (dtype == TCU_FLOAT32) {
    csr_gather32_kernel<<<grid_for(nnz / 4 + 1), 256, 0, st>>>((const float*)values, cols, (const float*)x, nnz,
                                                               x_len, (float*)z, h);
  } else {
    return TCU_ERR_DTYPE;
  }
  return launched("csr_gather");
}

tcu_status_t tcu_spmv_products(const void* values, tcu_dtype_t dtype, const int32_t* cols, int64_t nnz, const void* x,
                               int64_t x_len, float* prod, void* ws, void* stream) {
  if (nnz < 0 || x_len < 0) return TCU_ERR_ARG;
  if (nnz == 0) return TCU_OK;
  if (!values || !cols || !x || !prod) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  WsHeader* h = static_cast<WsHeader*>(ws);
  if (dtype == TCU_FLOAT16)
    spmv_products_kernel<__half><<<grid_for(nnz), 256, 0, st>>>((const __half*)values, cols, (const __half*)x, nnz,
                                                                 x_len, prod, h);
  else if (dtype == TCU_FLOAT32)
    spmv_products_kernel<float><<<grid_for(nnz), 256, 0, st>>>((const float*)values, cols, (const float*)x, nnz,
                                                                x_len, prod, h);
  else
    return TCU_ERR_DTYPE;
  return launched("spmv_products");
}

}  // extern "C"

namespace tcu {

tcu_status_t spmv_products_split(const void* values, tcu_dtype_t dtype, const int32_t* cols, int64_t nnz,
                                 const void* x, int64_t x_len, void* prod, void* ws, void* stream) {
  if (nnz < 0 || x_len < 0) return TCU_ERR_ARG;
  if (nnz == 0) return TCU_OK;
  if (!values || !cols || !x || !prod) return TCU_ERR_ARG;
  if (!aligned16(values) || !aligned16(cols) || !aligned16(prod)) return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  WsHeader* h = static_cast<WsHeader*>(ws);
  const int64_t groups = (nnz + 7) / 8;
  if (dtype == TCU_FLOAT16)
    spmv_products_split_kernel<__half><<<grid_for(groups), 256, 0, st>>>((const __half*)values, cols, (const __half*)x,
                                                                          nnz, x_len, (uint8_t*)prod, h);
  else if (dtype == TCU_FLOAT32)
    spmv_products_split_kernel<float><<<grid_for(groups), 256, 0, st>>>((const float*)values, cols, (const float*)x,
                                                                         nnz, x_len, (uint8_t*)prod, h);
  else
    return TCU_ERR_DTYPE;
  return launched("spmv_products_split");
}

}  // namespace tcu

extern "C" {

tcu_status_t tcu_gather_spmv(const void* values, int elem_bytes, int64_t n_values, const void* idxs,
                             tcu_dtype_t idx_dtype, int64_t n_idx, void* z, void* ws, void* stream) {
  if (n_values < 0 || n_idx < 0) return TCU_ERR_ARG;
  if (n_idx == 0) return TCU_OK;
  if (!idxs || !z || (n_values > 0 && !values)) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  WsHeader* h = static_cast<WsHeader*>(ws);
  const uint8_t* v = static_cast<const uint8_t*>(values);
  uint8_t* zo = static_cast<uint8_t*>(z);
  const int grid = grid_for(n_idx);
#define TCU_GS(EB, I) gather_spmv_kernel<EB, I><<<grid, 256, 0, st>>>(v, n_values, (const I*)idxs, n_idx, zo, h)
  const bool i32 = idx_dtype == TCU_INT32 || idx_dtype == TCU_UINT32;
  if (!i32 && idx_dtype != TCU_INT64) return TCU_ERR_DTYPE;
  switch (elem_bytes) {
    case 2: if (i32) TCU_GS(2, uint32_t); else TCU_GS(2, unsigned long long); break;
    case 4: if (i32) TCU_GS(4, uint32_t); else TCU_GS(4, unsigned long long); break;
    case 8: if (i32) TCU_GS(8, uint32_t); else TCU_GS(8, unsigned long long); break;
    default: return TCU_ERR_DTYPE;
  }
#undef TCU_GS
  return launched("gather_spmv");
}

tcu_status_t tcu_reduce_tiles(const void* x, tcu_dtype_t dtype, int64_t n, int64_t tile_len, int num_blocks, void* z,
                              void* ws, size_t ws_bytes, void* stream) {
  if (n < 0 || tile_len <= 0 || num_blocks <= 0) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t tiles = (n + tile_len - 1) / tile_len;
  const int64_t bl = tile_len * ((tiles + num_blocks - 1) / num_blocks);
  int splits = (sm_count() * 4 + num_blocks - 1) / num_blocks;
  if (splits < 1) splits = 1;
  if (splits > 64) splits = 64;
  const size_t need = 128 + (size_t)num_blocks * splits * 8;
  if (!ws || ws_bytes < need) return TCU_ERR_WORKSPACE;
  if (!z || (n > 0 && !x)) return TCU_ERR_ARG;
  unsigned long long* part = reinterpret_cast<unsigned long long*>(static_cast<uint8_t*>(ws) + 128);
  const int grid = num_blocks * splits;
  if (dtype == TCU_INT8) {
    reduce_tiles_partial_kernel<int8_t><<<grid, 256, 0, st>>>((const int8_t*)x, n, bl, num_blocks, splits, part);
    reduce_tiles_final_kernel<int><<<(num_blocks + 127) / 128, 128, 0, st>>>(part, num_blocks, splits, (int*)z);
  } else if (dtype == TCU_FLOAT16) {
    reduce_tiles_partial_kernel<__half><<<grid, 256, 0, st>>>((const __half*)x, n, bl, num_blocks, splits, part);
    reduce_tiles_final_kernel<float><<<(num_blocks + 127) / 128, 128, 0, st>>>(part, num_blocks, splits, (float*)z);
  } else {
    return TCU_ERR_DTYPE;
  }
  return clear_scratch(ws, need - 128, st, "reduce_tiles");
}

tcu_status_t tcu_complete_rows(const void* x, tcu_dtype_t dtype, int64_t n, const void* sums, int num_blocks,
                               int64_t width, void* z, void* ws, size_t ws_bytes, void* stream) {
  if (n < 0 || num_blocks <= 0 || width <= 0) return TCU_ERR_ARG;
  if (n % num_blocks != 0) return TCU_ERR_ARG;
  if (n == 0) return TCU_OK;
  if (!x || !sums || !z) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t bl = n / num_blocks;
  const int64_t rows = (bl + width - 1) / width;
  const size_t need = 128 + (size_t)num_blocks * rows * 8;
  if (!ws || ws_bytes < need) return TCU_ERR_WORKSPACE;
  unsigned long long* carry = reinterpret_cast<unsigned long long*>(static_cast<uint8_t*>(ws) + 128);
  if (dtype == TCU_FLOAT32) {
    complete_rows_carry_kernel<float><<<num_blocks, 1024, 0, st>>>((const float*)x, (const float*)sums, bl, width,
                                                                   num_blocks, carry);
    complete_rows_add_kernel<float><<<grid_for(n), 256, 0, st>>>((const float*)x, n, bl, width, carry, (float*)z);
  } else if (dtype == TCU_INT32) {
    complete_rows_carry_kernel<int><<<num_blocks, 1024, 0, st>>>((const int*)x, (const int*)sums, bl, width,
                                                                 num_blocks, carry);
    complete_rows_add_kernel<int><<<grid_for(n), 256, 0, st>>>((const int*)x, n, bl, width, carry, (int*)z);
  } else {
    return TCU_ERR_DTYPE;
  }
  return clear_scratch(ws, need - 128, st, "complete_rows");
}

tcu_status_t tcu_complete_blocks(const void* x, tcu_dtype_t dtype, int64_t n, const void* sums, int num_blocks,
                                 void* z, void* stream) {
  if (n < 0 || num_blocks <= 0 || n % num_blocks != 0) return TCU_ERR_ARG;
  if (num_blocks > 6000) return TCU_ERR_ARG;  // prefix table lives in shared memory
  if (n == 0) return TCU_OK;
  if (!x || !sums || !z) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t bl = n / num_blocks;
  const size_t smem = (size_t)num_blocks * 8;
  if (dtype == TCU_FLOAT32) {
    complete_blocks_kernel<float><<<grid_for(n), 256, smem, st>>>((const float*)x, (const float*)sums, n, bl,
                                                                  num_blocks, (float*)z);
  } else if (dtype == TCU_INT32) {
    complete_blocks_kernel<int><<<grid_for(n), 256, smem, st>>>((const int*)x, (const int*)sums, n, bl, num_blocks,
                                                                (int*)z);
  } else {
    return TCU_ERR_DTYPE;
  }
  return launched("complete_blocks");
}

tcu_status_t tcu_total(const void* x, tcu_dtype_t dtype, int64_t n, void* out, void* ws, size_t ws_bytes,
                       void* stream) {
  if (n < 0 || !out) return TCU_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(out) & 7u) return TCU_ERR_ALIGN;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, 8, st);
    return e == cudaSuccess ? TCU_OK : cuda_fail(e, "cudaMemsetAsync(total)");
  }
  if (!x) return TCU_ERR_ARG;
  if (!aligned16(x)) return TCU_ERR_ALIGN;
  switch (dtype) {
    case TCU_INT8: return run_total<int8_t>(x, n, out, ws, ws_bytes, st);
    case TCU_FLOAT16: return run_total<__half>(x, n, out, ws, ws_bytes, st);
    case TCU_FLOAT32: return run_total<float>(x, n, out, ws, ws_bytes, st);
    default: return TCU_ERR_DTYPE;
  }
}

tcu_status_t tcu_gen_lower(int64_t s, tcu_dtype_t dtype, void* z, void* stream) {
  if (s < 0) return TCU_ERR_ARG;
  if (s == 0) return TCU_OK;
  if (!z) return TCU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int g = grid_for(s * s);
  switch (dtype) {
    case TCU_INT8: gen_lower_kernel<int8_t><<<g, 256, 0, st>>>((int8_t*)z, s, (int8_t)1); break;
    case TCU_FLOAT16: gen_lower_kernel<uint16_t><<<g, 256, 0, st>>>((uint16_t*)z, s, (uint16_t)0x3C00); break;
    case TCU_BFLOAT16: gen_lower_kernel<uint16_t><<<g, 256, 0, st>>>((uint16_t*)z, s, (uint16_t)0x3F80); break;
    case TCU_FLOAT32: gen_lower_kernel<float><<<g, 256, 0, st>>>((float*)z, s, 1.0f); break;
    case TCU_INT32: gen_lower_kernel<int><<<g, 256, 0, st>>>((int*)z, s, 1); break;
    default: return TCU_ERR_DTYPE;
  }
  return launched("gen_lower");
}

}  // extern "C"

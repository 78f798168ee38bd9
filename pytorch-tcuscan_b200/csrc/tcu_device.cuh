// tcu_device.cuh -- sm_100a device primitives for the tcuscan kernels:
// mbarriers with bounded waits, TMA (cp.async.bulk.tensor) loads/stores,
// tcgen05 (TMEM alloc, MMA, commit, ld) and the decoupled look-back state.
//
// Every spin in this file is bounded by a %globaltimer deadline.  A wait that
// runs out records TCU_ERR_TIMEOUT in the workspace error word, raises the
// CTA's abort flag and returns false; callers then drain their own in-flight
// copies (again with bounded waits), free TMEM and exit.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <climits>

#include "tcuscan.h"

namespace tcu {

// ---------------------------------------------------------------------------
// Workspace header shared by every look-back kernel launch.  The tile
// counter and done counter are reset by the last CTA of each launch, and the
// epoch is bumped, so the per-tile descriptors of earlier launches read as
// stale without any memset between launches (CUDA-graph safe).
struct WsHeader {
  uint32_t tile_counter;   // dynamic tile assignment (atomicAdd)
  uint32_t done_ctas;      // CTAs finished in this launch
  uint32_t epoch;          // launch generation, tags the tile descriptors
  uint32_t error;          // first error code (sticky until read by the host)
  uint32_t err_site;       // where it happened (kernel-defined)
  uint32_t err_chunk;      // tile being processed
  uint32_t pad[10];
};
static_assert(sizeof(WsHeader) == 64, "header size");

// Look-back descriptor states: bits[1:0] state, bit 2 = the tile contains a
// segment start (its aggregate is already a complete carry), bits[31:3] =
// launch epoch.
enum : uint32_t { LB_INVALID = 0, LB_AGG = 1, LB_INC = 2, LB_SEGSTART = 4 };

// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Record the first error of a launch (sticky).
__device__ __forceinline__ void record_error(WsHeader* ws, uint32_t code, uint32_t site, uint32_t chunk) {
  if (atomicCAS(&ws->error, 0u, code) == 0u) {
    ws->err_site = site;
    ws->err_chunk = chunk;
  }
}

struct WaitCtx {
  WsHeader* ws;
  volatile int* abort_flag;  // in shared memory
  uint64_t timeout_ns;
};

__device__ __forceinline__ bool aborted(const WaitCtx& c) { return *c.abort_flag != 0; }

__device__ __forceinline__ void raise_abort(const WaitCtx& c, uint32_t site, uint32_t chunk) {
  record_error(c.ws, TCU_ERR_TIMEOUT, site, chunk);
  *c.abort_flag = 1;
}

// ---------------------------------------------------------------------------
// mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on the phase with the given parity.  Returns false on abort or
// timeout (and raises the abort flag on timeout).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const WaitCtx& c, uint32_t site,
                                          uint32_t chunk) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  uint32_t it = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (aborted(c)) return false;
    if ((++it & 63u) == 0u && globaltimer() - t0 > c.timeout_ns) {
      raise_abort(c, site, chunk);
      return false;
    }
  }
  return true;
}
// Drain wait used on the exit path: bounded, ignores the abort flag.
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity, uint64_t timeout_ns) {
  const uint64_t t0 = globaltimer();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer() - t0 > timeout_ns) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Named barriers for the epilogue warpgroups (id 0 is __syncthreads).
__device__ __forceinline__ void named_bar_sync(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// ---------------------------------------------------------------------------
// TMA (no multicast anywhere in this project).
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const void* tmap, int32_t c0, int32_t c1,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_2d(const void* tmap, int32_t c0, int32_t c1, const void* smem_src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tmap), "r"(c0),
               "r"(c1), "r"(smem_u32(smem_src))
               : "memory");
}
// Untiled bulk copy global -> shared (no multicast): both addresses 16-byte
// aligned, size a multiple of 16 bytes; completes `bytes` on the mbarrier.
__device__ __forceinline__ void bulk_load_1d(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void prefetch_tmap(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

// ---------------------------------------------------------------------------
// tcgen05 / TMEM
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// D[tmem] (+)= A[smem desc] * B[smem desc]; kind::f16 (f16/bf16 -> f32).
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// kind::i8 (s8/u8 -> s32).
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 lanes x 32 bit, 16 consecutive columns per thread.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// UMMA shared-memory descriptor, K-major, swizzled (32/64/128 B).
//   start address >> 4 in [0,14), LBO (=1, unused for swizzled K-major) in
//   [16,30), SBO = bytes between 8-row groups >> 4 in [32,46), version 1 at
//   [46,48), layout type at [61,64): 2 = 128B, 4 = 64B, 6 = 32B.
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t smem_addr, uint32_t swizzle_bytes) {
  const uint64_t layout = swizzle_bytes == 128 ? 2ull : (swizzle_bytes == 64 ? 4ull : 6ull);
  const uint64_t sbo = (8ull * swizzle_bytes) >> 4;
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (sbo & 0x3FFFull) << 32;
  d |= (uint64_t)1 << 46;
  d |= layout << 61;
  return d;
}

// Instruction descriptor: c_format [4,6), a_format [7,10), b_format [10,13),
// a/b K-major (bits 15/16 = 0), N>>3 at [17,23), M>>4 at [24,29).
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t c_fmt, uint32_t ab_fmt, uint32_t M, uint32_t N) {
  return (c_fmt << 4) | (ab_fmt << 7) | (ab_fmt << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
// c_format: F32 = 1, S32 = 2.  ab_format: kind::f16 -> F16 = 0, BF16 = 1;
// kind::i8 -> S8 = 1.
enum : uint32_t { CF_F32 = 1, CF_S32 = 2, AB_F16 = 0, AB_BF16 = 1, AB_S8 = 1 };

// Byte offset of the 16-byte chunk holding logical byte `o` inside a buffer
// laid out with the TMA/UMMA swizzle of the given span (32/64/128 B): bits
// [4, 4+log2(span/16)) are XORed with the bits three positions above.
__device__ __forceinline__ uint32_t swz(uint32_t o, uint32_t span) {
  const uint32_t mask = span == 128 ? 0x70u : (span == 64 ? 0x30u : 0x10u);
  return o ^ ((o >> 3) & mask);
}

// ---------------------------------------------------------------------------
// Warp helpers.
template <typename V>
__device__ __forceinline__ V warp_sum_any(V v) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }

// 4 mask bytes -> 4 selection bits (byte != 0).
__device__ __forceinline__ uint32_t sel4(uint32_t w) {
  const uint32_t u = __vsetne4(w, 0u);  // 0x01 per nonzero byte
  return (u & 1u) | ((u >> 7) & 2u) | ((u >> 14) & 4u) | ((u >> 21) & 8u);
}

// 32 lanes x 32 bit, one column per thread.
__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  return r;
}

// ---------------------------------------------------------------------------
// Global-memory acquire/release for the look-back flags.
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ long long ld_relaxed_s64(const long long* p) {
  long long v;
  asm volatile("ld.relaxed.gpu.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

}  // namespace tcu

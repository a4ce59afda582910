// mk_wave.cuh — inline PTX for the staged multiphase kernels (the fused
// one-launch loop and the row-staged collision): inter-CTA publication flags
// with acquire/release at GPU scope, bounded waits, mbarriers and the
// bulk-copy engine (cp.async.bulk, no multicast) staging rows into shared
// memory.
//
// Every wait here has an iteration limit.  When it runs out the wait records
// a code in the launch's error word and returns; later waits see the word and
// return at once, so a launch whose publication never comes ends in bounded
// time with an error the host reads (MK_ERR_TIMEOUT) instead of hanging.
#ifndef MK_WAVE_CUH
#define MK_WAVE_CUH

#include <stdint.h>

namespace mkw {

// Error codes written to the launch's error word.
enum { ERR_NONE = 0, ERR_FLAG_WAIT = 1, ERR_MBAR_WAIT = 2 };

// About one second of polling with the back-off below.
constexpr int kSpinLimit = 1 << 20;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Wait until *flag >= need (the publisher's count of finished planes).
// Returns false when the wait gave up or another wait of the launch already did.
__device__ __forceinline__ bool wait_count(const unsigned* flag, unsigned need, int* err) {
  for (int it = 0; it < kSpinLimit; ++it) {
    if (ld_acquire(flag) >= need) return true;
    if ((it & 15) == 15 && ld_volatile(err) != ERR_NONE) return false;
    if (it >= 32) __nanosleep(it < 1024 ? 64 : 1024);
  }
  atomicCAS(err, ERR_NONE, ERR_FLAG_WAIT);
  return false;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make initialised mbarriers visible to the bulk-copy engine.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of bulk-copy data for the phase.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// One plain arrival.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for the completion of the barrier phase with the given parity.
// Returns false (and records the code) when the wait gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err) {
  for (int it = 0; it < kSpinLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it >= 16) __nanosleep(64);
  }
  atomicCAS(err, ERR_NONE, ERR_MBAR_WAIT);
  return false;
}

// Order this thread's earlier generic-proxy accesses (and what it observed
// through acquire / barriers) before its later bulk copies.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bulk copy global -> this CTA's shared memory, completing on `bar`.  Both
// addresses 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// One 3-D tile of a tensor map (global) into this CTA's shared memory,
// completing on `bar`; coordinates (x, y, z) of the tile's first element,
// x times the element size a multiple of 16 bytes; elements outside the
// tensor read as zero.  `tmap` is the address of a __grid_constant__ kernel
// parameter.  No multicast.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace mkw

#endif

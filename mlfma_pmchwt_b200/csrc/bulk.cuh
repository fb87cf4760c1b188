// Shared-memory staging for sm_100a: mbarrier phases and TMA tensor copies
// (cp.async.bulk.tensor, tiled and tile::gather4) from global to shared
// memory.
// Every wait is bounded in time: after kWaitNs of polling it records a
// status bit in a global word and reports failure, so that a kernel whose
// producer stopped ends with an error the host can read instead of hanging.
#pragma once
#include <cstdint>

namespace mlfma {

constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s
constexpr int kStatusWaitTimeout = 1;
// which kernel's wait ran out (or'ed with kStatusWaitTimeout)
constexpr int kStatusAggTc = 2, kStatusLeafTc = 4, kStatusM2lGrp = 8;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async proxy (the bulk copies).
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int status_now(const int* status) {
  return *reinterpret_cast<const volatile int*>(status);
}

// Waits for the phase with the given parity to complete; false (and the
// status bit set) when it has not after kWaitNs. With give_up, the wait also
// ends early once another CTA has recorded a status bit, so that one failure
// does not cost every CTA of the launch its full wait; a wait for copies
// already issued passes give_up = false. site: the kernel's status bit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status, bool give_up = true,
                                          int site = 0) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (mbar_test(bar, parity)) return true;
    if (give_up && status_now(status) != 0) return false;
    if (global_ns() - t0 > kWaitNs) {
      atomicOr(status, kStatusWaitTimeout | site);
      return false;
    }
  }
}

// Tiled 2-D tensor copy (TMA) of the box at (x, y) of a tensor map into
// shared memory, completing on bar's transaction count. x (the innermost
// coordinate) times the element size must be a multiple of 16 bytes; dst
// 128-byte aligned. Parts of the box outside the tensor are zero-filled and
// count toward the transaction bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// Four rows (r0..r3, any order) of a 2-D tensor map whose box is one row
// high, from column x, into consecutive rows of dst (tile::gather4).
__device__ __forceinline__ void tma_gather4(void* dst, const void* map, int x, int r0, int r1, int r2, int r3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(smem_addr(bar))
      : "memory");
}

// Asynchronous global -> shared copy of 8 or 16 bytes (cached in L1), and the
// arrival on bar that follows this thread's earlier such copies (the arrival
// is not counted in advance: bar's expected count includes it).
template <int kBytes>
__device__ __forceinline__ void cp_async_ca(void* dst, const void* src) {
  static_assert(kBytes == 8 || kBytes == 16, "cp.async.ca takes 4, 8 or 16 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"(kBytes) : "memory");
}

__device__ __forceinline__ void cp_async_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const void* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

}  // namespace mlfma

#pragma once
// tma.cuh -- TMA tensor copies and mbarriers (inline PTX, sm_90+ forms used
// on sm_100a) shared by the TMA-fed kernels, and the host-side encoding of
// tensor maps through the driver entry point (no link against libcuda).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

namespace blgpu {
namespace tma {

constexpr int WAIT_LIMIT = 1 << 24;  // mbarrier polls (with back-off) before a copy counts as lost

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for phase `parity`: at most `limit` polls; false when the
// limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit = WAIT_LIMIT) {
  for (int it = 0; it < limit; ++it) {
    if (mbar_test(bar, parity)) return true;
    if (it >= 32) __nanosleep(64);
  }
  return false;
}
// bounded wait with the hardware-suspended try_wait (fewer issue slots
// than polling); false when the limit ran out
__device__ __forceinline__ bool mbar_wait_hw(uint64_t *bar, uint32_t parity) {
  for (int it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// plain arrival (count one) on an mbarrier
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// hardware-suspended wait that also gives up when *fail is set by another
// thread of the CTA (checked every 64 tries) or after WAIT_LIMIT tries (then
// it sets *fail); false when it gave up
__device__ __forceinline__ bool mbar_wait_or_fail(uint64_t *bar, uint32_t parity, volatile int *fail) {
  for (int it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 63) == 63 && *fail) return false;
  }
  *fail = 1;
  return false;
}
// generic-proxy shared-memory accesses before async-proxy ones (TMA)
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// untiled bulk copy global -> shared (both addresses 16-byte aligned, bytes
// a multiple of 16), completion counted on the mbarrier
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 2D tiled store from shared memory (coordinates in range, never negative)
__device__ __forceinline__ void store_2d(const CUtensorMap *map, const void *src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void store_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// wait until at most N bulk groups of this thread still read shared memory
template <int N> __device__ __forceinline__ void store_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// wait until all bulk groups of this thread have completed (writes done)
__device__ __forceinline__ void store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// 3D tiled store from shared memory (coordinates must be in range, never
// negative); completion through the bulk-group of the issuing thread
__device__ __forceinline__ void store_3d(const CUtensorMap *map, const void *src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void store_commit_and_wait_read() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// host: tiled tensor map, row-major dims[0] fastest; strides in bytes for
// dims 1..rank-1; false when the driver entry point or the encoding fails
bool encode(CUtensorMap *map, CUtensorMapDataType type, int rank, void *base, const cuuint64_t *dims,
            const cuuint64_t *strides, const cuuint32_t *box,
            CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE);

}  // namespace tma
}  // namespace blgpu

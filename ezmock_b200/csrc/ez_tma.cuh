// ez_tma.cuh -- Tensor Memory Accelerator (TMA) helpers for sm_100a: tensor
// maps encoded on the host through the driver entry point (no link-time
// dependency on libcuda), mbarrier waits with an iteration limit, and bulk
// tensor copies between global and shared memory.  Every tensor map covers
// this GPU's own buffers; no load here uses cluster multicast.
#ifndef EZ_TMA_CUH
#define EZ_TMA_CUH

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

// Encodes a tiled tensor map (cuTensorMapEncodeTiled, resolved once through
// cudaGetDriverEntryPoint).  Returns false on any error.
bool ez_tma_encode(CUtensorMap *map, CUtensorMapDataType type, int rank, void *base,
    const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
    CUtensorMapSwizzle swizzle);

// Iterations of an mbarrier wait before it gives up (a TMA copy lands within
// microseconds; the limit only bounds a wait that would otherwise not end).
#define EZ_TMA_SPIN_LIMIT (1u << 22)

__device__ __forceinline__ uint32_t ez_smem_addr(const void *p) {
  return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void ez_mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(ez_smem_addr(bar)), "r"(count)
               : "memory");
}

// Makes the barrier initialisation visible to the async proxy (TMA).
__device__ __forceinline__ void ez_fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void ez_mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(ez_smem_addr(bar)), "r"(bytes) : "memory");
}

// Waits for phase `parity` of the barrier to complete; false if the limit
// ran out first.
__device__ __forceinline__ bool ez_mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = ez_smem_addr(bar);
  for (uint32_t it = 0; it < EZ_TMA_SPIN_LIMIT; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// 3D tile load global -> shared, completion counted on `bar` (bytes).
__device__ __forceinline__ void ez_tma_load3(void *smem, const CUtensorMap *map,
    int c0, int c1, int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];"
      :: "r"(ez_smem_addr(smem)), "l"(map), "r"(c0), "r"(c1), "r"(c2),
         "r"(ez_smem_addr(bar)) : "memory");
}

// 3D tile store shared -> global (bulk async group of the issuing thread).
__device__ __forceinline__ void ez_tma_store3(const CUtensorMap *map, int c0, int c1, int c2,
    const void *smem) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
      :: "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(ez_smem_addr(smem)) : "memory");
}

__device__ __forceinline__ void ez_tma_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Waits until the issuing thread's committed stores have finished reading
// shared memory (all but the newest N groups).
template <int N>
__device__ __forceinline__ void ez_tma_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" :: "n"(N) : "memory");
}

// Waits until the issuing thread's committed stores are complete.
__device__ __forceinline__ void ez_tma_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (TMA) reads of them.
__device__ __forceinline__ void ez_fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void ez_prefetch_map(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" :: "l"(map) : "memory");
}

#endif

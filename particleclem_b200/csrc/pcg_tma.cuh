// pcg_tma.cuh -- Tensor Memory Accelerator (TMA) halo-tile loads for sm_100a, in inline PTX.
//
// A block stages one box of a 4-D FP32 array (x, y, z, component) from global memory into
// shared memory with one cp.async.bulk.tensor, completion tracked by an mbarrier in shared
// memory. No cluster multicast is used: every load reads this GPU's own memory into the
// issuing block's shared memory only. The tensor maps (CUtensorMap, 128 bytes, 64-byte
// aligned) are built on the host with cuTensorMapEncodeTiled and live in the launch tables
// in global memory.
//
// Rules the callers keep (the host checks them when it encodes a map): the global base is
// 16-byte aligned, the strides of dimensions 1..3 are multiples of 16 bytes, the box's x
// extent times 4 bytes is a multiple of 16, and every x coordinate a load starts at is a
// multiple of 4 elements (16 bytes); y, z and component coordinates may take any value,
// and the parts of a box outside the array read as zero.
#pragma once

#include <cstdint>

namespace PCG_TU {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  // make the initialised barrier visible to the async proxy (the TMA unit)
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive on the barrier announcing `bytes` of transaction data still to come.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// One bounded wait for phase `parity` of the barrier: true once the phase completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
    "{\n"
    ".reg .pred p;\n"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
    "selp.u32 %0, 1, 0, p;\n"
    "}\n"
    : "=r"(done)
    : "r"(smem_addr(bar)), "r"(parity)
    : "memory");
  return done != 0;
}

// Load the box at element coordinates (x, y, z, c) of the 4-D tensor map into shared
// memory dst (x fastest, then y, z, c: the box dense), completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, int x, int y, int z, int c, uint64_t* bar) {
  asm volatile(
    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
    "[%6];" ::"r"(smem_addr(dst)),
    "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_addr(bar))
    : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// Wait for phase `parity` of `bar` at most kTmaWaitLimit tries (each try suspends the
// thread for a hardware-chosen time); false when the limit is reached.
constexpr uint32_t kTmaWaitLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kTmaWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace PCG_TU

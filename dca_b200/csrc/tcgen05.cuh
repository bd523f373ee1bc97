// Minimal tcgen05 (5th-generation tensor core) building blocks for sm_100a, as inline PTX:
// tensor-memory allocation, shared-memory matrix descriptors for K-major 128-byte-swizzled
// operand tiles, the BF16 x BF16 -> FP32 MMA with the accumulator in tensor memory, the commit that
// signals an mbarrier when issued MMAs finish, and 32-lane x 16-column accumulator loads.
//
// Descriptor encodings follow the PTX ISA's tcgen05 "matrix descriptor" and "instruction
// descriptor" tables (also spelled out in CUTLASS's cute/arch/mma_sm100_desc.hpp):
//   smem descriptor  [0,14) start address >> 4, [16,30) leading byte offset >> 4,
//                    [32,46) stride byte offset >> 4, [46,48) version = 1, [61,64) layout
//                    (2 = 128-byte swizzle)
//   instr descriptor [4,6) D format (1 = F32), [7,10) A format (1 = BF16), [10,13) B format,
//                    [15] A major (0 = K), [16] B major, [17,23) N >> 3, [24,29) M >> 4
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "async_copy.cuh"

namespace dcaacc {
namespace tc {

// K-major operand tile with 128-byte swizzle: rows of 64 BF16 (128 bytes), 8-row atoms of 1 KB.
// Byte offset of element (row, k) inside a 64-column sub-tile whose base is 1024-byte aligned.
__host__ __device__ inline uint32_t sw128Offset(int row, int k) {
  const int chunk = (k >> 3) ^ (row & 7);
  return static_cast<uint32_t>(row * 128 + chunk * 16 + (k & 7) * 2);
}

__device__ inline uint64_t smemDescSw128(const void* tile_base) {
  const uint64_t addr = smemAddr(tile_base);
  return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// K-major operand tile with 64-byte swizzle: rows of 32 FP16 / BF16 (64 bytes), 8-row atoms of 512 B
// (the layout a TMA load with CU_TENSOR_MAP_SWIZZLE_64B writes).  Base 1024-byte aligned.
__device__ inline uint64_t smemDescSw64(const void* tile_base) {
  const uint64_t addr = smemAddr(tile_base);
  return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}

// Instruction descriptor bit that negates A (D += -A B^T).
constexpr uint32_t kNegateA = 1u << 13;

// Advance a descriptor's start address by `bytes` (a K step of 16 BF16 inside a swizzle atom is
// 32 bytes; the swizzle is applied on absolute address bits, so this is exact for 1 KB-aligned atoms).
__device__ inline uint64_t descAdvance(uint64_t desc, uint32_t bytes) {
  return desc + static_cast<uint64_t>(bytes >> 4);
}

// FP16 x FP16 -> FP32 (A and B formats 0).
__host__ __device__ constexpr uint32_t instrDescF16F32(int M, int N) {
  return (1u << 4) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

__host__ __device__ constexpr uint32_t instrDescBf16F32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

// Allocates `cols` tensor-memory columns (power of two >= 32); must be executed by one full warp.
// The base address is written to *slot (shared memory).
__device__ inline void tmemAlloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(slot)),
               "r"(cols)
               : "memory");
}

__device__ inline void tmemRelinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Frees the columns; executed by the same warp that allocated.
__device__ inline void tmemDealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

__device__ inline void fenceBeforeThreadSync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ inline void fenceAfterThreadSync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues (kind::f16: BF16 or FP16 operands, both
// the same type, as the instruction descriptor says).  accumulate = 0 overwrites D.
__device__ inline void mmaBf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                               uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives once on the mbarrier when all previously issued MMAs of this thread complete.
__device__ inline void commitTo(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smemAddr(bar))
               : "memory");
}

// Each thread of the warp reads 16 consecutive 32-bit columns of its own lane (the warp's lane
// quarter is selected by the address's lane field).
__device__ inline void ld32x32bx16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i)
    v[i] = __uint_as_float(r[i]);
}

// As ld32x32bx16, 32 consecutive columns.
__device__ inline void ld32x32bx32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i)
    v[i] = __uint_as_float(r[i]);
}

__device__ inline void waitLd() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16-byte asynchronous global -> shared copy (no mbarrier; completed by cpAsyncWaitAll).
__device__ inline void cpAsync16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smemAddr(smem_dst)), "l"(gmem_src) : "memory");
}

__device__ inline void cpAsyncWaitAll() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// ---- Tensor memory access (TMA) ----
// 3-D tiled load (box from the tensor map) into shared memory, completing `bytes` of the
// mbarrier's transaction count.  Plain (non-multicast) form only.  The innermost coordinate x
// must be a multiple of 16 bytes' worth of elements.
__device__ inline void tmaLoad3d(void* smem_dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smemAddr(smem_dst)), "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smemAddr(bar))
      : "memory");
}

__device__ inline void prefetchTensorMap(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

}  // namespace tc
}  // namespace dcaacc

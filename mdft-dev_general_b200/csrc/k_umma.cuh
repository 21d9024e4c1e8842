// tcgen05 (5th-generation tensor core) primitives for the angular contractions: tensor
// memory allocation, shared-memory matrix descriptors, the MMA issued by one thread with
// its completion signalled on an mbarrier, and the tensor-memory -> register loads of the
// epilogue.  Single-CTA forms only (cta_group::1), operands in this CTA's shared memory:
// nothing here reads another CTA's or another GPU's memory.
//
// Operand layout ("K-major, no swizzle" in the PTX ISA's terms): a tile of R rows (points,
// or output columns) by Kp reduction elements is stored as 8-row x 16-byte core matrices of
// 128 contiguous bytes, [R/8][Kp/CE][8 rows][CE elements] with CE = 16 / element size.  The
// two core matrices along K that one instruction reads (K = 32 bytes) are 128 bytes apart
// (the descriptor's leading byte offset) and successive 8-row groups are Kp/CE * 128 bytes
// apart (stride byte offset).
#pragma once

#include <cstdint>

#include <cuda_bf16.h>

#include "k_tma.cuh"

namespace mdft {
namespace umma {

// Bytes of a packed [R][Kp] operand tile of elements of `esize` bytes.
__host__ __device__ constexpr size_t tile_bytes(int R, int Kp, int esize) { return (size_t)R * Kp * esize; }

// Byte offset of element (r, k) of a packed [R][Kp] tile (CE = 16 / esize elements per chunk).
__host__ __device__ constexpr uint32_t elem_offset(int r, int k, int Kp, int esize) {
    return (uint32_t)((((r >> 3) * (Kp * esize / 16) + (k * esize) / 16) << 7) + ((r & 7) << 4) + ((k * esize) & 15));
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading byte offset
// (between the two 16-byte K halves of an instruction: 128), stride byte offset (between
// 8-row groups), version 1 in bits 46-47, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, A and B of format `fmt` (kind::f16: 1 = BF16;
// kind::tf32: 2 = TF32), both K-major, N = n (multiple of 16 for M = 128), M = 128.
__host__ __device__ constexpr uint32_t instr_desc(int fmt, int n) {
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// Allocate `ncols` (power of two, >= 32) tensor-memory columns for this CTA; the base
// address lands in *slot (shared memory).  Executed by one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, M = 128; issued by one thread.
template <int KIND>  // 0: kind::f16, 1: kind::tf32
__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
    if constexpr (KIND == 0) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(dtmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(dtmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z)
            : "memory");
    }
}

// Arrive once on `bar` when every tcgen05 operation issued so far by this thread is done.
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// 16 consecutive FP32 columns of this thread's lane (32x32b shape: warp w reads lanes
// 32 (w % 4) .. +31; the address carries the lane in bits 31..16 and the column in 15..0).
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Split of an FP32 value into two BF16 values with v ~ hi + lo (relative error ~2^-17).
__device__ __forceinline__ void split_bf16(float v, uint16_t &hi, uint16_t &lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

// The same split of two values with paired conversions (cvt.rn.bf16x2.f32): hi and lo
// receive (v0 | v1 << 16) as BF16 pairs.
__device__ __forceinline__ void split_bf16x2(float v0, float v1, uint32_t &hi, uint32_t &lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);  // .x = v0 (low half), .y = v1
    const float h0 = __low2float(h), h1 = __high2float(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(v0 - h0, v1 - h1);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

// Bounded wait on an mbarrier phase (false when the poll limit ran out).
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t parity) { return mbar_wait(bar, parity); }

}  // namespace umma
}  // namespace mdft

// Common device helpers for the dsa110-rt B200 fast-search kernels.
//
// Status words: every kernel that can give up (a bounded wait that ran out,
// an index that failed a bounds check in a checked build) records a code in
// a caller-provided device int; the host reads it after the stream syncs.
// No kernel traps.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "../../include/dsb200.h"

#define DSB_DEV __device__ __forceinline__

// Stage-2 ring element in the BF16 storage form: one 32-bit word per cell,
// the real part (bf16, nearest-even from float32) in the low half and the
// imaginary part in the high half.
DSB_DEV uint32_t bf16_pair(float re, float im) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);  // .x = re (low), .y = im (high)
  return *reinterpret_cast<const uint32_t*>(&h);
}
DSB_DEV float2 bf16_pair_to_f2(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}

// Packed float32 pairs (sm_100 add.rn.f32x2 / sub.rn.f32x2): one
// instruction for two independent float32 adds, each part rounded to
// nearest as the scalar add rounds it.
DSB_DEV unsigned long long f2_pack(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
DSB_DEV float2 f2_unpack(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
DSB_DEV float2 f2_add(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(b)));
  return f2_unpack(r);
}
DSB_DEV float2 f2_sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(b)));
  return f2_unpack(r);
}
DSB_DEV float4 f4_add(float4 a, float4 b) {
  const float2 lo = f2_add(make_float2(a.x, a.y), make_float2(b.x, b.y));
  const float2 hi = f2_add(make_float2(a.z, a.w), make_float2(b.z, b.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

// Iteration limit for every mbarrier spin (each try_wait may itself suspend
// for a hardware-chosen interval, so this bounds the wait to well under a
// few seconds on a healthy GPU).
#ifndef DSB_SPIN_LIMIT
#define DSB_SPIN_LIMIT (1u << 22)
#endif

DSB_DEV uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

DSB_DEV void dsb_flag(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// Bounds-checked build (-DDSB_CHECK): DSB_INB(i, n, status) is true when
// 0 <= i < n; otherwise it records DSB_E_BOUNDS in *status and is false, and
// the access it guards is skipped (no trap).  The normal build compiles it
// to true.  It guards the indices that come from host-built tables: ring
// slots and cells, gridding rows and baselines, combine targets.
#ifdef DSB_CHECK
DSB_DEV bool dsb_inb(long long i, long long n, int* status) {
  if (i >= 0 && i < n) return true;
  dsb_flag(status, DSB_E_BOUNDS);
  return false;
}
#define DSB_INB(i, n, st) dsb_inb((long long)(i), (long long)(n), (st))
#else
#define DSB_INB(i, n, st) true
#endif

// ---------------------------------------------------------------------------
// mbarrier
// ---------------------------------------------------------------------------
DSB_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
DSB_DEV void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
DSB_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Returns false if the barrier phase did not complete within the limit.
DSB_DEV bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < DSB_SPIN_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Arrive on `bar` expecting `bytes` of asynchronous copies in this phase.
DSB_DEV void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Arrive on `bar` with no asynchronous copy (completes a phase that carries
// no bytes).
DSB_DEV void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// One 3-D tile of a tensor map (this GPU's global memory, one CTA) into
// this CTA's shared memory, completing on `bar`.  The innermost coordinate
// times the element size must be a multiple of 16 bytes.
DSB_DEV void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// One 4-D tile of a tensor map (this GPU's global memory, one CTA) into
// this CTA's shared memory, completing on `bar`.  The innermost coordinate
// times the element size must be a multiple of 16 bytes.
DSB_DEV void tma_load_4d(void* dst, const void* tmap, int x, int y, int z, int w,
                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// tcgen05 (5th-generation tensor core, accumulators in tensor memory)
// ---------------------------------------------------------------------------
DSB_DEV void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
DSB_DEV void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
DSB_DEV void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Executed by one full warp.
DSB_DEV void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
DSB_DEV void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
DSB_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, signed int8 inputs, int32 accumulate.
DSB_DEV void umma_i8_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                        uint32_t accumulate) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2),
      "r"(m3)
      : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, float16 inputs (kind::f16; the
// instruction descriptor says f16 for both), float32 accumulate.
DSB_DEV void umma_f16_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                         uint32_t accumulate) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2),
      "r"(m3)
      : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, tf32 inputs (kind::tf32), float32 accumulate.
DSB_DEV void umma_tf32_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                          uint32_t accumulate) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2),
      "r"(m3)
      : "memory");
}

// Arrive on an mbarrier once every tcgen05.mma issued so far by this thread
// has completed.
DSB_DEV void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// Instruction descriptor: kind::i8, signed A and B, S32 accumulator,
// both operands K-major (bit layout of the sm_100 UMMA instruction
// descriptor: c_format [4,6), a_format [7,10), b_format [10,13),
// n_dim = N>>3 at [17,23), m_dim = M>>4 at [24,29)).
__host__ __device__ constexpr uint32_t idesc_i8(uint32_t M, uint32_t N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// Shared-memory matrix descriptor for a K-major operand in the 128-byte
// swizzle layout: rows of 128 B, 8-row atoms of 1024 B stacked at
// SBO = 1024 B, LBO unused (1), version 1, layout type SWIZZLE_128B (2).
DSB_DEV uint64_t sdesc_k_sw128(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// Byte offset of (row, k byte) inside a K-major SWIZZLE_128B tile whose
// 8-row atoms are 1024 B apart: the 16-byte chunk index is XOR-ed with the
// row's position inside its atom.
DSB_DEV uint32_t sw128_offset(uint32_t row, uint32_t kbyte) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + ((((kbyte >> 4) ^ (row & 7u)) & 7u) << 4) +
         (kbyte & 15u);
}

// Load 16 consecutive 32-bit TMEM columns of this warp's 32 lanes.
DSB_DEV void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
DSB_DEV void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Load 16 columns and wait for them in one statement, so that no use of r
// can be scheduled between the load and its wait.
DSB_DEV void tmem_ld16_wait(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

// Store 16 consecutive 32-bit TMEM columns of this warp's 32 lanes.
DSB_DEV void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 "
      "[%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}
DSB_DEV void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------------------
// int4 helpers: four packed (real | imag << 4) complex samples per 32-bit word
// ---------------------------------------------------------------------------
// Four two's-complement nibbles sign-extended to int8 bytes without byte
// SIMD: a nibble's bit 3 times 0x1E fills bits 4-7 of its own byte (0x08 *
// 0x1E = 0xF0, no carry into the next byte), and as those bits are clear in
// the nibble, adding is or-ing: one multiply-add after two masks.
DSB_DEV uint32_t nib_lo_s8x4(uint32_t w) {
  return (w & 0x08080808u) * 0x1Eu + (w & 0x0F0F0F0Fu);
}
DSB_DEV uint32_t nib_hi_s8x4(uint32_t w) {
  const uint32_t h = (w >> 4) & 0x0F0F0F0Fu;
  return (h & 0x08080808u) * 0x1Eu + h;
}
// Byte-wise 0 - v (v in -8..7 per byte): 0x80 - (v & 0x7F) cannot borrow
// across bytes, and xor-ing the complement of v's top bit restores the sign.
DSB_DEV uint32_t neg_s8x4(uint32_t v) {
  return (0x80808080u - (v & 0x7F7F7F7Fu)) ^ (~v & 0x80808080u);
}

DSB_DEV int upper_bls(int a, int b) { return a * (a + 1) / 2 + b; }

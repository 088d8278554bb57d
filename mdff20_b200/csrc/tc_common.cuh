// Helpers of the tcgen05 (5th-generation tensor core) kernels of sm_100a: shared-memory
// addresses, TF32 operand splitting, bounded mbarrier waits, matrix and instruction
// descriptors, MMA issue/commit, tensor-memory loads and bulk global->shared copies.
#pragma once
#include <cstdint>

#include "engine.cuh"

namespace mdffgpu {

constexpr long long TC_WAIT_CYCLES = 2000000000LL;   // bound of one mbarrier wait (about a second)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// x = h + l: h is x rounded to the TF32 grid (10 fraction bits; the half unit added to
// the magnitude bits, so ties round away from zero), l = x - h exactly; the MMA reads l to
// TF32 precision, so the pair carries about 21 bits of x
__device__ __forceinline__ float tf32_round(float x) { return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u); }
__device__ __forceinline__ void split2(float x, float &h, float &l) {
    h = tf32_round(x);
    l = x - h;
}

// one bounded probe of the phase (the hardware may block briefly before it returns false)
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// non-blocking test of the phase
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// polls until the phase completes or TC_WAIT_CYCLES SM clock cycles (about a second) pass
// (a phase already complete returns after one test, without reading the clock)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try(bar, parity))
        if (clock64() - t0 > TC_WAIT_CYCLES) return false;
    return true;
}

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance between the
// two 16-byte K chunks of one MMA, sbo = byte distance between 8-row groups
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version of sm_100
    return d;                 // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor, kind::tf32: D FP32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t addr, float *v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = __uint_as_float(r[k]);
}


// byte offset of element (row or column x, K index k) of a K-major no-swizzle operand
// whose 16-byte K chunks lie `lbo` bytes apart (8 x 16-byte core matrices)
__device__ __forceinline__ uint32_t kmaj(int x, int k, uint32_t lbo) {
    return (uint32_t)(k >> 2) * lbo + (uint32_t)((x >> 3) * 128 + (x & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// arrive on the barrier and add `bytes` to the transaction count its phase waits for
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// contiguous global -> shared copy of `bytes` (16-byte aligned addresses, a multiple of
// 16 bytes) that completes as transactions on the barrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

}  // namespace mdffgpu

// sm_100a tensor-core helpers shared by the tcgen05 kernels: shared-memory
// operand descriptors (canonical K-major layout, no swizzle), instruction
// descriptors, MMA issue and commit, bounded mbarrier waits and tensor-memory
// loads.
//
// K-major operand layout without swizzle: the operand is cut into core
// matrices of 8 rows x 16 bytes (8 BF16 or 4 TF32 elements of K), each 128
// contiguous bytes with row r at 16 r bytes; K-adjacent core matrices are
// `lbo` bytes apart and the 8-row groups `sbo` bytes apart.  One MMA consumes
// 32 bytes of K (two core matrices): K = 16 for kind::f16, K = 8 for
// kind::tf32.
#pragma once

#include <cstdint>

namespace fb200 {
namespace tc {

constexpr long long MMA_SPINS = 1ll << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row, k) in a K-major operand whose K extent is
// `kbytes` bytes per row (a multiple of 16), elements of `esize` bytes
__host__ __device__ __forceinline__ uint32_t core_offset(int row, int k, int kbytes, int esize) {
    const int per = 16 / esize;  // elements of K in one core-matrix row
    return (uint32_t)((row >> 3) * (kbytes / 16) * 128 + (k / per) * 128 + (row & 7) * 16 + (k % per) * esize);
}

// shared-memory matrix descriptor of a K-major, unswizzled operand starting
// at `addr` (16-byte aligned), K-adjacent core matrices `lbo` bytes apart,
// 8-row groups `sbo` bytes apart
__device__ __forceinline__ uint64_t operand_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, no swizzle
}

// instruction descriptor of kind::f16 / kind::tf32: FP32 accumulator, A and B
// of format `ab` (0 F16, 1 BF16, 2 TF32), both K-major, M x N
__host__ __device__ __forceinline__ uint32_t instr_desc(int ab, int m, int n) {
    return (1u << 4) | ((uint32_t)ab << 7) | ((uint32_t)ab << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}
constexpr int FORMAT_BF16 = 1;
constexpr int FORMAT_TF32 = 2;

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// wait for the phase `phase` of the mbarrier to complete; gives up after a
// bounded number of polls and returns false
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (long long spin = 0; spin < MMA_SPINS; spin++) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
        __nanosleep(32);
    }
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// tensor-memory allocation of `cols` columns (a power of two >= 32) by one
// whole warp; the address is written to shared memory at `slot`
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

// x rounded to TF32 (10 explicit mantissa bits, round to nearest, ties away)
// and the FP32 remainder: x = hi + lo exactly, |lo| <= 2^-11 |x|
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    lo = x - hi;
}

}  // namespace tc
}  // namespace fb200

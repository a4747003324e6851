// Tensor-core inference of the radial surrogate (surrogate.hpp) on sm_100a:
// tcgen05.mma with BF16 operands in shared memory and FP32 accumulators in
// tensor memory, 128 distances per tile, persistent CTAs of 4 warps.
//
// Every operand is a sum of three BF16 parts (hi + mid + lo, 24 significant
// bits): x = x0 + x1 + x2 with x0 = bf16(x), x1 = bf16(x - x0),
// x2 = bf16(x - x0 - x1).  A product a w is taken as the six products
// a_i w_j with i + j <= 2, each term below 2^-24 of a w being dropped, so
// the layers reproduce FP32 products to a few FP32 ulps.
//
// Per tile:
//   layer 1 (CUDA cores)  h1 = silu(w1 x + b1) and its r-derivative, split
//                         into three BF16 parts, the A operands [128 x 64]
//   layer 2 (tcgen05)     D = h1 W2^T and dh1 W2^T, 4 K-steps of 16, 6 MMAs
//                         each, M = 128, N = 64, two TMEM regions
//   epilogue              tcgen05.ld, h2 = silu(D + b2), dh2 = silu'(.) dD, split
//   layer 3 (tcgen05)     Y = h2 W3^T, dY = dh2 W3^T, N = outputs rounded up to 16
//   epilogue              R = s (Y + b3), dR/dr = s dY, staged in shared memory
//                         and stored row-contiguously
// One elected thread issues the MMAs and commits them to an mbarrier; every
// wait is bounded and sets an error flag instead of hanging.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8 x 8 BF16 core matrices of 128 contiguous bytes (row r at 16 r bytes),
// K-adjacent core matrices 128 bytes apart (leading byte offset), 8-row
// groups K/8 x 128 bytes apart (stride byte offset).
#include <cuda_bf16.h>

#include "engine.hpp"
#include "tcgen05.cuh"

namespace fb200 {

namespace {

constexpr int SH = 64;          // hidden units
constexpr int TILE = 128;       // distances per tile (MMA M)
constexpr int TMEM_COLS = 256;  // [0, N) values, [128, 128 + N) derivatives
using tc::fence_after;
using tc::fence_async_smem;
using tc::fence_before;
using tc::mbar_wait;
using tc::mma_bf16;
using tc::mma_commit;
using tc::smem_addr;
using tc::tmem_load16;

// byte offset of element (row, k) in a K-major [rows x 64] BF16 operand
__host__ __device__ __forceinline__ uint32_t core_offset(int row, int k) { return tc::core_offset(row, k, SH * 2, 2); }

__device__ __forceinline__ uint64_t operand_desc(uint32_t addr) { return tc::operand_desc(addr, 128, (SH / 8) * 128); }

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n
__device__ __forceinline__ uint32_t mma_idesc(int n) { return tc::instr_desc(tc::FORMAT_BF16, TILE, n); }

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + __expf(-z)); }

constexpr int PARTS = 3;                    // BF16 parts of every operand
constexpr int A_PART = TILE * SH * 2;       // bytes of one part of an A operand

// the three BF16 parts of v, at part p's copy of the K-major operand
__device__ __forceinline__ void store_split(unsigned char* base, int row, int k, float v) {
    const __nv_bfloat16 p0 = __float2bfloat16_rn(v);
    const float r1 = v - __bfloat162float(p0);
    const __nv_bfloat16 p1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 p2 = __float2bfloat16_rn(r1 - __bfloat162float(p1));
    const uint32_t o = core_offset(row, k);
    *reinterpret_cast<__nv_bfloat16*>(base + o) = p0;
    *reinterpret_cast<__nv_bfloat16*>(base + A_PART + o) = p1;
    *reinterpret_cast<__nv_bfloat16*>(base + 2 * A_PART + o) = p2;
}

// D (+)= A B^T for the operands split in three parts: the six products
// A_i B_j with i + j <= 2 of K-step s (32 bytes of K), `acc` for the first
__device__ __forceinline__ void mma_split(uint32_t d, uint32_t a, uint32_t a_part, uint32_t b, uint32_t b_part, int s,
                                          uint32_t idesc, uint32_t acc, uint32_t b_sbo) {
    const uint32_t k = 256 * s;
#pragma unroll
    for (int i = 0; i < PARTS; i++)
#pragma unroll
        for (int j = 0; j + i < PARTS; j++) {
            const uint64_t da = tc::operand_desc(a + i * a_part + k, 128, (SH / 8) * 128);
            const uint64_t db = tc::operand_desc(b + j * b_part + k, 128, b_sbo);
            mma_bf16(d, da, db, idesc, (i == 0 && j == 0) ? acc : 1u);
        }
}

struct MmaArgs {
    int O, out_pad;
    double rc;
    const float* master;  // w1 [64], b1 [64], W2, b2 [64], W3, b3 [O]
    const float* scale;
    const uint4* w2;      // packed BF16 B operand [3 parts][64 x 64]
    const uint4* w3;      // packed BF16 B operand [3 parts][out_pad x 64]
    const double* r;
    int64_t n;
    float* values;
    float* derivs;
    int64_t ld;
    int32_t* status;
    // when set, the hidden features h2 and dh2/dr of every distance are
    // written to features[i][0 .. 64) and [64 .. 128) and layer 3 is skipped
    // (the inputs of the output-layer fit, with the numerics of this kernel)
    float* features = nullptr;
};

__global__ void __launch_bounds__(TILE, 1) surrogate_mma_kernel(MmaArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned regions
    unsigned char* base = smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023);
    unsigned char* A_h = base;                           // 3 parts x 16 KB
    unsigned char* A_t = A_h + PARTS * A_PART;           // 3 parts x 16 KB
    unsigned char* B2 = A_t + PARTS * A_PART;            // 3 parts x 8 KB
    unsigned char* B3 = B2 + PARTS * SH * SH * 2;        // 3 parts x out_pad x 128 bytes
    float* prm = reinterpret_cast<float*>(B3 + PARTS * a.out_pad * SH * 2);  // w1, b1, b2, b3, scale
    float* w1 = prm;
    float* b1 = w1 + SH;
    float* b2 = b1 + SH;
    float* b3 = b2 + SH;
    float* sc = b3 + a.out_pad;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sc + a.out_pad + 2);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    __shared__ int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int O = a.O;
    const int offW2 = 2 * SH, offB2 = offW2 + SH * SH, offW3 = offB2 + SH, offB3 = offW3 + O * SH;
    for (int q = tid; q < PARTS * SH * SH * 2 / 16; q += TILE) reinterpret_cast<uint4*>(B2)[q] = a.w2[q];
    for (int q = tid; q < PARTS * a.out_pad * SH * 2 / 16; q += TILE) reinterpret_cast<uint4*>(B3)[q] = a.w3[q];
    for (int q = tid; q < SH; q += TILE) {
        w1[q] = a.master[q];
        b1[q] = a.master[SH + q];
        b2[q] = a.master[offB2 + q];
    }
    for (int q = tid; q < a.out_pad; q += TILE) {
        b3[q] = q < O ? a.master[offB3 + q] : 0.0f;
        sc[q] = q < O ? a.scale[q] : 0.0f;
    }
    if (tid == 0) {
        abort_flag = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const uint32_t bar_addr = smem_addr(bar);
    const float dxdr = (float)(2.0 / a.rc);
    uint32_t phase = 0;
    const int64_t tiles = (a.n + TILE - 1) / TILE;

    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t i = tile * TILE + tid;
        const bool valid = i < a.n;
        const float x = valid ? (float)(2.0 * a.r[i] / a.rc - 1.0) : 0.0f;
        for (int k = 0; k < SH; k++) {
            const float z = w1[k] * x + b1[k];
            const float sg = sigmoid(z);
            store_split(A_h, tid, k, z * sg);
            store_split(A_t, tid, k, sg * (1.0f + z * (1.0f - sg)) * w1[k] * dxdr);
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            const uint32_t id = mma_idesc(SH);
            const uint32_t aH = smem_addr(A_h), aT = smem_addr(A_t), b = smem_addr(B2);
            for (int s = 0; s < SH / 16; s++) {
                mma_split(tmem, aH, A_PART, b, SH * SH * 2, s, id, s > 0, (SH / 8) * 128);
                mma_split(tmem + 128, aT, A_PART, b, SH * SH * 2, s, id, s > 0, (SH / 8) * 128);
            }
            mma_commit(bar_addr);
        }
        if (mbar_wait(bar_addr, phase)) {
            phase ^= 1;
        } else {
            atomicOr(a.status, 1);
            abort_flag = 1;
        }
        __syncthreads();
        if (abort_flag) break;
        fence_after();
        for (int c = 0; c < SH; c += 16) {
            float d[16], t[16];
            tmem_load16(tmem + lane_base + c, d);
            tmem_load16(tmem + lane_base + 128 + c, t);
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const float z = d[q] + b2[c + q];
                const float sg = sigmoid(z);
                const float h2 = z * sg, dh2 = sg * (1.0f + z * (1.0f - sg)) * t[q];
                if (a.features) {
                    const int64_t gi = tile * TILE + tid;
                    if (gi < a.n) {
                        a.features[gi * 2 * SH + c + q] = h2;
                        a.features[gi * 2 * SH + SH + c + q] = dh2;
                    }
                } else {
                    store_split(A_h, tid, c + q, h2);
                    store_split(A_t, tid, c + q, dh2);
                }
            }
        }
        fence_before();
        fence_async_smem();
        __syncthreads();
        if (a.features) continue;  // no layer 3
        if (tid == 0) {
            fence_after();
            const uint32_t id = mma_idesc(a.out_pad);
            const uint32_t aH = smem_addr(A_h), aT = smem_addr(A_t), b = smem_addr(B3);
            for (int s = 0; s < SH / 16; s++) {
                mma_split(tmem, aH, A_PART, b, a.out_pad * SH * 2, s, id, s > 0, (SH / 8) * 128);
                mma_split(tmem + 128, aT, A_PART, b, a.out_pad * SH * 2, s, id, s > 0, (SH / 8) * 128);
            }
            mma_commit(bar_addr);
        }
        if (mbar_wait(bar_addr, phase)) {
            phase ^= 1;
        } else {
            atomicOr(a.status, 1);
            abort_flag = 1;
        }
        __syncthreads();
        if (abort_flag) break;
        fence_after();
        // The layer-3 MMAs have completed (mbarrier), so the A operands are
        // free: each warp stages its 32 rows x 16 columns there and stores
        // them row-contiguously (two rows of 64 bytes per instruction)
        // instead of one scattered element per lane.
        float* stage_v = reinterpret_cast<float*>(A_h) + warp * (2 * 32 * 17);
        float* stage_d = stage_v + 32 * 17;
        const int lane = tid & 31;
        for (int c = 0; c < a.out_pad; c += 16) {
            float y[16], t[16];
            tmem_load16(tmem + lane_base + c, y);
            tmem_load16(tmem + lane_base + 128 + c, t);
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int o = c + q;
                stage_v[lane * 17 + q] = sc[o] * (y[q] + b3[o]);
                stage_d[lane * 17 + q] = sc[o] * t[q];
            }
            __syncwarp();
            const int col = lane & 15, o = c + col;
#pragma unroll 4
            for (int it = 0; it < 16; it++) {
                const int row = 2 * it + (lane >> 4);
                const int64_t gi = tile * TILE + warp * 32 + row;
                if (gi < a.n && o < O) {
                    a.values[gi * a.ld + o] = stage_v[row * 17 + col];
                    if (a.derivs) a.derivs[gi * a.ld + o] = stage_d[row * 17 + col];
                }
            }
            __syncwarp();
        }
        fence_before();
        __syncthreads();
    }
    if (abort_flag) {
        // let the MMAs in flight finish (bounded) before freeing tensor memory
        mbar_wait(bar_addr, phase);
    }
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// the three BF16 parts of every weight, each part a K-major B operand
__global__ void pack_weights_kernel(const float* __restrict__ master, int O, int out_pad, unsigned char* w2,
                                    unsigned char* w3) {
    const int offW2 = 2 * SH, offW3 = offW2 + SH * SH + SH;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    auto split = [](float v, unsigned char* base, uint32_t o, int part_bytes) {
        const __nv_bfloat16 p0 = __float2bfloat16_rn(v);
        const float r1 = v - __bfloat162float(p0);
        const __nv_bfloat16 p1 = __float2bfloat16_rn(r1);
        const __nv_bfloat16 p2 = __float2bfloat16_rn(r1 - __bfloat162float(p1));
        *reinterpret_cast<__nv_bfloat16*>(base + o) = p0;
        *reinterpret_cast<__nv_bfloat16*>(base + part_bytes + o) = p1;
        *reinterpret_cast<__nv_bfloat16*>(base + 2 * part_bytes + o) = p2;
    };
    if (t < SH * SH) {
        const int row = t / SH, k = t % SH;
        split(master[offW2 + t], w2, core_offset(row, k), SH * SH * 2);
    }
    if (t < out_pad * SH) {
        const int row = t / SH, k = t % SH;
        split(row < O ? master[offW3 + row * SH + k] : 0.0f, w3, core_offset(row, k), out_pad * SH * 2);
    }
}

size_t mma_shared_bytes(int out_pad) {
    return 1024 + 2 * PARTS * (size_t)A_PART + PARTS * (size_t)SH * SH * 2 + PARTS * (size_t)out_pad * SH * 2 +
           4 * (size_t)(3 * SH + 2 * out_pad + 2) + 16 + 64;
}

}  // namespace

void pack_surrogate_weights(const float* master, int hidden, int O, int out_pad, void* w2_bf16, void* w3_bf16,
                            cudaStream_t stream) {
    if (hidden != SH) throw invalid_parameter("the tensor-core surrogate kernel needs 64 hidden units");
    const int total = std::max(SH * SH, out_pad * SH);
    pack_weights_kernel<<<(total + 255) / 256, 256, 0, stream>>>(master, O, out_pad, (unsigned char*)w2_bf16,
                                                                 (unsigned char*)w3_bf16);
    CUDA_CHECK(cudaGetLastError());
}

void launch_surrogate_mma(const float* master, int hidden, int O, int out_pad, double rc, const float* scale,
                          const void* w2_bf16, const void* w3_bf16, const double* r, int64_t n, float* values,
                          float* derivs, int64_t ld, int32_t* status, cudaStream_t stream, float* features) {
    if (hidden != SH) throw invalid_parameter("the tensor-core surrogate kernel needs 64 hidden units");
    if (out_pad > 128 || out_pad % 16 != 0)
        throw invalid_parameter("the tensor-core surrogate kernel supports at most 128 outputs");
    MmaArgs a{};
    a.O = O;
    a.out_pad = out_pad;
    a.rc = rc;
    a.master = master;
    a.scale = scale;
    a.w2 = (const uint4*)w2_bf16;
    a.w3 = (const uint4*)w3_bf16;
    a.r = r;
    a.n = n;
    a.values = values;
    a.derivs = derivs;
    a.ld = ld;
    a.status = status;
    a.features = features;
    const size_t smem = mma_shared_bytes(out_pad);
    // every CTA holds 256 of the SM's 512 tensor-memory columns for its whole
    // life: at most two CTAs may be resident on one SM, or a third would wait
    // in tcgen05.alloc for memory that is never freed (the shared-memory
    // request keeps a third off any SM)
    const size_t smem_request = std::max<size_t>(smem, 228 * 1024 / 3 + 1024);
    if (smem_request > 227 * 1024) throw invalid_parameter("the tensor-core surrogate kernel supports at most 128 outputs");
    CUDA_CHECK(cudaFuncSetAttribute(surrogate_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_request));
    // the largest shared-memory carveout
    CUDA_CHECK(cudaFuncSetAttribute(surrogate_mma_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
    int device = 0, sms = 0;
    CUDA_CHECK(cudaGetDevice(&device));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    // resident CTAs per SM from the shared-memory request (228 KB per SM,
    // 1 KB reserved per CTA): one with three-part operands at 112 outputs
    const int per_sm = std::max(1, std::min(2, (int)(228 * 1024 / (smem_request + 1024))));
    const int64_t tiles = (n + TILE - 1) / TILE;
    const int blocks = (int)std::min<int64_t>(tiles, (int64_t)sms * per_sm);
    surrogate_mma_kernel<<<blocks, TILE, smem_request, stream>>>(a);
    CUDA_CHECK(cudaGetLastError());
}

}  // namespace fb200

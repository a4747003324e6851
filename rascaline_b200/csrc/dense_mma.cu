// The two per-centre contractions of the FP32 dense power spectrum on the
// sm_100a tensor cores (tcgen05, TF32 operands split into hi + lo, FP32
// accumulation in tensor memory):
//
//   forward   P_l = X_l^T X_l,  X_l[m][(s, n)] = c[s][l m][n]
//             P_ab[l][n1][n2] = scale(l, a != b) P_l[(a, n1), (b, n2)]
//             (featomic's power_spectrum.rs:529-780)
//   adjoint   dL/dc_l[(a, n)][m] = sum_(b, q) G'_l[(a, n), (b, q)] X_l[m][(b, q)]
//             with G'_l the dL/dP block of the species pair (min, max) read
//             as is (a < b), transposed (a > b) or symmetrised (a == b),
//             times scale(l, a != b)
//
// A tile is G = 128 / SNP centres, SNP = S nmax rounded up to 32, 64 or 128:
// MMA row r = g SNP + s nmax + n.
//   forward  A = B = [X_l of the tile's centres]^T (rows r, K = m rounded up
//            to 8): D = A B^T is 128 x 128 and the diagonal SNP x SNP blocks
//            are the centres' P_l (the other blocks are not read).
//   adjoint  A = [G'_l of each centre] (rows r, K = (b, q) rounded up to 8),
//            B = [X_l of each centre, m padded to MP] (N = G MP rows):
//            D[(g, a, n), (g', m)] is dL/dc when g' = g.
// Every product is hi_a hi_b + hi_a lo_b + lo_a hi_b (three MMAs): the
// dropped lo lo term is below 2^-22 of the product, so the results are
// within a few FP32 ulps of the CUDA-core contractions.
//
// CTAs are persistent (grid = SMs x resident CTAs); every round of a tile
// builds the operands of `lpr` angular channels in shared memory (coalesced
// loads, 16-byte shared stores of four K elements), one thread issues the
// MMAs and commits them to an mbarrier (bounded wait, error flag instead of a
// hang), and the epilogue reads the accumulators with tcgen05.ld and writes
// the outputs.
#include "dense.hpp"
#include "tcgen05.cuh"

namespace fb200 {

namespace {

constexpr int ROWS = 128;
constexpr int THREADS = 256;

__device__ __forceinline__ int kpad_l(int l) { return (2 * l + 1 + 7) & ~7; }

// power spectrum normalisation 1 / ((-1)^l sqrt(2l + 1)), times sqrt(2) for
// two different neighbour species, evaluated in FP64 and rounded like the
// CUDA-core kernels do: [l] same species, [16 + l] mixed
__device__ __forceinline__ void fill_scales(float* table) {
    for (int i = threadIdx.x; i < 32; i += blockDim.x) {
        const int l = i & 15;
        const double s = sqrt((double)(2 * l + 1));
        table[i] = (float)(((i >= 16) ? 1.4142135623730951 : 1.0) * (1.0 / ((l % 2 == 0) ? s : -s)));
    }
}

__device__ __forceinline__ int key_of(int a, int b, int S) { return a * S - a * (a - 1) / 2 + (b - a); }

// store the hi and lo parts of four consecutive K elements (one 16-byte row
// of a core matrix)
__device__ __forceinline__ void store_quad(unsigned char* hi, unsigned char* lo, uint32_t offset, const float (&v)[4]) {
    float h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; e++) tc::split_tf32(v[e], h[e], l[e]);
    *reinterpret_cast<float4*>(hi + offset) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(lo + offset) = make_float4(l[0], l[1], l[2], l[3]);
}

struct MmaShape {
    int SN, SNP, G;   // rows per centre, padded; centres per tile
    int lpr;          // angular channels per round
    int tmem_cols;    // allocated tensor-memory columns
    int region;       // bytes of one operand part (hi or lo) of a round
    int MP, KP;       // adjoint: m padding per centre, K = (b, q) padding
};

// Shared prologue: aligned operand area, mbarrier, tensor memory
struct Ctx {
    unsigned char* hi;
    unsigned char* lo;
    uint32_t bar;
    uint32_t tmem;
};

__device__ __forceinline__ Ctx setup(unsigned char* smem_raw, const MmaShape& sh, uint64_t* bar, uint32_t* slot) {
    unsigned char* base = smem_raw + ((1024 - (tc::smem_addr(smem_raw) & 1023)) & 1023);
    Ctx c;
    c.hi = base;
    c.lo = base + sh.region;
    c.bar = tc::smem_addr(bar);
    if (threadIdx.x == 0) tc::mbar_init(c.bar, 1);
    if (threadIdx.x < 32) tc::tmem_alloc(slot, (uint32_t)sh.tmem_cols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    c.tmem = *slot;
    return c;
}

__device__ __forceinline__ void teardown(const Ctx& c, const MmaShape& sh, bool aborted, uint32_t phase) {
    // let MMAs still in flight finish (bounded) before freeing tensor memory
    if (aborted) tc::mbar_wait(c.bar, phase);
    tc::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after();
        tc::tmem_dealloc(c.tmem, (uint32_t)sh.tmem_cols);
    }
}

// wait for the round's MMAs; false (and the error flag set) when the wait
// gives up
__device__ __forceinline__ bool round_wait(const Ctx& c, uint32_t& phase, int32_t* status, int* abort_flag) {
    if (tc::mbar_wait(c.bar, phase)) {
        phase ^= 1;
    } else {
        atomicOr(status, 1);
        *abort_flag = 1;
    }
    __syncthreads();
    if (*abort_flag) return false;
    tc::fence_after();
    return true;
}

__global__ void __launch_bounds__(THREADS) dense_contraction_mma(DenseArgs<float> a, MmaShape sh) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ float scales[32];
    if (threadIdx.x == 0) abort_flag = 0;
    fill_scales(scales);
    const Ctx ctx = setup(smem_raw, sh, &bar, &tmem_slot);
    const int S = a.n_species, N = a.nmax, K = a.K, NN = N * N, lmax = a.lmax;
    const int SN = sh.SN, SNP = sh.SNP, G = sh.G;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = warp & 3, half = warp >> 2;
    const int64_t tiles = (a.n_atoms + G - 1) / G;
    uint32_t phase = 0;
    bool aborted = false;
    // the operand row this thread builds: r = g SNP + s nmax + n
    const int row = threadIdx.x & (ROWS - 1), kh = threadIdx.x >> 7;
    const int row_g = row / SNP, row_rr = row - row_g * SNP;
    const int row_s = row_rr / N, row_n = row_rr - row_s * N;
    for (int64_t tile = blockIdx.x; tile < tiles && !aborted; tile += gridDim.x) {
        const int64_t c0 = tile * G;
        const int ng = (int)min((int64_t)G, a.n_atoms - c0);
        const bool row_ok = row_g < ng && row_rr < SN;
        const float* row_src = a.coef + ((c0 + (row_ok ? row_g : 0)) * S + row_s) * (int64_t)K + row_n;
        for (int l0 = 0; l0 <= lmax; l0 += sh.lpr) {
            const int l1 = min(lmax, l0 + sh.lpr - 1);
            // operands: for each channel of the round, rows r, K = m padded
            // to 8; thread = (row, half of the K quads)
            int off = 0;
            for (int l = l0; l <= l1; l++) {
                const int kp = kpad_l(l), M = 2 * l + 1;
                const float* src = row_src + (int64_t)l * l * N;
                for (int k4 = kh; k4 < kp / 4; k4 += 2) {
                    float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    if (row_ok) {
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const int m = 4 * k4 + e;
                            if (m < M) v[e] = __ldg(src + m * N);
                        }
                    }
                    store_quad(ctx.hi, ctx.lo, off + tc::core_offset(row, 4 * k4, kp * 4, 4), v);
                }
                off += ROWS * kp * 4;
            }
            tc::fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tc::fence_after();
                const uint32_t idesc = tc::instr_desc(tc::FORMAT_TF32, ROWS, ROWS);
                const uint32_t hi = tc::smem_addr(ctx.hi), lo = tc::smem_addr(ctx.lo);
                int o = 0;
                for (int l = l0; l <= l1; l++) {
                    const int kp = kpad_l(l);
                    const uint32_t sbo = (uint32_t)(kp / 4) * 128;
                    const uint32_t d = ctx.tmem + (uint32_t)((l - l0) * ROWS);
                    for (int ks = 0; ks < kp / 8; ks++) {
                        const uint64_t ah = tc::operand_desc(hi + o + 256 * ks, 128, sbo);
                        const uint64_t al = tc::operand_desc(lo + o + 256 * ks, 128, sbo);
                        tc::mma_tf32(d, ah, ah, idesc, ks > 0);
                        tc::mma_tf32(d, ah, al, idesc, 1);
                        tc::mma_tf32(d, al, ah, idesc, 1);
                    }
                    o += ROWS * kp * 4;
                }
                tc::mma_commit(ctx.bar);
            }
            if (!round_wait(ctx, phase, a.status, &abort_flag)) {
                aborted = true;
                break;
            }
            // epilogue: warp (q, half) reads rows 32 q .. 32 q + 31 of its
            // centre's diagonal block, 16 columns at a time
            const int r = 32 * q + lane;
            const int g = (32 * q) / SNP;
            const int rr = r - g * SNP;
            const int s = rr / N, n1 = rr - s * N;
            const bool out_ok = g < ng && rr < SN;
            const int chunks = (SN + 15) / 16;
            const int items = (l1 - l0 + 1) * chunks;
            for (int item = half; item < items; item += 2) {
                const int j = item / chunks, ch = item - j * chunks;
                const int l = l0 + j;
                float v[16];
                tc::tmem_load16(ctx.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(j * ROWS + g * SNP + 16 * ch), v);
                if (!out_ok) continue;
                float* out = a.values + (c0 + g) * (int64_t)a.n_keys * a.n_props + (int64_t)l * NN + n1 * N;
                if ((N & 3) == 0) {
#pragma unroll
                    for (int t = 0; t < 16; t += 4) {
                        const int col = 16 * ch + t;
                        const int sb = col / N, n2 = col - sb * N;
                        if (col < SN && sb >= s) {
                            const float sc = scales[(sb != s ? 16 : 0) + l];
                            float* dst = out + (int64_t)key_of(s, sb, S) * a.n_props + n2;
                            *reinterpret_cast<float4*>(dst) =
                                make_float4(v[t] * sc, v[t + 1] * sc, v[t + 2] * sc, v[t + 3] * sc);
                        }
                    }
                } else {
#pragma unroll
                    for (int t = 0; t < 16; t++) {
                        const int col = 16 * ch + t;
                        const int sb = col / N, n2 = col - sb * N;
                        if (col < SN && sb >= s)
                            out[(int64_t)key_of(s, sb, S) * a.n_props + n2] = v[t] * scales[(sb != s ? 16 : 0) + l];
                    }
                }
            }
            tc::fence_before();
            __syncthreads();
        }
    }
    teardown(ctx, sh, aborted, phase);
}

__global__ void __launch_bounds__(THREADS) dense_grad_coef_mma(DenseArgs<float> a, MmaShape sh) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ float scales[32];
    if (threadIdx.x == 0) abort_flag = 0;
    fill_scales(scales);
    const Ctx ctx = setup(smem_raw, sh, &bar, &tmem_slot);
    const int S = a.n_species, N = a.nmax, K = a.K, NN = N * N, lmax = a.lmax;
    const int SN = sh.SN, SNP = sh.SNP, G = sh.G, MP = sh.MP, KP = sh.KP, NB = G * MP;
    const int64_t KPROPS = (int64_t)a.n_keys * a.n_props;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = warp & 3, half = warp >> 2;
    const int64_t tiles = (a.n_atoms + G - 1) / G;
    // operand bytes of one channel: A [128 x KP], then B [NB x KP]
    const int a_bytes = ROWS * KP * 4, b_bytes = NB * KP * 4;
    uint32_t phase = 0;
    bool aborted = false;
    // species and radial index of every K position (b, q) of A and B
    __shared__ int kk_species[ROWS], kk_radial[ROWS];
    for (int kk = threadIdx.x; kk < KP; kk += THREADS) {
        kk_species[kk] = kk < SN ? kk / N : 0;
        kk_radial[kk] = kk < SN ? kk - (kk / N) * N : 0;
    }
    __syncthreads();
    // 16-byte loads of quads: one species per quad and aligned rows
    const bool vec = (N & 3) == 0 && (K & 3) == 0 && (a.n_props & 3) == 0 && (uintptr_t)a.coef % 16 == 0 &&
                     (uintptr_t)a.grad_values % 16 == 0;
    // the A row this thread builds: (g, a, n)
    const int row = threadIdx.x & (ROWS - 1), kh = threadIdx.x >> 7;
    const int row_g = row / SNP, row_rr = row - row_g * SNP;
    const int sa = row_rr / N, n = row_rr - sa * N;
    // the B row this thread builds: (g, m)
    const int b_row = threadIdx.x % NB, b_k0 = threadIdx.x / NB, b_step = THREADS / NB;
    const int b_g = b_row / MP, b_m = b_row - b_g * MP;
    const int kq = KP / 4;
    for (int64_t tile = blockIdx.x; tile < tiles && !aborted; tile += gridDim.x) {
        const int64_t c0 = tile * G;
        const int ng = (int)min((int64_t)G, a.n_atoms - c0);
        const bool row_ok = row_g < ng && row_rr < SN;
        const int64_t row_c = c0 + (row_ok ? row_g : 0);
        const float* Gc = a.grad_values + (a.grad_species ? (int64_t)a.grad_species[row_c] : row_c) * KPROPS;
        for (int l0 = 0; l0 <= lmax; l0 += sh.lpr) {
            const int l1 = min(lmax, l0 + sh.lpr - 1);
            const int nl = l1 - l0 + 1;
            // A: G'_l rows (g, a, n), K = (b, q) in quads; thread = (row,
            // half of the quads)
            for (int j = 0; j < nl; j++) {
                const int l = l0 + j;
                const float* gl = Gc + l * NN;
                const float sc_same = scales[l], sc_mixed = scales[16 + l];
                for (int k4 = kh; k4 < kq; k4 += 2) {
                    float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    if (row_ok && 4 * k4 < SN) {
                        if (vec) {
                            // the quad is (b, q0 .. q0 + 3) of one species b
                            const int sb = kk_species[4 * k4], q0 = kk_radial[4 * k4];
                            if (sa < sb) {
                                const float4 x = __ldg(reinterpret_cast<const float4*>(
                                    gl + key_of(sa, sb, S) * a.n_props + n * N + q0));
                                v[0] = x.x * sc_mixed;
                                v[1] = x.y * sc_mixed;
                                v[2] = x.z * sc_mixed;
                                v[3] = x.w * sc_mixed;
                            } else if (sa > sb) {
                                const float* gk = gl + key_of(sb, sa, S) * a.n_props + q0 * N + n;
#pragma unroll
                                for (int e = 0; e < 4; e++) v[e] = __ldg(gk + e * N) * sc_mixed;
                            } else {
                                const float* gk = gl + key_of(sa, sa, S) * a.n_props;
                                const float4 x = __ldg(reinterpret_cast<const float4*>(gk + n * N + q0));
                                v[0] = (x.x + __ldg(gk + (q0 + 0) * N + n)) * sc_same;
                                v[1] = (x.y + __ldg(gk + (q0 + 1) * N + n)) * sc_same;
                                v[2] = (x.z + __ldg(gk + (q0 + 2) * N + n)) * sc_same;
                                v[3] = (x.w + __ldg(gk + (q0 + 3) * N + n)) * sc_same;
                            }
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; e++) {
                                const int kk = 4 * k4 + e;
                                if (kk < SN) {
                                    const int sb = kk_species[kk], qn = kk_radial[kk];
                                    float x;
                                    if (sa < sb) {
                                        x = __ldg(gl + key_of(sa, sb, S) * a.n_props + n * N + qn);
                                    } else if (sa > sb) {
                                        x = __ldg(gl + key_of(sb, sa, S) * a.n_props + qn * N + n);
                                    } else {
                                        const float* gk = gl + key_of(sa, sa, S) * a.n_props;
                                        x = __ldg(gk + n * N + qn) + __ldg(gk + qn * N + n);
                                    }
                                    v[e] = x * (sa != sb ? sc_mixed : sc_same);
                                }
                            }
                        }
                    }
                    store_quad(ctx.hi, ctx.lo, j * (a_bytes + b_bytes) + tc::core_offset(row, 4 * k4, KP * 4, 4), v);
                }
            }
            // B: X_l rows (g, m) with m < MP, K = (b, q); thread = (B row,
            // every b_step-th quad)
            for (int j = 0; j < nl; j++) {
                const int l = l0 + j;
                const bool b_ok = b_g < ng && b_m < 2 * l + 1;
                const float* src = a.coef + (c0 + (b_ok ? b_g : 0)) * S * (int64_t)K + (int64_t)(l * l + b_m) * N;
                for (int k4 = b_k0; k4 < kq; k4 += b_step) {
                    float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    if (b_ok && 4 * k4 < SN) {
                        if (vec) {
                            const float4 x = __ldg(reinterpret_cast<const float4*>(
                                src + (int64_t)kk_species[4 * k4] * K + kk_radial[4 * k4]));
                            v[0] = x.x;
                            v[1] = x.y;
                            v[2] = x.z;
                            v[3] = x.w;
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; e++) {
                                const int kk = 4 * k4 + e;
                                if (kk < SN) v[e] = __ldg(src + (int64_t)kk_species[kk] * K + kk_radial[kk]);
                            }
                        }
                    }
                    store_quad(ctx.hi, ctx.lo, j * (a_bytes + b_bytes) + a_bytes + tc::core_offset(b_row, 4 * k4, KP * 4, 4),
                               v);
                }
            }
            tc::fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tc::fence_after();
                const uint32_t idesc = tc::instr_desc(tc::FORMAT_TF32, ROWS, NB);
                const uint32_t hi = tc::smem_addr(ctx.hi), lo = tc::smem_addr(ctx.lo);
                const uint32_t sbo = (uint32_t)(KP / 4) * 128;
                for (int j = 0; j < nl; j++) {
                    const uint32_t oa = (uint32_t)(j * (a_bytes + b_bytes)), ob = oa + (uint32_t)a_bytes;
                    const uint32_t d = ctx.tmem + (uint32_t)(j * NB);
                    for (int ks = 0; ks < KP / 8; ks++) {
                        const uint64_t ah = tc::operand_desc(hi + oa + 256 * ks, 128, sbo);
                        const uint64_t al = tc::operand_desc(lo + oa + 256 * ks, 128, sbo);
                        const uint64_t bh = tc::operand_desc(hi + ob + 256 * ks, 128, sbo);
                        const uint64_t bl = tc::operand_desc(lo + ob + 256 * ks, 128, sbo);
                        tc::mma_tf32(d, ah, bh, idesc, ks > 0);
                        tc::mma_tf32(d, ah, bl, idesc, 1);
                        tc::mma_tf32(d, al, bh, idesc, 1);
                    }
                }
                tc::mma_commit(ctx.bar);
            }
            if (!round_wait(ctx, phase, a.status, &abort_flag)) {
                aborted = true;
                break;
            }
            // epilogue: row (g, a, n) holds dL/dc for m = 0 .. 2l at columns
            // j NB + g MP + m
            const int r = 32 * q + lane;
            const int g = (32 * q) / SNP;
            const int rr = r - g * SNP;
            const int ea = rr / N, en = rr - ea * N;
            const bool out_ok = g < ng && rr < SN;
            const int chunks = MP / 16;
            for (int item = half; item < nl * chunks; item += 2) {
                const int j = item / chunks, ch = item - j * chunks;
                const int l = l0 + j, M = 2 * l + 1;
                float v[16];
                tc::tmem_load16(ctx.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(j * NB + g * MP + 16 * ch), v);
                if (!out_ok) continue;
                float* out = a.grad_coef + ((c0 + g) * S + ea) * (int64_t)K + (int64_t)l * l * N + en;
#pragma unroll
                for (int t = 0; t < 16; t++) {
                    const int m = 16 * ch + t;
                    if (m < M) out[(int64_t)m * N] = v[t];
                }
            }
            tc::fence_before();
            __syncthreads();
        }
    }
    teardown(ctx, sh, aborted, phase);
}

int sm_count() {
    int device = 0, sms = 0;
    CUDA_CHECK(cudaGetDevice(&device));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    return sms;
}

MmaShape base_shape(const DenseArgs<float>& a) {
    MmaShape sh{};
    sh.SN = a.n_species * a.nmax;
    sh.SNP = sh.SN <= 32 ? 32 : (sh.SN <= 64 ? 64 : 128);
    sh.G = ROWS / sh.SNP;
    return sh;
}

// Launch with at most 512 / tmem_cols CTAs per SM (a CTA waiting in
// tcgen05.alloc for columns that a co-resident CTA holds until it exits would
// only serialise), through a shared-memory request that keeps more off.
template <typename Kernel>
void launch_persistent(Kernel kernel, const DenseArgs<float>& a, const MmaShape& sh, size_t smem, int64_t tiles,
                       cudaStream_t stream) {
    const int max_ctas = std::min(4, 512 / sh.tmem_cols);
    const size_t request = std::max<size_t>(smem + 1024, 228 * 1024 / (max_ctas + 1) + 1024);
    CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)request));
    CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
    // resident CTAs per SM from the shared-memory request (228 KB per SM,
    // 1 KB reserved per CTA) and the tensor-memory budget; the occupancy
    // query may answer before the carveout preference applies
    const int per_sm = std::max(1, std::min<int>(max_ctas, (int)(228 * 1024 / (request + 1024))));
    const int blocks = (int)std::min<int64_t>(tiles, (int64_t)sm_count() * per_sm);
    kernel<<<blocks, THREADS, request, stream>>>(a, sh);
    CUDA_CHECK(cudaGetLastError());
}

int tmem_columns(int used) {
    int cols = 32;
    while (cols < used) cols *= 2;
    return cols;
}

}  // namespace

int dense_mma_channels_per_round = 1;

bool dense_mma_supported(const DenseArgs<float>& a) {
    // the epilogue's 16-byte stores need 16-byte aligned rows
    return a.n_atoms > 0 && a.n_species * a.nmax <= ROWS && 2 * a.lmax + 1 <= 32 && a.lmax < 16 &&
           (uintptr_t)a.values % 16 == 0;
}

void launch_dense_contraction_mma(const DenseArgs<float>& a, cudaStream_t stream) {
    MmaShape sh = base_shape(a);
    sh.lpr = std::max(1, std::min(dense_mma_channels_per_round, 4));
    // the largest round: sum of K paddings of lpr consecutive channels
    auto round_k = [&](int lpr) {
        int kmax = 0;
        for (int l0 = 0; l0 <= a.lmax; l0 += lpr) {
            int k = 0;
            for (int l = l0; l <= std::min(a.lmax, l0 + lpr - 1); l++) k += (2 * l + 1 + 7) & ~7;
            kmax = std::max(kmax, k);
        }
        return kmax;
    };
    // at most 200 KB of operands per round
    while (sh.lpr > 1 && 2 * ROWS * round_k(sh.lpr) * 4 > 200 * 1024) sh.lpr--;
    sh.tmem_cols = tmem_columns(sh.lpr * ROWS);
    const int kmax = round_k(sh.lpr);
    sh.region = ROWS * kmax * 4;
    const int64_t tiles = (a.n_atoms + sh.G - 1) / sh.G;
    launch_persistent(dense_contraction_mma, a, sh, 2 * (size_t)sh.region, tiles, stream);
}

void launch_dense_grad_coef_mma(const DenseArgs<float>& a, cudaStream_t stream) {
    MmaShape sh = base_shape(a);
    sh.MP = 2 * a.lmax + 1 <= 16 ? 16 : 32;
    sh.KP = (sh.SN + 7) & ~7;
    const int nb = sh.G * sh.MP;
    sh.lpr = std::max(1, std::min(dense_mma_channels_per_round, 4));
    // at most 512 tensor-memory columns and 200 KB of operands per round
    while (sh.lpr > 1 && (sh.lpr * nb > 512 || 2 * sh.lpr * (ROWS + nb) * sh.KP * 4 > 200 * 1024)) sh.lpr--;
    sh.tmem_cols = tmem_columns(sh.lpr * nb);
    sh.region = sh.lpr * (ROWS + nb) * sh.KP * 4;
    const int64_t tiles = (a.n_atoms + sh.G - 1) / sh.G;
    launch_persistent(dense_grad_coef_mma, a, sh, 2 * (size_t)sh.region, tiles, stream);
}

}  // namespace fb200

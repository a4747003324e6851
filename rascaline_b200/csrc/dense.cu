// Dense power spectrum (FP64 or FP32) and its adjoint backward pass.
//
// Forward, per call:
//   directions   every half pair gives two directions (pair << 1 | reversed);
//                a stable radix sort on (centre, species of the other atom)
//                keeps pair order inside each segment, the order of
//                featomic's accumulate_all_pairs (spherical_expansion.rs:
//                101-358); segment starts by binary search
//   features     thread per pair: cutoff, Y_lm, R_nl in T
//   expansion    CTA per (centre, species), thread per (l, m, n), segment reduced in
//                registers (no atomics), inverse pairs with (-1)^l
//                (spherical_expansion_pair.rs:130-163), self term on l = 0
//   contraction  CTA per centre, coefficients in shared memory, thread per
//                (species pair a <= b, l, n1) with a register row over n2:
//                P[l n1 n2] = sum_m c_a[l m n1] c_b[l m n2] / ((-1)^l sqrt(2l+1)),
//                times sqrt(2) when a != b (power_spectrum.rs:529-780)
//
// Backward (adjoint of the above for a loss L with dL/dP given):
//   dL/dc        CTA per centre, coefficients and dL/dP in shared memory,
//                thread per (a, l, n) with a register row over m:
//                dL/dc_a[l m n] = sum over the species pairs containing a of
//                scale * sum_n' G[n n'] c_b[l m n']
//   dL/dr_ij     thread per pair, Y_lm, dY_lm, R_nl, dR_nl recomputed in
//                registers and contracted at once:
//                D = dL/dc_i[s_j] + (-1)^l dL/dc_j[s_i],
//                dL/dr_ij = sum_lm Y A u + f/r dY B, A = sum_n D (f' R + f R'),
//                B = sum_n D R  (the pair gradient of spherical_expansion_pair.rs:323-422)
//   (lmax > 8 or nmax > 16: warp-per-item kernels over stored pair records)
//   atoms        thread per atom: dL/dr_a = sum over its directions of
//                -+dL/dr_ij (self images cancel and are skipped), plus the
//                strain (r_ij x dL/dr_ij) and cell (shift x dL/dr_ij) sums of
//                its own pairs
//   systems      CTA per system: strain and cell derivatives summed over atoms
// Every reduction has a fixed order: results are deterministic.
#include <cub/cub.cuh>
#include <cstdlib>
#include <type_traits>

#include "dense.hpp"
#include "pair_math.cuh"

namespace fb200 {

namespace {

constexpr int DENSE_LMAX_SMALL = 8;
constexpr int DENSE_LMAX_LARGE = 24;
constexpr int DENSE_CHUNK = 32;

__device__ __forceinline__ int isqrt_lm(int lm) {
    int l = (int)sqrtf((float)lm);
    while (l * l > lm) l--;
    while ((l + 1) * (l + 1) <= lm) l++;
    return l;
}

// power spectrum normalisation 1 / ((-1)^l sqrt(2l + 1)), times sqrt(2) for
// two different neighbour species
__device__ __forceinline__ double ps_scale(int l, bool mixed) {
    const double s = sqrt((double)(2 * l + 1));
    const double norm = (l % 2 == 0) ? s : -s;
    return (mixed ? 1.4142135623730951 : 1.0) * (1.0 / norm);
}

__device__ __forceinline__ void key_species(int key, int S, int* a, int* b) {
    int x = 0;
    while (key >= S - x) {
        key -= S - x;
        x++;
    }
    *a = x;
    *b = x + key;
}

__device__ __forceinline__ int key_index(int a, int b, int S) { return a * S - a * (a - 1) / 2 + (b - a); }

__global__ void dense_direction_keys(const int32_t* __restrict__ first, const int32_t* __restrict__ second,
                                     const int32_t* __restrict__ species, int64_t n_pairs, int S,
                                     int32_t* __restrict__ keys, int32_t* __restrict__ codes) {
    const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= 2 * n_pairs) return;
    const int64_t p = d >> 1;
    const bool reversed = d & 1;
    const int32_t centre = reversed ? second[p] : first[p];
    const int32_t other = reversed ? first[p] : second[p];
    keys[d] = centre * S + species[other];
    codes[d] = (int32_t)d;
}

__global__ void dense_segments(const int32_t* __restrict__ sorted, int64_t n_dirs, int64_t n_segments,
                               int64_t* __restrict__ seg_offset) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > n_segments) return;
    int64_t lo = 0, hi = n_dirs;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)sorted[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    seg_offset[k] = lo;
}

// The record of pair p (cutoff, direction, Y_lm [, dY_lm], R_nl [, dR_nl]) into f
template <typename T, int LCAP, bool GRAD>
__device__ __forceinline__ void pair_record(const DevicePairs& pairs, int64_t p, const DeviceRadial& exact,
                                            const DenseTables<T>& tab, const CutoffParams& cut, const FeatureLayout& L,
                                            T* __restrict__ f, int32_t* __restrict__ status, int radial_external) {
    const double r = pairs.distance[p];
    const double v0 = pairs.vector[3 * p], v1 = pairs.vector[3 * p + 1], v2 = pairs.vector[3 * p + 2];
    double u0 = v0 / r, u1 = v1 / r, u2 = v2 / r;
    if (r < 1e-6) {
        u0 = 0.0;
        u1 = 0.0;
        u2 = 1.0;
    }
    double fc, dfc;
    soap::cutoff_function(cut.smoothing, cut.rc, cut.width, r, &fc, &dfc);
    double sc = 1.0, dsc = 0.0;
    if (cut.scaling) soap::willatt2018(cut.scale, cut.rate, cut.exponent, r, &sc, &dsc);
    f[0] = (T)(sc * fc);
    f[1] = (T)(dfc * sc + fc * dsc);
    f[2] = (T)r;
    f[3] = (T)u0;
    f[4] = (T)u1;
    f[5] = (T)u2;
    if constexpr (LCAP <= 8) {
        // row by row in registers, stored straight into the pair record
        T* __restrict__ Y = f + L.off_y;
        T* __restrict__ G = f + L.off_dy;
        const int L2 = L.L2;
        ylm_rows<T, LCAP, GRAD>(tab.ylm, (T)u0, (T)u1, (T)u2, [](int) {},
                                [&](int l, int m, T yp, T ym, const T* gp, const T* gm) {
                                    const int ip = l * l + l + m, im = l * l + l - m;
                                    Y[ip] = yp;
                                    if (m > 0) Y[im] = ym;
                                    if (GRAD) {
#pragma unroll
                                        for (int x = 0; x < 3; x++) {
                                            G[x * L2 + ip] = gp[x];
                                            if (m > 0) G[x * L2 + im] = gm[x];
                                        }
                                    }
                                });
    } else if (GRAD) {
        ylm_compute<T, LCAP>(tab.ylm, (T)u0, (T)u1, (T)u2, f + L.off_y, f + L.off_dy, f + L.off_dy + L.L2,
                             f + L.off_dy + 2 * L.L2);
    } else {
        ylm_compute<T, LCAP>(tab.ylm, (T)u0, (T)u1, (T)u2, f + L.off_y, nullptr, nullptr, nullptr);
    }
    if (radial_external) return;
    bool ok = true;
    for (int l = 0; l <= L.lmax; l++)
        ok &= radial_eval<T>(exact, tab.spline, l, r, f + L.off_r + l * L.nmax, GRAD ? f + L.off_dr + l * L.nmax : nullptr);
    if (!ok) atomicExch(status, 1);
}

// Thread per pair.  STAGED: the records of the CTA are built in shared
// memory (row pitch stride + 1) and written out as one contiguous block, so
// that the stores are coalesced instead of one scattered element per lane
// (the records of consecutive pairs are adjacent in HBM).
template <typename T, int LCAP, bool GRAD, bool STAGED>
__global__ void dense_pair_features(DevicePairs pairs, DeviceRadial exact, DenseTables<T> tab, CutoffParams cut,
                                    FeatureLayout L, T* __restrict__ features, int32_t* __restrict__ status,
                                    int radial_external) {
    extern __shared__ __align__(16) unsigned char feature_smem[];
    const int64_t p0 = (int64_t)blockIdx.x * blockDim.x;
    const int64_t p = p0 + threadIdx.x;
    const int pitch = L.stride + 1;
    T* f = STAGED ? reinterpret_cast<T*>(feature_smem) + threadIdx.x * pitch : features + p * L.stride;
    if (p < pairs.count) pair_record<T, LCAP, GRAD>(pairs, p, exact, tab, cut, L, f, status, radial_external);
    if (!STAGED) return;
    __syncthreads();
    const int count = (int)min((int64_t)blockDim.x, pairs.count - p0);
    const int total = count * L.stride;
    const T* src = reinterpret_cast<const T*>(feature_smem);
    T* dst = features + p0 * L.stride;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int rec = i / L.stride;
        dst[i] = src[rec * pitch + (i - rec * L.stride)];
    }
}

// Thread per (l, m) and pair of radial functions (n0 = 2j, n1 = 2j + 1): the
// direction scalars and Y_lm are loaded once for both, which halves the loads
// of this load-issue-bound kernel; each coefficient is still summed over the
// directions in pair order.
template <typename T>
__global__ void __launch_bounds__(256) dense_expansion(DenseArgs<T> a) {
    __shared__ int64_t dir_feature[DENSE_CHUNK];
    __shared__ T dir_f[DENSE_CHUNK];
    __shared__ int dir_inv[DENSE_CHUNK];
    const FeatureLayout L = a.layout;
    // one CTA per (centre, neighbour species) segment
    const int S = a.n_species;
    const int64_t c = blockIdx.x / S;
    const int t = (int)(blockIdx.x - c * S);
    const int K = a.K, N = L.nmax, NH = (N + 1) / 2;
    const int items = L.L2 * NH;
    const int tc = a.atom_species[c];
    const int64_t d0 = a.seg_offset[c * S + t], d1 = a.seg_offset[c * S + t + 1];
    for (int k0 = 0; k0 < items; k0 += blockDim.x) {
        const int k = k0 + threadIdx.x;
        const bool active = k < items;
        const int lm = active ? k / NH : 0;
        const int n0 = active ? 2 * (k - lm * NH) : 0;
        const bool has1 = n0 + 1 < N;
        const int l = isqrt_lm(lm);
        const T sign_l = (l & 1) ? T(-1) : T(1);
        const int ri = l * N + n0;
        T acc0 = T(0), acc1 = T(0);
        for (int64_t dc = d0; dc < d1; dc += DENSE_CHUNK) {
            const int nd = (int)min((int64_t)DENSE_CHUNK, d1 - dc);
            __syncthreads();
            if (threadIdx.x < nd) {
                const int32_t code = a.dir_code[dc + threadIdx.x];
                const int64_t p = code >> 1;
                dir_feature[threadIdx.x] = p * L.stride;
                dir_inv[threadIdx.x] = code & 1;
                dir_f[threadIdx.x] = a.features[p * L.stride];
            }
            __syncthreads();
            if (!active) continue;
            for (int q = 0; q < nd; q++) {
                const T* __restrict__ F = a.features + dir_feature[q];
                const T fy = dir_f[q] * F[L.off_y + lm];
                const T v0 = fy * F[L.off_r + ri];
                const T v1 = has1 ? fy * F[L.off_r + ri + 1] : T(0);
                const bool inv = dir_inv[q];
                acc0 += inv ? sign_l * v0 : v0;
                acc1 += inv ? sign_l * v1 : v1;
            }
        }
        if (!active) continue;
        const bool self = t == tc && l == 0;
        T* out = a.coef + (c * S + t) * K + lm * N + n0;
        out[0] = (self ? a.tab.self_contribution[n0] : T(0)) + acc0;
        if (has1) out[1] = (self ? a.tab.self_contribution[n0 + 1] : T(0)) + acc1;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) dense_contraction(DenseArgs<T> a) {
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * warps + warp;
    if (item >= a.n_atoms * a.n_keys) return;
    const int64_t c = item / a.n_keys;
    const int key = (int)(item - c * a.n_keys);
    int sa, sb;
    key_species(key, a.n_species, &sa, &sb);
    const int N = a.nmax, NN = N * N;
    const T* ca = a.coef + (c * a.n_species + sa) * a.K;
    const T* cb = a.coef + (c * a.n_species + sb) * a.K;
    T* out = a.values + item * a.n_props;
    for (int o = lane; o < a.n_props; o += 32) {
        const int l = o / NN;
        const int rem = o - l * NN;
        const int n1 = rem / N, n2 = rem - n1 * N;
        const int base = l * l * N;
        T s = T(0);
        for (int m = 0; m < 2 * l + 1; m++) s += ca[base + m * N + n1] * cb[base + m * N + n2];
        out[o] = s * (T)ps_scale(l, sa != sb);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) dense_grad_coef(DenseArgs<T> a) {
    extern __shared__ __align__(16) unsigned char dense_smem[];
    T* cs = reinterpret_cast<T*>(dense_smem);
    const int64_t c = blockIdx.x;
    const int S = a.n_species, K = a.K, N = a.nmax, NN = N * N;
    for (int i = threadIdx.x; i < S * K; i += blockDim.x) cs[i] = a.coef[c * S * K + i];
    __syncthreads();
    const T* G = a.grad_values + (a.grad_species ? (int64_t)a.grad_species[c] : c) * a.n_keys * a.n_props;
    for (int o = threadIdx.x; o < S * K; o += blockDim.x) {
        const int sa = o / K;
        const int k = o - sa * K;
        const int lm = k / N;
        const int n = k - lm * N;
        const int l = isqrt_lm(lm);
        T acc = T(0);
        for (int b = 0; b < S; b++) {
            const T* cb = cs + b * K + lm * N;
            T s = T(0);
            if (sa < b) {
                const T* g = G + (int64_t)key_index(sa, b, S) * a.n_props + l * NN + n * N;
                for (int q = 0; q < N; q++) s += g[q] * cb[q];
                acc += (T)ps_scale(l, true) * s;
            } else if (sa > b) {
                const T* g = G + (int64_t)key_index(b, sa, S) * a.n_props + l * NN + n;
                for (int q = 0; q < N; q++) s += g[q * N] * cb[q];
                acc += (T)ps_scale(l, true) * s;
            } else {
                const T* g = G + (int64_t)key_index(sa, sa, S) * a.n_props + l * NN;
                for (int q = 0; q < N; q++) s += (g[n * N + q] + g[q * N + n]) * cb[q];
                acc += (T)ps_scale(l, false) * s;
            }
        }
        a.grad_coef[c * S * K + o] = acc;
    }
}

// global -> shared copy of n elements, in 16-byte vectors when both ends and
// the length allow it
template <typename T>
__device__ __forceinline__ void stage_copy(T* __restrict__ dst, const T* __restrict__ src, int64_t n) {
    if (((uintptr_t)dst % 16) == 0 && ((uintptr_t)src % 16) == 0 && (n * (int64_t)sizeof(T)) % 16 == 0) {
        const int64_t nv = n * (int64_t)sizeof(T) / 16;
        for (int64_t i = threadIdx.x; i < nv; i += blockDim.x)
            reinterpret_cast<float4*>(dst)[i] = __ldg(reinterpret_cast<const float4*>(src) + i);
    } else {
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    }
}

// The two per-centre contractions with the centre's coefficients (and, for
// the adjoint, its dL/dP row) staged in shared memory and register tiles,
// for nmax <= NCAP and 2 lmax + 1 <= MCAP.  Same sums in the same order as
// dense_contraction / dense_grad_coef, so the results are identical; the
// tiles cut the loads per multiply-add from 2 to about 1 / NCAP
// (contraction) and 1 / (2l + 1) (adjoint).
//
// P_ab[l][n1][n2] = scale(l, a != b) sum_m c_a[l m n1] c_b[l m n2]
// (power_spectrum.rs:529-780), one thread per (key, l, n1), NCAP outputs.
template <typename T, int NCAP>
__global__ void __launch_bounds__(128) dense_contraction_tiled(DenseArgs<T> a) {
    extern __shared__ __align__(16) unsigned char dense_smem[];
    T* cs = reinterpret_cast<T*>(dense_smem);
    const int64_t c = blockIdx.x;
    const int S = a.n_species, K = a.K, N = a.nmax, NN = N * N, LN = (a.lmax + 1) * N;
    stage_copy(cs, a.coef + c * S * K, (int64_t)S * K);
    __syncthreads();
    const int items = a.n_keys * LN;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int key = it / LN;
        const int rem = it - key * LN;
        const int l = rem / N, n1 = rem - l * N;
        int sa, sb;
        key_species(key, S, &sa, &sb);
        const T* ca = cs + sa * K + l * l * N;
        const T* cb = cs + sb * K + l * l * N;
        T acc[NCAP];
#pragma unroll
        for (int q = 0; q < NCAP; q++) acc[q] = T(0);
        for (int m = 0; m < 2 * l + 1; m++) {
            const T x = ca[m * N + n1];
#pragma unroll
            for (int q = 0; q < NCAP; q++)
                if (q < N) acc[q] += x * cb[m * N + q];
        }
        const T scale = (T)ps_scale(l, sa != sb);
        T* out = a.values + (c * a.n_keys + key) * a.n_props + l * NN + n1 * N;
#pragma unroll
        for (int q = 0; q < NCAP; q++)
            if (q < N) out[q] = acc[q] * scale;
    }
}

// dL/dc_a[l m n] = sum_b scale(l, a != b) sum_q G_ab[l](n, q) c_b[l m q], with
// G_ab the dL/dP block of the key (min(a, b), max(a, b)) read as is (a < b),
// transposed (a > b) or symmetrised (a == b); one thread per (a, l, n), all m.
template <typename T, int MCAP>
__global__ void __launch_bounds__(128) dense_grad_coef_tiled(DenseArgs<T> a) {
    extern __shared__ __align__(16) unsigned char dense_smem[];
    T* cs = reinterpret_cast<T*>(dense_smem);
    const int64_t c = blockIdx.x;
    const int S = a.n_species, K = a.K, N = a.nmax, NN = N * N, LN = (a.lmax + 1) * N;
    const int64_t KP = (int64_t)a.n_keys * a.n_props;
    T* gs = cs + S * K;
    stage_copy(cs, a.coef + c * S * K, (int64_t)S * K);
    stage_copy(gs, a.grad_values + (a.grad_species ? (int64_t)a.grad_species[c] : c) * KP, KP);
    __syncthreads();
    for (int it = threadIdx.x; it < S * LN; it += blockDim.x) {
        const int sa = it / LN;
        const int rem = it - sa * LN;
        const int l = rem / N, n = rem - l * N;
        const int M = 2 * l + 1;
        T acc[MCAP];
#pragma unroll
        for (int m = 0; m < MCAP; m++) acc[m] = T(0);
        for (int b = 0; b < S; b++) {
            const T* cb = cs + b * K + l * l * N;
            T s[MCAP];
#pragma unroll
            for (int m = 0; m < MCAP; m++) s[m] = T(0);
            const T* g;
            int row, col;
            if (sa < b) {
                g = gs + (int64_t)key_index(sa, b, S) * a.n_props + l * NN;
                row = n * N;
                col = 1;
            } else {
                g = gs + (int64_t)key_index(b, sa, S) * a.n_props + l * NN;
                row = n;
                col = N;
            }
            for (int q = 0; q < N; q++) {
                const T gq = sa == b ? g[n * N + q] + g[q * N + n] : g[row + q * col];
#pragma unroll
                for (int m = 0; m < MCAP; m++)
                    if (m < M) s[m] += gq * cb[m * N + q];
            }
            const T scale = (T)ps_scale(l, sa != b);
#pragma unroll
            for (int m = 0; m < MCAP; m++) acc[m] += scale * s[m];
        }
        T* out = a.grad_coef + c * S * K + sa * K + l * l * N + n;
#pragma unroll
        for (int m = 0; m < MCAP; m++)
            if (m < M) out[m * N] = acc[m];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) dense_pair_adjoint(DenseArgs<T> a, int64_t n_pairs) {
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t p = (int64_t)blockIdx.x * warps + warp;
    if (p >= n_pairs) return;
    const FeatureLayout L = a.layout;
    const T* __restrict__ F = a.features + p * L.stride;
    const T f = F[0], fg = F[1], r = F[2];
    const T u0 = F[3], u1 = F[4], u2 = F[5];
    const T f_over_r = f / r;
    const int i = a.pairs.first[p], j = a.pairs.second[p];
    const int S = a.n_species, N = a.nmax;
    const T* Di = a.grad_coef + ((int64_t)i * S + a.atom_species[j]) * a.K;
    const T* Dj = a.grad_coef + ((int64_t)j * S + a.atom_species[i]) * a.K;
    T g0 = T(0), g1 = T(0), g2 = T(0);
    for (int lm = lane; lm < L.L2; lm += 32) {
        const int l = isqrt_lm(lm);
        const T sign = (l & 1) ? T(-1) : T(1);
        T A = T(0), B = T(0);
        for (int n = 0; n < N; n++) {
            const T D = Di[lm * N + n] + sign * Dj[lm * N + n];
            const T R = F[L.off_r + l * N + n];
            const T dR = F[L.off_dr + l * N + n];
            A += D * (fg * R + f * dR);
            B += D * R;
        }
        const T AY = A * F[L.off_y + lm];
        const T Bf = B * f_over_r;
        g0 += AY * u0 + Bf * F[L.off_dy + lm];
        g1 += AY * u1 + Bf * F[L.off_dy + L.L2 + lm];
        g2 += AY * u2 + Bf * F[L.off_dy + 2 * L.L2 + lm];
    }
    for (int off = 16; off > 0; off >>= 1) {
        g0 += __shfl_down_sync(0xffffffffu, g0, off);
        g1 += __shfl_down_sync(0xffffffffu, g1, off);
        g2 += __shfl_down_sync(0xffffffffu, g2, off);
    }
    if (lane == 0) {
        a.pair_grad[3 * p] = g0;
        a.pair_grad[3 * p + 1] = g1;
        a.pair_grad[3 * p + 2] = g2;
    }
}

// Spline R_nl(r) and dR_nl/dr of one angular channel into registers: the
// arithmetic of radial_eval (featomic/src/math/splines.rs:225-289), unrolled
// over at most NCAP radial functions.
template <typename T, int NCAP>
__device__ __forceinline__ void spline_row(const DeviceSplineT<T>& S, int l, double r, T (&R)[NCAP], T (&dR)[NCAP]) {
    const int N = S.nmax;
    const double* pos = S.positions + S.knot_offset[l];
    const int k = soap::spline_interval(pos, S.knot_count[l], r);
    const soap::HermiteWeights w = soap::hermite_weights(pos[k], pos[k + 1], r);
    const T* pv = S.values + ((size_t)S.knot_offset[l] + k) * N;
    const T* pd = S.derivs + ((size_t)S.knot_offset[l] + k) * N;
    const T h00 = (T)w.h00, h10 = (T)(w.h10 * w.delta), h01 = (T)w.h01, h11 = (T)(w.h11 * w.delta);
    const T d00 = (T)(w.d00 * w.dxdt), d10 = (T)w.d10, d01 = (T)(w.d01 * w.dxdt), d11 = (T)w.d11;
#pragma unroll
    for (int n = 0; n < NCAP; n++) {
        if (n < N) {
            const T p0 = pv[n], m0 = pd[n], p1 = pv[N + n], m1 = pd[N + n];
            R[n] = h00 * p0 + h10 * m0 + h01 * p1 + h11 * m1;
            dR[n] = d00 * p0 + d10 * m0 + d01 * p1 + d11 * m1;
        } else {
            R[n] = T(0);
            dR[n] = T(0);
        }
    }
}

// dense_pair_features<GRAD> + dense_pair_adjoint in one pass, one pair per
// thread, nothing written but dL/dr_ij: the cutoff, Y_lm and dY_lm (row by
// row in registers) and the spline R_nl, dR_nl (one channel at a time in
// registers) are contracted at once with
//   D_lmn = dL/dc_i[s_j][lmn] + (-1)^l dL/dc_j[s_i][lmn]
// (the pair term of both centres, spherical_expansion_pair.rs:130-163, 323-422):
//   dL/dr_ij = sum_lm [A_lm Y_lm u + B_lm f / r dY_lm/du],
//   A_lm = sum_n D_lmn (f' R_ln + f dR_ln),  B_lm = sum_n D_lmn R_ln.
// Pairs are ordered by first atom, so the Di rows of a warp are mostly the
// same (broadcast loads).  Used when lmax <= 8, nmax <= NCAP, the radial
// integral is splined and no learned surrogate replaces it.
template <typename T, int NCAP>
__global__ void __launch_bounds__(128) dense_pair_adjoint_fused(DenseArgs<T> a, int64_t n_pairs) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_pairs) return;
    const double r = a.pairs.distance[p];
    const double v0 = a.pairs.vector[3 * p], v1 = a.pairs.vector[3 * p + 1], v2 = a.pairs.vector[3 * p + 2];
    double ud0 = v0 / r, ud1 = v1 / r, ud2 = v2 / r;
    if (r < 1e-6) {
        ud0 = 0.0;
        ud1 = 0.0;
        ud2 = 1.0;
    }
    double fc, dfc;
    soap::cutoff_function(a.cut.smoothing, a.cut.rc, a.cut.width, r, &fc, &dfc);
    double sc = 1.0, dsc = 0.0;
    if (a.cut.scaling) soap::willatt2018(a.cut.scale, a.cut.rate, a.cut.exponent, r, &sc, &dsc);
    const T f = (T)(sc * fc), fg = (T)(dfc * sc + fc * dsc);
    const T u0 = (T)ud0, u1 = (T)ud1, u2 = (T)ud2;
    const T f_over_r = f / (T)r;
    const int i = a.pairs.first[p], j = a.pairs.second[p];
    const int S = a.n_species, N = a.nmax;
    const T* __restrict__ Di = a.grad_coef + ((int64_t)i * S + a.atom_species[j]) * a.K;
    const T* __restrict__ Dj = a.grad_coef + ((int64_t)j * S + a.atom_species[i]) * a.K;
    T R[NCAP], dR[NCAP], P[NCAP];
    T sign = T(1);
    T g0 = T(0), g1 = T(0), g2 = T(0);
    // With N == NCAP the rows are read as 16-byte vectors (K N-aligned rows
    // of 4 or 2 elements): the kernel is bound by L1 load throughput.
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    constexpr int W = 16 / sizeof(T);
    const bool vec = N == NCAP && (a.K * (int)sizeof(T)) % 16 == 0;
    auto term = [&](int lm, T y, const T* gy) {
        T A = T(0), B = T(0);
        const T* di = Di + lm * N;
        const T* dj = Dj + lm * N;
        if (vec) {
#pragma unroll
            for (int q = 0; q < NCAP / W; q++) {
                const V x4 = __ldg(reinterpret_cast<const V*>(di) + q);
                const V z4 = __ldg(reinterpret_cast<const V*>(dj) + q);
                const T* xs = reinterpret_cast<const T*>(&x4);
                const T* zs = reinterpret_cast<const T*>(&z4);
#pragma unroll
                for (int e = 0; e < W; e++) {
                    const T D = xs[e] + sign * zs[e];
                    A += D * P[q * W + e];
                    B += D * R[q * W + e];
                }
            }
        } else {
#pragma unroll
            for (int n = 0; n < NCAP; n++) {
                if (n < N) {
                    const T D = di[n] + sign * dj[n];
                    A += D * P[n];
                    B += D * R[n];
                }
            }
        }
        const T AY = A * y;
        const T Bf = B * f_over_r;
        g0 += AY * u0 + Bf * gy[0];
        g1 += AY * u1 + Bf * gy[1];
        g2 += AY * u2 + Bf * gy[2];
    };
    ylm_rows<T, 8, true>(
        a.tab.ylm, u0, u1, u2,
        [&](int l) {
            spline_row<T, NCAP>(a.tab.spline, l, r, R, dR);
#pragma unroll
            for (int n = 0; n < NCAP; n++) P[n] = fg * R[n] + f * dR[n];
            sign = (l & 1) ? T(-1) : T(1);
        },
        [&](int l, int m, T yp, T ym, const T* gp, const T* gm) {
            term(l * l + l + m, yp, gp);
            if (m > 0) term(l * l + l - m, ym, gm);
        });
    a.pair_grad[3 * p] = g0;
    a.pair_grad[3 * p + 1] = g1;
    a.pair_grad[3 * p + 2] = g2;
}

template <typename T>
__global__ void dense_atom_reduce(DenseArgs<T> a, int with_partials) {
    const int64_t atom = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (atom >= a.n_atoms) return;
    const int S = a.n_species;
    const int64_t d0 = a.seg_offset[atom * S], d1 = a.seg_offset[(atom + 1) * S];
    T g[3] = {T(0), T(0), T(0)};
    for (int64_t d = d0; d < d1; d++) {
        const int32_t code = a.dir_code[d];
        const int64_t p = code >> 1;
        if (a.pairs.first[p] == a.pairs.second[p]) continue;
        const T* pg = a.pair_grad + 3 * p;
        if (code & 1) {
            g[0] += pg[0];
            g[1] += pg[1];
            g[2] += pg[2];
        } else {
            g[0] -= pg[0];
            g[1] -= pg[1];
            g[2] -= pg[2];
        }
    }
    a.grad_positions[3 * atom] = g[0];
    a.grad_positions[3 * atom + 1] = g[1];
    a.grad_positions[3 * atom + 2] = g[2];
    if (!with_partials) return;
    T w[18];
#pragma unroll
    for (int x = 0; x < 18; x++) w[x] = T(0);
    for (int64_t p = a.pair_start[atom]; p < a.pair_start[atom + 1]; p++) {
        const T* pg = a.pair_grad + 3 * p;
#pragma unroll
        for (int x = 0; x < 3; x++) {
            const T v = (T)a.pairs.vector[3 * p + x];
            const T sh = (T)a.pairs.shift[3 * p + x];
#pragma unroll
            for (int y = 0; y < 3; y++) {
                w[x * 3 + y] += v * pg[y];
                w[9 + x * 3 + y] += sh * pg[y];
            }
        }
    }
    T* out = a.atom_partial + 18 * atom;
#pragma unroll
    for (int x = 0; x < 18; x++) out[x] = w[x];
}

template <typename T>
__global__ void __launch_bounds__(256) dense_system_reduce(DenseArgs<T> a) {
    __shared__ T red[256];
    const int64_t s = blockIdx.x;
    const int64_t a0 = a.atom_offset[s], a1 = a.atom_offset[s + 1];
    for (int x = 0; x < 18; x++) {
        T acc = T(0);
        for (int64_t atom = a0 + threadIdx.x; atom < a1; atom += blockDim.x) acc += a.atom_partial[18 * atom + x];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int width = blockDim.x / 2; width > 0; width >>= 1) {
            if ((int)threadIdx.x < width) red[threadIdx.x] += red[threadIdx.x + width];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            if (x < 9 && a.grad_strain) a.grad_strain[9 * s + x] = red[0];
            if (x >= 9 && a.grad_cell) a.grad_cell[9 * s + x - 9] = red[0];
        }
        __syncthreads();
    }
}

// Forward-mode derivative (tangent) of the expansion along a displacement of
// the positions (tangent_positions [atoms][3]) and cells (tangent_cell
// [systems][3][3], rows = cell vectors, may be null): the pair vector moves by
//   delta_ij = t[second] - t[first] + shift . T_cell[system]
// (positions held fixed when the cell moves, as in featomic's cell gradient),
// and each pair term c_ij[l m n] = f R_ln Y_lm moves by
//   (f' R_ln + f R'_ln) Y_lm (u . delta) + f / r R_ln (dY_lm . delta)
// (spherical_expansion_pair.rs:323-422).  Thread per (pair, lm), from the
// pair records with gradients; writes tangent[pair][lm][n].
template <typename T>
__global__ void dense_pair_tangent(DenseArgs<T> a, int64_t n_pairs, const T* __restrict__ tpos,
                                   const T* __restrict__ tcell, T* __restrict__ tangent) {
    const FeatureLayout L = a.layout;
    const int64_t item = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= n_pairs * L.L2) return;
    const int64_t p = item / L.L2;
    const int lm = (int)(item - p * L.L2);
    const int l = isqrt_lm(lm);
    const int N = a.nmax;
    const int i = a.pairs.first[p], j = a.pairs.second[p];
    T d[3];
#pragma unroll
    for (int x = 0; x < 3; x++) d[x] = tpos[3 * j + x] - tpos[3 * i + x];
    if (tcell) {
        // system of the pair: the last system that starts at or before atom i
        int64_t lo = 0, hi = a.n_systems - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if (a.atom_offset[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        const T* U = tcell + 9 * lo;
#pragma unroll
        for (int x = 0; x < 3; x++)
            d[x] += (T)a.pairs.shift[3 * p] * U[x] + (T)a.pairs.shift[3 * p + 1] * U[3 + x] +
                    (T)a.pairs.shift[3 * p + 2] * U[6 + x];
    }
    const T* __restrict__ F = a.features + p * L.stride;
    const T f = F[0], fg = F[1], r = F[2];
    const T ud = F[3] * d[0] + F[4] * d[1] + F[5] * d[2];
    const T yd = F[L.off_dy + lm] * d[0] + F[L.off_dy + L.L2 + lm] * d[1] + F[L.off_dy + 2 * L.L2 + lm] * d[2];
    const T y = F[L.off_y + lm];
    const T A = y * ud, B = f / r * yd;
    T* out = tangent + p * a.K + lm * N;
    for (int n = 0; n < N; n++) {
        const T R = F[L.off_r + l * N + n], dR = F[L.off_dr + l * N + n];
        out[n] = (fg * R + f * dR) * A + R * B;
    }
}

// tangent of the coefficients: sum over each (centre, species) segment of
// the pair tangents in pair order, (-1)^l for the reversed direction
template <typename T>
__global__ void __launch_bounds__(256) dense_tangent_expansion(DenseArgs<T> a, const T* __restrict__ tangent,
                                                               T* __restrict__ tcoef) {
    const int S = a.n_species, N = a.nmax;
    const int64_t c = blockIdx.x / S;
    const int t = (int)(blockIdx.x - c * S);
    const int64_t d0 = a.seg_offset[c * S + t], d1 = a.seg_offset[c * S + t + 1];
    for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
        const int l = isqrt_lm(k / N);
        const T sign = (l & 1) ? T(-1) : T(1);
        T acc = T(0);
        for (int64_t d = d0; d < d1; d++) {
            const int32_t code = a.dir_code[d];
            const T v = tangent[(int64_t)(code >> 1) * a.K + k];
            acc += (code & 1) ? sign * v : v;
        }
        tcoef[(c * S + t) * a.K + k] = acc;
    }
}

// tangent of the power spectrum: warp per (centre, key), lane per property
//   dP[l n1 n2] = scale sum_m (dc_a[l m n1] c_b[l m n2] + c_a[l m n1] dc_b[l m n2])
template <typename T>
__global__ void __launch_bounds__(256) dense_tangent_contraction(DenseArgs<T> a, const T* __restrict__ tcoef,
                                                                 T* __restrict__ tvalues) {
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * warps + warp;
    if (item >= a.n_atoms * a.n_keys) return;
    const int64_t c = item / a.n_keys;
    const int key = (int)(item - c * a.n_keys);
    int sa, sb;
    key_species(key, a.n_species, &sa, &sb);
    const int N = a.nmax, NN = N * N;
    const T* ca = a.coef + (c * a.n_species + sa) * a.K;
    const T* cb = a.coef + (c * a.n_species + sb) * a.K;
    const T* ta = tcoef + (c * a.n_species + sa) * a.K;
    const T* tb = tcoef + (c * a.n_species + sb) * a.K;
    T* out = tvalues + item * a.n_props;
    for (int o = lane; o < a.n_props; o += 32) {
        const int l = o / NN;
        const int rem = o - l * NN;
        const int n1 = rem / N, n2 = rem - n1 * N;
        const int base = l * l * N;
        T s = T(0);
        for (int m = 0; m < 2 * l + 1; m++)
            s += ta[base + m * N + n1] * cb[base + m * N + n2] + ca[base + m * N + n1] * tb[base + m * N + n2];
        out[o] = s * (T)ps_scale(l, sa != sb);
    }
}

template <typename T, bool GRAD>
void launch_features(const DenseArgs<T>& a, int64_t n_pairs, cudaStream_t stream) {
    if (n_pairs == 0) return;
    DevicePairs pairs = a.pairs;
    pairs.count = n_pairs;
    const int external = a.surrogate != nullptr ? 1 : 0;
    // staged records: as many threads (multiple of 32, at most 128) as fit in
    // 48 KB of shared memory
    const size_t record = sizeof(T) * (size_t)(a.layout.stride + 1);
    const int staged_threads = (int)std::min<size_t>(128, (48 * 1024 / record) / 32 * 32);
    if (a.lmax <= DENSE_LMAX_SMALL && !external && staged_threads >= 32) {
        const unsigned blocks = (unsigned)((n_pairs + staged_threads - 1) / staged_threads);
        dense_pair_features<T, DENSE_LMAX_SMALL, GRAD, true><<<blocks, staged_threads, record * staged_threads, stream>>>(
            pairs, a.exact, a.tab, a.cut, a.layout, a.features, a.status, external);
    } else {
        const int threads = 64;
        const unsigned blocks = (unsigned)((n_pairs + threads - 1) / threads);
        if (a.lmax <= DENSE_LMAX_SMALL) {
            dense_pair_features<T, DENSE_LMAX_SMALL, GRAD, false><<<blocks, threads, 0, stream>>>(
                pairs, a.exact, a.tab, a.cut, a.layout, a.features, a.status, external);
        } else {
            dense_pair_features<T, DENSE_LMAX_LARGE, GRAD, false><<<blocks, threads, 0, stream>>>(
                pairs, a.exact, a.tab, a.cut, a.layout, a.features, a.status, external);
        }
    }
    CUDA_CHECK(cudaGetLastError());
    if constexpr (sizeof(T) == 4) {
        if (a.surrogate) {
            float* f = reinterpret_cast<float*>(a.features);
            surrogate_fill(a.surrogate, a.pairs.distance, n_pairs, f + a.layout.off_r,
                           GRAD ? f + a.layout.off_dr : nullptr, a.layout.stride, stream);
        }
    }
}

int coefficient_threads(int K) { return std::max(DENSE_CHUNK, std::min(256, (K + 31) / 32 * 32)); }

}  // namespace

namespace {
int mma_state = -1;  // -1: not read from the environment yet
}

bool dense_mma_enabled() {
    if (mma_state < 0) {
        const char* env = std::getenv("FEATOMIC_B200_DENSE_MMA");
        mma_state = (env && env[0] == '0') ? 0 : 1;
        const char* channels = std::getenv("FEATOMIC_B200_MMA_CHANNELS");
        if (channels && channels[0] >= '1' && channels[0] <= '4') dense_mma_channels_per_round = channels[0] - '0';
    }
    return mma_state == 1;
}

void set_dense_mma_enabled(bool enabled) { mma_state = enabled ? 1 : 0; }

void launch_dense_directions(const DevicePairs& pairs, const int32_t* atom_species, int n_species, int64_t n_atoms,
                             int32_t* dir_code, int64_t* seg_offset, DeviceArena& arena, cudaStream_t stream) {
    const int64_t n_dirs = 2 * pairs.count;
    const int64_t n_segments = n_atoms * n_species;
    if (n_segments >= (int64_t)INT32_MAX) throw invalid_parameter("too many atoms x species for the dense layout");
    if (n_dirs > 0) {
        int32_t* keys = arena.alloc<int32_t>("dense.keys", n_dirs);
        int32_t* sorted = arena.alloc<int32_t>("dense.sorted_keys", n_dirs);
        int32_t* codes = arena.alloc<int32_t>("dense.codes", n_dirs);
        const int threads = 256;
        dense_direction_keys<<<(unsigned)((n_dirs + threads - 1) / threads), threads, 0, stream>>>(
            pairs.first, pairs.second, atom_species, pairs.count, n_species, keys, codes);
        CUDA_CHECK(cudaGetLastError());
        int end_bit = 1;
        while (end_bit < 31 && ((int64_t)1 << end_bit) <= n_segments) end_bit++;
        size_t temp = 0;
        CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys, sorted, codes, dir_code, (int)n_dirs, 0, end_bit,
                                                   stream));
        void* t = arena.alloc_bytes("dense.sort_temp", temp);
        CUDA_CHECK(cub::DeviceRadixSort::SortPairs(t, temp, keys, sorted, codes, dir_code, (int)n_dirs, 0, end_bit,
                                                   stream));
        dense_segments<<<(unsigned)((n_segments + 1 + threads - 1) / threads), threads, 0, stream>>>(
            sorted, n_dirs, n_segments, seg_offset);
        CUDA_CHECK(cudaGetLastError());
    } else {
        CUDA_CHECK(cudaMemsetAsync(seg_offset, 0, sizeof(int64_t) * (n_segments + 1), stream));
    }
}

template <typename T>
void launch_dense_forward(const DenseArgs<T>& a, int64_t n_pairs, cudaStream_t stream) {
    auto mark = [&](int k) {
        if (a.marks) CUDA_CHECK(cudaEventRecord(a.marks[k], stream));
    };
    mark(0);
    if (a.gradient_features) launch_features<T, true>(a, n_pairs, stream);
    else launch_features<T, false>(a, n_pairs, stream);
    mark(1);
    if (a.n_atoms == 0) {
        mark(2);
        mark(3);
        return;
    }
    dense_expansion<T><<<(unsigned)(a.n_atoms * a.n_species),
                         coefficient_threads(a.layout.L2 * ((a.nmax + 1) / 2)), 0, stream>>>(a);
    CUDA_CHECK(cudaGetLastError());
    mark(2);
    if (a.values == nullptr) {  // the expansion alone
        mark(3);
        return;
    }
    if constexpr (sizeof(T) == 4) {
        if (dense_mma_enabled() && dense_mma_supported(a)) {
            launch_dense_contraction_mma(a, stream);
            mark(3);
            return;
        }
    }
    const size_t smem = sizeof(T) * (size_t)a.n_species * a.K;
    if (a.nmax <= 16 && smem <= 48 * 1024) {
        if (a.nmax <= 8) dense_contraction_tiled<T, 8><<<(unsigned)a.n_atoms, 128, smem, stream>>>(a);
        else dense_contraction_tiled<T, 16><<<(unsigned)a.n_atoms, 128, smem, stream>>>(a);
    } else {
        const int64_t items = a.n_atoms * a.n_keys;
        const int warps = 8;
        dense_contraction<T><<<(unsigned)((items + warps - 1) / warps), 32 * warps, 0, stream>>>(a);
    }
    CUDA_CHECK(cudaGetLastError());
    mark(3);
}

template <typename T>
void launch_dense_grad_coef(const DenseArgs<T>& a, cudaStream_t stream) {
    const size_t smem = sizeof(T) * (size_t)a.n_species * a.K;
    if (smem > 200 * 1024) throw invalid_parameter("too many species x coefficients for the adjoint kernel");
    static bool configured[2] = {false, false};
    const int which = sizeof(T) == 8 ? 1 : 0;
    if (!configured[which]) {
        CUDA_CHECK(cudaFuncSetAttribute(dense_grad_coef<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CUDA_CHECK(cudaFuncSetAttribute(dense_grad_coef_tiled<T, 17>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024));
        configured[which] = true;
    }
    const size_t tiled_smem = smem + sizeof(T) * (size_t)a.n_keys * a.n_props;
    bool mma = false;
    if constexpr (sizeof(T) == 4) mma = dense_mma_enabled() && dense_mma_supported(a);
    if (mma) {
        if constexpr (sizeof(T) == 4) launch_dense_grad_coef_mma(a, stream);
    } else if (a.lmax <= DENSE_LMAX_SMALL && tiled_smem <= 200 * 1024) {
        dense_grad_coef_tiled<T, 17><<<(unsigned)a.n_atoms, 128, tiled_smem, stream>>>(a);
    } else {
        dense_grad_coef<T><<<(unsigned)a.n_atoms, 256, smem, stream>>>(a);
    }
    CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void launch_dense_backward(const DenseArgs<T>& a, int64_t n_pairs, cudaStream_t stream, bool coef_grad_given) {
    auto mark = [&](int k) {
        if (a.marks) CUDA_CHECK(cudaEventRecord(a.marks[k], stream));
    };
    mark(4);
    if (a.n_atoms == 0) {
        for (int k = 5; k < 8; k++) mark(k);
        return;
    }
    if (!coef_grad_given) launch_dense_grad_coef(a, stream);
    mark(5);
    bool fused = a.lmax <= DENSE_LMAX_SMALL && a.nmax <= 16 && a.tab.spline.splined;
    if constexpr (sizeof(T) == 4) fused = fused && a.surrogate == nullptr;
    if (n_pairs > 0 && fused) {
        const int threads = 128;
        const unsigned blocks = (unsigned)((n_pairs + threads - 1) / threads);
        if (a.nmax <= 8) dense_pair_adjoint_fused<T, 8><<<blocks, threads, 0, stream>>>(a, n_pairs);
        else dense_pair_adjoint_fused<T, 16><<<blocks, threads, 0, stream>>>(a, n_pairs);
        CUDA_CHECK(cudaGetLastError());
    } else if (n_pairs > 0) {
        if (!a.gradient_features) launch_features<T, true>(a, n_pairs, stream);
        const int warps = 8;
        dense_pair_adjoint<T><<<(unsigned)((n_pairs + warps - 1) / warps), 32 * warps, 0, stream>>>(a, n_pairs);
        CUDA_CHECK(cudaGetLastError());
    }
    mark(6);
    const bool partials = a.grad_strain || a.grad_cell;
    const int threads = 128;
    dense_atom_reduce<T><<<(unsigned)((a.n_atoms + threads - 1) / threads), threads, 0, stream>>>(a, partials ? 1 : 0);
    CUDA_CHECK(cudaGetLastError());
    if (partials && a.n_systems > 0) {
        dense_system_reduce<T><<<(unsigned)a.n_systems, 256, 0, stream>>>(a);
        CUDA_CHECK(cudaGetLastError());
    }
    mark(7);
}

template <typename T>
void launch_dense_jvp(const DenseArgs<T>& a, int64_t n_pairs, const T* tangent_positions, const T* tangent_cell,
                      T* pair_tangent, T* tangent_coef, T* tangent_values, cudaStream_t stream) {
    if (a.n_atoms == 0) return;
    if (n_pairs > 0) {
        launch_features<T, true>(a, n_pairs, stream);
        const int threads = 128;
        const int64_t items = n_pairs * a.layout.L2;
        dense_pair_tangent<T><<<(unsigned)((items + threads - 1) / threads), threads, 0, stream>>>(
            a, n_pairs, tangent_positions, tangent_cell, pair_tangent);
        CUDA_CHECK(cudaGetLastError());
    }
    dense_tangent_expansion<T><<<(unsigned)(a.n_atoms * a.n_species), 128, 0, stream>>>(a, pair_tangent, tangent_coef);
    CUDA_CHECK(cudaGetLastError());
    if (tangent_values) {
        const int warps = 8;
        const int64_t items = a.n_atoms * a.n_keys;
        dense_tangent_contraction<T><<<(unsigned)((items + warps - 1) / warps), 32 * warps, 0, stream>>>(
            a, tangent_coef, tangent_values);
        CUDA_CHECK(cudaGetLastError());
    }
}

template void launch_dense_forward<float>(const DenseArgs<float>&, int64_t, cudaStream_t);
template void launch_dense_forward<double>(const DenseArgs<double>&, int64_t, cudaStream_t);
template void launch_dense_backward<float>(const DenseArgs<float>&, int64_t, cudaStream_t, bool);
template void launch_dense_backward<double>(const DenseArgs<double>&, int64_t, cudaStream_t, bool);
template void launch_dense_jvp<float>(const DenseArgs<float>&, int64_t, const float*, const float*, float*, float*,
                                      float*, cudaStream_t);
template void launch_dense_jvp<double>(const DenseArgs<double>&, int64_t, const double*, const double*, double*,
                                       double*, double*, cudaStream_t);

}  // namespace fb200

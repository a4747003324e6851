// Batched form of the power spectrum and its adjoint: many small
// non-periodic systems (molecules) in ONE persistent launch.
//
// Phase A, one centre per warp, centres taken from a work queue ordered by
// decreasing system size:
//   * the centre's neighbours are the atoms of its own system closer than the
//     cutoff (no cell list is needed for molecules of at most a few thousand
//     atoms); each lane evaluates one direction: cutoff, Y_lm (row by row, the
//     recursion of featomic/src/math/spherical_harmonics.rs:228-424) and the
//     spline R_nl (featomic/src/math/splines.rs:225-289), staged in shared
//     memory;
//   * the warp accumulates the centre's coefficients c[species][l m n] in
//     shared memory (spherical_expansion.rs:101-358), in a fixed order;
//   * the power spectrum row P[(a, b)][l n1 n2] (power_spectrum.rs:529-780)
//     and, for a loss L, dL/dc from dL/dP (a linear model's weights per
//     centre species, or any dL/dP per atom);
//   * for every direction a -> b, h_ab = sum_lmn dL/dc_a[s_b][l m n]
//     d(f R Y)/dr_ab, evaluated by one lane with Y_lm and dY_lm recomputed
//     row by row in registers.  The pair term of the spherical expansion of
//     the other atom is the same with the roles swapped, so
//     dL/dr_i = sum_j (h_ji - h_ij) needs no other centre's dL/dc.
// Grid barrier (bounded wait, error flag on timeout).
// Phase B, one system per warp: dL/dr_i from the h of the system, the energy
// and the strain derivative sum_ab r_ab x h_ab.
//
// FP32 arithmetic; positions, distances and the spline interval search in
// FP64.  Deterministic: no floating-point atomics.
//
// This header holds the device code; batched_kernels_*.cu instantiate the
// kernel variants in separate translation units (compiled in parallel) and
// batched.cu holds the host side.
#pragma once

#include "batched.hpp"
#include "pair_math.cuh"

namespace fb200 {
namespace batched_detail {


constexpr int BLCAP = 8;
constexpr long long BARRIER_SPINS = 1ll << 25;  // x ~100 ns: a few seconds

__device__ __forceinline__ int isqrt_lm(int lm) {
    int l = (int)sqrtf((float)lm);
    while (l * l > lm) l--;
    while ((l + 1) * (l + 1) <= lm) l++;
    return l;
}

__device__ __forceinline__ void key_pair(int key, int S, int* a, int* b) {
    int x = 0;
    while (key >= S - x) {
        key -= S - x;
        x++;
    }
    *a = x;
    *b = x + key;
}

__device__ __forceinline__ int key_index(int a, int b, int S) { return a * S - a * (a - 1) / 2 + (b - a); }

// R_nl(r) (and dR/dr) of one angular channel into registers
template <int NCAP>
__device__ __forceinline__ bool radial_row(const BatchArgs& a, int l, double r, float (&R)[NCAP], float (&dR)[NCAP],
                                           bool grad) {
    const int N = a.nmax;
    const DeviceSplineT<float>& S = a.tab.spline;
    if (S.splined) {
        const double* pos = S.positions + S.knot_offset[l];
        const int k = soap::spline_interval(pos, S.knot_count[l], r);
        const soap::HermiteWeights w = soap::hermite_weights(pos[k], pos[k + 1], r);
        const float* pv = S.values + ((size_t)S.knot_offset[l] + k) * N;
        const float* pd = S.derivs + ((size_t)S.knot_offset[l] + k) * N;
        const float h00 = (float)w.h00, h10 = (float)(w.h10 * w.delta), h01 = (float)w.h01,
                    h11 = (float)(w.h11 * w.delta);
        const float d00 = (float)(w.d00 * w.dxdt), d10 = (float)w.d10, d01 = (float)(w.d01 * w.dxdt),
                    d11 = (float)w.d11;
#pragma unroll
        for (int n = 0; n < NCAP; n++) {
            if (n < N) {
                const float q0 = pv[n], m0 = pd[n], q1 = pv[N + n], m1 = pd[N + n];
                R[n] = h00 * q0 + h10 * m0 + h01 * q1 + h11 * m1;
                dR[n] = grad ? d00 * q0 + d10 * m0 + d01 * q1 + d11 * m1 : 0.0f;
            } else {
                R[n] = 0.0f;
                dR[n] = 0.0f;
            }
        }
        return true;
    }
    double v[64], g[64];
    const bool ok = radial_compute(a.exact, l, r, v, grad ? g : nullptr);
#pragma unroll
    for (int n = 0; n < NCAP; n++) {
        R[n] = n < N ? (float)v[n] : 0.0f;
        dR[n] = (grad && n < N) ? (float)g[n] : 0.0f;
    }
    return ok;
}

struct Direction {
    bool keep;
    double r, u[3], d[3];
    float f, fg;
};

// direction centre -> atom j: r_ij = r_j - r_i, cutoff function and radial
// scaling (featomic's f and df/dr)
__device__ __forceinline__ Direction direction(const BatchArgs& a, double xi, double yi, double zi, int64_t j) {
    Direction D;
    D.d[0] = a.positions[3 * j] - xi;
    D.d[1] = a.positions[3 * j + 1] - yi;
    D.d[2] = a.positions[3 * j + 2] - zi;
    const double r2 = D.d[0] * D.d[0] + D.d[1] * D.d[1] + D.d[2] * D.d[2];
    D.keep = r2 < a.rc2;
    D.r = sqrt(r2);
    if (D.r < 1e-6) {
        // coincident atoms: spherical_expansion_pair.rs:337-339
        D.u[0] = 0.0;
        D.u[1] = 0.0;
        D.u[2] = 1.0;
    } else {
        for (int x = 0; x < 3; x++) D.u[x] = D.d[x] / D.r;
    }
    double fc = 0.0, dfc = 0.0, sc = 1.0, dsc = 0.0;
    if (D.keep) {
        soap::cutoff_function(a.cut.smoothing, a.cut.rc, a.cut.width, D.r, &fc, &dfc);
        if (a.cut.scaling) soap::willatt2018(a.cut.scale, a.cut.rate, a.cut.exponent, D.r, &sc, &dsc);
    }
    D.f = (float)(sc * fc);
    D.fg = (float)(dfc * sc + fc * dsc);
    return D;
}

// Grid-wide barrier with a bounded wait.  Returns false (and sets bit 1 of
// *status) when the other CTAs did not arrive in time.
__device__ inline bool grid_barrier(unsigned int* bar, int32_t* status) {
    __shared__ int ok_shared;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* generation = bar + 1;
        const unsigned int mine = *generation;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*generation == mine) {
                if (++spins > BARRIER_SPINS) {
                    atomicOr(status, 2);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_shared = ok;
    }
    __syncthreads();
    return ok_shared != 0;
}

template <int CHUNK, int LAYOUT, int NCAP>
__global__ void __launch_bounds__(256) batched_kernel(BatchArgs a) {
    extern __shared__ __align__(16) float bsmem[];
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const int S = a.n_species, K = a.K, N = a.nmax, NN = N * N;
    const int L2 = (a.lmax + 1) * (a.lmax + 1), RN = (a.lmax + 1) * N;
    const int KP = a.n_keys * a.n_props;
    const int SK = S * K;
    const int feat = CHUNK * (L2 + RN) > SK ? CHUNK * (L2 + RN) : SK;
    const int per_warp = SK + feat + CHUNK;

    float* scale = bsmem;  // [2 (lmax + 1)]: unmixed then mixed species
    float* C = bsmem + 64 + warp * per_warp;
    float* Fr = C + SK;
    float* Yd = Fr;
    float* Rd = Fr + CHUNK * L2;
    float* dC = Fr;
    int* dsp = reinterpret_cast<int*>(Fr + feat);
    for (int t = threadIdx.x; t < 2 * (a.lmax + 1); t += blockDim.x) {
        const int l = t % (a.lmax + 1);
        const double s = sqrt((double)(2 * l + 1));
        scale[t] = (float)((t > a.lmax ? 1.4142135623730951 : 1.0) / ((l % 2 == 0) ? s : -s));
    }
    __syncthreads();
    const bool backward = a.weights != nullptr || a.grad_values != nullptr;

    // ---------------- phase A: one centre per warp ----------------
    while (true) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(a.queue, 1);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= a.n_atoms) break;
        const int64_t i = a.order[idx];
        const int sys = a.atom_system[i];
        const int64_t a0 = a.atom_offset[sys];
        const int n = (int)(a.atom_offset[sys + 1] - a0);
        const int si = a.species[i];
        const double xi = a.positions[3 * i], yi = a.positions[3 * i + 1], zi = a.positions[3 * i + 2];
        for (int k = lane; k < SK; k += 32) C[k] = 0.0f;
        __syncwarp();

        // spherical expansion of the centre
        for (int j0 = 0; j0 < n; j0 += CHUNK) {
            const int jl = j0 + lane;
            bool keep = false;
            if (lane < CHUNK && jl < n && a0 + jl != i) {
                const int64_t j = a0 + jl;
                const Direction D = direction(a, xi, yi, zi, j);
                if (D.keep) {
                    keep = true;
                    dsp[lane] = a.species[j];
                    float* y = Yd + lane * L2;
                    ylm_rows<float, BLCAP, false>(
                        a.tab.ylm, (float)D.u[0], (float)D.u[1], (float)D.u[2], [&](int) {},
                        [&](int l, int m, float yp, float ym, const float*, const float*) {
                            y[l * l + l + m] = yp;
                            if (m > 0) y[l * l + l - m] = ym;
                        });
                    float R[NCAP], dR[NCAP];
                    float* rr = Rd + lane * RN;
                    for (int l = 0; l <= a.lmax; l++) {
                        if (!radial_row<NCAP>(a, l, D.r, R, dR, false)) atomicOr(a.status, 1);
#pragma unroll
                        for (int q = 0; q < NCAP; q++)
                            if (q < N) rr[l * N + q] = D.f * R[q];
                    }
                }
            }
            const unsigned mask = __ballot_sync(FULL, keep);
            __syncwarp();
            if (LAYOUT == 0) {
                for (int k = lane; k < K; k += 32) {
                    const int lm = k / N, nn = k - lm * N, l = isqrt_lm(lm);
                    unsigned mm = mask;
                    while (mm) {
                        const int q = __ffs(mm) - 1;
                        mm &= mm - 1;
                        C[dsp[q] * K + k] += Yd[q * L2 + lm] * Rd[q * RN + l * N + nn];
                    }
                }
            } else {
                for (int lm = lane; lm < L2; lm += 32) {
                    const int l = isqrt_lm(lm);
                    unsigned mm = mask;
                    while (mm) {
                        const int q = __ffs(mm) - 1;
                        mm &= mm - 1;
                        const float y = Yd[q * L2 + lm];
                        float* c = C + dsp[q] * K + lm * N;
                        const float* rr = Rd + q * RN + l * N;
#pragma unroll
                        for (int nn = 0; nn < NCAP; nn++)
                            if (nn < N) c[nn] += y * rr[nn];
                    }
                }
            }
            __syncwarp();
        }
        if (lane < N) C[si * K + lane] += a.tab.self_contribution[lane];
        __syncwarp();

        // power spectrum row and the linear energy
        const float* Wi = a.grad_values ? a.grad_values + i * KP : (a.weights ? a.weights + (int64_t)si * KP : nullptr);
        float energy = 0.0f;
        if (a.values || a.weights) {
            for (int o = lane; o < KP; o += 32) {
                const int key = o / a.n_props;
                const int p = o - key * a.n_props;
                int sa, sb;
                key_pair(key, S, &sa, &sb);
                const int l = p / NN;
                const int n1 = (p - l * NN) / N, n2 = p - l * NN - n1 * N;
                const float* ca = C + sa * K + l * l * N + n1;
                const float* cb = C + sb * K + l * l * N + n2;
                float s = 0.0f;
                for (int m = 0; m < 2 * l + 1; m++) s += ca[m * N] * cb[m * N];
                const float P = s * scale[(sa != sb ? a.lmax + 1 : 0) + l];
                if (a.values) a.values[i * KP + o] = P;
                if (a.weights) energy += Wi[o] * P;
            }
        }
        if (!backward) continue;

        // dL/dc of the centre (the staged directions are no longer needed)
        for (int o = lane; o < SK; o += 32) {
            const int sa = o / K;
            const int k = o - sa * K;
            const int lm = k / N, nn = k - lm * N, l = isqrt_lm(lm);
            float acc = 0.0f;
            for (int b = 0; b < S; b++) {
                const float* cb = C + b * K + lm * N;
                float s = 0.0f;
                if (sa < b) {
                    const float* g = Wi + key_index(sa, b, S) * a.n_props + l * NN + nn * N;
                    for (int q = 0; q < N; q++) s += g[q] * cb[q];
                    acc += scale[a.lmax + 1 + l] * s;
                } else if (sa > b) {
                    const float* g = Wi + key_index(b, sa, S) * a.n_props + l * NN + nn;
                    for (int q = 0; q < N; q++) s += g[q * N] * cb[q];
                    acc += scale[a.lmax + 1 + l] * s;
                } else {
                    const float* g = Wi + key_index(sa, sa, S) * a.n_props + l * NN;
                    for (int q = 0; q < N; q++) s += (g[nn * N + q] + g[q * N + nn]) * cb[q];
                    acc += scale[l] * s;
                }
            }
            dC[o] = acc;
        }
        __syncwarp();

        // h for every direction of the centre, one direction per lane
        float vir[9];
#pragma unroll
        for (int x = 0; x < 9; x++) vir[x] = 0.0f;
        for (int j0 = 0; j0 < n; j0 += 32) {
            const int jl = j0 + lane;
            if (jl >= n) continue;
            float h[3] = {0.0f, 0.0f, 0.0f};
            const int64_t j = a0 + jl;
            Direction D;
            D.keep = false;
            if (j != i) D = direction(a, xi, yi, zi, j);
            if (D.keep) {
                const float* Dc = dC + a.species[j] * K;
                const float u0 = (float)D.u[0], u1 = (float)D.u[1], u2 = (float)D.u[2];
                const float f_over_r = D.f / (float)D.r;
                float R[NCAP], dR[NCAP], Rg[NCAP];
                ylm_rows<float, BLCAP, true>(
                    a.tab.ylm, u0, u1, u2,
                    [&](int l) {
                        if (!radial_row<NCAP>(a, l, D.r, R, dR, true)) atomicOr(a.status, 1);
#pragma unroll
                        for (int q = 0; q < NCAP; q++) Rg[q] = D.fg * R[q] + D.f * dR[q];
                    },
                    [&](int l, int m, float yp, float ym, const float* gp, const float* gm) {
                        {
                            const float* d = Dc + (l * l + l + m) * N;
                            float A = 0.0f, B = 0.0f;
#pragma unroll
                            for (int q = 0; q < NCAP; q++)
                                if (q < N) {
                                    A += d[q] * Rg[q];
                                    B += d[q] * R[q];
                                }
                            const float Ay = A * yp, Bf = B * f_over_r;
                            h[0] += Ay * u0 + Bf * gp[0];
                            h[1] += Ay * u1 + Bf * gp[1];
                            h[2] += Ay * u2 + Bf * gp[2];
                        }
                        if (m > 0) {
                            const float* d = Dc + (l * l + l - m) * N;
                            float A = 0.0f, B = 0.0f;
#pragma unroll
                            for (int q = 0; q < NCAP; q++)
                                if (q < N) {
                                    A += d[q] * Rg[q];
                                    B += d[q] * R[q];
                                }
                            const float Ay = A * ym, Bf = B * f_over_r;
                            h[0] += Ay * u0 + Bf * gm[0];
                            h[1] += Ay * u1 + Bf * gm[1];
                            h[2] += Ay * u2 + Bf * gm[2];
                        }
                    });
#pragma unroll
                for (int x = 0; x < 3; x++)
#pragma unroll
                    for (int y = 0; y < 3; y++) vir[x * 3 + y] += (float)D.d[x] * h[y];
            }
            float* hp = a.h + 3 * (a.h_offset[sys] + (i - a0) * n + jl);
            hp[0] = h[0];
            hp[1] = h[1];
            hp[2] = h[2];
        }
        for (int off = 16; off > 0; off >>= 1) {
            energy += __shfl_down_sync(FULL, energy, off);
#pragma unroll
            for (int x = 0; x < 9; x++) vir[x] += __shfl_down_sync(FULL, vir[x], off);
        }
        if (lane == 0) {
            a.atom_energy[i] = energy;
#pragma unroll
            for (int x = 0; x < 9; x++) a.atom_strain[9 * i + x] = vir[x];
        }
        __syncwarp();
    }
    if (!backward) return;

    // ---------------- phase B: one system per warp ----------------
    if (!grid_barrier(a.barrier, a.status)) return;
    const int64_t gw = (int64_t)blockIdx.x * nwarps + warp;
    const int64_t total = (int64_t)gridDim.x * nwarps;
    for (int64_t s = gw; s < a.n_systems; s += total) {
        const int64_t a0 = a.atom_offset[s];
        const int n = (int)(a.atom_offset[s + 1] - a0);
        const int64_t hb = a.h_offset[s];
        float energy = 0.0f, st[9];
#pragma unroll
        for (int x = 0; x < 9; x++) st[x] = 0.0f;
        for (int il = lane; il < n; il += 32) {
            float g[3] = {0.0f, 0.0f, 0.0f};
            // written by other CTAs before the barrier: read through L2
            for (int jl = 0; jl < n; jl++) {
                const float* hij = a.h + 3 * (hb + (int64_t)il * n + jl);
                const float* hji = a.h + 3 * (hb + (int64_t)jl * n + il);
                g[0] += __ldcg(hji) - __ldcg(hij);
                g[1] += __ldcg(hji + 1) - __ldcg(hij + 1);
                g[2] += __ldcg(hji + 2) - __ldcg(hij + 2);
            }
            if (a.grad_positions) {
                a.grad_positions[3 * (a0 + il)] = g[0];
                a.grad_positions[3 * (a0 + il) + 1] = g[1];
                a.grad_positions[3 * (a0 + il) + 2] = g[2];
            }
            energy += __ldcg(a.atom_energy + a0 + il);
#pragma unroll
            for (int x = 0; x < 9; x++) st[x] += __ldcg(a.atom_strain + 9 * (a0 + il) + x);
        }
        for (int off = 16; off > 0; off >>= 1) {
            energy += __shfl_down_sync(FULL, energy, off);
#pragma unroll
            for (int x = 0; x < 9; x++) st[x] += __shfl_down_sync(FULL, st[x], off);
        }
        if (lane == 0) {
            if (a.energies) a.energies[s] = energy;
            if (a.grad_strain)
#pragma unroll
                for (int x = 0; x < 9; x++) a.grad_strain[9 * s + x] = st[x];
        }
    }
}

using KernelFn = void (*)(BatchArgs);

// the kernel variants of one CHUNK x LAYOUT pair, NCAP = 8 (small) or 16
KernelFn kernel_16_0(bool small);
KernelFn kernel_16_1(bool small);
KernelFn kernel_32_0(bool small);
KernelFn kernel_32_1(bool small);

}  // namespace batched_detail
}  // namespace fb200

// Kernel (b): SOAP spherical expansion on the GPU, FP64.
//
// Two launches (or, for lmax <= 8, one: se_fused_kernel builds the pair
// terms of each chunk of directions in shared memory instead of reading the
// per-pair records from HBM):
//
// * `pair_features` -- one thread per half pair: cutoff / radial scaling,
//   real spherical harmonics Y_lm (and their Cartesian gradients) by the
//   Legendre recursion of featomic/src/math/spherical_harmonics.rs:228-424,
//   and the radial integral R_nl(r) (and dR/dr) from the Hermite spline
//   tables (featomic/src/math/splines.rs:225-289) or, when the spline is
//   disabled, analytically (radial_integral/gto.rs:115-205).  The result is a
//   per-pair feature record in HBM.
//
// * `se_accumulate` -- one CTA per (centre, neighbour species), one thread per coefficient
//   (l, m, n).  Directions (pair, orientation) are sorted by
//   (centre, neighbour species, pair), so every (centre, species) segment is a
//   contiguous run reduced in registers: no atomics, deterministic order.  It
//   reproduces accumulate_all_pairs (featomic/src/calculators/soap/
//   spherical_expansion.rs:101-358): values, the per-pair gradient of the
//   first->second orientation, the self (centre) gradient, and the strain and
//   cell gradients, with the (-1)^l / -(-1)^l factors of the reversed pair
//   (spherical_expansion_pair.rs:130-163).
#include <algorithm>
#include <cstdlib>

#include "engine.hpp"
#include "pair_math.cuh"
#include "soap_math.cuh"

namespace fb200 {

namespace {

constexpr int LMAX_SMALL = 8;
constexpr int LMAX_LARGE = 24;

template <int LCAP>
__global__ void pair_features_kernel(DevicePairs pairs, DeviceRadial radial, DeviceYlm ylm, CutoffParams cut,
                                     FeatureLayout L, double* __restrict__ features, int32_t* __restrict__ status) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pairs.count) return;
    double* f = features + p * L.stride;
    double r = pairs.distance[p];
    double v0 = pairs.vector[3 * p], v1 = pairs.vector[3 * p + 1], v2 = pairs.vector[3 * p + 2];
    double u0 = v0 / r, u1 = v1 / r, u2 = v2 / r;
    if (r < 1e-6) {
        // coincident atoms: spherical_expansion_pair.rs:337-339
        u0 = 0.0;
        u1 = 0.0;
        u2 = 1.0;
    }
    double fc, dfc;
    soap::cutoff_function(cut.smoothing, cut.rc, cut.width, r, &fc, &dfc);
    double sc = 1.0, dsc = 0.0;
    if (cut.scaling) soap::willatt2018(cut.scale, cut.rate, cut.exponent, r, &sc, &dsc);
    f[0] = sc * fc;
    f[1] = dfc * sc + fc * dsc;
    f[2] = r;
    f[3] = u0;
    f[4] = u1;
    f[5] = u2;
    f[6] = v0;
    f[7] = v1;
    f[8] = v2;
    f[9] = pairs.first[p] == pairs.second[p] ? 1.0 : 0.0;
    f[10] = (double)pairs.shift[3 * p];
    f[11] = (double)pairs.shift[3 * p + 1];
    f[12] = (double)pairs.shift[3 * p + 2];
    if (L.with_grad) {
        ylm_compute<double, LCAP>(ylm, u0, u1, u2, f + L.off_y, f + L.off_dy, f + L.off_dy + L.L2,
                                  f + L.off_dy + 2 * L.L2);
    } else {
        ylm_compute<double, LCAP>(ylm, u0, u1, u2, f + L.off_y, nullptr, nullptr, nullptr);
    }
    bool ok = true;
    for (int l = 0; l <= L.lmax; l++) {
        ok &= radial_compute(radial, l, r, f + L.off_r + l * L.nmax, L.with_grad ? f + L.off_dr + l * L.nmax : nullptr);
    }
    if (!ok) atomicExch(status, 1);
}

// Per-direction scalars staged in shared memory for a chunk of directions
struct DirScalars {
    double f, fg, r, rinv, u[3], v[3], sh[3];
    int64_t feature;  // offset of the pair's feature record
    int inv, self_image;
};

constexpr int SE_CHUNK = 32;

template <bool POS, bool STRAIN, bool CELL>
__global__ void __launch_bounds__(256) se_accumulate_kernel(SeArgs a) {
    constexpr bool GRAD = POS || STRAIN || CELL;
    __shared__ DirScalars dirs[SE_CHUNK];
    const FeatureLayout L = a.layout;
    // one CTA per (centre, neighbour species) segment: the segments are
    // independent, and S times more CTAs keep more of them in flight
    const int S = a.n_species;
    const int64_t c = blockIdx.x / S;
    const int t_block = (int)(blockIdx.x - c * S);
    const int K = L.L2 * L.nmax;
    const int tc = a.centre_species[c];

    for (int k0 = 0; k0 < K; k0 += blockDim.x) {
        const int k = k0 + threadIdx.x;
        const bool active = k < K;
        const int lm = active ? k / L.nmax : 0;
        const int n = active ? k - lm * L.nmax : 0;
        int l = (int)sqrt((double)lm);
        while (l * l > lm) l--;
        while ((l + 1) * (l + 1) <= lm) l++;
        const double sign_l = (l & 1) ? -1.0 : 1.0;
        const int ri = l * L.nmax + n;

        for (int t = t_block; t == t_block; t++) {
            const int64_t d0 = a.seg_offset[c * S + t], d1 = a.seg_offset[c * S + t + 1];
            double acc = 0.0;
            double sg[3] = {0.0, 0.0, 0.0};
            double st[9], ce[9];
#pragma unroll
            for (int x = 0; x < 9; x++) {
                st[x] = 0.0;
                ce[x] = 0.0;
            }
            for (int64_t dc = d0; dc < d1; dc += SE_CHUNK) {
                const int nd = (int)min((int64_t)SE_CHUNK, d1 - dc);
                __syncthreads();
                if (threadIdx.x < nd) {
                    const int32_t code = a.dir_code[dc + threadIdx.x];
                    const int64_t p = code >> 1;
                    const double* F = a.features + p * L.stride;
                    DirScalars& D = dirs[threadIdx.x];
                    D.feature = p * L.stride;
                    D.inv = code & 1;
                    D.f = F[0];
                    if (GRAD) {
                        D.fg = F[1];
                        D.r = F[2];
                        D.rinv = 1.0 / D.r;
                        for (int x = 0; x < 3; x++) {
                            D.u[x] = F[3 + x];
                            D.v[x] = F[6 + x];
                            D.sh[x] = F[10 + x];
                        }
                        D.self_image = F[9] != 0.0;
                    }
                }
                __syncthreads();
                if (!active) continue;
#pragma unroll 2
                for (int q = 0; q < nd; q++) {
                    const DirScalars& D = dirs[q];
                    const double* __restrict__ F = a.features + D.feature;
                    const double Yv = __ldg(F + L.off_y + lm);
                    const double Rv = __ldg(F + L.off_r + ri);
                    const double val = D.f * Yv * Rv;
                    acc += D.inv ? sign_l * val : val;
                    if (!GRAD) continue;
                    const double dR = __ldg(F + L.off_dr + ri);
                    double g[3];
#pragma unroll
                    for (int x = 0; x < 3; x++) {
                        const double dY = __ldg(F + L.off_dy + x * L.L2 + lm);
                        g[x] = D.fg * D.u[x] * Rv * Yv + D.f * dR * D.u[x] * Yv + D.f * Rv * dY * D.rinv;
                    }
                    if (POS && !D.inv) {
                        double* pg = a.pair_grad + (D.feature / L.stride) * 3 * K;
                        pg[k] = g[0];
                        pg[K + k] = g[1];
                        pg[2 * K + k] = g[2];
                    }
                    const double gf = D.inv ? -sign_l : 1.0;
                    const double gi[3] = {gf * g[0], gf * g[1], gf * g[2]};
                    if (POS && !D.self_image) {
                        sg[0] -= gi[0];
                        sg[1] -= gi[1];
                        sg[2] -= gi[2];
                    }
                    if (STRAIN) {
#pragma unroll
                        for (int x = 0; x < 3; x++) {
                            const double vx = D.inv ? -D.v[x] : D.v[x];
#pragma unroll
                            for (int y = 0; y < 3; y++) st[x * 3 + y] += vx * gi[y];
                        }
                    }
                    if (CELL) {
#pragma unroll
                        for (int x = 0; x < 3; x++) {
                            const double sx = D.inv ? -D.sh[x] : D.sh[x];
#pragma unroll
                            for (int y = 0; y < 3; y++) ce[x * 3 + y] += sx * gi[y];
                        }
                    }
                }
            }
            if (!active) continue;
            const int64_t base = (c * S + t);
            const double self = (t == tc && l == 0) ? a.self_contribution[n] : 0.0;
            a.coef[base * K + k] = self + acc;
            if (POS) {
                double* sgp = a.self_grad + base * 3 * K;
                sgp[k] = sg[0];
                sgp[K + k] = sg[1];
                sgp[2 * K + k] = sg[2];
            }
            if (STRAIN) {
                double* o = a.strain + base * 9 * K;
#pragma unroll
                for (int x = 0; x < 9; x++) o[x * K + k] = st[x];
            }
            if (CELL) {
                double* o = a.cellg + base * 9 * K;
#pragma unroll
                for (int x = 0; x < 9; x++) o[x * K + k] = ce[x];
            }
        }
    }
}

// Fused form of pair_features + se_accumulate (lmax <= 8): one CTA per
// (centre, neighbour species) segment.  For each chunk of FUSED_CHUNK
// directions (32: nearly every segment is one chunk, and 86 KB of shared
// memory still fits the two CTAs per SM the registers allow) the pair terms
// are built in shared memory instead of being read
// back from per-pair records in HBM: one thread per (direction, m) evaluates
// column m of the Legendre table and then Y_l^{+-m} (+ gradients), one thread
// per (direction, l) the radial integral R_nl (+ dR/dr), one thread per
// direction the cutoff and radial scaling; then every thread accumulates two
// radial functions of one (l, m) over the chunk's directions in pair order.
// The same functions in the same order as the two-kernel path, so the results
// are bit-identical to it; no atomics.
constexpr int FUSED_CHUNK = 32;

struct FusedDir {
    // rinv = 1 / r, computed once per direction: the angular gradient term
    // f R dY / r is evaluated as f R dY * rinv (one extra rounding against
    // featomic's division, far inside the 1e-10 parity bound; an FP64 divide
    // per coefficient was most of this kernel's instruction stream)
    double f, fg, r, rinv, u[3], v[3], sh[3];
    int64_t pair;
    int inv, self_image;
};

__host__ __device__ inline size_t fused_shared_doubles(int lmax, int nmax, bool grad) {
    const int L2 = (lmax + 1) * (lmax + 1), LR = (lmax + 1) * nmax, NP = (lmax + 1) * (lmax + 2) / 2;
    return (size_t)FUSED_CHUNK * (L2 * (grad ? 4 : 1) + LR * (grad ? 2 : 1) + NP);
}

template <bool POS, bool STRAIN, bool CELL>
__global__ void __launch_bounds__(256, 2) se_fused_kernel(SeArgs a, DevicePairs pairs, DeviceRadial radial, DeviceYlm ylm,
                                                        CutoffParams cut) {
    constexpr bool GRAD = POS || STRAIN || CELL;
    extern __shared__ double fsm[];
    __shared__ FusedDir dirs[FUSED_CHUNK];
    const FeatureLayout L = a.layout;
    const int L2 = L.L2, N = L.nmax, LR = (L.lmax + 1) * N, NH = (N + 1) / 2, NP = (L.lmax + 1) * (L.lmax + 2) / 2;
    double* Ys = fsm;                                      // [chunk][L2]
    double* dYs = Ys + FUSED_CHUNK * L2;                   // [chunk][3][L2]
    double* Rs = dYs + (GRAD ? FUSED_CHUNK * 3 * L2 : 0);  // [chunk][LR]
    double* dRs = Rs + FUSED_CHUNK * LR;                   // [chunk][LR]
    double* Ps = dRs + (GRAD ? FUSED_CHUNK * LR : 0);      // [chunk][NP] Legendre table
    const int S = a.n_species;
    const int64_t c = blockIdx.x / S;
    const int t = (int)(blockIdx.x - c * S);
    const int K = L2 * N;
    const int tc = a.centre_species[c];
    const int64_t d0 = a.seg_offset[c * S + t], d1 = a.seg_offset[c * S + t + 1];
    // this thread's coefficients: (l, m) = lm and n = n0, n0 + 1
    const int item = threadIdx.x;
    const bool active = item < L2 * NH;
    const int lm = active ? item / NH : 0;
    const int n0 = active ? 2 * (item - lm * NH) : 0;
    const bool has1 = n0 + 1 < N;
    int l = (int)sqrt((double)lm);
    while (l * l > lm) l--;
    while ((l + 1) * (l + 1) <= lm) l++;
    const double sign_l = (l & 1) ? -1.0 : 1.0;
    const int ri = l * N + n0;
    double acc[2] = {0.0, 0.0};
    double sg[2][3], st[2][9], ce[2][9];
#pragma unroll
    for (int j = 0; j < 2; j++) {
#pragma unroll
        for (int x = 0; x < 3; x++) sg[j][x] = 0.0;
#pragma unroll
        for (int x = 0; x < 9; x++) {
            st[j][x] = 0.0;
            ce[j][x] = 0.0;
        }
    }
    for (int64_t dc = d0; dc < d1; dc += FUSED_CHUNK) {
        const int nd = (int)min((int64_t)FUSED_CHUNK, d1 - dc);
        const int lcols = L.lmax + 1;
        __syncthreads();
        // threads [0, nd * lcols): direction q, Legendre column m (the m = 0
        // thread also writes the direction's scalars); threads
        // [nd * lcols, 2 nd * lcols): direction q, radial channel l
        for (int w = threadIdx.x; w < 2 * nd * lcols; w += blockDim.x) {
            const bool column = w < nd * lcols;
            const int wq = column ? w : w - nd * lcols;
            const int q = wq / lcols, j = wq - q * lcols;
            const int32_t code = a.dir_code[dc + q];
            const int64_t p = code >> 1;
            const double r = pairs.distance[p];
            if (!column) {
                radial_spline_compute(radial, j, r, Rs + q * LR + j * N, GRAD ? dRs + q * LR + j * N : nullptr);
                continue;
            }
            // the direction's unit vector and scalars, as pair_features_kernel computes them
            const double v0 = pairs.vector[3 * p], v1 = pairs.vector[3 * p + 1], v2 = pairs.vector[3 * p + 2];
            double u0 = v0 / r, u1 = v1 / r, u2 = v2 / r;
            if (r < 1e-6) {
                // coincident atoms: spherical_expansion_pair.rs:337-339
                u0 = 0.0;
                u1 = 0.0;
                u2 = 1.0;
            }
            ylm_legendre_column(ylm, ylm_angles(u0, u1, u2), j, Ps + q * NP);
            if (j != 0) continue;
            double fc, dfc;
            soap::cutoff_function(cut.smoothing, cut.rc, cut.width, r, &fc, &dfc);
            double sc = 1.0, dsc = 0.0;
            if (cut.scaling) soap::willatt2018(cut.scale, cut.rate, cut.exponent, r, &sc, &dsc);
            FusedDir& D = dirs[q];
            D.f = sc * fc;
            D.fg = dfc * sc + fc * dsc;
            D.r = r;
            D.rinv = 1.0 / r;
            D.u[0] = u0;
            D.u[1] = u1;
            D.u[2] = u2;
            D.v[0] = v0;
            D.v[1] = v1;
            D.v[2] = v2;
            for (int x = 0; x < 3; x++) D.sh[x] = (double)pairs.shift[3 * p + x];
            D.pair = p;
            D.inv = code & 1;
            D.self_image = pairs.first[p] == pairs.second[p];
        }
        __syncthreads();
        // Y_l^{+-m} (+ gradients) of every (direction, m) from the complete table
        for (int w = threadIdx.x; w < nd * lcols; w += blockDim.x) {
            const int q = w / lcols, m = w - q * lcols;
            const FusedDir& D = dirs[q];
            double* Y = Ys + q * L2;
            double* G = GRAD ? dYs + q * 3 * L2 : nullptr;
            ylm_column_outputs(ylm, ylm_angles(D.u[0], D.u[1], D.u[2]), m, Ps + q * NP, Y, G,
                               GRAD ? G + L2 : nullptr, GRAD ? G + 2 * L2 : nullptr);
        }
        __syncthreads();
        if (!active) continue;
        for (int q = 0; q < nd; q++) {
            const FusedDir& D = dirs[q];
            const double Yv = Ys[q * L2 + lm];
            double dY[3] = {0.0, 0.0, 0.0};
            if (GRAD) {
#pragma unroll
                for (int x = 0; x < 3; x++) dY[x] = dYs[(q * 3 + x) * L2 + lm];
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (j == 1 && !has1) break;
                const double Rv = Rs[q * LR + ri + j];
                const double val = D.f * Yv * Rv;
                acc[j] += D.inv ? sign_l * val : val;
                if (!GRAD) continue;
                const double dR = dRs[q * LR + ri + j];
                double g[3];
#pragma unroll
                for (int x = 0; x < 3; x++) g[x] = D.fg * D.u[x] * Rv * Yv + D.f * dR * D.u[x] * Yv + D.f * Rv * dY[x] * D.rinv;
                const int k = lm * N + n0 + j;
                if (POS && !D.inv) {
                    double* pg = a.pair_grad + D.pair * 3 * K;
                    pg[k] = g[0];
                    pg[K + k] = g[1];
                    pg[2 * K + k] = g[2];
                }
                const double gf = D.inv ? -sign_l : 1.0;
                const double gi[3] = {gf * g[0], gf * g[1], gf * g[2]};
                if (POS && !D.self_image) {
                    sg[j][0] -= gi[0];
                    sg[j][1] -= gi[1];
                    sg[j][2] -= gi[2];
                }
                if (STRAIN) {
#pragma unroll
                    for (int x = 0; x < 3; x++) {
                        const double vx = D.inv ? -D.v[x] : D.v[x];
#pragma unroll
                        for (int y = 0; y < 3; y++) st[j][x * 3 + y] += vx * gi[y];
                    }
                }
                if (CELL) {
#pragma unroll
                    for (int x = 0; x < 3; x++) {
                        const double sx = D.inv ? -D.sh[x] : D.sh[x];
#pragma unroll
                        for (int y = 0; y < 3; y++) ce[j][x * 3 + y] += sx * gi[y];
                    }
                }
            }
        }
    }
    if (!active) return;
    const int64_t base = c * S + t;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        if (j == 1 && !has1) break;
        const int n = n0 + j, k = lm * N + n;
        const double self = (t == tc && l == 0) ? a.self_contribution[n] : 0.0;
        a.coef[base * K + k] = self + acc[j];
        if (POS) {
            double* sgp = a.self_grad + base * 3 * K;
            sgp[k] = sg[j][0];
            sgp[K + k] = sg[j][1];
            sgp[2 * K + k] = sg[j][2];
        }
        if (STRAIN) {
            double* o = a.strain + base * 9 * K;
#pragma unroll
            for (int x = 0; x < 9; x++) o[x * K + k] = st[j][x];
        }
        if (CELL) {
            double* o = a.cellg + base * 9 * K;
#pragma unroll
            for (int x = 0; x < 9; x++) o[x * K + k] = ce[j][x];
        }
    }
}

// spherical_expansion calculator output: values / strain / cell of one
// (block, sample) row per CTA
__global__ void se_output_rows_kernel(SeOutArgs a, int do_strain, int do_cell) {
    const int64_t row = blockIdx.x;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    const int c = a.row_centre[row];
    const int blk = a.row_block[row];
    const int s = a.row_sample[row];
    const int l = a.block_l[blk];
    const int t = a.block_species[blk];
    const int width = (2 * l + 1) * a.nmax;
    const int64_t src = ((int64_t)c * a.n_species + t);
    const int start = l * l * a.nmax;
    for (int q = threadIdx.x; q < width; q += blockDim.x)
        a.out[a.off_values[blk] + (int64_t)s * width + q] = a.coef[src * K + start + q];
    if (do_strain) {
        for (int q = threadIdx.x; q < 9 * width; q += blockDim.x) {
            int x = q / width, w = q - x * width;
            a.out[a.off_strain[blk] + (int64_t)s * 9 * width + q] = a.strain[(src * 9 + x) * K + start + w];
        }
    }
    if (do_cell) {
        for (int q = threadIdx.x; q < 9 * width; q += blockDim.x) {
            int x = q / width, w = q - x * width;
            a.out[a.off_cell[blk] + (int64_t)s * 9 * width + q] = a.cellg[(src * 9 + x) * K + start + w];
        }
    }
}

// positions gradient rows: self gradient for the centre, sum over the pairs
// between centre and neighbour otherwise (spherical_expansion.rs:468-521)
__global__ void se_output_gradients_kernel(SeOutArgs a) {
    const int64_t row = blockIdx.x;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    const int blk = a.grad_block[row];
    const int l = a.block_l[blk];
    const int t = a.block_species[blk];
    const int c = a.grad_centre[row];
    const int j = a.grad_atom[row];
    const int width = (2 * l + 1) * a.nmax;
    const int start = l * l * a.nmax;
    const double sign_l = (l & 1) ? -1.0 : 1.0;
    double* out = a.out + a.off_positions[blk] + a.grad_row[row] * 3 * width;
    for (int q = threadIdx.x; q < 3 * width; q += blockDim.x) {
        int x = q / width, w = q - x * width;
        double v;
        if (c == j) {
            v = a.self_grad[(((int64_t)c * a.n_species + t) * 3 + x) * K + start + w];
        } else {
            v = 0.0;
            for (int d = a.grad_d0[row]; d < a.grad_d1[row]; d++) {
                int32_t code = a.dir_code[d];
                int64_t p = code >> 1;
                double factor = (code & 1) ? -sign_l : 1.0;
                v += factor * a.pair_grad[(p * 3 + x) * K + start + w];
            }
        }
        out[q] = v;
    }
}

}  // namespace

void launch_pair_features(const DevicePairs& pairs, const DeviceRadial& radial, const DeviceYlm& ylm,
                          const CutoffParams& cut, const FeatureLayout& layout, double* features, int32_t* status,
                          cudaStream_t stream) {
    if (pairs.count == 0) return;
    int threads = 64;
    int blocks = (int)((pairs.count + threads - 1) / threads);
    if (ylm.lmax <= LMAX_SMALL) {
        pair_features_kernel<LMAX_SMALL><<<blocks, threads, 0, stream>>>(pairs, radial, ylm, cut, layout, features, status);
    } else {
        pair_features_kernel<LMAX_LARGE><<<blocks, threads, 0, stream>>>(pairs, radial, ylm, cut, layout, features, status);
    }
    CUDA_CHECK(cudaGetLastError());
}

void launch_se_accumulate(const SeArgs& args, cudaStream_t stream) {
    if (args.n_centres == 0) return;
    int K = args.layout.L2 * args.layout.nmax;
    int threads = std::max(SE_CHUNK, std::min(256, (K + 31) / 32 * 32));
    const bool grad = args.layout.with_grad;
    const bool p = grad && args.do_positions, st = grad && args.do_strain, ce = grad && args.do_cell;
    const unsigned blocks = (unsigned)(args.n_centres * args.n_species);
#define SE_LAUNCH(P, ST, CE) se_accumulate_kernel<P, ST, CE><<<blocks, threads, 0, stream>>>(args)
    if (!p && !st && !ce) SE_LAUNCH(false, false, false);
    else if (p && !st && !ce) SE_LAUNCH(true, false, false);
    else if (p && st && !ce) SE_LAUNCH(true, true, false);
    else if (p && st && ce) SE_LAUNCH(true, true, true);
    else if (p && !st && ce) SE_LAUNCH(true, false, true);
    else if (!p && st && !ce) SE_LAUNCH(false, true, false);
    else if (!p && !st && ce) SE_LAUNCH(false, false, true);
    else SE_LAUNCH(false, true, true);
#undef SE_LAUNCH
    CUDA_CHECK(cudaGetLastError());
}

namespace {
int fused_state = -1;  // -1: not read from the environment yet
}

bool se_fused_enabled() {
    if (fused_state < 0) {
        const char* env = std::getenv("FEATOMIC_B200_FUSED_SE");
        fused_state = (env && env[0] == '0') ? 0 : 1;
    }
    return fused_state == 1;
}

void set_se_fused_enabled(bool enabled) { fused_state = enabled ? 1 : 0; }

bool se_fused_supported(const FeatureLayout& layout, const DeviceRadial& radial) {
    const size_t bytes = sizeof(double) * fused_shared_doubles(layout.lmax, layout.nmax, layout.with_grad);
    const int items = layout.L2 * ((layout.nmax + 1) / 2);
    return radial.splined && layout.lmax <= LMAX_SMALL && items <= 256 && bytes <= 160 * 1024;
}

void launch_se_fused(const SeArgs& args, const DevicePairs& pairs, const DeviceRadial& radial, const DeviceYlm& ylm,
                     const CutoffParams& cut, cudaStream_t stream) {
    if (args.n_centres == 0) return;
    const FeatureLayout& L = args.layout;
    const int items = L.L2 * ((L.nmax + 1) / 2);
    const int threads = std::max(32, (items + 31) / 32 * 32);
    const size_t smem = sizeof(double) * fused_shared_doubles(L.lmax, L.nmax, L.with_grad);
    const bool grad = L.with_grad;
    const bool p = grad && args.do_positions, st = grad && args.do_strain, ce = grad && args.do_cell;
    const unsigned blocks = (unsigned)(args.n_centres * args.n_species);
#define SE_FUSED(P, ST, CE)                                                                                           \
    do {                                                                                                              \
        CUDA_CHECK(cudaFuncSetAttribute(se_fused_kernel<P, ST, CE>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                        (int)smem));                                                                  \
        se_fused_kernel<P, ST, CE><<<blocks, threads, smem, stream>>>(args, pairs, radial, ylm, cut);                 \
    } while (0)
    if (!p && !st && !ce) SE_FUSED(false, false, false);
    else if (p && !st && !ce) SE_FUSED(true, false, false);
    else if (p && st && !ce) SE_FUSED(true, true, false);
    else if (p && st && ce) SE_FUSED(true, true, true);
    else if (p && !st && ce) SE_FUSED(true, false, true);
    else if (!p && st && !ce) SE_FUSED(false, true, false);
    else if (!p && !st && ce) SE_FUSED(false, false, true);
    else SE_FUSED(false, true, true);
#undef SE_FUSED
    CUDA_CHECK(cudaGetLastError());
}

namespace {

// One warp per direction d = 2 pair + reversed.  The pair contribution of
// spherical_expansion_pair.rs:323-422 from the pair record, reversed by
// PairContribution::inverse_pair (:130-163: values x (-1)^l, gradients x
// -(-1)^l, vector and shifts negated), written like accumulate_in_block
// (:424-540) into rows that no other direction touches: values; positions
// rows first -= g, second += g (one row, left at zero, for an i-i image);
// strain vector[x1] g[x2]; cell shift[abc] g[xyz].  Each row receives one
// contribution, so the sums of the reference reduce to these stores.
template <bool POS, bool STRAIN, bool CELL>
__global__ void __launch_bounds__(256) by_pair_kernel(ByPairArgs a) {
    constexpr bool GRAD = POS || STRAIN || CELL;
    const int warps = blockDim.x >> 5, lane = threadIdx.x & 31;
    const int64_t d = (int64_t)blockIdx.x * warps + (threadIdx.x >> 5);
    if (d >= a.n_dirs) return;
    const FeatureLayout L = a.layout;
    const int64_t p = d >> 1;
    const bool inv = d & 1;
    const double* __restrict__ F = a.features + p * L.stride;
    const double f = F[0];
    const int N = L.nmax;
    const int K = L.L2 * N;
    const int blk0 = a.dir_block0[d];
    const int64_t row0 = a.dir_row0[d], row1 = a.dir_row1[d];
    const int64_t grow = GRAD ? a.dir_grow[d] : 0;
    const bool same_atom = a.pairs.first[p] == a.pairs.second[p];
    double fg = 0.0, rinv = 1.0, u[3] = {0.0, 0.0, 0.0}, vd[3] = {0.0, 0.0, 0.0}, sd[3] = {0.0, 0.0, 0.0};
    if (GRAD) {
        fg = F[1];
        rinv = 1.0 / F[2];  // multiplied into the angular term, as in se_fused_kernel
#pragma unroll
        for (int x = 0; x < 3; x++) {
            u[x] = F[3 + x];
            vd[x] = inv ? -a.pairs.vector[3 * p + x] : a.pairs.vector[3 * p + x];
            sd[x] = (double)(inv ? -a.pairs.shift[3 * p + x] : a.pairs.shift[3 * p + x]);
        }
    }
    for (int q = lane; q < K; q += 32) {
        const int lm = q / N, n = q - lm * N;
        int l = (int)sqrt((double)lm);
        while (l * l > lm) l--;
        while ((l + 1) * (l + 1) <= lm) l++;
        const int mm = lm - l * l, w = 2 * l + 1;
        const double m1 = (l & 1) ? -1.0 : 1.0;
        const int blk = blk0 + l;
        const int64_t row = l == 0 ? row0 : row1;
        const double Yv = F[L.off_y + lm];
        const double Rv = F[L.off_r + l * N + n];
        double val = f * Yv * Rv;
        if (inv) val *= m1;
        a.out[a.off_values[blk] + (row * w + mm) * N + n] = val;
        if (!GRAD) continue;
        const double dR = F[L.off_dr + l * N + n];
        double g[3];
#pragma unroll
        for (int x = 0; x < 3; x++) {
            const double dY = F[L.off_dy + x * L.L2 + lm];
            g[x] = fg * u[x] * Rv * Yv + f * dR * u[x] * Yv + f * Rv * dY * rinv;
            if (inv) g[x] *= -m1;
        }
        if (POS && !same_atom) {
            double* o = a.out + a.off_positions[blk];
#pragma unroll
            for (int x = 0; x < 3; x++) {
                o[((grow * 3 + x) * w + mm) * N + n] = 0.0 - g[x];
                o[(((grow + 1) * 3 + x) * w + mm) * N + n] = g[x];
            }
        }
        if (STRAIN) {
            double* o = a.out + a.off_strain[blk] + row * 9 * w * N + mm * N + n;
#pragma unroll
            for (int x1 = 0; x1 < 3; x1++)
#pragma unroll
                for (int x2 = 0; x2 < 3; x2++) o[(x1 * 3 + x2) * w * N] = vd[x1] * g[x2];
        }
        if (CELL) {
            double* o = a.out + a.off_cell[blk] + row * 9 * w * N + mm * N + n;
#pragma unroll
            for (int x1 = 0; x1 < 3; x1++)
#pragma unroll
                for (int x2 = 0; x2 < 3; x2++) o[(x1 * 3 + x2) * w * N] = sd[x1] * g[x2];
        }
    }
}

// self pairs (i, i, 0 0 0) of the l = 0 blocks: the centre's own density
// (spherical_expansion_pair.rs:222-313)
__global__ void by_pair_self_kernel(ByPairArgs a, int nmax) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n_self * nmax) return;
    const int64_t s = k / nmax;
    const int n = (int)(k - s * nmax);
    a.out[a.off_values[a.self_block[s]] + a.self_row[s] * nmax + n] = a.self_contribution[n];
}

}  // namespace

void launch_by_pair(const ByPairArgs& args, bool positions, bool strain, bool cell, cudaStream_t stream) {
    if (args.n_dirs > 0) {
        const int warps = 8;
        const unsigned blocks = (unsigned)((args.n_dirs + warps - 1) / warps);
        const int which = (positions ? 1 : 0) | (strain ? 2 : 0) | (cell ? 4 : 0);
        switch (which) {
            case 0: by_pair_kernel<false, false, false><<<blocks, 32 * warps, 0, stream>>>(args); break;
            case 1: by_pair_kernel<true, false, false><<<blocks, 32 * warps, 0, stream>>>(args); break;
            case 2: by_pair_kernel<false, true, false><<<blocks, 32 * warps, 0, stream>>>(args); break;
            case 3: by_pair_kernel<true, true, false><<<blocks, 32 * warps, 0, stream>>>(args); break;
            case 4: by_pair_kernel<false, false, true><<<blocks, 32 * warps, 0, stream>>>(args); break;
            case 5: by_pair_kernel<true, false, true><<<blocks, 32 * warps, 0, stream>>>(args); break;
            case 6: by_pair_kernel<false, true, true><<<blocks, 32 * warps, 0, stream>>>(args); break;
            default: by_pair_kernel<true, true, true><<<blocks, 32 * warps, 0, stream>>>(args); break;
        }
        CUDA_CHECK(cudaGetLastError());
    }
    if (args.n_self > 0) {
        const int64_t items = args.n_self * args.layout.nmax;
        by_pair_self_kernel<<<(unsigned)((items + 255) / 256), 256, 0, stream>>>(args, args.layout.nmax);
        CUDA_CHECK(cudaGetLastError());
    }
}

void launch_se_output(const SeOutArgs& args, bool positions, bool strain, bool cell, cudaStream_t stream) {
    if (args.n_rows > 0) {
        se_output_rows_kernel<<<(unsigned)args.n_rows, 128, 0, stream>>>(args, strain, cell);
        CUDA_CHECK(cudaGetLastError());
    }
    if (positions && args.n_grad_rows > 0) {
        se_output_gradients_kernel<<<(unsigned)args.n_grad_rows, 128, 0, stream>>>(args);
        CUDA_CHECK(cudaGetLastError());
    }
}

// rows and property columns of one output array for a selection
__global__ void gather_rows_kernel(const double* __restrict__ src, const int64_t* __restrict__ rows, int64_t n_rows,
                                   int64_t inner, int64_t src_props, const int64_t* __restrict__ props,
                                   int64_t n_props, double* __restrict__ dst) {
    const int64_t total = n_rows * inner * n_props;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i % n_props, rm = i / n_props;
        const int64_t m = rm % inner, r = rows[rm / inner];
        dst[i] = r < 0 ? 0.0 : src[(r * inner + m) * src_props + props[p]];
    }
}

void launch_gather_rows(const double* src, const int64_t* rows, int64_t n_rows, int64_t inner, int64_t src_props,
                        const int64_t* props, int64_t n_props, double* dst) {
    const int64_t total = n_rows * inner * n_props;
    if (total == 0) return;
    const int threads = 256;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + threads - 1) / threads, 148 * 16);
    gather_rows_kernel<<<blocks, threads>>>(src, rows, n_rows, inner, src_props, props, n_props, dst);
}

}  // namespace fb200

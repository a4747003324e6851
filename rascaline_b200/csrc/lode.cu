// LODE spherical expansion (featomic/src/calculators/lode/spherical_expansion.rs)
// on the GPU.  For every periodic system:
//
//   host    k-vectors of the cell inside the k_cutoff ball (one of each +-k
//           pair), the density's Fourier transform f(k) and the radial
//           integral R_nl(|k|) (spline or analytic) per k-vector
//   kernel  lode_projection_kernel: T[k][lm][n] = R_nl(|k|) Y_lm(k^)
//   kernel  lode_phases_kernel: cos(k.r_i), sin(k.r_i) for every atom and k
//   kernel  lode_type_sums_kernel: the same summed over the atoms of each type
//   kernel  lode_values_kernel: one CTA per (centre, neighbour type), every
//           thread a few (l, m, n) coefficients, sum over k of
//           4 pi / V f(k) S_i^t(k) T[k][lm][n] with the structure factor
//           S_i^t (real part for even l, imaginary for odd l)
//   kernel  lode_gradients_kernel: one CTA per gradient row (centre i,
//           atom j, neighbour type t), the pair factor of (i, j) against the
//           same table times the k-vector
//
// Every coefficient is summed over k in featomic's order with featomic's
// expressions (the sign (-1)^{l/2}, (-1)^{(l+1)/2} applied at the end, which
// is exact), then the central-atom and k = 0 terms in featomic's order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <set>

#include "lode.hpp"
#include "pair_math.cuh"
#include "soap_math.cuh"

namespace fb200 {

// ---------------------------------------------------------------------------
// host math
// ---------------------------------------------------------------------------
namespace {
constexpr double EULER_GAMMA = 0.5772156649015329;
}

// E1(x) = int_x^inf e^-t / t dt: power series -gamma - ln x - sum (-x)^k /
// (k k!) for x <= 1 (Abramowitz & Stegun 5.1.11), continued fraction
// e^-x / (x + 1 - 1 / (x + 3 - 4 / (x + 5 - ...))) evaluated by the modified
// Lentz method beyond (A&S 5.1.22)
double exp1(double x) {
    if (x == 0.0) return INFINITY;
    if (!(x > 0.0)) return NAN;
    if (x <= 1.0) {
        double term = 1.0, sum = 0.0;
        for (int k = 1; k < 200; k++) {
            term *= -x / (double)k;
            const double add = term / (double)k;
            sum += add;
            if (std::fabs(add) <= 1e-17 * std::fabs(sum)) break;
        }
        return -EULER_GAMMA - std::log(x) - sum;
    }
    const double tiny = 1e-300;
    double b = x + 1.0, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 10000; i++) {
        const double a = -(double)i * (double)i;
        b += 2.0;
        d = 1.0 / (a * d + b);
        c = b + a / c;
        const double del = c * d;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-16) break;
    }
    return h * std::exp(-x);
}

// Ei(x) = -E1(-x) for x < 0; power series gamma + ln x + sum x^k / (k k!)
// for 0 < x <= 40, asymptotic e^x / x sum k! / x^k beyond
double expi(double x) {
    if (x == 0.0) return -INFINITY;
    if (x < 0.0) return -exp1(-x);
    if (x <= 40.0) {
        double term = 1.0, sum = 0.0;
        for (int k = 1; k < 500; k++) {
            term *= x / (double)k;
            const double add = term / (double)k;
            sum += add;
            if (std::fabs(add) <= 1e-17 * std::fabs(sum)) break;
        }
        return EULER_GAMMA + std::log(x) + sum;
    }
    double term = 1.0, sum = 1.0;
    for (int k = 1; k <= 20; k++) {
        term *= (double)k / x;
        sum += term;
    }
    return std::exp(x) / x * sum;
}

// 2F1(1, b; c; z) = sum_k (b)_k / (c)_k z^k, every term positive for
// b, c > 0 and 0 <= z < 1
double hyp2f1_one(double b, double c, double z) {
    double term = 1.0, sum = 1.0;
    for (int k = 0; k < 2000000; k++) {
        term *= (b + (double)k) / (c + (double)k) * z;
        sum += term;
        if (term <= 1e-17 * sum) break;
    }
    return sum;
}

// math/k_vectors.rs:19-87: the reciprocal cell 2 pi (H^T)^-1, lattice points
// (n1, n2, n3) in featomic's order with |k| < k_cutoff, n1 > 0, or n1 = 0 and
// n2 > 0, or n1 = n2 = 0 and n3 > 0
KVectors compute_k_vectors(const double cell[9], double k_cutoff) {
    // inverse of the transposed cell (rows of `cell` are the cell vectors)
    const double* H = cell;
    double T[9] = {H[0], H[3], H[6], H[1], H[4], H[7], H[2], H[5], H[8]};
    const double det = T[0] * (T[4] * T[8] - T[5] * T[7]) - T[1] * (T[3] * T[8] - T[5] * T[6]) +
                       T[2] * (T[3] * T[7] - T[4] * T[6]);
    if (det == 0.0) throw invalid_parameter("LODE can only be used with periodic systems");
    double inv[9] = {(T[4] * T[8] - T[5] * T[7]) / det, (T[2] * T[7] - T[1] * T[8]) / det,
                     (T[1] * T[5] - T[2] * T[4]) / det, (T[5] * T[6] - T[3] * T[8]) / det,
                     (T[0] * T[8] - T[2] * T[6]) / det, (T[2] * T[3] - T[0] * T[5]) / det,
                     (T[3] * T[7] - T[4] * T[6]) / det, (T[1] * T[6] - T[0] * T[7]) / det,
                     (T[0] * T[4] - T[1] * T[3]) / det};
    double R[9];
    for (int k = 0; k < 9; k++) R[k] = 2.0 * M_PI * inv[k];
    const double* b1 = R;
    const double* b2 = R + 3;
    const double* b3 = R + 6;
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const double m00 = dot(b1, b1), m11 = dot(b2, b2), m22 = dot(b3, b3);
    const double m01 = dot(b1, b2), m02 = dot(b1, b3), m12 = dot(b2, b3);
    const double volume = R[0] * (R[4] * R[8] - R[5] * R[7]) - R[1] * (R[3] * R[8] - R[5] * R[6]) +
                          R[2] * (R[3] * R[7] - R[4] * R[6]);
    const long n1_max = (long)(std::sqrt(m11 * m22 - m12 * m12) / volume * k_cutoff);
    const long n2_max = (long)(std::sqrt(m22 * m00 - m02 * m02) / volume * k_cutoff);
    const long n3_max = (long)(std::sqrt(m00 * m11 - m01 * m01) / volume * k_cutoff);
    const double cutoff2 = k_cutoff * k_cutoff;
    KVectors out;
    auto add = [&](long n1, long n2, long n3) {
        double k[3];
        for (int x = 0; x < 3; x++) k[x] = (double)n1 * b1[x] + (double)n2 * b2[x] + (double)n3 * b3[x];
        const double n2k = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        if (n2k < cutoff2) {
            const double norm = std::sqrt(n2k);
            out.norm.push_back(norm);
            for (int x = 0; x < 3; x++) out.direction.push_back(k[x] / norm);
        }
    };
    for (long n3 = 1; n3 <= n3_max; n3++) add(0, 0, n3);
    for (long n2 = 1; n2 <= n2_max; n2++)
        for (long n3 = -n3_max; n3 <= n3_max; n3++) add(0, n2, n3);
    for (long n1 = 1; n1 <= n1_max; n1++)
        for (long n2 = -n2_max; n2 <= n2_max; n2++)
            for (long n3 = -n3_max; n3 <= n3_max; n3++) add(n1, n2, n3);
    return out;
}

namespace {

// lode/radial_integral/gto.rs:62-131 before the orthonormalisation:
// sqrt(pi / 2) sigma_n^{n+3} sqrt2^n (k sigma_n / sqrt2)^l G(a, b, -k^2 sigma_n^2 / 2)
// with G = Gamma(a) / Gamma(b) 1F1(a, b, z), a = (n + l + 3) / 2, b = l + 3/2,
// and its derivative in k
void lode_radial_raw(const LodeTables& t, int l, double k, double* values, double* grads) {
    const double global = std::sqrt(M_PI) / M_SQRT2;
    const int N = t.h.nmax();
    for (int n = 0; n < N; n++) {
        const double sigma = t.widths[n];
        const double ksig = k * sigma / M_SQRT2;
        const double factor = global * soap::powi(sigma, n + 3) * soap::powi(M_SQRT2, n) * soap::powi(ksig, l);
        const double kns2 = -k * sigma * sigma;
        const double z = 0.5 * k * kns2;
        const double a = 0.5 * (double)(n + l + 3), b = (double)l + 1.5;
        const double ratio = soap::gamma_fn(a) / soap::gamma_fn(b);
        values[n] = ratio * soap::hyp1f1(a, b, z);
        if (grads) grads[n] = ratio * (a / b * soap::hyp1f1(a + 1.0, b + 1.0, z));
        values[n] *= factor;
        if (grads) {
            grads[n] *= kns2 * factor;
            grads[n] += (double)l / k * values[n];
        }
    }
    // at k = 0 the expression above is 0 / 0 for the gradients: zero except
    // for l = 1 (gto.rs:107-124)
    if (k == 0.0 && grads) {
        for (int n = 0; n < N; n++) grads[n] = 0.0;
        if (l == 1) {
            for (int n = 0; n < N; n++) {
                const double sigma = t.widths[n];
                const double a = 0.5 * (double)(n + l) + 1.5, b = 2.5;
                const double factor = global * soap::powi(sigma, n + l + 3) * soap::powi(M_SQRT2, n - l);
                grads[n] = soap::gamma_fn(a) / soap::gamma_fn(b) * factor;
            }
        }
    }
}

void orthonormalize(const LodeTables& t, double* v) {
    const int N = t.h.nmax();
    double tmp[64];
    for (int k = 0; k < N; k++) {
        double s = 0.0;
        for (int n = 0; n < N; n++) s += v[n] * t.ortho[(size_t)k * N + n];
        tmp[k] = s;
    }
    for (int k = 0; k < N; k++) v[k] = tmp[k];
}

}  // namespace

void LodeTables::radial(int l, double k, double* v, double* g) const {
    const int N = h.nmax();
    if (!positions.empty()) {
        const double* pos = positions.data() + knot_offset[l];
        const int count = knot_count[l];
        const int kk = soap::spline_interval(pos, count, k);
        const soap::HermiteWeights w = soap::hermite_weights(pos[kk], pos[kk + 1], k);
        const double* pv = values.data() + ((size_t)knot_offset[l] + kk) * N;
        const double* pd = derivs.data() + ((size_t)knot_offset[l] + kk) * N;
        for (int n = 0; n < N; n++) {
            v[n] = soap::hermite_value(w, pv[n], pd[n], pv[N + n], pd[N + n]);
            if (g) g[n] = soap::hermite_derivative(w, pv[n], pd[n], pv[N + n], pd[N + n]);
        }
        return;
    }
    lode_radial_raw(*this, l, k, v, g);
    orthonormalize(*this, v);
    if (g) orthonormalize(*this, g);
}

// lode/spherical_expansion.rs:276-335
double LodeTables::density_fourier(double k) const {
    const int p = h.exponent;
    const double s2 = h.smearing * h.smearing;
    if (p == 0) return std::pow(4.0 * M_PI * s2, 0.75) * std::exp(-0.5 * k * k * s2);
    if (p == 1) {
        const double k2 = k * k;
        return 4.0 * M_PI * (std::exp(-0.5 * k2 * s2) / k2);
    }
    const double p_eff = 3.0 - (double)p;
    const double factor = std::pow(M_PI, 1.5) * std::pow(2.0 * s2, 0.5 * p_eff) / soap::gamma_fn(0.5 * (double)p);
    const double x = 0.5 * (k * k) * s2;
    const double sqrt_pi = std::sqrt(M_PI);
    double value = 0.0;
    switch (p) {
    case 2: value = std::sqrt(M_PI / x) * std::erfc(std::sqrt(x)); break;
    case 3: value = -expi(-x); break;
    case 4: value = 2.0 * (std::exp(-x) - std::sqrt(M_PI * x) * std::erfc(std::sqrt(x))); break;
    case 5: value = std::exp(-x) + x * expi(-x); break;
    case 6:
        value = ((2.0 - 4.0 * x) * std::exp(-x) + 4.0 * sqrt_pi * std::pow(x, 1.5) * std::erfc(std::sqrt(x))) / 3.0;
        break;
    case 7: value = (1.0 - x) * std::exp(-x) / 2.0 - x * x / 2.0 * expi(-x); break;
    case 8:
        value = -2.0 / 15.0 * ((-3.0 + 2.0 * x - 4.0 * x * x) * std::exp(-x) +
                               4.0 * sqrt_pi * std::pow(x, 2.5) * std::erfc(std::sqrt(x)));
        break;
    case 9: value = (x * x - x + 2.0) * std::exp(-x) / 6.0 + x * x * x / 6.0 * expi(-x); break;
    default: throw invalid_parameter("potential_exponent = " + std::to_string(p) + " is not implemented");
    }
    return factor * value;
}

LodeTables build_lode_tables(const LodeHypers& h) {
    LodeTables t;
    t.h = h;
    const int N = h.nmax();
    t.widths = gto_basis_widths(N, h.radius);
    t.ortho = gto_basis_orthonormalization(N, h.radius);
    if (h.splined) {
        // one spline per angular channel over [0, k_cutoff] (radial_integral/
        // spline.rs:28-68, featomic/src/math/splines.rs:79-193)
        std::vector<double> pos, val, der;
        for (int l = 0; l <= h.max_angular; l++) {
            build_spline_knots([&](double k, double* v, double* g) {
                lode_radial_raw(t, l, k, v, g);
                orthonormalize(t, v);
                orthonormalize(t, g);
            }, h.k_cutoff, N, N, h.spline_accuracy, pos, val, der);
            t.knot_offset.push_back((int32_t)t.positions.size());
            t.knot_count.push_back((int32_t)pos.size());
            t.positions.insert(t.positions.end(), pos.begin(), pos.end());
            t.values.insert(t.values.end(), val.begin(), val.end());
            t.derivs.insert(t.derivs.end(), der.begin(), der.end());
        }
    }
    // central-atom contribution <n 0 0> (gto.rs:133-181), from the analytic
    // expressions whether or not the integral is splined
    std::vector<double> c(N);
    const double s = h.smearing, p = (double)h.exponent;
    for (int n = 0; n < N; n++) {
        const double n_eff = 0.5 * (3.0 + (double)n);
        if (h.exponent == 0) {
            const double factor = std::pow(M_PI, -0.25) / std::pow(s * s, 0.75);
            const double alpha = 0.5 * (1.0 / (s * s) + 1.0 / (t.widths[n] * t.widths[n]));
            c[n] = factor * soap::gamma_fn(n_eff) / std::pow(alpha, n_eff);
        } else {
            const double factor = 2.0 * std::sqrt(4.0 * M_PI) / soap::gamma_fn(p / 2.0) / p;
            const double q = s / t.widths[n];
            const double hyparg = 1.0 / (1.0 + q * q);
            c[n] = factor * std::pow(2.0, (1.0 + (double)n - p) / 2.0) * soap::powi(s, 3 + n - h.exponent) *
                   soap::gamma_fn(n_eff) * hyp2f1_one(n_eff, (p + 2.0) / 2.0, hyparg) * std::pow(hyparg, n_eff);
        }
    }
    orthonormalize(t, c.data());
    t.center = c;
    // k = 0 term (spherical_expansion.rs:337-376): factor times R_n0(0)
    double factor = 0.0;
    if (h.exponent == 0) {
        const double s2 = s * s;
        factor = std::pow(2.0 * M_PI * s2, 1.5) / std::pow(M_PI * s2, 0.75) / std::sqrt(4.0 * M_PI);
    } else if (h.exponent > 3) {
        const double p_eff = 3.0 - p;
        factor = 0.5 * M_PI * std::pow(2.0, p_eff) / soap::gamma_fn(0.5 * p) * std::pow(2.0, (p - 1.0) / 2.0) / -p_eff *
                 std::pow(s, -p_eff) / std::pow(s, 2.0 * p - 6.0);
    }
    std::vector<double> r0(N);
    t.radial(0, 0.0, r0.data(), nullptr);
    t.k0.resize(N);
    for (int n = 0; n < N; n++) t.k0[n] = factor * r0[n];
    return t;
}

}  // namespace fb200

namespace fb200 {

namespace {

constexpr int LODE_LCAP = 16;
constexpr int LODE_CHUNK = 128;  // k-vectors staged in shared memory at a time
constexpr int LODE_GROUP = 8;    // centres of one neighbour type per values CTA
constexpr int LODE_THREADS = 128;
constexpr int LODE_Q = 4;        // coefficients per thread

__host__ __device__ inline int l_of(int lm) {
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) l++;
    return l;
}

// T[k][lm N + n] = R_nl(|k|) Y_lm(k^) (spherical_expansion.rs:226-274):
// one thread per k-vector
__global__ void lode_projection_kernel(int K, int L, int N, const double* __restrict__ dir,
                                       const double* __restrict__ radial, DeviceYlm ylm, double* __restrict__ T) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    double Y[(LODE_LCAP + 1) * (LODE_LCAP + 1)];
    ylm_compute<double, LODE_LCAP>(ylm, dir[3 * k], dir[3 * k + 1], dir[3 * k + 2], Y, nullptr, nullptr, nullptr);
    const int L2 = (L + 1) * (L + 1);
    double* out = T + (size_t)k * L2 * N;
    for (int lm = 0; lm < L2; lm++) {
        const int l = l_of(lm);
        const double* R = radial + ((size_t)k * (L + 1) + l) * N;
        for (int n = 0; n < N; n++) out[lm * N + n] = R[n] * Y[lm];
    }
}

// cos and sin of k.r for every (atom, k) (spherical_expansion.rs:92-111),
// k.r = (|k| k^) . r in featomic's order
__global__ void lode_phases_kernel(int n_atoms, int K, const double* __restrict__ positions,
                                   const double* __restrict__ kvec, double* __restrict__ C, double* __restrict__ S) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n_atoms * K) return;
    const int i = (int)(idx / K), k = (int)(idx - (int64_t)i * K);
    const double* p = positions + 3 * i;
    const double* q = kvec + 3 * k;
    const double s = q[0] * p[0] + q[1] * p[1] + q[2] * p[2];
    double sn, cs;
    sincos(s, &sn, &cs);
    C[idx] = cs;
    S[idx] = sn;
}

// sum of cos(k.r_j), sin(k.r_j) over the atoms j of each type, in atom order
// (spherical_expansion.rs:125-141)
__global__ void lode_type_sums_kernel(int n_atoms, int K, int n_species, const int32_t* __restrict__ species,
                                      const double* __restrict__ C, const double* __restrict__ S,
                                      double* __restrict__ Ct, double* __restrict__ St) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n_species * K) return;
    const int t = idx / K, k = idx - t * K;
    double sc = 0.0, ss = 0.0;
    for (int j = 0; j < n_atoms; j++) {
        if (species[j] != t) continue;
        sc += C[(size_t)j * K + k];
        ss += S[(size_t)j * K + k];
    }
    Ct[idx] = sc;
    St[idx] = ss;
}

struct LodeArgs {
    int n_atoms, K, S, L, N;
    const int32_t* species;     // [n_atoms] species index of the system's atoms
    const double *C, *Sn;       // [n_atoms][K]
    const double *Ct, *St;      // [S][K]
    const double* gdf;          // [K] 4 pi / V f(k)
    const double* T;            // [K][(L + 1)^2][N]
    const double* kvec;         // [K][3] |k| k^ (unused by the values)
    const double* knorm;        // [K]
    const double* kdir;         // [K][3]
    // values
    const int32_t* row;         // [n_atoms][S] sample row of atom i in the blocks (type_i, t), -1: none
    const int64_t* off_values;  // [S][S][L + 1] offset of each block's values
    const int32_t* type_count;  // [S] atoms of each type in the system
    const double* center;       // [N] central-atom contribution
    const double* k0;           // [N] 4 pi / V times the k = 0 term
    double center_factor;       // 1 - center_atom_weight
    int add_k0;
    // gradients
    const int32_t* tasks;       // [n_tasks][4] (i, j, t, row)
    const int64_t* off_positions;
    double* out;
};

__device__ inline double lode_phase(int l) {
    // spherical_expansion.rs:667-671
    return (l % 2 == 0) ? ((l / 2) % 2 == 0 ? 1.0 : -1.0) : (((l + 1) / 2) % 2 == 0 ? 1.0 : -1.0);
}

// values (spherical_expansion.rs:616-723): CTA (neighbour type t, group of
// LODE_GROUP centres of one type, tile of coefficients); each thread sums
// LODE_Q coefficients of every centre of the group over k
__global__ void __launch_bounds__(LODE_THREADS) lode_values_kernel(LodeArgs a, const int32_t* __restrict__ groups,
                                                                    int n_groups) {
    const int t = blockIdx.x % a.S;
    const int g = blockIdx.x / a.S;
    if (g >= n_groups) return;
    const int32_t* centres = groups + (size_t)g * LODE_GROUP;  // -1 padded, all of one type
    const int L2 = (a.L + 1) * (a.L + 1), outs = L2 * a.N;
    const int o0 = blockIdx.y * LODE_THREADS * LODE_Q;
    __shared__ double wr[LODE_GROUP][LODE_CHUNK], wi[LODE_GROUP][LODE_CHUNK];
    double acc[LODE_GROUP][LODE_Q];
#pragma unroll
    for (int c = 0; c < LODE_GROUP; c++)
#pragma unroll
        for (int q = 0; q < LODE_Q; q++) acc[c][q] = 0.0;
    int parity[LODE_Q];
#pragma unroll
    for (int q = 0; q < LODE_Q; q++) {
        const int o = o0 + q * LODE_THREADS + threadIdx.x;
        parity[q] = o < outs ? (l_of(o / a.N) & 1) : 0;
    }
    for (int k0 = 0; k0 < a.K; k0 += LODE_CHUNK) {
        const int nk = min(LODE_CHUNK, a.K - k0);
        __syncthreads();
        for (int w = threadIdx.x; w < LODE_GROUP * nk; w += blockDim.x) {
            const int c = w / nk, kk = w - c * nk, k = k0 + kk;
            const int i = centres[c];
            if (i < 0 || a.row[(size_t)i * a.S + t] < 0) {
                wr[c][kk] = 0.0;
                wi[c][kk] = 0.0;
                continue;
            }
            const double ci = a.C[(size_t)i * a.K + k], si = a.Sn[(size_t)i * a.K + k];
            const double ct = a.Ct[(size_t)t * a.K + k], st = a.St[(size_t)t * a.K + k];
            // structure factor per centre (:143-155), real and imaginary part
            const double real = 2.0 * (ci * ct + si * st);
            const double imag = 2.0 * (si * ct - ci * st);
            wr[c][kk] = a.gdf[k] * real;
            wi[c][kk] = a.gdf[k] * imag;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < LODE_Q; q++) {
            const int o = o0 + q * LODE_THREADS + threadIdx.x;
            if (o >= outs) continue;
            const double* Tk = a.T + (size_t)k0 * outs + o;
            const double(*w)[LODE_CHUNK] = parity[q] ? wi : wr;
            int kk = 0;
            // four k-vectors per step: the loads first, then each sum in k order
            for (; kk + 4 <= nk; kk += 4) {
                double tv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) tv[u] = Tk[(size_t)(kk + u) * outs];
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int c = 0; c < LODE_GROUP; c++) acc[c][q] += w[c][kk + u] * tv[u];
            }
            for (; kk < nk; kk++) {
                const double tv = Tk[(size_t)kk * outs];
#pragma unroll
                for (int c = 0; c < LODE_GROUP; c++) acc[c][q] += w[c][kk] * tv;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < LODE_Q; q++) {
        const int o = o0 + q * LODE_THREADS + threadIdx.x;
        if (o >= outs) continue;
        const int lm = o / a.N, n = o - lm * a.N, l = l_of(lm), mi = lm - l * l;
        const double phase = lode_phase(l);
#pragma unroll
        for (int c = 0; c < LODE_GROUP; c++) {
            const int i = centres[c];
            if (i < 0) continue;
            const int r = a.row[(size_t)i * a.S + t];
            if (r < 0) continue;
            const int ti = a.species[i];
            double x = 0.0;
            if (l == 0) {
                // central atom (:378-426), then the k = 0 term once per atom
                // of type t (:635-661)
                if (t == ti) x -= a.center_factor * a.center[n];
                if (a.add_k0)
                    for (int j = 0; j < a.type_count[t]; j++) x += a.k0[n];
            }
            x += phase * acc[c][q];
            const int64_t off = a.off_values[((size_t)ti * a.S + t) * (a.L + 1) + l];
            a.out[off + ((int64_t)r * (2 * l + 1) + mi) * a.N + n] = x;
        }
    }
}

// positions gradients (spherical_expansion.rs:725-873): CTA (gradient row,
// tile of coefficients); the pair factor of (i, j) per k staged in shared
// memory with |k| and k^
__global__ void __launch_bounds__(LODE_THREADS) lode_gradients_kernel(LodeArgs a, int n_tasks) {
    const int task = blockIdx.x;
    if (task >= n_tasks) return;
    const int i = a.tasks[4 * task], j = a.tasks[4 * task + 1], t = a.tasks[4 * task + 2], r = a.tasks[4 * task + 3];
    const int ti = a.species[i];
    const int L2 = (a.L + 1) * (a.L + 1), outs = L2 * a.N;
    const int o0 = blockIdx.y * LODE_THREADS * LODE_Q;
    __shared__ double pe[LODE_CHUNK], po[LODE_CHUNK], kn[LODE_CHUNK], kd[LODE_CHUNK][3];
    double acc[LODE_Q][3];
#pragma unroll
    for (int q = 0; q < LODE_Q; q++) acc[q][0] = acc[q][1] = acc[q][2] = 0.0;
    for (int k0 = 0; k0 < a.K; k0 += LODE_CHUNK) {
        const int nk = min(LODE_CHUNK, a.K - k0);
        __syncthreads();
        for (int kk = threadIdx.x; kk < nk; kk += blockDim.x) {
            const int k = k0 + kk;
            const double ci = a.C[(size_t)i * a.K + k], si = a.Sn[(size_t)i * a.K + k];
            const double cj = a.C[(size_t)j * a.K + k], sj = a.Sn[(size_t)j * a.K + k];
            // real / imaginary part of i e^{i k (r_i - r_j)}
            double even = 2.0 * (si * cj - ci * sj);
            double odd = -2.0 * (ci * cj + si * sj);
            if (i == j) {
                // -sum_{j != i}: from the structure factor per centre
                const double ct = a.Ct[(size_t)t * a.K + k], st = a.St[(size_t)t * a.K + k];
                const double real = 2.0 * (ci * ct + si * st);
                const double imag = 2.0 * (si * ct - ci * st);
                if (t == ti) {
                    even = -(1.0 * imag - even);
                    odd = -(-1.0 * real - odd);
                } else {
                    even = -1.0 * imag;
                    odd = -(-1.0) * real;
                }
            }
            pe[kk] = even * a.gdf[k];
            po[kk] = odd * a.gdf[k];
            kn[kk] = a.knorm[k];
            kd[kk][0] = a.kdir[3 * k];
            kd[kk][1] = a.kdir[3 * k + 1];
            kd[kk][2] = a.kdir[3 * k + 2];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < LODE_Q; q++) {
            const int o = o0 + q * LODE_THREADS + threadIdx.x;
            if (o >= outs) continue;
            const bool oddl = l_of(o / a.N) & 1;
            const double* p = oddl ? po : pe;
            const double* Tk = a.T + (size_t)k0 * outs + o;
            int kk = 0;
            for (; kk + 4 <= nk; kk += 4) {
                double tv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) tv[u] = Tk[(size_t)(kk + u) * outs];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const double s = p[kk + u] * tv[u] * kn[kk + u];
                    acc[q][0] += s * kd[kk + u][0];
                    acc[q][1] += s * kd[kk + u][1];
                    acc[q][2] += s * kd[kk + u][2];
                }
            }
            for (; kk < nk; kk++) {
                const double s = p[kk] * Tk[(size_t)kk * outs] * kn[kk];
                acc[q][0] += s * kd[kk][0];
                acc[q][1] += s * kd[kk][1];
                acc[q][2] += s * kd[kk][2];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < LODE_Q; q++) {
        const int o = o0 + q * LODE_THREADS + threadIdx.x;
        if (o >= outs) continue;
        const int lm = o / a.N, n = o - lm * a.N, l = l_of(lm), mi = lm - l * l;
        const double phase = lode_phase(l);
        const int64_t off = a.off_positions[((size_t)ti * a.S + t) * (a.L + 1) + l];
        for (int x = 0; x < 3; x++)
            a.out[off + (((int64_t)r * 3 + x) * (2 * l + 1) + mi) * a.N + n] = phase * acc[q][x];
    }
}

}  // namespace

}  // namespace fb200

namespace fb200 {

LodeEngine::LodeEngine(const LodeHypers& h) : tables_(build_lode_tables(h)), ylm_(build_ylm_tables(h.max_angular)) {}

LodeEngine::~LodeEngine() {
    for (void* p : table_buffers_) cudaFree(p);
}

void LodeEngine::upload_tables() {
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    if (tables_ready_ && dev == device_) return;
    if (tables_ready_) throw invalid_parameter("a calculator can only be used on the device it first ran on");
    device_ = dev;
    auto putv = [&](const std::vector<double>& v) {
        void* d = nullptr;
        CUDA_CHECK(cudaMalloc(&d, std::max<size_t>(8, v.size() * sizeof(double))));
        if (!v.empty()) CUDA_CHECK(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
        table_buffers_.push_back(d);
        return (const double*)d;
    };
    d_ylm_.lmax = ylm_.lmax;
    d_ylm_.A = putv(ylm_.A);
    d_ylm_.B = putv(ylm_.B);
    d_ylm_.sq_plus = putv(ylm_.sq_plus);
    d_ylm_.sq_minus = putv(ylm_.sq_minus);
    d_ylm_.sq_2l1 = putv(ylm_.sq_2l1);
    d_ylm_.sq_half = putv(ylm_.sq_half);
    d_ylm_.sq_ll1 = putv(ylm_.sq_ll1);
    d_ylm_.inv_ll = putv(ylm_.inv_ll);
    tables_ready_ = true;
}

namespace {

template <typename T>
T* put(DeviceArena& arena, const std::string& name, const std::vector<T>& v, cudaStream_t stream) {
    T* d = arena.alloc<T>(name, (int64_t)v.size());
    if (!v.empty()) CUDA_CHECK(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream));
    return d;
}

Labels labels_xyz() {
    Labels l;
    l.names = {"xyz"};
    l.values = {0, 1, 2};
    return l;
}

}  // namespace

// keys AllTypesPairsKeys x angular channels (spherical_expansion.rs:448-460,
// labels/keys.rs:36-57), samples and gradient samples LongRangeSamplesPerAtom
// (labels/samples/long_range.rs:21-74), then the kernels system by system
std::unique_ptr<TensorMap> LodeEngine::compute(const std::vector<HostSystem>& systems, const GradientOptions& g,
                                               bool device_output, const double* d_positions, cudaStream_t stream) {
    auto t_start = std::chrono::steady_clock::now();
    if (g.strain) throw invalid_parameter("the lode spherical expansion calculator does not support gradients with respect to strain");
    if (g.cell) throw invalid_parameter("the lode spherical expansion calculator does not support gradients with respect to cell");
    upload_tables();
    const LodeHypers& h = tables_.h;
    const int L = h.max_angular, N = h.nmax(), L2 = (L + 1) * (L + 1);

    // species and key pairs
    std::vector<int32_t> types;
    for (auto& s : systems) types.insert(types.end(), s.types.begin(), s.types.end());
    std::sort(types.begin(), types.end());
    types.erase(std::unique(types.begin(), types.end()), types.end());
    const int S = (int)types.size();
    auto species_of = [&](int32_t t) { return (int)(std::lower_bound(types.begin(), types.end(), t) - types.begin()); };
    std::vector<int32_t> pair_present((size_t)S * S, 0);
    std::vector<std::vector<int32_t>> sys_species(systems.size());
    for (size_t s = 0; s < systems.size(); s++) {
        std::vector<int32_t> present(S, 0);
        for (int32_t t : systems[s].types) present[species_of(t)] = 1;
        for (int a = 0; a < S; a++)
            for (int b = 0; b < S; b++)
                if (present[a] && present[b]) pair_present[(size_t)a * S + b] = 1;
        for (int32_t t : systems[s].types) sys_species[s].push_back(species_of(t));
        if (!systems[s].types.empty()) {
            const double* c = systems[s].cell;
            bool zero = true;
            for (int k = 0; k < 9; k++) zero &= c[k] == 0.0;
            if (zero) throw invalid_parameter("LODE can only be used with periodic systems");
        }
    }
    // blocks: pairs (a, b) in order, then l; per pair: samples and gradient rows
    struct PairPlan {
        Labels samples, grad_samples;
        int64_t n_samples = 0, n_grad = 0;
    };
    std::vector<PairPlan> pairs((size_t)S * S);
    std::vector<int32_t> keys_values;
    for (int a = 0; a < S; a++)
        for (int b = 0; b < S; b++) {
            if (!pair_present[(size_t)a * S + b]) continue;
            auto& pp = pairs[(size_t)a * S + b];
            pp.samples.names = {"system", "atom"};
            pp.grad_samples.names = {"sample", "system", "atom"};
            for (int l = 0; l <= L; l++) keys_values.insert(keys_values.end(), {l, 1, types[a], types[b]});
        }
    // per system: sample rows of every (atom, neighbour type) and gradient tasks
    std::vector<std::vector<int32_t>> rows(systems.size()), tasks(systems.size());
    for (size_t s = 0; s < systems.size(); s++) {
        const auto& sp = sys_species[s];
        const int n = (int)sp.size();
        std::vector<int32_t> count(S, 0);
        for (int32_t t : sp) count[t]++;
        rows[s].assign((size_t)n * S, -1);
        for (int i = 0; i < n; i++)
            for (int t = 0; t < S; t++) {
                if (!count[t]) continue;
                auto& pp = pairs[(size_t)sp[i] * S + t];
                const int32_t r = (int32_t)pp.n_samples++;
                rows[s][(size_t)i * S + t] = r;
                pp.samples.values.insert(pp.samples.values.end(), {(int32_t)s, i});
                if (!g.positions) continue;
                for (int j = 0; j < n; j++) {
                    if (sp[j] != t && j != i) continue;
                    tasks[s].insert(tasks[s].end(), {i, j, t, (int32_t)pp.n_grad});
                    pp.grad_samples.values.insert(pp.grad_samples.values.end(), {r, (int32_t)s, j});
                    pp.n_grad++;
                }
            }
    }
    // the samples of a block are ordered by system, then atom: rows above
    // were numbered per (atom, type) in that order within each system
    // offsets: per block values, then positions gradients
    std::vector<int64_t> off_values((size_t)S * S * (L + 1), -1), off_positions((size_t)S * S * (L + 1), -1);
    int64_t total = 0;
    for (int a = 0; a < S; a++)
        for (int b = 0; b < S; b++) {
            if (!pair_present[(size_t)a * S + b]) continue;
            const auto& pp = pairs[(size_t)a * S + b];
            for (int l = 0; l <= L; l++) {
                const size_t k = ((size_t)a * S + b) * (L + 1) + l;
                off_values[k] = total;
                total += pp.n_samples * (2 * l + 1) * N;
                if (g.positions) {
                    off_positions[k] = total;
                    total += pp.n_grad * 3 * (2 * l + 1) * N;
                }
            }
        }

    double* d_out = nullptr;
    std::shared_ptr<void> storage;
    {
        void* p = nullptr;
        CUDA_CHECK(cudaMallocAsync(&p, std::max<size_t>(8, sizeof(double) * (size_t)total), stream));
        CUDA_CHECK(cudaMemsetAsync(p, 0, std::max<size_t>(8, sizeof(double) * (size_t)total), stream));
        storage = std::shared_ptr<void>(p, [](void* q) { cudaFreeAsync(q, nullptr); });
        d_out = (double*)p;
    }
    cudaEvent_t ev0, ev1;
    CUDA_CHECK(cudaEventCreate(&ev0));
    CUDA_CHECK(cudaEventCreate(&ev1));
    CUDA_CHECK(cudaEventRecord(ev0, stream));

    int64_t atom_offset = 0;
    const int64_t* d_offv = put(arena_, "lode.off_values", off_values, stream);
    const int64_t* d_offp = put(arena_, "lode.off_positions", off_positions, stream);
    for (size_t s = 0; s < systems.size(); s++) {
        const HostSystem& sys = systems[s];
        const int n = (int)sys.n_atoms;
        if (n == 0) continue;
        KVectors kv = compute_k_vectors(sys.cell, h.k_cutoff);
        const int K = (int)kv.count();
        if (K == 0) throw invalid_parameter("No k-vectors for current combination of hyper parameters.");
        const double* c = sys.cell;
        const double volume = std::fabs(c[0] * (c[4] * c[8] - c[5] * c[7]) - c[1] * (c[3] * c[8] - c[5] * c[6]) +
                                        c[2] * (c[3] * c[7] - c[4] * c[6]));
        const double global = 4.0 * M_PI / volume;
        std::vector<double> kvec(3 * (size_t)K), gdf(K), radial((size_t)K * (L + 1) * N);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < K; k++) {
            for (int x = 0; x < 3; x++) kvec[3 * k + x] = kv.norm[k] * kv.direction[3 * k + x];
            gdf[k] = global * tables_.density_fourier(kv.norm[k]);
            for (int l = 0; l <= L; l++) tables_.radial(l, kv.norm[k], &radial[((size_t)k * (L + 1) + l) * N], nullptr);
        }
        std::vector<double> k0(N), center = tables_.center;
        for (int q = 0; q < N; q++) k0[q] = global * tables_.k0[q];
        std::vector<int32_t> count(S, 0);
        for (int32_t t : sys_species[s]) count[t]++;

        LodeArgs a{};
        a.n_atoms = n;
        a.K = K;
        a.S = S;
        a.L = L;
        a.N = N;
        a.species = put(arena_, "lode.species", sys_species[s], stream);
        double* d_kvec = put(arena_, "lode.kvec", kvec, stream);
        a.kvec = d_kvec;
        a.knorm = put(arena_, "lode.knorm", kv.norm, stream);
        a.kdir = put(arena_, "lode.kdir", kv.direction, stream);
        a.gdf = put(arena_, "lode.gdf", gdf, stream);
        const double* d_radial = put(arena_, "lode.radial", radial, stream);
        double* T = arena_.alloc<double>("lode.T", (int64_t)K * L2 * N);
        double* C = arena_.alloc<double>("lode.cos", (int64_t)n * K);
        double* Sn = arena_.alloc<double>("lode.sin", (int64_t)n * K);
        double* Ct = arena_.alloc<double>("lode.cos_sum", (int64_t)S * K);
        double* St = arena_.alloc<double>("lode.sin_sum", (int64_t)S * K);
        a.T = T;
        a.C = C;
        a.Sn = Sn;
        a.Ct = Ct;
        a.St = St;
        a.row = put(arena_, "lode.rows", rows[s], stream);
        a.off_values = d_offv;
        a.off_positions = d_offp;
        a.type_count = put(arena_, "lode.type_count", count, stream);
        a.center = put(arena_, "lode.center", center, stream);
        a.k0 = put(arena_, "lode.k0", k0, stream);
        a.center_factor = 1.0 - h.center_atom_weight;
        a.add_k0 = (h.exponent == 0 || h.exponent > 3) ? 1 : 0;
        a.out = d_out;

        const double* positions = nullptr;
        if (d_positions) {
            positions = d_positions + 3 * atom_offset;
        } else {
            positions = put(arena_, "lode.positions", sys.positions, stream);
        }
        lode_projection_kernel<<<(K + 127) / 128, 128, 0, stream>>>(K, L, N, a.kdir, d_radial, d_ylm_, T);
        CUDA_CHECK(cudaGetLastError());
        const int64_t nk = (int64_t)n * K;
        lode_phases_kernel<<<(unsigned)((nk + 255) / 256), 256, 0, stream>>>(n, K, positions, d_kvec, C, Sn);
        CUDA_CHECK(cudaGetLastError());
        lode_type_sums_kernel<<<(S * K + 255) / 256, 256, 0, stream>>>(n, K, S, a.species, C, Sn, Ct, St);
        CUDA_CHECK(cudaGetLastError());
        // groups of LODE_GROUP centres of one species
        std::vector<int32_t> groups;
        for (int t = 0; t < S; t++) {
            std::vector<int32_t> members;
            for (int i = 0; i < n; i++)
                if (sys_species[s][i] == t) members.push_back(i);
            for (size_t q = 0; q < members.size(); q += LODE_GROUP)
                for (int c2 = 0; c2 < LODE_GROUP; c2++)
                    groups.push_back(q + c2 < members.size() ? members[q + c2] : -1);
        }
        const int n_groups = (int)(groups.size() / LODE_GROUP);
        const int32_t* d_groups = put(arena_, "lode.groups", groups, stream);
        const unsigned tiles = (unsigned)((L2 * N + LODE_THREADS * LODE_Q - 1) / (LODE_THREADS * LODE_Q));
        if (n_groups > 0) {
            lode_values_kernel<<<dim3((unsigned)(n_groups * S), tiles), LODE_THREADS, 0, stream>>>(a, d_groups, n_groups);
            CUDA_CHECK(cudaGetLastError());
        }
        if (g.positions && !tasks[s].empty()) {
            const int n_tasks = (int)(tasks[s].size() / 4);
            a.tasks = put(arena_, "lode.tasks", tasks[s], stream);
            lode_gradients_kernel<<<dim3((unsigned)n_tasks, tiles), LODE_THREADS, 0, stream>>>(a, n_tasks);
            CUDA_CHECK(cudaGetLastError());
        }
        // the per-system buffers are reused by the next system
        CUDA_CHECK(cudaStreamSynchronize(stream));
        atom_offset += n;
    }
    CUDA_CHECK(cudaEventRecord(ev1, stream));

    auto tm = std::make_unique<TensorMap>();
    tm->on_device = device_output;
    tm->device = device_;
    tm->keys.names = {"o3_lambda", "o3_sigma", "center_type", "neighbor_type"};
    tm->keys.values = keys_values;
    double* base = d_out;
    if (device_output) {
        tm->storage = storage;
    } else {
        double* host = static_cast<double*>(std::malloc(std::max<size_t>(8, sizeof(double) * (size_t)total)));
        if (!host) throw std::bad_alloc();
        tm->storage = std::shared_ptr<void>(host, std::free);
        if (total) CUDA_CHECK(cudaMemcpyAsync(host, d_out, sizeof(double) * total, cudaMemcpyDeviceToHost, stream));
        base = host;
    }
    CUDA_CHECK(cudaStreamSynchronize(stream));
    Labels properties;
    properties.names = {"n"};
    for (int q = 0; q < N; q++) properties.values.push_back(q);
    for (int a = 0; a < S; a++)
        for (int b = 0; b < S; b++) {
            if (!pair_present[(size_t)a * S + b]) continue;
            const auto& pp = pairs[(size_t)a * S + b];
            for (int l = 0; l <= L; l++) {
                const size_t k = ((size_t)a * S + b) * (L + 1) + l;
                Labels mu;
                mu.names = {"o3_mu"};
                for (int m = -l; m <= l; m++) mu.values.push_back(m);
                auto blk = std::make_unique<Block>();
                blk->samples = pp.samples;
                blk->components = {mu};
                blk->properties = properties;
                blk->shape = {(size_t)pp.n_samples, (size_t)(2 * l + 1), (size_t)N};
                blk->data = base + off_values[k];
                if (g.positions) {
                    auto gb = std::make_unique<Block>();
                    gb->samples = pp.grad_samples;
                    gb->components = {labels_xyz(), mu};
                    gb->properties = properties;
                    gb->shape = {(size_t)pp.n_grad, 3, (size_t)(2 * l + 1), (size_t)N};
                    gb->data = base + off_positions[k];
                    blk->gradients.emplace_back("positions", std::move(gb));
                }
                tm->blocks.push_back(std::move(blk));
            }
        }
    float ms = 0.0f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    times_ = PhaseTimes{};
    times_.expansion = ms;
    times_.total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return tm;
}

}  // namespace fb200

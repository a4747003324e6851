// Clebsch-Gordan tensor products of spherical-expansion blocks: the real CG
// coefficients (host) and the coupling kernel behind
// featomic_b200_cg_coefficients / featomic_b200_cg_product.
//
// Follows python/featomic/featomic/clebsch_gordan/_coefficients.py:
// complex CG coefficients (the `wigners` package there, Racah's closed form
// here), turned real with the real<->complex harmonic transforms of
// _coefficients.py:336-384 (U(l) on m1 and m2, U(lambda)^H on mu) and the real
// or imaginary part kept by the parity of l1 + l2 + lambda
// (_coefficients.py:137-224); the product of two blocks is
// out[s, mu, p * n2 + q] = sum_{m1 m2} C[m1, m2, mu] a[s, m1, p] b[s, m2, q]
// (_coefficients.py:628-709, properties p-major as
// _utils.py:_compute_labels_full_cartesian_product).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/featomic_b200.h"
#include "clebsch_gordan.hpp"
#include "engine.hpp"

namespace fb200 {

namespace {

long double factorial(int n) {
    long double f = 1.0L;
    for (int k = 2; k <= n; k++) f *= (long double)k;
    return f;
}

// <j1 m1 j2 m2 | J M> by Racah's formula (Racah 1942; e.g. Varshalovich et
// al., "Quantum Theory of Angular Momentum", 8.2.1 eq. 3), Condon-Shortley
// phase convention.
long double complex_cg(int j1, int m1, int j2, int m2, int J, int M) {
    if (m1 + m2 != M || std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(M) > J) return 0.0L;
    if (J < std::abs(j1 - j2) || J > j1 + j2) return 0.0L;
    const long double pre = std::sqrt((2.0L * J + 1.0L) * factorial(J + j1 - j2) * factorial(J - j1 + j2) *
                                      factorial(j1 + j2 - J) / factorial(j1 + j2 + J + 1));
    const long double norm = std::sqrt(factorial(J + M) * factorial(J - M) * factorial(j1 - m1) *
                                       factorial(j1 + m1) * factorial(j2 - m2) * factorial(j2 + m2));
    long double sum = 0.0L;
    const int kmin = std::max({0, j2 - J - m1, j1 - J + m2});
    const int kmax = std::min({j1 + j2 - J, j1 - m1, j2 + m2});
    for (int k = kmin; k <= kmax; k++) {
        const long double d = factorial(k) * factorial(j1 + j2 - J - k) * factorial(j1 - m1 - k) *
                              factorial(j2 + m2 - k) * factorial(J - j2 + m1 + k) * factorial(J - j1 - m2 + k);
        sum += ((k & 1) ? -1.0L : 1.0L) / d;
    }
    return pre * norm * sum;
}

using cplx = std::complex<long double>;

// U(l)[l + m, l + m'] with complex Y = U . real Y (real harmonics in
// featomic's m order -l..l, _coefficients.py:336-369).
std::vector<cplx> real_to_complex(int l) {
    const int M = 2 * l + 1;
    std::vector<cplx> u((size_t)M * M, cplx(0, 0));
    const long double r = 1.0L / std::sqrt(2.0L);
    for (int m = -l; m <= l; m++) {
        const long double sign = (m & 1) ? -1.0L : 1.0L;
        if (m < 0) {
            u[(size_t)(l + m) * M + (l + m)] = cplx(0, -r);
            u[(size_t)(l + m) * M + (l - m)] = cplx(0, r * sign);
        } else if (m == 0) {
            u[(size_t)l * M + l] = cplx(1, 0);
        } else {
            u[(size_t)(l + m) * M + (l - m)] = cplx(r, 0);
            u[(size_t)(l + m) * M + (l + m)] = cplx(r * sign, 0);
        }
    }
    return u;
}

}  // namespace

// Real CG coefficients, dense [2 l1 + 1][2 l2 + 1][2 lambda + 1].
std::vector<double> real_cg_coefficients(int l1, int l2, int lambda) {
    if (l1 < 0 || l2 < 0 || lambda < 0) throw invalid_parameter("angular orders must be non-negative");
    if (lambda < std::abs(l1 - l2) || lambda > l1 + l2)
        throw invalid_parameter("lambda = " + std::to_string(lambda) + " can not couple l1 = " + std::to_string(l1) +
                                " and l2 = " + std::to_string(l2));
    if (l1 + l2 > 40) throw invalid_parameter("angular orders above 40 are not supported");
    const int A = 2 * l1 + 1, B = 2 * l2 + 1, C = 2 * lambda + 1;
    std::vector<cplx> cg((size_t)A * B * C);
    for (int a = 0; a < A; a++)
        for (int b = 0; b < B; b++)
            for (int c = 0; c < C; c++)
                cg[((size_t)a * B + b) * C + c] = cplx(complex_cg(l1, a - l1, l2, b - l2, lambda, c - lambda), 0);
    const auto u1 = real_to_complex(l1), u2 = real_to_complex(l2), ul = real_to_complex(lambda);
    // x1[a', b, c] = sum_a U1[a', a] cg[a, b, c]
    std::vector<cplx> x1((size_t)A * B * C, cplx(0, 0)), x2((size_t)A * B * C, cplx(0, 0));
    for (int ap = 0; ap < A; ap++)
        for (int a = 0; a < A; a++) {
            const cplx u = u1[(size_t)ap * A + a];
            if (u == cplx(0, 0)) continue;
            for (size_t bc = 0; bc < (size_t)B * C; bc++) x1[(size_t)ap * B * C + bc] += u * cg[(size_t)a * B * C + bc];
        }
    // x2[a, b', c] = sum_b U2[b', b] x1[a, b, c]
    for (int a = 0; a < A; a++)
        for (int bp = 0; bp < B; bp++)
            for (int b = 0; b < B; b++) {
                const cplx u = u2[(size_t)bp * B + b];
                if (u == cplx(0, 0)) continue;
                for (int c = 0; c < C; c++) x2[((size_t)a * B + bp) * C + c] += u * x1[((size_t)a * B + b) * C + c];
            }
    // real[a, b, c'] = sum_c x2[a, b, c] conj(U_lambda)[c', c]  (x2 @ U_lambda^H)
    const bool even = ((l1 + l2 + lambda) & 1) == 0;
    std::vector<double> out((size_t)A * B * C);
    for (size_t ab = 0; ab < (size_t)A * B; ab++)
        for (int cp = 0; cp < C; cp++) {
            cplx s(0, 0);
            for (int c = 0; c < C; c++) s += x2[ab * C + c] * std::conj(ul[(size_t)cp * C + c]);
            out[ab * C + cp] = (double)(even ? s.real() : s.imag());
        }
    return out;
}

namespace {

struct DeviceCgTask {
    const void* first;
    const void* second;
    void* output;
    int64_t n_samples;
    int64_t block_start;  // first CTA of this task
    int64_t out_stride;   // elements between (sample, mu) rows of the output
    int32_t n_first, n_second, lambda;
    int32_t m1_count, m2_count;
    int32_t entries;      // offset of the task's (mu-sorted) coefficient list
    int32_t mu_offsets;   // offset of its [2 lambda + 2] per-mu starts
    int32_t vector;       // rows of `second` / `output` take 4-wide vector accesses
    int32_t vector_first; // rows of `first` take 8-wide vector loads
};

struct CgEntry {
    int16_t m1, m2;
    float pad;
    double value;
};

constexpr int CG_THREADS = 256;
constexpr int CG_PV = 8;  // first-block properties per thread
constexpr int CG_QV = 4;  // second-block properties per thread

__device__ inline void load4(const float* p, float (&x)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
}
__device__ inline void load4(const double* p, double (&x)[4]) {
    const double2 u = reinterpret_cast<const double2*>(p)[0], v = reinterpret_cast<const double2*>(p)[1];
    x[0] = u.x, x[1] = u.y, x[2] = v.x, x[3] = v.y;
}
__device__ inline void load8(const float* p, float (&x)[8]) {
    const float4 u = reinterpret_cast<const float4*>(p)[0], v = reinterpret_cast<const float4*>(p)[1];
    x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w, x[4] = v.x, x[5] = v.y, x[6] = v.z, x[7] = v.w;
}
__device__ inline void load8(const double* p, double (&x)[8]) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double2 u = reinterpret_cast<const double2*>(p)[k];
        x[2 * k] = u.x, x[2 * k + 1] = u.y;
    }
}
__device__ inline void store4(float* p, const float (&x)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
}
__device__ inline void store4(double* p, const double (&x)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(x[0], x[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(x[2], x[3]);
}

// One thread per (sample, 8 first-block properties, 4 second-block
// properties) of one task: each coefficient and first-block value is loaded
// once for 4 or 32 products, the first-block row (8 wide), the second-block
// row and the output row (4 wide) are vector accesses when the task allows, and every output value is written
// once.  Each output is sum_k (C_k * a[m1_k]) * b[m2_k] over the task's
// non-zero coefficients of that mu, in the table order.
template <typename T>
__global__ void __launch_bounds__(CG_THREADS)
cg_product_kernel(const DeviceCgTask* __restrict__ tasks, int n_tasks, const CgEntry* __restrict__ entries,
                  const int32_t* __restrict__ mu_starts) {
    int lo = 0, hi = n_tasks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (tasks[mid].block_start <= (int64_t)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    const DeviceCgTask t = tasks[lo];
    const int nqt = (t.n_second + CG_QV - 1) / CG_QV, npt = (t.n_first + CG_PV - 1) / CG_PV;
    const int64_t tiles = (int64_t)npt * nqt;
    const int64_t item = ((int64_t)blockIdx.x - t.block_start) * CG_THREADS + threadIdx.x;
    if (item >= t.n_samples * tiles) return;
    const int64_t s = item / tiles;
    const int64_t r = item - s * tiles;
    const int pt = (int)(r / nqt), qt = (int)(r - (int64_t)pt * nqt);
    const int p0 = pt * CG_PV, q0 = qt * CG_QV;
    const int np = min(CG_PV, t.n_first - p0), nq = min(CG_QV, t.n_second - q0);
    const T* __restrict__ a = static_cast<const T*>(t.first) + s * t.m1_count * t.n_first + p0;
    const T* __restrict__ b = static_cast<const T*>(t.second) + s * t.m2_count * t.n_second + q0;
    T* __restrict__ out = static_cast<T*>(t.output) + s * (2 * t.lambda + 1) * t.out_stride +
                          (int64_t)p0 * t.n_second + q0;
    const bool vec = t.vector && nq == CG_QV;
    const bool vec_first = CG_PV == 8 && t.vector_first && np == CG_PV;
    const int32_t* starts = mu_starts + t.mu_offsets;
    const CgEntry* e = entries + t.entries;
    for (int mu = 0; mu <= 2 * t.lambda; mu++) {
        T acc[CG_PV][CG_QV];
#pragma unroll
        for (int i = 0; i < CG_PV; i++)
#pragma unroll
            for (int j = 0; j < CG_QV; j++) acc[i][j] = T(0);
        for (int k = starts[mu]; k < starts[mu + 1]; k++) {
            const CgEntry c = e[k];
            const T* brow = b + (int64_t)c.m2 * t.n_second;
            T bv[CG_QV];
            if (vec) {
                load4(brow, bv);
            } else {
#pragma unroll
                for (int j = 0; j < CG_QV; j++) bv[j] = j < nq ? brow[j] : T(0);
            }
            T av[CG_PV];
            if (vec_first) {
                load8(a + (int64_t)c.m1 * t.n_first, av);
            } else {
#pragma unroll
                for (int i = 0; i < CG_PV; i++) av[i] = i < np ? a[(int64_t)c.m1 * t.n_first + i] : T(0);
            }
#pragma unroll
            for (int i = 0; i < CG_PV; i++) {
                const T ca = T(c.value) * av[i];
#pragma unroll
                for (int j = 0; j < CG_QV; j++) acc[i][j] += ca * bv[j];
            }
        }
        T* orow = out + mu * t.out_stride;
#pragma unroll
        for (int i = 0; i < CG_PV; i++) {
            if (i >= np) break;
            if (vec) {
                store4(orow + (int64_t)i * t.n_second, acc[i]);
            } else {
#pragma unroll
                for (int j = 0; j < CG_QV; j++)
                    if (j < nq) orow[(int64_t)i * t.n_second + j] = acc[i][j];
            }
        }
    }
}

struct DeviceCoupleTask {
    const void* input;
    void* output;
    int64_t n_outer, n_inner;
    int64_t block_start;
    int32_t m1_count, m2_count, lambda;
    int32_t entries, mu_offsets;
};

// Coupling of two spherical axes of one array: one thread per (outer,
// inner) index, out[o, mu, i] = sum_k C_k * x[o, m1_k, m2_k, i] over the
// non-zero coefficients of mu in table order; loads and stores coalesced
// along the inner index.
template <typename T>
__global__ void __launch_bounds__(CG_THREADS)
cg_couple_kernel(const DeviceCoupleTask* __restrict__ tasks, int n_tasks, const CgEntry* __restrict__ entries,
                 const int32_t* __restrict__ mu_starts) {
    int lo = 0, hi = n_tasks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (tasks[mid].block_start <= (int64_t)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    const DeviceCoupleTask t = tasks[lo];
    const int64_t item = ((int64_t)blockIdx.x - t.block_start) * CG_THREADS + threadIdx.x;
    if (item >= t.n_outer * t.n_inner) return;
    const int64_t o = item / t.n_inner, i = item - o * t.n_inner;
    const T* __restrict__ x = static_cast<const T*>(t.input) + o * t.m1_count * t.m2_count * t.n_inner + i;
    T* __restrict__ out = static_cast<T*>(t.output) + o * (2 * t.lambda + 1) * t.n_inner + i;
    const int32_t* starts = mu_starts + t.mu_offsets;
    const CgEntry* e = entries + t.entries;
    for (int mu = 0; mu <= 2 * t.lambda; mu++) {
        T acc = T(0);
        for (int k = starts[mu]; k < starts[mu + 1]; k++) {
            const CgEntry c = e[k];
            acc += T(c.value) * x[((int64_t)c.m1 * t.m2_count + c.m2) * t.n_inner];
        }
        out[mu * t.n_inner] = acc;
    }
}

// Non-zero real CG coefficients of (l1, l2, lambda), grouped by mu, cached.
struct SparseCg {
    std::vector<CgEntry> entries;
    std::vector<int32_t> mu_starts;  // [2 lambda + 2], relative to entries
};

const SparseCg& sparse_cg(int l1, int l2, int lambda) {
    static std::mutex mutex;
    static std::map<std::tuple<int, int, int>, SparseCg> cache;
    std::lock_guard<std::mutex> lock(mutex);
    auto it = cache.find({l1, l2, lambda});
    if (it != cache.end()) return it->second;
    const auto dense = real_cg_coefficients(l1, l2, lambda);
    const int A = 2 * l1 + 1, B = 2 * l2 + 1, C = 2 * lambda + 1;
    SparseCg sp;
    sp.mu_starts.push_back(0);
    for (int c = 0; c < C; c++) {
        for (int a = 0; a < A; a++)
            for (int b = 0; b < B; b++) {
                const double v = dense[((size_t)a * B + b) * C + c];
                if (std::fabs(v) > 1e-15) sp.entries.push_back(CgEntry{(int16_t)a, (int16_t)b, 0.0f, v});
            }
        sp.mu_starts.push_back((int32_t)sp.entries.size());
    }
    return cache.emplace(std::make_tuple(l1, l2, lambda), std::move(sp)).first->second;
}

}  // namespace

void cg_product(const featomic_b200_cg_task_t* tasks, size_t n_tasks, int precision, cudaStream_t stream) {
    if (precision != 32 && precision != 64) throw invalid_parameter("precision must be 32 or 64");
    std::vector<DeviceCgTask> dev;
    std::vector<CgEntry> entries;
    std::vector<int32_t> mu_starts;
    int64_t blocks = 0;
    for (size_t i = 0; i < n_tasks; i++) {
        const auto& t = tasks[i];
        if (t.n_samples < 0 || t.n_first < 0 || t.n_second < 0)
            throw invalid_parameter("negative size in Clebsch-Gordan task " + std::to_string(i));
        const int64_t items = t.n_samples * (int64_t)t.n_first * t.n_second;
        if (items == 0) continue;
        if (!t.first || !t.second || !t.output)
            throw invalid_parameter("NULL array in Clebsch-Gordan task " + std::to_string(i));
        const SparseCg& sp = sparse_cg(t.l1, t.l2, t.lambda);
        DeviceCgTask d;
        d.first = t.first;
        d.second = t.second;
        d.output = t.output;
        d.n_samples = t.n_samples;
        d.block_start = blocks;
        const int64_t pq = (int64_t)t.n_first * t.n_second;
        if (t.output_stride != 0 && t.output_stride < pq)
            throw invalid_parameter("output_stride of Clebsch-Gordan task " + std::to_string(i) +
                                    " is smaller than n_first * n_second");
        d.out_stride = t.output_stride == 0 ? pq : t.output_stride;
        d.n_first = t.n_first;
        d.n_second = t.n_second;
        d.lambda = t.lambda;
        d.m1_count = 2 * t.l1 + 1;
        d.m2_count = 2 * t.l2 + 1;
        d.entries = (int32_t)entries.size();
        d.mu_offsets = (int32_t)mu_starts.size();
        const size_t align = 4 * (precision == 64 ? sizeof(double) : sizeof(float));
        d.vector = t.n_second % CG_QV == 0 && d.out_stride % CG_QV == 0 && reinterpret_cast<uintptr_t>(t.second) % std::min<size_t>(align, 16) == 0 &&
                   reinterpret_cast<uintptr_t>(t.output) % std::min<size_t>(align, 16) == 0;
        d.vector_first = t.n_first % CG_PV == 0 && reinterpret_cast<uintptr_t>(t.first) % 16 == 0;
        entries.insert(entries.end(), sp.entries.begin(), sp.entries.end());
        mu_starts.insert(mu_starts.end(), sp.mu_starts.begin(), sp.mu_starts.end());
        dev.push_back(d);
        const int64_t threads = t.n_samples * ((t.n_first + CG_PV - 1) / CG_PV) * ((t.n_second + CG_QV - 1) / CG_QV);
        blocks += (threads + CG_THREADS - 1) / CG_THREADS;
    }
    if (dev.empty()) return;
    if (blocks > 0x7fffffffLL) throw invalid_parameter("Clebsch-Gordan product too large for one launch");
    // one device buffer for the three tables, released in stream order
    const size_t tb = dev.size() * sizeof(DeviceCgTask);
    const size_t eb = std::max<size_t>(entries.size(), 1) * sizeof(CgEntry);
    const size_t mb = mu_starts.size() * sizeof(int32_t);
    const size_t e_off = (tb + 15) / 16 * 16, m_off = e_off + (eb + 15) / 16 * 16, total = m_off + mb;
    std::vector<unsigned char> host(total, 0);
    std::memcpy(host.data(), dev.data(), tb);
    if (!entries.empty()) std::memcpy(host.data() + e_off, entries.data(), entries.size() * sizeof(CgEntry));
    std::memcpy(host.data() + m_off, mu_starts.data(), mb);
    unsigned char* buffer = nullptr;
    CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&buffer), total, stream));
    // a copy from pageable host memory returns once the source has been
    // staged, so `host` may be released when this function returns
    CUDA_CHECK(cudaMemcpyAsync(buffer, host.data(), total, cudaMemcpyHostToDevice, stream));
    const auto* d_tasks = reinterpret_cast<const DeviceCgTask*>(buffer);
    const auto* d_entries = reinterpret_cast<const CgEntry*>(buffer + e_off);
    const auto* d_mu = reinterpret_cast<const int32_t*>(buffer + m_off);
    if (precision == 64)
        cg_product_kernel<double><<<(unsigned)blocks, CG_THREADS, 0, stream>>>(d_tasks, (int)dev.size(), d_entries, d_mu);
    else
        cg_product_kernel<float><<<(unsigned)blocks, CG_THREADS, 0, stream>>>(d_tasks, (int)dev.size(), d_entries, d_mu);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaFreeAsync(buffer, stream));
}

void cg_couple(const featomic_b200_cg_couple_task_t* tasks, size_t n_tasks, int precision, cudaStream_t stream) {
    if (precision != 32 && precision != 64) throw invalid_parameter("precision must be 32 or 64");
    std::vector<DeviceCoupleTask> dev;
    std::vector<CgEntry> entries;
    std::vector<int32_t> mu_starts;
    int64_t blocks = 0;
    for (size_t i = 0; i < n_tasks; i++) {
        const auto& t = tasks[i];
        if (t.n_outer < 0 || t.n_inner < 0)
            throw invalid_parameter("negative size in Clebsch-Gordan coupling task " + std::to_string(i));
        const int64_t items = t.n_outer * t.n_inner;
        const SparseCg& sp = sparse_cg(t.l1, t.l2, t.lambda);
        if (items == 0) continue;
        if (!t.input || !t.output)
            throw invalid_parameter("NULL array in Clebsch-Gordan coupling task " + std::to_string(i));
        DeviceCoupleTask d;
        d.input = t.input;
        d.output = t.output;
        d.n_outer = t.n_outer;
        d.n_inner = t.n_inner;
        d.block_start = blocks;
        d.m1_count = 2 * t.l1 + 1;
        d.m2_count = 2 * t.l2 + 1;
        d.lambda = t.lambda;
        d.entries = (int32_t)entries.size();
        d.mu_offsets = (int32_t)mu_starts.size();
        entries.insert(entries.end(), sp.entries.begin(), sp.entries.end());
        mu_starts.insert(mu_starts.end(), sp.mu_starts.begin(), sp.mu_starts.end());
        dev.push_back(d);
        blocks += (items + CG_THREADS - 1) / CG_THREADS;
    }
    if (dev.empty()) return;
    if (blocks > 0x7fffffffLL) throw invalid_parameter("Clebsch-Gordan coupling too large for one launch");
    const size_t tb = dev.size() * sizeof(DeviceCoupleTask);
    const size_t eb = std::max<size_t>(entries.size(), 1) * sizeof(CgEntry);
    const size_t mb = mu_starts.size() * sizeof(int32_t);
    const size_t e_off = (tb + 15) / 16 * 16, m_off = e_off + (eb + 15) / 16 * 16, total = m_off + mb;
    std::vector<unsigned char> host(total, 0);
    std::memcpy(host.data(), dev.data(), tb);
    if (!entries.empty()) std::memcpy(host.data() + e_off, entries.data(), entries.size() * sizeof(CgEntry));
    std::memcpy(host.data() + m_off, mu_starts.data(), mb);
    unsigned char* buffer = nullptr;
    CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&buffer), total, stream));
    // staged before the call returns (pageable source), as above
    CUDA_CHECK(cudaMemcpyAsync(buffer, host.data(), total, cudaMemcpyHostToDevice, stream));
    const auto* d_tasks = reinterpret_cast<const DeviceCoupleTask*>(buffer);
    const auto* d_entries = reinterpret_cast<const CgEntry*>(buffer + e_off);
    const auto* d_mu = reinterpret_cast<const int32_t*>(buffer + m_off);
    if (precision == 64)
        cg_couple_kernel<double><<<(unsigned)blocks, CG_THREADS, 0, stream>>>(d_tasks, (int)dev.size(), d_entries, d_mu);
    else
        cg_couple_kernel<float><<<(unsigned)blocks, CG_THREADS, 0, stream>>>(d_tasks, (int)dev.size(), d_entries, d_mu);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaFreeAsync(buffer, stream));
}

}  // namespace fb200

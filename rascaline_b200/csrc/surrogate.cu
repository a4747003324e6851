// Learned radial surrogate (see surrogate.hpp): training set from the exact
// analytic GTO radial integral (featomic/src/calculators/soap/radial_integral/
// gto.rs:115-205 through radial_compute), training kernels on the CUDA
// cores, inference on the tensor cores (surrogate_mma.cu) or the CUDA cores.
//
// Training step (one CUDA graph replay):
//   samples   thread per minibatch sample: forward with the FP32 master
//             weights, carrying the x-derivative of every activation; loss =
//             mean squared error of the normalised outputs + lambda times
//             that of their x-derivatives (x = 2 r / r_c - 1); backward pass,
//             second derivatives of the SiLU included, to the per-sample
//             deltas, stored
//   gradient  thread per (parameter, chunk of samples), then a fixed-order
//             sum over the chunks: deterministic, no atomics
//   adam      FP32 master weights, cosine learning-rate decay
//
// Output-layer fit (after the Adam steps): the output layer is linear in the
// hidden features, so W3 and b3 are refitted by least squares over the whole
// training set, on values and x-derivatives:
//   min sum_i |[h2_i, 1] W - y_i|^2 + lambda |[dh2_i/dx, 0] W - dy_i/dx|^2
// with the features h2, dh2 of the tensor-core kernel itself (so that its
// outputs are the fitted ones), normal equations accumulated in FP64
// (features of a chunk of samples, then a fixed-order sum: deterministic),
// solved by a Cholesky factorisation in one CTA.
//
// The tensor cores (surrogate_mma.cu) read W2 and W3 as sums of three BF16
// matrices (hi + mid + lo, 24 significant bits); the CUDA-core evaluation
// reads the FP32 weights, or (the single-BF16 control) their BF16 roundings.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>

#include "dense.hpp"
#include "pair_math.cuh"
#include "surrogate.hpp"

namespace fb200 {

namespace {

constexpr int MLP_H = 64;
constexpr int GRAD_CHUNK = 256;

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + __expf(-z)); }

struct Offsets {
    int w1, b1, w2, b2, w3, b3, total;
    __host__ __device__ static Offsets make(int H, int O) {
        Offsets o;
        o.w1 = 0;
        o.b1 = H;
        o.w2 = 2 * H;
        o.b2 = 2 * H + H * H;
        o.w3 = 3 * H + H * H;
        o.b3 = 3 * H + H * H + O * H;
        o.total = o.b3 + O;
        return o;
    }
};

// training set: r uniform in [0, rc], targets R_o(r), o = l nmax + n
__global__ void surrogate_dataset_kernel(DeviceRadial exact, int64_t n, double rc, uint64_t seed, float* __restrict__ r,
                                         float* __restrict__ targets, float* __restrict__ dtargets,
                                         int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double u = (double)(splitmix64(seed ^ (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
    // the stored FP32 distance is the one the targets are computed at
    const float rf = (float)(rc * u);
    const double ri = (double)rf;
    r[i] = rf;
    const int N = exact.nmax, O = (exact.lmax + 1) * N;
    double v[64], g[64];
    for (int l = 0; l <= exact.lmax; l++) {
        if (!radial_compute(exact, l, ri, v, g)) atomicExch(status, 1);
        for (int q = 0; q < N; q++) {
            targets[i * O + l * N + q] = (float)v[q];
            dtargets[i * O + l * N + q] = (float)g[q];
        }
    }
}

// largest |target| of every output (block per output)
__global__ void surrogate_scale_kernel(const float* __restrict__ t, int64_t n, int O, float* __restrict__ scale) {
    __shared__ float red[256];
    const int o = blockIdx.x;
    float m = 0.0f;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, fabsf(t[i * O + o]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) scale[o] = red[0] > 0.0f ? red[0] : 1.0f;
}

__global__ void surrogate_normalise_kernel(float* __restrict__ t, int64_t n, int O, const float* __restrict__ scale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * O) return;
    t[i] /= scale[i % O];
}

struct TrainArgs {
    int O;
    double rc;
    const float* master;
    const float* r;        // [n]
    const float* targets;  // [n][O]
    const float* dtargets; // [n][O] their r-derivatives
    float deriv_weight;    // lambda: weight of the derivative term of the loss
    int64_t n, batch;
    int sample;            // random minibatch (1) or the first `batch` samples (0)
    uint64_t seed;
    const int64_t* step;
    // per sample: input, activations and their x-derivatives, deltas
    float *x, *h1, *dh1, *dz1, *gw1, *h2, *dh2, *dz2, *ddz2, *dy, *df;
    float* loss_part;      // [blocks]
};

// silu(z), silu'(z), silu''(z)
__device__ __forceinline__ void silu_terms(float z, float& s, float& s1, float& s2) {
    const float sg = sigmoid(z);
    s = z * sg;
    s1 = sg * (1.0f + z * (1.0f - sg));
    s2 = sg * (1.0f - sg) * (2.0f + z * (1.0f - 2.0f * sg));
}

// forward and backward of one sample per thread; weights in shared memory
__global__ void __launch_bounds__(128) surrogate_sample_kernel(TrainArgs a) {
    extern __shared__ float wsm[];
    constexpr int H = MLP_H;
    const int O = a.O;
    const Offsets off = Offsets::make(H, O);
    for (int p = threadIdx.x; p < off.total; p += blockDim.x) wsm[p] = a.master[p];
    __syncthreads();
    const float* w1 = wsm + off.w1;
    const float* b1 = wsm + off.b1;
    const float* W2 = wsm + off.w2;
    const float* b2 = wsm + off.b2;
    const float* W3 = wsm + off.w3;
    const float* b3 = wsm + off.b3;

    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float loss = 0.0f;
    if (b < a.batch) {
        int64_t s = b;
        if (a.sample) s = (int64_t)(splitmix64(a.seed ^ ((uint64_t)(*a.step) * 0xD1B54A32D192ED03ull) ^ (uint64_t)b) %
                                    (uint64_t)a.n);
        const float x = (float)(2.0 * a.r[s] / a.rc - 1.0);
        a.x[b] = x;
        float* h1r = a.h1 + b * H;
        float* dh1r = a.dh1 + b * H;
        float* h2r = a.h2 + b * H;
        float* dh2r = a.dh2 + b * H;
        float* dz2r = a.dz2 + b * H;
        float* ddz2r = a.ddz2 + b * H;
        // layer 1: h1 and dh1/dx
        float h[H], dh[H];
#pragma unroll
        for (int k = 0; k < H; k++) {
            float sv, s1, s2;
            silu_terms(w1[k] * x + b1[k], sv, s1, s2);
            h[k] = sv;
            dh[k] = s1 * w1[k];
            h1r[k] = h[k];
            dh1r[k] = dh[k];
        }
        // layer 2: h2 and dh2/dx; silu' and silu'' dz2 kept for the backward pass
        for (int j = 0; j < H; j++) {
            float z = b2[j], dz = 0.0f;
#pragma unroll
            for (int k = 0; k < H; k++) {
                z += W2[j * H + k] * h[k];
                dz += W2[j * H + k] * dh[k];
            }
            float sv, s1, s2;
            silu_terms(z, sv, s1, s2);
            h2r[j] = sv;
            dh2r[j] = s1 * dz;
            dz2r[j] = s1;
            ddz2r[j] = s2 * dz;
        }
        // layer 3, loss, output deltas e (values) and f (x-derivatives)
#pragma unroll
        for (int k = 0; k < H; k++) {
            h[k] = h2r[k];
            dh[k] = dh2r[k];
        }
        const float* t = a.targets + s * O;
        const float* dt = a.dtargets + s * O;
        const float dxscale = (float)(0.5 * a.rc);  // dt/dx = dt/dr * rc / 2
        const float gscale = 2.0f / (float)(a.batch * O);
        const float lam = a.deriv_weight;
        float* e = a.dy + b * O;
        float* f = a.df + b * O;
        for (int o = 0; o < O; o++) {
            float y = b3[o], dy = 0.0f;
#pragma unroll
            for (int k = 0; k < H; k++) {
                y += W3[o * H + k] * h[k];
                dy += W3[o * H + k] * dh[k];
            }
            const float d = y - t[o];
            const float dd = dy - dt[o] * dxscale;
            loss += d * d + lam * dd * dd;
            e[o] = gscale * d;
            f[o] = gscale * lam * dd;
        }
        // back to layer 2: delta of z2 and of dz2
        for (int k = 0; k < H; k++) {
            float gh2 = 0.0f, gdh2 = 0.0f;
            for (int o = 0; o < O; o++) {
                gh2 += W3[o * H + k] * e[o];
                gdh2 += W3[o * H + k] * f[o];
            }
            const float s1 = dz2r[k], s2dz = ddz2r[k];
            dz2r[k] = s1 * gh2 + s2dz * gdh2;
            ddz2r[k] = s1 * gdh2;
        }
        // back to layer 1: delta of z1 and the gradient of w1
        for (int k = 0; k < H; k++) {
            float gh1 = 0.0f, gdh1 = 0.0f;
#pragma unroll 8
            for (int j = 0; j < H; j++) {
                gh1 += W2[j * H + k] * dz2r[j];
                gdh1 += W2[j * H + k] * ddz2r[j];
            }
            float sv, s1, s2;
            silu_terms(w1[k] * x + b1[k], sv, s1, s2);
            const float d1 = s1 * gh1 + s2 * w1[k] * gdh1;
            a.dz1[b * H + k] = d1;
            a.gw1[b * H + k] = d1 * x + s1 * gdh1;
        }
    }
    // per-block loss, fixed-order tree
    __shared__ float red[128];
    red[threadIdx.x] = loss;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) a.loss_part[blockIdx.x] = red[0];
}

// partial gradient of parameter p over one chunk of samples
__global__ void surrogate_gradient_kernel(TrainArgs a, float* __restrict__ partial, int n_chunks) {
    constexpr int H = MLP_H;
    const int O = a.O;
    const Offsets off = Offsets::make(H, O);
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    if (p >= off.total) return;
    const int64_t b0 = (int64_t)chunk * GRAD_CHUNK;
    const int64_t b1 = b0 + GRAD_CHUNK < a.batch ? b0 + GRAD_CHUNK : a.batch;
    float acc = 0.0f;
    if (p < off.b1) {
        const int j = p - off.w1;
        for (int64_t b = b0; b < b1; b++) acc += a.gw1[b * H + j];
    } else if (p < off.w2) {
        const int j = p - off.b1;
        for (int64_t b = b0; b < b1; b++) acc += a.dz1[b * H + j];
    } else if (p < off.b2) {
        const int j = (p - off.w2) / H, k = (p - off.w2) % H;
        for (int64_t b = b0; b < b1; b++)
            acc += a.dz2[b * H + j] * a.h1[b * H + k] + a.ddz2[b * H + j] * a.dh1[b * H + k];
    } else if (p < off.w3) {
        const int j = p - off.b2;
        for (int64_t b = b0; b < b1; b++) acc += a.dz2[b * H + j];
    } else if (p < off.b3) {
        const int o = (p - off.w3) / H, k = (p - off.w3) % H;
        for (int64_t b = b0; b < b1; b++) acc += a.dy[b * O + o] * a.h2[b * H + k] + a.df[b * O + o] * a.dh2[b * H + k];
    } else {
        const int o = p - off.b3;
        for (int64_t b = b0; b < b1; b++) acc += a.dy[b * O + o];
    }
    partial[(int64_t)chunk * off.total + p] = acc;
}

__global__ void surrogate_sum_kernel(const float* __restrict__ partial, int n_chunks, int total, float* __restrict__ grad,
                                     const float* __restrict__ loss_part, int n_loss, float* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < total) {
        float acc = 0.0f;
        for (int c = 0; c < n_chunks; c++) acc += partial[(int64_t)c * total + p];
        grad[p] = acc;
    }
    if (p == 0) {
        float s = 0.0f;
        for (int c = 0; c < n_loss; c++) s += loss_part[c];
        *loss = s;
    }
}

__global__ void surrogate_adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                                      float* __restrict__ v, int total, const int64_t* __restrict__ step,
                                      int64_t total_steps, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= total) return;
    const double t = (double)(*step) + 1.0;
    const double decay = 0.5 * (1.0 + cos(3.141592653589793 * fmin(t / (double)total_steps, 1.0)));
    const float rate = lr * (float)(0.01 + 0.99 * decay);
    const float b1 = 0.9f, b2 = 0.999f;
    const float gi = g[p];
    const float mi = b1 * m[p] + (1.0f - b1) * gi;
    const float vi = b2 * v[p] + (1.0f - b2) * gi * gi;
    m[p] = mi;
    v[p] = vi;
    const float mh = mi / (float)(1.0 - pow(0.9, t));
    const float vh = vi / (float)(1.0 - pow(0.999, t));
    w[p] -= rate * mh / (sqrtf(vh) + 1e-8f);
}

__global__ void surrogate_step_kernel(int64_t* step) { *step += 1; }

// R_o(r), dR_o/dr on the CUDA cores, FP32 arithmetic with the FP32 weights
// or, with `bf16_weights` (the single-BF16 control), W2 and W3 rounded to one
// BF16 each
__global__ void __launch_bounds__(128) surrogate_eval_kernel(const float* __restrict__ master, int O, double rc,
                                                             const float* __restrict__ scale, const double* __restrict__ r,
                                                             int64_t n, float* __restrict__ values,
                                                             float* __restrict__ derivs, int64_t ld, int bf16_weights) {
    extern __shared__ float wsm[];
    constexpr int H = MLP_H;
    const Offsets off = Offsets::make(H, O);
    for (int p = threadIdx.x; p < off.total; p += blockDim.x) {
        const float v = master[p];
        const bool bf = bf16_weights && ((p >= off.w2 && p < off.b2) || (p >= off.w3 && p < off.b3));
        wsm[p] = bf ? bf16_round(v) : v;
    }
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* w1 = wsm + off.w1;
    const float* b1 = wsm + off.b1;
    const float* W2 = wsm + off.w2;
    const float* b2 = wsm + off.b2;
    const float* W3 = wsm + off.w3;
    const float* b3 = wsm + off.b3;
    const float x = (float)(2.0 * r[i] / rc - 1.0);
    const float dxdr = (float)(2.0 / rc);
    float h[H], dh[H];
#pragma unroll
    for (int k = 0; k < H; k++) {
        const float z = w1[k] * x + b1[k];
        const float sg = sigmoid(z);
        h[k] = z * sg;
        dh[k] = sg * (1.0f + z * (1.0f - sg)) * w1[k] * dxdr;
    }
    float h2[H], dh2[H];
    for (int j = 0; j < H; j++) {
        float z = b2[j], dz = 0.0f;
#pragma unroll
        for (int k = 0; k < H; k++) {
            z += W2[j * H + k] * h[k];
            dz += W2[j * H + k] * dh[k];
        }
        const float sg = sigmoid(z);
        h2[j] = z * sg;
        dh2[j] = sg * (1.0f + z * (1.0f - sg)) * dz;
    }
    for (int o = 0; o < O; o++) {
        float y = b3[o], dy = 0.0f;
#pragma unroll
        for (int k = 0; k < H; k++) {
            y += W3[o * H + k] * h2[k];
            dy += W3[o * H + k] * dh2[k];
        }
        values[i * ld + o] = scale[o] * y;
        if (derivs) derivs[i * ld + o] = scale[o] * dy;
    }
}

// Rows of the least-squares problem of the output layer for the samples
// [s0, s0 + count), from the hidden features of the tensor-core kernel
// (h2 and dh2/dr, [count][2 H]): row 2 j = ([h2, 1], y) and row 2 j + 1 =
// sqrt(lambda) r_c / 2 ([dh2/dr, 0], dy/dr) of sample s0 + j (derivatives
// with respect to x = 2 r / r_c - 1, as in the training loss), features of
// width H + 1 then targets of width O, FP64
__global__ void __launch_bounds__(128) surrogate_fit_rows_kernel(const float* __restrict__ features, int O,
                                                                 const float* __restrict__ targets,
                                                                 const float* __restrict__ dtargets, int64_t s0,
                                                                 int64_t count, double dweight,
                                                                 double* __restrict__ rows) {
    constexpr int H = MLP_H;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const int64_t i = s0 + j;
    const int W = H + 1 + O;
    double* v = rows + (2 * j) * W;
    double* d = v + W;
    const float* f = features + j * 2 * H;
    for (int q = 0; q < H; q++) {
        v[q] = (double)f[q];
        d[q] = dweight * (double)f[H + q];
    }
    v[H] = 1.0;
    d[H] = 0.0;
    for (int o = 0; o < O; o++) {
        v[H + 1 + o] = (double)targets[i * O + o];
        d[H + 1 + o] = dweight * (double)dtargets[i * O + o];
    }
}

// the FP32 training distances as FP64 (the input of the tensor-core kernel)
__global__ void surrogate_widen_kernel(const float* __restrict__ r, int64_t n, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)r[i];
}

// M[a][b] += sum over the rows of F[row][a] X[row][b], a < H + 1 (features),
// b < H + 1 + O (features then targets): thread per entry, rows in order
__global__ void surrogate_normal_kernel(const double* __restrict__ rows, int64_t n_rows, int O,
                                        double* __restrict__ M) {
    const int W = MLP_H + 1 + O;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)(MLP_H + 1) * W) return;
    const int a = (int)(e / W), b = (int)(e - (int64_t)a * W);
    double acc = 0.0;
    for (int64_t q = 0; q < n_rows; q++) acc += rows[q * W + a] * rows[q * W + b];
    M[e] += acc;
}

// Solve A [W3^T; b3^T] = B (A = M[:, :H + 1], B = M[:, H + 1:]) by a Cholesky
// factorisation in one CTA, FP64 in shared memory; a relative ridge of 1e-13
// keeps the factorisation defined for features that are linearly dependent
// to rounding.  Writes W3 and b3 into the master weights; status 2 if a
// pivot is not positive.
__global__ void __launch_bounds__(256) surrogate_solve_kernel(const double* __restrict__ M, int O,
                                                              float* __restrict__ master, int32_t* __restrict__ status) {
    extern __shared__ double sm[];
    constexpr int F = MLP_H + 1;
    const int W = F + O;
    double* A = sm;          // [F][F]
    double* B = sm + F * F;  // [F][O]
    for (int e = threadIdx.x; e < F * W; e += blockDim.x) {
        const int a = e / W, b = e - a * W;
        if (b < F) A[a * F + b] = M[e];
        else B[a * O + (b - F)] = M[e];
    }
    __syncthreads();
    __shared__ double ridge;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < F; k++) t += A[k * F + k];
        ridge = 1e-13 * t / F;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < F; k += blockDim.x) A[k * F + k] += ridge;
    __syncthreads();
    // right-looking Cholesky: A = L L^T, L in the lower triangle
    for (int k = 0; k < F; k++) {
        if (threadIdx.x == 0) {
            const double p = A[k * F + k];
            if (!(p > 0.0)) atomicExch(status, 2);
            A[k * F + k] = p > 0.0 ? sqrt(p) : 1.0;
        }
        __syncthreads();
        const double piv = A[k * F + k];
        for (int i = k + 1 + threadIdx.x; i < F; i += blockDim.x) A[i * F + k] /= piv;
        __syncthreads();
        const int m = F - k - 1;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            const int i = k + 1 + e / m, j = k + 1 + e % m;
            if (j <= i) A[i * F + j] -= A[i * F + k] * A[j * F + k];
        }
        __syncthreads();
    }
    // L Z = B, then L^T X = Z: one thread per right-hand side
    for (int o = threadIdx.x; o < O; o += blockDim.x) {
        for (int i = 0; i < F; i++) {
            double v = B[i * O + o];
            for (int k = 0; k < i; k++) v -= A[i * F + k] * B[k * O + o];
            B[i * O + o] = v / A[i * F + i];
        }
        for (int i = F - 1; i >= 0; i--) {
            double v = B[i * O + o];
            for (int k = i + 1; k < F; k++) v -= A[k * F + i] * B[k * O + o];
            B[i * O + o] = v / A[i * F + i];
        }
    }
    __syncthreads();
    const Offsets off = Offsets::make(MLP_H, O);
    for (int e = threadIdx.x; e < O * MLP_H; e += blockDim.x) {
        const int o = e / MLP_H, k = e - o * MLP_H;
        master[off.w3 + e] = (float)B[k * O + o];
    }
    for (int o = threadIdx.x; o < O; o += blockDim.x) master[off.b3 + o] = (float)B[MLP_H * O + o];
}

// the radial integral the surrogate replaces: FP64 spline or analytic GTO
__global__ void radial_reference_kernel(DeviceRadial radial, const double* __restrict__ r, int64_t n,
                                        float* __restrict__ values, float* __restrict__ derivs, int64_t ld,
                                        int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int N = radial.nmax;
    double v[64], g[64];
    for (int l = 0; l <= radial.lmax; l++) {
        if (!radial_compute(radial, l, r[i], v, derivs ? g : nullptr)) atomicExch(status, 1);
        for (int q = 0; q < N; q++) {
            values[i * ld + l * N + q] = (float)v[q];
            if (derivs) derivs[i * ld + l * N + q] = (float)g[q];
        }
    }
}

}  // namespace

void launch_radial_reference(const DeviceRadial& radial, const double* r, int64_t n, float* values, float* derivs,
                             int64_t ld, int32_t* status, cudaStream_t stream) {
    if (n == 0) return;
    const int threads = 128;
    radial_reference_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, stream>>>(radial, r, n, values,
                                                                                          derivs, ld, status);
    CUDA_CHECK(cudaGetLastError());
}

void launch_surrogate_mma(const float* master, int hidden, int O, int out_pad, double rc, const float* scale,
                          const void* w2_bf16, const void* w3_bf16, const double* r, int64_t n, float* values,
                          float* derivs, int64_t ld, int32_t* status, cudaStream_t stream, float* features = nullptr);
void pack_surrogate_weights(const float* master, int hidden, int O, int out_pad, void* w2_bf16, void* w3_bf16,
                            cudaStream_t stream);

RadialSurrogate::RadialSurrogate(Engine& engine, int hidden, uint64_t seed) : engine_(engine), H_(hidden), seed_(seed) {
    if (hidden != MLP_H) throw invalid_parameter("the radial surrogate supports 64 hidden units");
    const Hypers& h = engine.hypers();
    O_ = (h.max_angular + 1) * h.nmax();
    if (O_ > 256) throw invalid_parameter("the radial surrogate supports at most 256 outputs ((max_angular + 1) * (max_radial + 1))");
    out_pad_ = (O_ + 15) / 16 * 16;
    rc_ = h.cutoff;
    CUDA_CHECK(cudaGetDevice(&device_));
    const Offsets off = Offsets::make(H_, O_);
    n_params_ = off.total;
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
        buffers_.push_back(p);
        return p;
    };
    d_master_ = (float*)alloc(4 * n_params_);
    d_grad_ = (float*)alloc(4 * n_params_);
    d_m_ = (float*)alloc(4 * n_params_);
    d_v_ = (float*)alloc(4 * n_params_);
    d_step_ = (int64_t*)alloc(8);
    d_loss_ = (float*)alloc(8);
    d_scale_ = (float*)alloc(4 * O_);
    // hi, mid and lo BF16 parts of W2 and W3 in the tensor-core layout
    d_w2_bf16_ = alloc(3 * 2 * (size_t)H_ * H_);
    d_w3_bf16_ = alloc(3 * 2 * (size_t)out_pad_ * H_);
    // initial weights: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)), w1 wider so that
    // the first layer covers the input range
    std::vector<float> p(n_params_, 0.0f);
    uint64_t state = seed;
    auto uniform = [&](float a) {
        state = splitmix64(state);
        return (float)(((state >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * a;
    };
    for (int k = 0; k < H_; k++) {
        p[off.w1 + k] = uniform(4.0f);
        p[off.b1 + k] = uniform(2.0f);
    }
    for (int k = 0; k < H_ * H_; k++) p[off.w2 + k] = uniform(1.0f / std::sqrt((float)H_));
    for (int k = 0; k < O_ * H_; k++) p[off.w3 + k] = uniform(1.0f / std::sqrt((float)H_));
    CUDA_CHECK(cudaMemcpy(d_master_, p.data(), 4 * n_params_, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_m_, 0, 4 * n_params_));
    CUDA_CHECK(cudaMemset(d_v_, 0, 4 * n_params_));
    CUDA_CHECK(cudaMemset(d_step_, 0, 8));
    scale_.assign(O_, 1.0f);
    CUDA_CHECK(cudaMemcpy(d_scale_, scale_.data(), 4 * O_, cudaMemcpyHostToDevice));
}

RadialSurrogate::~RadialSurrogate() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (void* p : buffers_) cudaFree(p);
}

void RadialSurrogate::make_dataset(int64_t n, uint64_t seed, cudaStream_t stream) {
    if (n < 1 || n > ((int64_t)1 << 26)) throw invalid_parameter("the training set must hold 1 to 2^26 samples");
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
        buffers_.push_back(p);
        return p;
    };
    n_samples_ = n;
    d_r_ = (float*)alloc(4 * n);
    d_t_ = (float*)alloc(4 * (size_t)n * O_);
    d_dt_ = (float*)alloc(4 * (size_t)n * O_);
    int32_t* status = (int32_t*)alloc(4);
    CUDA_CHECK(cudaMemsetAsync(status, 0, 4, stream));
    DeviceRadial exact = engine_.device_radial();
    exact.splined = 0;
    const int threads = 128;
    surrogate_dataset_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, stream>>>(exact, n, rc_, seed, d_r_,
                                                                                             d_t_, d_dt_, status);
    CUDA_CHECK(cudaGetLastError());
    surrogate_scale_kernel<<<O_, 256, 0, stream>>>(d_t_, n, O_, d_scale_);
    CUDA_CHECK(cudaGetLastError());
    // values and r-derivatives normalised by each output's largest |value|
    surrogate_normalise_kernel<<<(unsigned)((n * O_ + 255) / 256), 256, 0, stream>>>(d_t_, n, O_, d_scale_);
    CUDA_CHECK(cudaGetLastError());
    surrogate_normalise_kernel<<<(unsigned)((n * O_ + 255) / 256), 256, 0, stream>>>(d_dt_, n, O_, d_scale_);
    CUDA_CHECK(cudaGetLastError());
    int32_t h_status = 0;
    CUDA_CHECK(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaMemcpyAsync(scale_.data(), d_scale_, 4 * O_, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status) throw internal_error("the analytic radial integral did not converge for the training set");
}

void RadialSurrogate::batch_step(int64_t batch, bool sample, cudaStream_t stream, double lr) {
    const Offsets off = Offsets::make(H_, O_);
    TrainArgs a{};
    a.O = O_;
    a.rc = rc_;
    a.master = d_master_;
    a.r = d_r_;
    a.targets = d_t_;
    a.dtargets = d_dt_;
    a.deriv_weight = (float)deriv_weight_;
    a.n = n_samples_;
    a.batch = batch;
    a.sample = sample ? 1 : 0;
    a.seed = seed_;
    a.step = d_step_;
    a.x = bufs_.x;
    a.h1 = bufs_.h1;
    a.dh1 = bufs_.dh1;
    a.dz1 = bufs_.dz1;
    a.gw1 = bufs_.gw1;
    a.h2 = bufs_.h2;
    a.dh2 = bufs_.dh2;
    a.dz2 = bufs_.dz2;
    a.ddz2 = bufs_.ddz2;
    a.dy = bufs_.dy;
    a.df = bufs_.df;
    a.loss_part = bufs_.loss_part;
    const int threads = 128;
    const int blocks = (int)((batch + threads - 1) / threads);
    const size_t smem = 4 * (size_t)off.total;
    surrogate_sample_kernel<<<blocks, threads, smem, stream>>>(a);
    CUDA_CHECK(cudaGetLastError());
    const int chunks = (int)((batch + GRAD_CHUNK - 1) / GRAD_CHUNK);
    float* partial = bufs_.partial;
    surrogate_gradient_kernel<<<dim3((off.total + 127) / 128, chunks), 128, 0, stream>>>(a, partial, chunks);
    CUDA_CHECK(cudaGetLastError());
    surrogate_sum_kernel<<<(off.total + 127) / 128, 128, 0, stream>>>(partial, chunks, off.total, d_grad_,
                                                                       bufs_.loss_part, blocks, d_loss_);
    CUDA_CHECK(cudaGetLastError());
    if (lr > 0.0) {
        surrogate_adam_kernel<<<(off.total + 127) / 128, 128, 0, stream>>>(d_master_, d_grad_, d_m_, d_v_, off.total,
                                                                           d_step_, graph_steps_ > 0 ? graph_steps_ : 1,
                                                                           (float)lr);
        CUDA_CHECK(cudaGetLastError());
        surrogate_step_kernel<<<1, 1, 0, stream>>>(d_step_);
        CUDA_CHECK(cudaGetLastError());
    }
}

void RadialSurrogate::ensure_batch(int64_t batch) {
    if (batch <= batch_cap_) return;
    auto alloc = [&](size_t count) {
        void* p = nullptr;
        CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(4 * count, 16)));
        buffers_.push_back(p);
        return (float*)p;
    };
    const int64_t chunks = (batch + GRAD_CHUNK - 1) / GRAD_CHUNK;
    const size_t bh = (size_t)batch * H_, bo = (size_t)batch * O_;
    bufs_.x = alloc(batch);
    bufs_.h1 = alloc(bh);
    bufs_.dh1 = alloc(bh);
    bufs_.dz1 = alloc(bh);
    bufs_.gw1 = alloc(bh);
    bufs_.h2 = alloc(bh);
    bufs_.dh2 = alloc(bh);
    bufs_.dz2 = alloc(bh);
    bufs_.ddz2 = alloc(bh);
    bufs_.dy = alloc(bo);
    bufs_.df = alloc(bo);
    bufs_.partial = alloc((size_t)chunks * n_params_);
    bufs_.loss_part = alloc((batch + 127) / 128);
    batch_cap_ = batch;
}

double RadialSurrogate::train(int64_t steps, int64_t batch, double lr, cudaStream_t stream) {
    if (n_samples_ == 0) throw invalid_parameter("make the training set before training");
    if (batch < 1 || batch > ((int64_t)1 << 20)) throw invalid_parameter("the minibatch must hold 1 to 2^20 samples");
    if (steps < 1) return 0.0;
    const bool rebuild = !graph_exec_ || graph_steps_ != steps || batch > batch_cap_ || graph_lr_ != lr ||
                         graph_deriv_weight_ != deriv_weight_;
    ensure_batch(batch);
    if (rebuild) {
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (graph_) cudaGraphDestroy(graph_);
        graph_exec_ = nullptr;
        graph_ = nullptr;
        graph_steps_ = steps;  // decay horizon of the learning rate
        graph_lr_ = lr;
        graph_deriv_weight_ = deriv_weight_;
        cudaStream_t cap = nullptr;
        CUDA_CHECK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        CUDA_CHECK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        try {
            batch_step(batch, true, cap, lr);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(cap, &g);
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cap);
            throw;
        }
        CUDA_CHECK(cudaStreamEndCapture(cap, &graph_));
        CUDA_CHECK(cudaStreamDestroy(cap));
        CUDA_CHECK(cudaGraphInstantiate(&graph_exec_, graph_, 0));
    }
    CUDA_CHECK(cudaMemsetAsync(d_step_, 0, 8, stream));
    CUDA_CHECK(cudaMemsetAsync(d_m_, 0, 4 * n_params_, stream));
    CUDA_CHECK(cudaMemsetAsync(d_v_, 0, 4 * n_params_, stream));
    for (int64_t s = 0; s < steps; s++) CUDA_CHECK(cudaGraphLaunch(graph_exec_, stream));
    float loss = 0.0f;
    CUDA_CHECK(cudaMemcpyAsync(&loss, d_loss_, 4, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    return (double)loss / (double)(batch * O_);
}

double RadialSurrogate::loss_and_gradient(int64_t n, std::vector<float>& gradient, cudaStream_t stream) {
    if (n_samples_ == 0) throw invalid_parameter("make the training set first");
    if (n < 1 || n > n_samples_) throw invalid_parameter("the gradient batch must be within the training set");
    ensure_batch(n);
    batch_step(n, false, stream, 0.0);
    gradient.resize(n_params_);
    float loss = 0.0f;
    CUDA_CHECK(cudaMemcpyAsync(gradient.data(), d_grad_, 4 * n_params_, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaMemcpyAsync(&loss, d_loss_, 4, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    return (double)loss / (double)(n * O_);
}

std::vector<float> RadialSurrogate::parameters(cudaStream_t stream) const {
    std::vector<float> p(n_params_);
    CUDA_CHECK(cudaMemcpyAsync(p.data(), d_master_, 4 * n_params_, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    return p;
}

void RadialSurrogate::set_parameters(const std::vector<float>& p, cudaStream_t stream) {
    if ((int64_t)p.size() != n_params_) throw invalid_parameter("wrong number of surrogate parameters");
    CUDA_CHECK(cudaMemcpyAsync(d_master_, p.data(), 4 * n_params_, cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

std::vector<float> RadialSurrogate::dataset_r(cudaStream_t stream) const {
    std::vector<float> r(n_samples_);
    if (n_samples_) {
        CUDA_CHECK(cudaMemcpyAsync(r.data(), d_r_, 4 * n_samples_, cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
    }
    return r;
}

void RadialSurrogate::evaluate_reference(const double* r, int64_t n, float* values, float* derivs, int64_t ld,
                                         bool analytic, cudaStream_t stream) {
    if (ld < O_) throw invalid_parameter("the output row stride must be at least the number of outputs");
    DeviceRadial radial = engine_.device_radial();
    if (analytic) radial.splined = 0;
    else if (!radial.splined) throw invalid_parameter("this calculator has no spline (spline_accuracy is null)");
    int32_t* status = (int32_t*)d_loss_ + 1;
    CUDA_CHECK(cudaMemsetAsync(status, 0, 4, stream));
    launch_radial_reference(radial, r, n, values, derivs, ld, status, stream);
    int32_t h_status = 0;
    CUDA_CHECK(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status) throw internal_error("the analytic radial integral did not converge");
}

void RadialSurrogate::evaluate(const double* r, int64_t n, float* values, float* derivs, int64_t ld, bool tensor_cores,
                               cudaStream_t stream, bool check, bool bf16_weights) {
    if (n == 0) return;
    if (ld < O_) throw invalid_parameter("the output row stride must be at least the number of outputs");
    if (!tensor_cores) {
        const Offsets off = Offsets::make(H_, O_);
        const int threads = 128;
        surrogate_eval_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 4 * (size_t)off.total, stream>>>(
            d_master_, O_, rc_, d_scale_, r, n, values, derivs, ld, bf16_weights ? 1 : 0);
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    pack_surrogate_weights(d_master_, H_, O_, out_pad_, d_w2_bf16_, d_w3_bf16_, stream);
    int32_t* status = (int32_t*)d_loss_ + 1;
    CUDA_CHECK(cudaMemsetAsync(status, 0, 4, stream));
    launch_surrogate_mma(d_master_, H_, O_, out_pad_, rc_, d_scale_, d_w2_bf16_, d_w3_bf16_, r, n, values, derivs, ld,
                         status, stream);
    if (!check) return;
    int32_t h_status = 0;
    CUDA_CHECK(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status) throw internal_error("the tensor-core surrogate kernel timed out waiting for its MMAs");
}

void RadialSurrogate::fit_output_layer(double lambda, cudaStream_t stream) {
    if (n_samples_ == 0) throw invalid_parameter("make the training set before fitting the output layer");
    if (!(lambda >= 0.0 && std::isfinite(lambda))) throw invalid_parameter("the derivative weight must be >= 0");
    const int F = H_ + 1, W = H_ + 1 + O_;
    const int64_t chunk = std::min<int64_t>(n_samples_, 1 << 16);
    std::vector<void*> scratch;
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        CUDA_CHECK(cudaMallocAsync(&p, std::max<size_t>(bytes, 16), stream));
        scratch.push_back(p);
        return p;
    };
    double* rows = (double*)alloc(sizeof(double) * 2 * (size_t)chunk * W);
    double* M = (double*)alloc(sizeof(double) * (size_t)F * W);
    float* features = (float*)alloc(sizeof(float) * 2 * (size_t)chunk * H_);
    double* r = (double*)alloc(sizeof(double) * (size_t)chunk);
    int32_t* status = (int32_t*)alloc(4);
    CUDA_CHECK(cudaMemsetAsync(M, 0, sizeof(double) * (size_t)F * W, stream));
    CUDA_CHECK(cudaMemsetAsync(status, 0, 4, stream));
    const double dweight = std::sqrt(lambda) * 0.5 * rc_;
    pack_surrogate_weights(d_master_, H_, O_, out_pad_, d_w2_bf16_, d_w3_bf16_, stream);
    for (int64_t s0 = 0; s0 < n_samples_; s0 += chunk) {
        const int64_t count = std::min(chunk, n_samples_ - s0);
        // the hidden features with the numerics of the tensor-core kernel
        surrogate_widen_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(d_r_ + s0, count, r);
        CUDA_CHECK(cudaGetLastError());
        launch_surrogate_mma(d_master_, H_, O_, out_pad_, rc_, d_scale_, d_w2_bf16_, d_w3_bf16_, r, count, nullptr,
                             nullptr, O_, status, stream, features);
        surrogate_fit_rows_kernel<<<(unsigned)((count + 127) / 128), 128, 0, stream>>>(features, O_, d_t_, d_dt_, s0,
                                                                                       count, dweight, rows);
        CUDA_CHECK(cudaGetLastError());
        const int64_t entries = (int64_t)F * W;
        surrogate_normal_kernel<<<(unsigned)((entries + 127) / 128), 128, 0, stream>>>(rows, 2 * count, O_, M);
        CUDA_CHECK(cudaGetLastError());
    }
    const size_t smem = sizeof(double) * (size_t)F * W;
    CUDA_CHECK(cudaFuncSetAttribute(surrogate_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    surrogate_solve_kernel<<<1, 256, smem, stream>>>(M, O_, d_master_, status);
    CUDA_CHECK(cudaGetLastError());
    int32_t h_status = 0;
    CUDA_CHECK(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, stream));
    for (void* p : scratch) CUDA_CHECK(cudaFreeAsync(p, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status & 1) throw internal_error("the tensor-core surrogate kernel timed out waiting for its MMAs");
    if (h_status) throw internal_error("the least-squares fit of the surrogate's output layer is singular");
}

void surrogate_fill(RadialSurrogate* surrogate, const double* distance, int64_t n, float* values, float* derivs,
                    int64_t ld, cudaStream_t stream) {
    surrogate->evaluate(distance, n, values, derivs, ld, surrogate->out_pad() <= 128, stream, false);
}

}  // namespace fb200

// Kernel (c): SOAP power spectrum and its gradients on the GPU, FP64.
//
//   P[l, n1, n2] = sum_m c_a[l m n1] c_b[l m n2] * (sqrt 2 if a != b) / ((-1)^l sqrt(2l+1))
//
// featomic/src/calculators/soap/power_spectrum.rs:571-764.  One CTA per
// centre keeps the centre's expansion coefficients (all neighbour species) in
// shared memory.  Every output row is a set of per-l products
//
//   G[x][n1][n2] = sum_m v[l m n2] g[x][l m n1]  (+ sum_m v'[l m n1] g'[x][l m n2])
//
// evaluated one l at a time by a warp: all lanes share l (so the m-loops do
// not diverge) and each lane accumulates two consecutive (n1, n2) outputs for
// every component.  Sums run over m in featomic's order with fused
// multiply-adds (one rounding per term instead of two; the results stay
// within 1e-10 relative + 1e-12 of the largest magnitude of featomic's
// unfused sums), and each row is written exactly once, with 512-byte
// contiguous streaming stores, into the final TensorMap block layout ([sample][property], [gradient row][xyz]
// [property], [sample][3][3][property]).
//
// positions gradient of row (centre i, atom j):
//   j == i : sum_m c_b dself_a + c_a dself_b
//   j != i : sum_m c_b dc_a(i<-j) [type(j) == a] + c_a dc_b(i<-j) [type(j) == b]
// with dc(i<-j) = sum over the pairs between i and j of g_pair (i first) or
// -(-1)^l g_pair (i second), in pair order, read in place.  The row index
// inside a block is
// the slot's first row plus the rank of the neighbour among the rows of that
// sample (prefix counts per species).

#include <cub/cub.cuh>

#include <map>
#include <mutex>

#include "engine.hpp"

namespace fb200 {

namespace {

constexpr double SQRT_2 = 1.4142135623730951;

__device__ __forceinline__ int isqrt_lm(int lm) {
    int l = (int)sqrt((double)lm);
    while (l * l > lm) l--;
    while ((l + 1) * (l + 1) <= lm) l++;
    return l;
}

__device__ __forceinline__ double ps_norm(int l) {
    double s = sqrt((double)(2 * l + 1));
    return (l % 2 == 0) ? s : -s;
}

// Sources of the "gradient" operand of a tile.  Multiplying by
// -(-1)^l (the reversed orientation of a pair) is exact, so reading a pair
// gradient in place equals staging its flipped copy; several periodic images
// are summed element by element in pair order, like featomic's
// positions-gradient block.
struct DirectSource {
    const double* p;
    bool flip;
    __device__ __forceinline__ double load(int idx, double sl) const { return flip ? sl * p[idx] : p[idx]; }
};

struct ImagesSource {
    const int32_t* codes;
    int n;
    const double* pair_grad;
    int64_t stride;  // 3 K
    __device__ __forceinline__ double load(int idx, double sl) const {
        double v = 0.0;
        for (int d = 0; d < n; d++) {
            const int32_t code = codes[d];
            const double g = pair_grad[(int64_t)(code >> 1) * stride + idx];
            v += (code & 1) ? sl * g : g;
        }
        return v;
    }
};

// m-sum of one (l, lane) tile from raw pointers (already offset to the
// lane's n1 / n2 and to the first m of l).  NEG subtracts the products, which
// equals adding the products with the operand negated (negation is exact).
template <int NC, bool NEG, bool PAIRED>
__device__ __forceinline__ void sum_term1(int nm, int nmax, int stride, const double* __restrict__ g,
                                          const double* __restrict__ v, double (&acc)[NC][2]) {
    // acc[x][j] += v[m][n2_j] * g[x][m][n1]   (PAIRED: both outputs share n1)
    for (int m = 0; m < nm; m++, g += nmax, v += nmax) {
        const double va = v[0], vb = v[1];
#pragma unroll
        for (int x = 0; x < NC; x++) {
            const double gx = g[x * stride];
            if (NEG) {
                acc[x][0] = __fma_rn(-va, gx, acc[x][0]);
                acc[x][1] = __fma_rn(-vb, gx, acc[x][1]);
            } else {
                acc[x][0] = __fma_rn(va, gx, acc[x][0]);
                acc[x][1] = __fma_rn(vb, gx, acc[x][1]);
            }
        }
    }
}

template <int NC, bool NEG>
__device__ __forceinline__ void sum_term2(int nm, int nmax, int stride, const double* __restrict__ g,
                                          const double* __restrict__ v, double (&acc)[NC][2]) {
    // acc[x][j] += v[m][n1] * g[x][m][n2_j]
    for (int m = 0; m < nm; m++, g += nmax, v += nmax) {
        const double u = v[0];
#pragma unroll
        for (int x = 0; x < NC; x++) {
            const double ga = g[x * stride], gb = g[x * stride + 1];
            if (NEG) {
                acc[x][0] = __fma_rn(-u, ga, acc[x][0]);
                acc[x][1] = __fma_rn(-u, gb, acc[x][1]);
            } else {
                acc[x][0] = __fma_rn(u, ga, acc[x][0]);
                acc[x][1] = __fma_rn(u, gb, acc[x][1]);
            }
        }
    }
}

// Tile rows of one output row, even nmax: every lane of the warp shares l
// (uniform m-loop trip counts) and owns the two consecutive outputs
// q = 2 lane, 2 lane + 1 (+ 64 k) of q = n1 nmax + n2, for all NC components:
//   acc[x][j] = sum_m v2[l m n2] * g1[x][l m n1]   (if g1)
//             + sum_m v1[l m n1] * g2[x][l m n2]   (if g2)
// with g1 / g2 negated on even l when flip1 / flip2 (the -(-1)^l factor of a
// reversed pair).  Each element is summed over m in featomic's order; the
// scaling (sqrt 2 if a != b) / ((-1)^l sqrt(2l+1)) is applied at the end.
template <int NC>
__device__ __forceinline__ void rows_even(int lane, int lmax, int nmax, int stride, const double* g1, bool flip1,
                                          const double* v2, const double* v1, const double* g2, bool flip2,
                                          double* __restrict__ out, int64_t xstride, const double* scale_l) {
    const int nn = nmax * nmax;
    for (int qa = 2 * lane; qa < nn; qa += 64) {
        const int n1 = qa / nmax, n2 = qa - n1 * nmax;
        for (int l = 0; l <= lmax; l++) {
            const int base = l * l * nmax;
            const int nm = 2 * l + 1;
            const bool even = (l & 1) == 0;
            double acc[NC][2];
#pragma unroll
            for (int x = 0; x < NC; x++) acc[x][0] = acc[x][1] = 0.0;
            if (g1) {
                if (flip1 && even) sum_term1<NC, true, true>(nm, nmax, stride, g1 + base + n1, v2 + base + n2, acc);
                else sum_term1<NC, false, true>(nm, nmax, stride, g1 + base + n1, v2 + base + n2, acc);
            }
            if (g2) {
                if (flip2 && even) sum_term2<NC, true>(nm, nmax, stride, g2 + base + n2, v1 + base + n1, acc);
                else sum_term2<NC, false>(nm, nmax, stride, g2 + base + n2, v1 + base + n1, acc);
            }
            const double scale = scale_l[l];
            double* o = out + (int64_t)l * nn + qa;
#pragma unroll
            for (int x = 0; x < NC; x++) {
                double2 w;
                w.x = acc[x][0] * scale;
                w.y = acc[x][1] * scale;
                __stcs(reinterpret_cast<double2*>(o + x * xstride), w);
            }
        }
    }
}

// Generic tile of one l (odd nmax, or several periodic images summed on the
// fly): the lane owns outputs q = 2 lane, 2 lane + 1 (+ 64 k).
template <int NC, typename G1, typename G2>
__device__ __forceinline__ void l_tile(int lane, int l, int nmax, int stride, bool use1, const G1& g1,
                                       const double* __restrict__ v2, const double* __restrict__ v1, bool use2,
                                       const G2& g2, double* __restrict__ out, int64_t xstride, double scale) {
    const int nn = nmax * nmax;
    const int base = l * l * nmax;
    const int nm = 2 * l + 1;
    const double sl = (l & 1) ? 1.0 : -1.0;
    double* o = out + (int64_t)l * nn;
    for (int qa = 2 * lane; qa < nn; qa += 64) {
        const int qb = qa + 1;
        const bool hasb = qb < nn;
        const int n1a = qa / nmax, n2a = qa - n1a * nmax;
        const int n1b = hasb ? qb / nmax : n1a, n2b = hasb ? qb - n1b * nmax : n2a;
        double acc[NC][2];
#pragma unroll
        for (int x = 0; x < NC; x++) acc[x][0] = acc[x][1] = 0.0;
        if (use1) {
            for (int m = 0; m < nm; m++) {
                const int row = base + m * nmax;
                const double va = v2[row + n2a], vb = v2[row + n2b];
#pragma unroll
                for (int x = 0; x < NC; x++) {
                    const double ga = g1.load(x * stride + row + n1a, sl);
                    const double gb = (n1b == n1a) ? ga : g1.load(x * stride + row + n1b, sl);
                    acc[x][0] = __fma_rn(va, ga, acc[x][0]);
                    acc[x][1] = __fma_rn(vb, gb, acc[x][1]);
                }
            }
        }
        if (use2) {
            for (int m = 0; m < nm; m++) {
                const int row = base + m * nmax;
                const double ua = v1[row + n1a], ub = v1[row + n1b];
#pragma unroll
                for (int x = 0; x < NC; x++) {
                    acc[x][0] = __fma_rn(ua, g2.load(x * stride + row + n2a, sl), acc[x][0]);
                    acc[x][1] = __fma_rn(ub, g2.load(x * stride + row + n2b, sl), acc[x][1]);
                }
            }
        }
#pragma unroll
        for (int x = 0; x < NC; x++) {
            o[x * xstride + qa] = acc[x][0] * scale;
            if (hasb) o[x * xstride + qb] = acc[x][1] * scale;
        }
    }
}

// one output row (all l): the fast even-nmax path for in-place operands,
// the generic path otherwise
template <int NC, typename G1, typename G2>
__device__ __forceinline__ void rows(int lane, int lmax, int nmax, int stride, bool use1, const G1& g1,
                                     const double* v2, const double* v1, bool use2, const G2& g2, double* out,
                                     int64_t xstride, const double* scale_l) {
    for (int l = 0; l <= lmax; l++)
        l_tile<NC>(lane, l, nmax, stride, use1, g1, v2, v1, use2, g2, out, xstride, scale_l[l]);
}

template <int NC>
__device__ __forceinline__ void rows(int lane, int lmax, int nmax, int stride, bool use1, const DirectSource& g1,
                                     const double* v2, const double* v1, bool use2, const DirectSource& g2, double* out,
                                     int64_t xstride, const double* scale_l) {
    if ((nmax & 1) == 0 && ((xstride & 1) == 0) && ((((uintptr_t)out) & 15) == 0)) {
        rows_even<NC>(lane, lmax, nmax, stride, use1 ? g1.p : nullptr, g1.flip, v2, v1, use2 ? g2.p : nullptr, g2.flip,
                      out, xstride, scale_l);
    } else {
        for (int l = 0; l <= lmax; l++)
            l_tile<NC>(lane, l, nmax, stride, use1, g1, v2, v1, use2, g2, out, xstride, scale_l[l]);
    }
}

// (sqrt 2 if mixed) / ((-1)^l sqrt(2l+1)) for l = 0..lmax, in shared memory:
// entries [0, L] unmixed, [L + 1, 2L + 1] mixed
__device__ __forceinline__ void load_scales(int lmax, double* scale_s) {
    for (int i = threadIdx.x; i < 2 * (lmax + 1); i += blockDim.x) {
        const int l = i % (lmax + 1);
        const double s = sqrt((double)(2 * l + 1));
        const double norm = (l % 2 == 0) ? s : -s;
        scale_s[i] = (i > lmax ? SQRT_2 : 1.0) * (1.0 / norm);
    }
}

__device__ __forceinline__ void load_coefficients(const PsArgs& a, int64_t c, double* coef_s, int SK) {
    const double* src = a.coef + c * SK;
    for (int i = threadIdx.x; i < SK; i += blockDim.x) coef_s[i] = src[i];
}

template <int MAXN>
__global__ void __launch_bounds__(256) ps_values_kernel(PsArgs a) {
    extern __shared__ double smem[];
    const int64_t c = blockIdx.x;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    double* coef_s = smem;
    double* scale_s = smem + a.n_species * K;
    load_coefficients(a, c, coef_s, a.n_species * K);
    load_scales(a.lmax, scale_s);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int64_t s0 = a.slot_offset[c], ns = a.slot_offset[c + 1] - s0;
    for (int64_t s = warp; s < ns; s += nwarps) {
        const PsKeySlot slot = a.slots[s0 + s];
        double* out = a.out + a.off_values[slot.block] + (int64_t)slot.sample * a.n_props;
        DirectSource ca{coef_s + slot.a * K, false};
        rows<1>(lane, a.lmax, a.nmax, K, true, ca, coef_s + slot.b * K, nullptr, false, ca, out, a.n_props,
                scale_s + (slot.a != slot.b ? a.lmax + 1 : 0));
    }
}

// one positions-gradient row (both kinds of source)
template <typename G>
__device__ __forceinline__ void positions_row(const PsArgs& a, int lane, int K, const double* coef_s,
                                              const double* scale_s, const PsKeySlot& slot, bool self, int species,
                                              const G& g, const double* self_a, const double* self_b, double* out) {
    const double* scales = scale_s + (slot.a != slot.b ? a.lmax + 1 : 0);
    const double* ca = coef_s + slot.a * K;
    const double* cb = coef_s + slot.b * K;
    if (self) {
        DirectSource s1{self_a, false}, s2{self_b, false};
        rows<3>(lane, a.lmax, a.nmax, K, true, s1, cb, ca, true, s2, out, a.n_props, scales);
    } else {
        rows<3>(lane, a.lmax, a.nmax, K, species == slot.a, g, cb, ca, species == slot.b, g, out, a.n_props, scales);
    }
}

// D[n1][n2] += sum_k A[n1][k] B[k][n2] on the FP64 tensor cores (DMMA,
// 8 x 8 x 4): lane t holds A[t / 4][t % 4] and B[t % 4][t / 4] and the two
// outputs D[t / 4][2 (t % 4) + {0, 1}]
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

constexpr int DMMA_SLOTS = 4;

// Positions-gradient rows of one neighbour entry that shares a single pair
// with the centre, nmax <= 8, on the FP64 tensor cores.  For a slot (a, b)
// and the entry's species s, per l:
//   s == a:  rows += G^T C_b   (sum_m g[x][l m][n1] c_b[l m][n2])
//   s == b:  rows += C_a^T G   (sum_m c_a[l m][n1] g[x][l m][n2])
// with G the pair gradient (times -(-1)^l for a reversed pair).  Lane t owns
// m = m0 + t % 4, n = t / 4 of every fragment: the same register of G is the
// A operand of the first product and the B operand of the second.  Up to
// DMMA_SLOTS slots share the loads of G.
__device__ void positions_entry_dmma(const PsArgs& a, int lane, int K, const double* __restrict__ coef_s,
                                     const double* __restrict__ scale_s, const double* __restrict__ g, bool flip,
                                     int species, const int32_t* slot_ab, const int64_t* slot_base,
                                     const int32_t* cum_w, int64_t ns) {
    const int S = a.n_species, N = a.nmax;
    const int tm = lane & 3, tn = lane >> 2;
    const bool n_ok = tn < N;
    const int n2 = 2 * tm;
    int64_t s = 0;
    while (s < ns) {
        // the next chunk of slots that contain the entry's species
        int sa[DMMA_SLOTS], sb[DMMA_SLOTS];
        double* out[DMMA_SLOTS];
        int count = 0;
#pragma unroll
        for (int i = 0; i < DMMA_SLOTS; i++) {
            sa[i] = sb[i] = -1;
            out[i] = nullptr;
            while (s < ns) {
                const int x = slot_ab[2 * s], y = slot_ab[2 * s + 1];
                const int64_t here = s++;
                if (species != x && species != y) continue;
                const int64_t rank = cum_w[x] + (x != y ? cum_w[y] : 0) + cum_w[S];
                sa[i] = x;
                sb[i] = y;
                out[i] = a.out + slot_base[here] + rank * 3 * a.n_props;
                count = i + 1;
                break;
            }
        }
        if (count == 0) break;
        for (int l = 0; l <= a.lmax; l++) {
            const int M = 2 * l + 1, base = l * l * N;
            const double sign = (flip && (l & 1) == 0) ? -1.0 : 1.0;
            double acc[DMMA_SLOTS][3][2];
#pragma unroll
            for (int i = 0; i < DMMA_SLOTS; i++)
#pragma unroll
                for (int x = 0; x < 3; x++) acc[i][x][0] = acc[i][x][1] = 0.0;
            for (int m0 = 0; m0 < M; m0 += 4) {
                const int m = m0 + tm;
                const bool ok = n_ok && m < M;
                const int idx = base + m * N + tn;
                double gx[3];
#pragma unroll
                for (int x = 0; x < 3; x++) gx[x] = ok ? sign * g[x * K + idx] : 0.0;
#pragma unroll
                for (int i = 0; i < DMMA_SLOTS; i++) {
                    if (i < count) {
                        if (species == sa[i]) {
                            const double cb = ok ? coef_s[sb[i] * K + idx] : 0.0;
#pragma unroll
                            for (int x = 0; x < 3; x++) dmma_8x8x4(acc[i][x], gx[x], cb);
                        }
                        if (species == sb[i]) {
                            const double ca = ok ? coef_s[sa[i] * K + idx] : 0.0;
#pragma unroll
                            for (int x = 0; x < 3; x++) dmma_8x8x4(acc[i][x], ca, gx[x]);
                        }
                    }
                }
            }
            const int64_t o = (int64_t)l * N * N + (int64_t)tn * N + n2;
#pragma unroll
            for (int i = 0; i < DMMA_SLOTS; i++) {
                if (i < count && n_ok) {
                    const double scale = scale_s[(sa[i] != sb[i] ? a.lmax + 1 : 0) + l];
#pragma unroll
                    for (int x = 0; x < 3; x++) {
                        double* dst = out[i] + x * a.n_props + o;
                        if (N == 8) {
                            double2 w;
                            w.x = acc[i][x][0] * scale;
                            w.y = acc[i][x][1] * scale;
                            __stcs(reinterpret_cast<double2*>(dst), w);
                        } else {
                            if (n2 < N) dst[0] = acc[i][x][0] * scale;
                            if (n2 + 1 < N) dst[1] = acc[i][x][1] * scale;
                        }
                    }
                }
            }
        }
    }
}

constexpr int POS_WARPS = 4;
// resident CTAs per SM the register budget is set for (128 registers)
constexpr int POS_MIN_BLOCKS = 4;
// CTAs per centre, each taking every POS_SPLIT-th group of POS_WARPS entries:
// more, smaller CTAs shorten the last wave
constexpr int POS_SPLIT = 2;
// per-centre slot tables staged in shared memory (centres with at most this
// many slots; more read them from global memory) and per-warp entry counts
constexpr int POS_SLOT_CAP = 64;
constexpr int POS_CUM_CAP = 65;
constexpr size_t POS_TABLE_BYTES = POS_SLOT_CAP * (8 + 2 * 4) + POS_WARPS * POS_CUM_CAP * 4;

template <int MAXN>
__global__ void __launch_bounds__(POS_WARPS * 32, POS_MIN_BLOCKS) ps_positions_kernel(PsArgs a) {
    extern __shared__ double smem[];
    const int64_t c = blockIdx.x / POS_SPLIT;
    const int part = (int)(blockIdx.x - c * POS_SPLIT);
    const int S = a.n_species;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int64_t head = (S * K + 2 * (a.lmax + 1) + 1) & ~1;
    double* coef_s = smem;
    double* scale_s = smem + S * K;
    // output-row tables: the first output element of every slot and its
    // species pair, then each warp's copy of its entry's counts, so that the
    // slot loop reads shared memory instead of a chain of dependent global
    // loads (slot -> counts -> first row -> block offset)
    int64_t* slot_base = reinterpret_cast<int64_t*>(smem + head);
    int32_t* slot_ab = reinterpret_cast<int32_t*>(slot_base + POS_SLOT_CAP);
    int32_t* cum_w = slot_ab + 2 * POS_SLOT_CAP + warp * POS_CUM_CAP;
    load_coefficients(a, c, coef_s, S * K);
    load_scales(a.lmax, scale_s);
    const int64_t s0 = a.slot_offset[c], ns = a.slot_offset[c + 1] - s0;
    const bool tables = ns <= POS_SLOT_CAP;
    if (tables) {
        for (int64_t i = threadIdx.x; i < ns; i += blockDim.x) {
            const PsKeySlot slot = a.slots[s0 + i];
            slot_base[i] = a.off_positions[slot.block] + a.slot_row[s0 + i] * 3 * a.n_props;
            slot_ab[2 * i] = slot.a;
            slot_ab[2 * i + 1] = slot.b;
        }
    }
    __syncthreads();
    const int64_t e0 = a.entry_offset[c], ne = a.entry_offset[c + 1] - e0;
    for (int64_t e = warp + part * nwarps; e < ne; e += (int64_t)nwarps * POS_SPLIT) {
        const PsEntry entry = a.entries[e0 + e];
        const bool self = entry.atom == (int32_t)c;
        const int32_t* cum = a.entry_cum + (e0 + e) * (S + 1);
        const bool single = entry.d1 - entry.d0 <= 1;
        if (tables) {
            for (int i = lane; i <= S; i += 32) cum_w[i] = cum[i];
            __syncwarp();
        }
        if (tables && !self && entry.d1 - entry.d0 == 1 && a.nmax <= 8) {
            // the common entry: FP64 tensor cores, the pair gradient read in place
            const int32_t code = a.dir_code[entry.d0];
            positions_entry_dmma(a, lane, K, coef_s, scale_s, a.pair_grad + (int64_t)(code >> 1) * 3 * K, code & 1,
                                 entry.species, slot_ab, slot_base, cum_w, ns);
            __syncwarp();
            continue;
        }
        DirectSource direct{nullptr, false};
        ImagesSource images{a.dir_code + entry.d0, entry.d1 - entry.d0, a.pair_grad, 3 * (int64_t)K};
        if (!self && single && entry.d1 > entry.d0) {
            const int32_t code = a.dir_code[entry.d0];
            direct.p = a.pair_grad + (int64_t)(code >> 1) * 3 * K;
            direct.flip = code & 1;
        }
        for (int64_t s = 0; s < ns; s++) {
            PsKeySlot slot;
            double* out;
            if (tables) {
                slot = PsKeySlot{0, 0, slot_ab[2 * s], slot_ab[2 * s + 1]};
                if (!self && entry.species != slot.a && entry.species != slot.b) continue;
                const int64_t rank = cum_w[slot.a] + (slot.a != slot.b ? cum_w[slot.b] : 0) + cum_w[S];
                out = a.out + slot_base[s] + rank * 3 * a.n_props;
            } else {
                slot = a.slots[s0 + s];
                if (!self && entry.species != slot.a && entry.species != slot.b) continue;
                const int64_t rank = cum[slot.a] + (slot.a != slot.b ? cum[slot.b] : 0) + cum[S];
                const int64_t row = a.slot_row[s0 + s] + rank;
                out = a.out + a.off_positions[slot.block] + row * 3 * a.n_props;
            }
            const double* self_a = a.self_grad + ((int64_t)c * S + slot.a) * 3 * K;
            const double* self_b = a.self_grad + ((int64_t)c * S + slot.b) * 3 * K;
            if (self || single) {
                positions_row(a, lane, K, coef_s, scale_s, slot, self, entry.species, direct, self_a, self_b, out);
            } else {
                positions_row(a, lane, K, coef_s, scale_s, slot, self, entry.species, images, self_a, self_b, out);
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Positions-gradient rows, staged form (nmax <= 8, at most 10 species).
//
// A CTA owns a contiguous range of one centre's neighbour entries (the rows
// of consecutive entries in a slot are consecutive in memory).  Its four
// warps share, in shared memory:
//   * the centre's coefficients of every species in DMMA fragment order,
//     zero-padded to 4 m and 8 n per l (so that padding contributes nothing);
//   * two pair-gradient buffers, the next entry's filled by cp.async while
//     the current one is computed.  For nmax = 8 a buffer holds
//     [3][step][4 m][8 n] (m padded to 4 per l like the coefficients, the
//     padding kept at zero), with the 16-byte chunks of the rows m = 2, 3 of
//     each step swapped pairwise, so that a fragment load is one offset per
//     lane plus a warp-uniform step offset and its 32 lanes hit 32 distinct
//     banks in each half warp; other nmax keep featomic's [3][(l m)][n];
//   * the slot tables, the slots of each neighbour species, and the entry
//     metadata of up to STG_CHUNK entries.
// Every (entry, slot) is one item: a warp computes the whole gradient row
// (3 x (lmax + 1) tiles of 8 x 8, written front to back with 512-byte
// streaming stores) on the FP64 tensor cores, so each row leaves the SM in
// one short burst.  The per-l products and their order equal the per-warp
// DMMA form above.  Entries with several periodic images of one neighbour
// take the CUDA-core rows with global operands; the centre's own rows are
// written by ps_centre_rows_kernel on the side stream.
constexpr int STG_WARPS = 4;
constexpr int STG_RING = 2;
constexpr int STG_CHUNK = 64;
constexpr int STG_SPLIT = 2;
constexpr int STG_MAX_SPECIES = 10;
constexpr int STG_MAX_SLOTS = STG_MAX_SPECIES * (STG_MAX_SPECIES + 1) / 2;
constexpr int STG_MAX_STEPS = 5;
constexpr int STG_G_PAD = 32;  // doubles after an unpadded gradient buffer, read by the padded last m step

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// DMMA steps of 4 m values over l = 0..lmax
__host__ __device__ __forceinline__ int stg_steps(int lmax) {
    int n = 0;
    for (int l = 0; l <= lmax; l++) n += (2 * l + 1 + 3) / 4;
    return n;
}

// offset of lane (m = lane % 4, n = lane / 4) inside a 32-double step block
// of the swizzled nmax = 8 buffer: chunk n / 2 of rows m = 2, 3 is stored at
// (n / 2) ^ 2
__device__ __forceinline__ int stg_lane_offset8(int lane) {
    const int tm = lane & 3, tn = lane >> 2;
    return tm * 8 + ((((tn >> 1) ^ (((tm >> 1) & 1) << 1))) << 1) + (tn & 1);
}

struct StgLayout {
    int P;        // doubles per species of the fragment-ordered coefficients (32 per step)
    int GB;       // doubles per gradient buffer (even)
    size_t cf, scale, ring, rows, slot_base, slot_ab, sp_count, sp_slot, meta_entry, meta_code, meta_cum, bytes;
};

__host__ __device__ inline StgLayout stg_layout(int S, int lmax, int nmax) {
    StgLayout L{};
    const int RB = (lmax + 1) * (lmax + 1);
    const int K = RB * nmax;
    L.P = 32 * stg_steps(lmax);
    L.GB = nmax == 8 ? 3 * L.P : (3 * K + STG_G_PAD + 1) & ~1;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 15) & ~(size_t)15;
        return at;
    };
    L.cf = take(sizeof(double) * S * L.P);
    L.scale = take(sizeof(double) * 2 * (lmax + 1));
    L.ring = take(sizeof(double) * STG_RING * L.GB);
    L.rows = take(sizeof(int32_t) * 3 * RB);
    L.slot_base = take(sizeof(int64_t) * STG_MAX_SLOTS);
    L.slot_ab = take(sizeof(int32_t) * 2 * STG_MAX_SLOTS);
    L.sp_count = take(sizeof(int32_t) * STG_MAX_SPECIES);
    L.sp_slot = take(sizeof(int32_t) * STG_MAX_SPECIES * STG_MAX_SPECIES);
    L.meta_entry = take(sizeof(PsEntry) * STG_CHUNK);
    L.meta_code = take(sizeof(int32_t) * STG_CHUNK);
    L.meta_cum = take(sizeof(int32_t) * STG_CHUNK * (S + 1));
    L.bytes = off;
    return L;
}

// one (entry, slot) row from a staged pair gradient: per l, the three 8 x 8
// tiles G^T C_b (entry species == a) and C_a^T G (entry species == b)
template <bool N8>
__device__ __forceinline__ void stg_row(int lane, int lmax, int nmax, int64_t n_props, const double* __restrict__ gs,
                                        const double* __restrict__ cf, int P, const double* __restrict__ scale_s,
                                        int a, int b, int s, bool flip, double* __restrict__ out) {
    const int tm = lane & 3, tn = lane >> 2;
    const bool t1 = s == a, t2 = s == b;
    const double* ca = cf + a * P + lane;
    const double* cb = cf + b * P + lane;
    const int RB = (lmax + 1) * (lmax + 1);  // rows (l, m) of one component
    const int N = N8 ? 8 : nmax;
    const bool vec = N8 && ((((uintptr_t)out) & 15) == 0);
    const double* scales = scale_s + (a != b ? lmax + 1 : 0);
    // N8: component x of step st starts at (x P + 32 st) + the lane's offset
    const double* g0 = gs + (N8 ? stg_lane_offset8(lane) : 0);
    int step = 0;
    for (int l = 0; l <= lmax; l++) {
        const int steps = (2 * l + 1 + 3) >> 2;
        double acc[3][2];
#pragma unroll
        for (int x = 0; x < 3; x++) acc[x][0] = acc[x][1] = 0.0;
        // at most STG_MAX_STEPS steps per l (lmax <= 9: the launch condition),
        // unrolled so that the fragment loads of later steps are issued early
#pragma unroll
        for (int st = 0; st < STG_MAX_STEPS; st++) {
            if (st >= steps) break;
            double g[3];
            if (N8) {
                const double* gp = g0 + (step + st) * 32;
#pragma unroll
                for (int x = 0; x < 3; x++) g[x] = gp[x * P];
            } else {
                const int r = l * l + 4 * st + tm;
#pragma unroll
                for (int x = 0; x < 3; x++) g[x] = gs[(x * RB + r) * N + tn];
            }
            if (t1) {
                const double c = cb[(step + st) * 32];
#pragma unroll
                for (int x = 0; x < 3; x++) dmma_8x8x4(acc[x], g[x], c);
            }
            if (t2) {
                const double c = ca[(step + st) * 32];
#pragma unroll
                for (int x = 0; x < 3; x++) dmma_8x8x4(acc[x], c, g[x]);
            }
        }
        step += steps;
        // -(-1)^l of a reversed pair, exact, folded into the scale
        const double scale = (flip && (l & 1) == 0) ? -scales[l] : scales[l];
        const int n2 = 2 * tm;
        if (vec) {
            double* o = out + (int64_t)l * 64 + tn * 8 + n2;
#pragma unroll
            for (int x = 0; x < 3; x++) {
                double2 w;
                w.x = acc[x][0] * scale;
                w.y = acc[x][1] * scale;
                __stcs(reinterpret_cast<double2*>(o + x * n_props), w);
            }
        } else if (tn < N) {
            double* o = out + (int64_t)l * N * N + tn * N + n2;
#pragma unroll
            for (int x = 0; x < 3; x++) {
                if (n2 < N) __stcs(o + x * n_props, acc[x][0] * scale);
                if (n2 + 1 < N) __stcs(o + x * n_props + 1, acc[x][1] * scale);
            }
        }
    }
}

// (l, step offset) of row lm = l^2 + m
__device__ __forceinline__ void stg_row_position(int lm, int& l, int& m, int& step) {
    l = 0;
    step = 0;
    while ((l + 1) * (l + 1) <= lm) {
        step += (2 * l + 1 + 3) >> 2;
        l++;
    }
    m = lm - l * l;
}

template <bool N8>
__global__ void __launch_bounds__(STG_WARPS * 32, 4) ps_positions_staged_kernel(PsArgs a) {
    extern __shared__ __align__(16) unsigned char stg_smem[];
    const int64_t c = blockIdx.x / STG_SPLIT;
    const int part = (int)(blockIdx.x - c * STG_SPLIT);
    const int S = a.n_species, L = a.lmax, N = a.nmax;
    const int RB = (L + 1) * (L + 1);
    const int K = RB * N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e_first = a.entry_offset[c], n_entries = a.entry_offset[c + 1] - e_first;
    const int64_t eb = e_first + n_entries * part / STG_SPLIT;
    const int64_t ee = e_first + n_entries * (part + 1) / STG_SPLIT;
    if (eb >= ee) return;

    const StgLayout lay = stg_layout(S, L, N);
    double* cf = reinterpret_cast<double*>(stg_smem + lay.cf);
    double* scale_s = reinterpret_cast<double*>(stg_smem + lay.scale);
    double* ring = reinterpret_cast<double*>(stg_smem + lay.ring);
    int32_t* rows = reinterpret_cast<int32_t*>(stg_smem + lay.rows);
    int64_t* slot_base = reinterpret_cast<int64_t*>(stg_smem + lay.slot_base);
    int32_t* slot_ab = reinterpret_cast<int32_t*>(stg_smem + lay.slot_ab);
    int32_t* sp_count = reinterpret_cast<int32_t*>(stg_smem + lay.sp_count);
    int32_t* sp_slot = reinterpret_cast<int32_t*>(stg_smem + lay.sp_slot);
    PsEntry* meta_entry = reinterpret_cast<PsEntry*>(stg_smem + lay.meta_entry);
    int32_t* meta_code = reinterpret_cast<int32_t*>(stg_smem + lay.meta_code);
    int32_t* meta_cum = reinterpret_cast<int32_t*>(stg_smem + lay.meta_cum);

    // coefficients in fragment order: element (step, lane) of species sp is
    // c[l, m = 4 st + lane % 4, n = lane / 4], zero outside m < 2l+1, n < nmax
    const double* coef = a.coef + c * S * K;
    for (int i = threadIdx.x; i < S * lay.P; i += blockDim.x) {
        const int sp = i / lay.P, rem = i - sp * lay.P;
        int g = rem >> 5;
        const int t = rem & 31;
        int l = 0;
        while (g >= ((2 * l + 1 + 3) >> 2)) {
            g -= (2 * l + 1 + 3) >> 2;
            l++;
        }
        const int m = 4 * g + (t & 3), n = t >> 2;
        cf[i] = (m < 2 * l + 1 && n < N) ? coef[sp * K + (l * l + m) * N + n] : 0.0;
    }
    load_scales(L, scale_s);
    if (N8) {
        // padded rows stay zero; rows[r]: first double of source row r
        // (x, l, m) in the buffer, times 2, plus the row's chunk swap bit
        for (int i = threadIdx.x; i < STG_RING * lay.GB; i += blockDim.x) ring[i] = 0.0;
        for (int r = threadIdx.x; r < 3 * RB; r += blockDim.x) {
            const int x = r / RB;
            int l, m, step;
            stg_row_position(r - x * RB, l, m, step);
            const int dest = x * lay.P + (step + (m >> 2)) * 32 + (m & 3) * 8;
            rows[r] = 2 * dest + ((m >> 1) & 1);
        }
    } else {
        // the padded last m step reads past the gradient: keep that tail finite
        for (int i = threadIdx.x; i < STG_RING * (lay.GB - 3 * K); i += blockDim.x) {
            const int buf = i / (lay.GB - 3 * K), j = i - buf * (lay.GB - 3 * K);
            ring[buf * lay.GB + 3 * K + j] = 0.0;
        }
    }
    const int64_t s0 = a.slot_offset[c];
    // one slot per species pair a <= b of the centre's keys: at most
    // STG_MAX_SLOTS for the species counts this kernel is launched with
    const int ns = (int)(a.slot_offset[c + 1] - s0);
    if (ns > STG_MAX_SLOTS) return;
    for (int i = threadIdx.x; i < ns; i += blockDim.x) {
        const PsKeySlot slot = a.slots[s0 + i];
        slot_base[i] = a.off_positions[slot.block] + a.slot_row[s0 + i] * 3 * a.n_props;
        slot_ab[2 * i] = slot.a;
        slot_ab[2 * i + 1] = slot.b;
    }
    __syncthreads();
    if (threadIdx.x < S) {
        const int sp = threadIdx.x;
        int n = 0;
        for (int i = 0; i < ns; i++)
            if (slot_ab[2 * i] == sp || slot_ab[2 * i + 1] == sp) sp_slot[sp * STG_MAX_SPECIES + n++] = i;
        sp_count[sp] = n;
    }

    const bool aligned16 = ((3 * K) & 1) == 0;
    for (int64_t chunk = eb; chunk < ee; chunk += STG_CHUNK) {
        const int nc = (int)min((int64_t)STG_CHUNK, ee - chunk);
        for (int i = threadIdx.x; i < nc; i += blockDim.x) {
            const PsEntry entry = a.entries[chunk + i];
            meta_entry[i] = entry;
            meta_code[i] = (entry.d1 - entry.d0 == 1) ? a.dir_code[entry.d0] : 0;
        }
        for (int i = threadIdx.x; i < nc * (S + 1); i += blockDim.x) meta_cum[i] = a.entry_cum[chunk * (S + 1) + i];
        __syncthreads();

        // pair gradient of entry k into ring buffer k % STG_RING (regular
        // entries only: one pair, not the centre)
        auto issue = [&](int k) {
            if (k < nc) {
                const PsEntry entry = meta_entry[k];
                if (entry.atom != (int32_t)c && entry.d1 - entry.d0 == 1) {
                    const double* src = a.pair_grad + (int64_t)(meta_code[k] >> 1) * 3 * K;
                    double* dst = ring + (k % STG_RING) * lay.GB;
                    if (N8) {
                        for (int q = threadIdx.x; q < 3 * K / 2; q += blockDim.x) {
                            const int e = rows[q >> 2], ch = q & 3;
                            cp_async16(dst + (e >> 1) + ((ch ^ ((e & 1) << 1)) << 1), src + 2 * q);
                        }
                    } else if (aligned16) {
                        for (int q = threadIdx.x; q < 3 * K / 2; q += blockDim.x) cp_async16(dst + 2 * q, src + 2 * q);
                    } else {
                        for (int q = threadIdx.x; q < 3 * K; q += blockDim.x) cp_async8(dst + q, src + q);
                    }
                }
            }
            cp_async_commit();
        };
        issue(0);
        for (int k = 0; k < nc; k++) {
            cp_async_wait<0>();
            // entry k's gradient is visible to every warp, and every warp is
            // done with entry k - 1, whose buffer the next issue reuses
            __syncthreads();
            issue(k + 1);
            const PsEntry entry = meta_entry[k];
            if (entry.atom == (int32_t)c) continue;  // the centre's own rows: ps_centre_rows_kernel
            const int32_t* cum = meta_cum + k * (S + 1);
            const bool regular = entry.d1 - entry.d0 == 1;
            const int n_items = sp_count[entry.species];
            for (int it = warp; it < n_items; it += STG_WARPS) {
                const int si = sp_slot[entry.species * STG_MAX_SPECIES + it];
                const int sa = slot_ab[2 * si], sb = slot_ab[2 * si + 1];
                const int64_t rank = cum[sa] + (sa != sb ? cum[sb] : 0) + cum[S];
                double* out = a.out + slot_base[si] + rank * 3 * a.n_props;
                if (regular) {
                    stg_row<N8>(lane, L, N, a.n_props, ring + (k % STG_RING) * lay.GB, cf, lay.P, scale_s, sa, sb,
                                entry.species, meta_code[k] & 1, out);
                } else {
                    const PsKeySlot slot{0, 0, sa, sb};
                    ImagesSource images{a.dir_code + entry.d0, entry.d1 - entry.d0, a.pair_grad, 3 * (int64_t)K};
                    positions_row(a, lane, K, coef, scale_s, slot, false, entry.species, images, nullptr, nullptr, out);
                }
            }
        }
        cp_async_wait<0>();
        __syncthreads();  // metadata and ring are reused by the next chunk
    }
}

// Rows of one centre and one slot (a, b) built from two operands of three
// components each, D_a and D_b ([3][(l m)][n] in global memory):
//   tile[x] = sum_m D_a[x][l m][n1] c_b[l m][n2] + c_a[l m][n1] D_b[x][l m][n2]
// on the FP64 tensor cores, per l all fragment loads issued together (at most
// CR_MAX_STEPS steps of 4 m, lmax <= 8).  The centre's own positions rows use
// the self gradients, the strain / cell rows three components of the 3 x 3
// gradients at a time.
constexpr int CR_MAX_STEPS = 5;
constexpr int CR_SPLIT = 2;

__device__ __forceinline__ void centre_row(int lane, int lmax, int nmax, int K, int64_t n_props,
                                           const double* __restrict__ da, const double* __restrict__ db,
                                           const double* __restrict__ cf, int P, const double* __restrict__ scales,
                                           int a, int b, double* __restrict__ out) {
    const int tm = lane & 3, tn = lane >> 2;
    const double* ca = cf + a * P + lane;
    const double* cb = cf + b * P + lane;
    const int N = nmax;
    const bool vec = N == 8 && ((((uintptr_t)out) & 15) == 0);
    int step = 0;
    for (int l = 0; l <= lmax; l++) {
        const int M = 2 * l + 1, steps = (M + 3) >> 2;
        double ga[CR_MAX_STEPS][3], gb[CR_MAX_STEPS][3], va[CR_MAX_STEPS], vb[CR_MAX_STEPS];
#pragma unroll
        for (int st = 0; st < CR_MAX_STEPS; st++) {
            if (st < steps) {
                const int m = 4 * st + tm;
                const bool ok = m < M && tn < N;
                const int idx = (l * l + m) * N + tn;
#pragma unroll
                for (int x = 0; x < 3; x++) {
                    ga[st][x] = ok ? da[x * K + idx] : 0.0;
                    gb[st][x] = ok ? db[x * K + idx] : 0.0;
                }
                va[st] = ca[(step + st) * 32];
                vb[st] = cb[(step + st) * 32];
            }
        }
        double acc[3][2];
#pragma unroll
        for (int x = 0; x < 3; x++) acc[x][0] = acc[x][1] = 0.0;
#pragma unroll
        for (int st = 0; st < CR_MAX_STEPS; st++) {
            if (st < steps) {
#pragma unroll
                for (int x = 0; x < 3; x++) dmma_8x8x4(acc[x], ga[st][x], vb[st]);
#pragma unroll
                for (int x = 0; x < 3; x++) dmma_8x8x4(acc[x], va[st], gb[st][x]);
            }
        }
        step += steps;
        const double scale = scales[l];
        const int n2 = 2 * tm;
        if (vec) {
            double* o = out + (int64_t)l * 64 + tn * 8 + n2;
#pragma unroll
            for (int x = 0; x < 3; x++) {
                double2 w;
                w.x = acc[x][0] * scale;
                w.y = acc[x][1] * scale;
                __stcs(reinterpret_cast<double2*>(o + x * n_props), w);
            }
        } else if (tn < N) {
            double* o = out + (int64_t)l * N * N + tn * N + n2;
#pragma unroll
            for (int x = 0; x < 3; x++) {
                if (n2 < N) __stcs(o + x * n_props, acc[x][0] * scale);
                if (n2 + 1 < N) __stcs(o + x * n_props + 1, acc[x][1] * scale);
            }
        }
    }
}

// The centre's rows, on the side stream beside the staged positions kernel:
// its own positions-gradient rows (CR_SELF; featomic's
// sum_m c_b dself_a + c_a dself_b) and its strain / cell rows (CR_STRAIN,
// CR_CELL; three passes of three components).  CR_SPLIT CTAs per centre with the
// coefficients in fragment order in shared memory; items (slot, kind, pass)
// are spread over their warps.
constexpr int CR_SELF = 1, CR_STRAIN = 2, CR_CELL = 4, CR_VALUES = 8;

// the values row of one centre and slot (a, b): per l the 8 x 8 tile
// sum_m c_a[l m][n1] c_b[l m][n2] from the fragment-ordered coefficients
__device__ __forceinline__ void values_row(int lane, int lmax, int nmax, const double* __restrict__ cf, int P,
                                           const double* __restrict__ scales, int a, int b, double* __restrict__ out) {
    const int tm = lane & 3, tn = lane >> 2;
    const double* ca = cf + a * P + lane;
    const double* cb = cf + b * P + lane;
    const int N = nmax;
    const bool vec = N == 8 && ((((uintptr_t)out) & 15) == 0);
    int step = 0;
    for (int l = 0; l <= lmax; l++) {
        const int steps = (2 * l + 1 + 3) >> 2;
        double acc[2] = {0.0, 0.0};
#pragma unroll
        for (int st = 0; st < CR_MAX_STEPS; st++) {
            if (st >= steps) break;
            dmma_8x8x4(acc, ca[(step + st) * 32], cb[(step + st) * 32]);
        }
        step += steps;
        const double scale = scales[l];
        const int n2 = 2 * tm;
        if (vec) {
            double2 w;
            w.x = acc[0] * scale;
            w.y = acc[1] * scale;
            __stcs(reinterpret_cast<double2*>(out + (int64_t)l * 64 + tn * 8 + n2), w);
        } else if (tn < N) {
            double* o = out + (int64_t)l * N * N + tn * N + n2;
            if (n2 < N) __stcs(o, acc[0] * scale);
            if (n2 + 1 < N) __stcs(o + 1, acc[1] * scale);
        }
    }
}

__global__ void __launch_bounds__(128) ps_centre_rows_kernel(PsArgs a, int kinds) {
    extern __shared__ __align__(16) double cr_smem[];
    __shared__ int64_t self_entry;
    // CR_SPLIT CTAs per centre share its items
    const int64_t c = blockIdx.x / CR_SPLIT;
    const int part = (int)(blockIdx.x - c * CR_SPLIT);
    const int S = a.n_species, L = a.lmax, N = a.nmax;
    const int K = (L + 1) * (L + 1) * N;
    const int P = 32 * stg_steps(L);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    double* cf = cr_smem;
    double* scale_s = cr_smem + S * P;
    const double* coef = a.coef + c * S * K;
    for (int i = threadIdx.x; i < S * P; i += blockDim.x) {
        const int sp = i / P, rem = i - sp * P;
        int g = rem >> 5;
        const int t = rem & 31;
        int l = 0;
        while (g >= ((2 * l + 1 + 3) >> 2)) {
            g -= (2 * l + 1 + 3) >> 2;
            l++;
        }
        const int m = 4 * g + (t & 3), n = t >> 2;
        cf[i] = (m < 2 * l + 1 && n < N) ? coef[sp * K + (l * l + m) * N + n] : 0.0;
    }
    load_scales(L, scale_s);
    // the centre's entry among its neighbour entries (sorted by atom index)
    const int64_t e0 = a.entry_offset[c], ne = a.entry_offset[c + 1] - e0;
    if (warp == 0) {
        int64_t found = -1;
        if (kinds & CR_SELF) {
            for (int64_t base = 0; base < ne && found < 0; base += 32) {
                const bool hit = base + lane < ne && a.entries[e0 + base + lane].atom == (int32_t)c;
                const unsigned mask = __ballot_sync(0xffffffffu, hit);
                if (mask) found = e0 + base + __ffs(mask) - 1;
            }
        }
        if (lane == 0) self_entry = found;
    }
    __syncthreads();
    const int64_t s0 = a.slot_offset[c];
    const int ns = (int)(a.slot_offset[c + 1] - s0);
    // per slot: the self row (if requested and the centre's entry exists),
    // then 3 strain passes, then 3 cell passes
    const int n_values = (kinds & CR_VALUES) ? 1 : 0, n_self = (kinds & CR_SELF) && self_entry >= 0 ? 1 : 0;
    const int n_strain = (kinds & CR_STRAIN) ? 3 : 0, n_cell = (kinds & CR_CELL) ? 3 : 0;
    const int per_slot = n_values + n_self + n_strain + n_cell;
    for (int it = part * nwarps + warp; it < ns * per_slot; it += CR_SPLIT * nwarps) {
        const int si = it / per_slot;
        int kind = it - si * per_slot;
        const PsKeySlot slot = a.slots[s0 + si];
        const double* scales = scale_s + (slot.a != slot.b ? L + 1 : 0);
        if (kind < n_values) {
            values_row(lane, L, N, cf, P, scales, slot.a, slot.b,
                       a.out + a.off_values[slot.block] + (int64_t)slot.sample * a.n_props);
            continue;
        }
        kind -= n_values;
        const double *da, *db;
        double* out;
        if (kind < n_self) {
            const int32_t* cum = a.entry_cum + self_entry * (S + 1);
            const int64_t rank = cum[slot.a] + (slot.a != slot.b ? cum[slot.b] : 0) + cum[S];
            out = a.out + a.off_positions[slot.block] + (a.slot_row[s0 + si] + rank) * 3 * a.n_props;
            da = a.self_grad + ((int64_t)c * S + slot.a) * 3 * K;
            db = a.self_grad + ((int64_t)c * S + slot.b) * 3 * K;
        } else {
            kind -= n_self;
            const bool strain = kind < n_strain;
            const int xr = strain ? kind : kind - n_strain;
            const double* src = strain ? a.strain : a.cellg;
            const int64_t* offs = strain ? a.off_strain : a.off_cell;
            out = a.out + offs[slot.block] + ((int64_t)slot.sample * 9 + 3 * xr) * a.n_props;
            da = src + (((int64_t)c * S + slot.a) * 9 + 3 * xr) * K;
            db = src + (((int64_t)c * S + slot.b) * 9 + 3 * xr) * K;
        }
        centre_row(lane, L, N, K, a.n_props, da, db, cf, P, scales, slot.a, slot.b, out);
    }
}

// strain (which = 0) or cell (which = 1) rows: 9 components, done as three
// passes of 3 to bound the register tile
template <int MAXN>
__global__ void __launch_bounds__(256) ps_strain_cell_kernel(PsArgs a, int which) {
    extern __shared__ double smem[];
    const int64_t c = blockIdx.x;
    const int S = a.n_species;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    double* coef_s = smem;
    double* scale_s = smem + S * K;
    load_coefficients(a, c, coef_s, S * K);
    load_scales(a.lmax, scale_s);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const double* src = which == 0 ? a.strain : a.cellg;
    const int64_t* offs = which == 0 ? a.off_strain : a.off_cell;
    const int64_t s0 = a.slot_offset[c], ns = a.slot_offset[c + 1] - s0;
    for (int64_t task = warp; task < 3 * ns; task += nwarps) {
        const int64_t s = task / 3;
        const int xr = (int)(task - s * 3);
        const PsKeySlot slot = a.slots[s0 + s];
        DirectSource ga{src + (((int64_t)c * S + slot.a) * 9 + 3 * xr) * K, false};
        DirectSource gb{src + (((int64_t)c * S + slot.b) * 9 + 3 * xr) * K, false};
        double* out = a.out + offs[slot.block] + ((int64_t)slot.sample * 9 + 3 * xr) * a.n_props;
        rows<3>(lane, a.lmax, a.nmax, K, true, ga, coef_s + slot.b * K, coef_s + slot.a * K, true, gb, out, a.n_props,
                scale_s + (slot.a != slot.b ? a.lmax + 1 : 0));
    }
}

// A second stream per device for the values and strain / cell kernels, which
// run beside the positions kernel and fill the SMs its last wave leaves idle.
// Dependencies go through events created per call, so concurrent callers that
// share this stream stay correctly ordered.
cudaStream_t side_stream() {
    static std::mutex mutex;
    static std::map<int, cudaStream_t> streams;
    int device = 0;
    CUDA_CHECK(cudaGetDevice(&device));
    std::lock_guard<std::mutex> lock(mutex);
    auto it = streams.find(device);
    if (it != streams.end()) return it->second;
    // default priority: with the highest one its kernels delay the positions
    // kernel more than they gain (1.89 against 1.85 ms per 1000-atom step)
    cudaStream_t s = nullptr;
    CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    streams[device] = s;
    return s;
}

template <int MAXN>
void launch_all(const PsArgs& args, bool values, bool positions, bool strain, bool cell, cudaStream_t stream,
                const PsEvents& events) {
    const int K = (args.lmax + 1) * (args.lmax + 1) * args.nmax;
    const size_t coef_bytes = sizeof(double) * ((size_t)args.n_species * K + 2 * (args.lmax + 1));
    const int threads = 256;
    static bool configured = false;
    if (!configured) {
        CUDA_CHECK(cudaFuncSetAttribute(ps_values_kernel<MAXN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CUDA_CHECK(cudaFuncSetAttribute(ps_positions_kernel<MAXN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CUDA_CHECK(cudaFuncSetAttribute(ps_strain_cell_kernel<MAXN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CUDA_CHECK(cudaFuncSetAttribute(ps_positions_staged_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CUDA_CHECK(cudaFuncSetAttribute(ps_positions_staged_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CUDA_CHECK(cudaFuncSetAttribute(ps_centre_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        configured = true;
    }
    if (coef_bytes > 200 * 1024) throw invalid_parameter("too many species / radial / angular functions for the power spectrum kernels");
    const size_t pos_bytes =
        sizeof(double) * (((size_t)args.n_species * K + 2 * (args.lmax + 1) + 1) / 2 * 2) + POS_TABLE_BYTES;
    if (positions && pos_bytes > 200 * 1024)
        throw invalid_parameter("too many radial / angular functions for the positions gradient kernel");

    // side stream: values, strain, cell
    cudaStream_t side = side_stream();
    cudaEvent_t fork = nullptr, join = nullptr;
    CUDA_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CUDA_CHECK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    CUDA_CHECK(cudaEventRecord(fork, stream));
    CUDA_CHECK(cudaStreamWaitEvent(side, fork, 0));
    // nmax <= 8, lmax <= 9: the staged positions kernel, and the values rows
    // with the centres' own positions rows and the strain / cell rows in
    // ps_centre_rows_kernel (values alone keep ps_values_kernel)
    const StgLayout stg = stg_layout(args.n_species, args.lmax, args.nmax);
    const bool dmma_rows = args.nmax <= 8 && (2 * args.lmax + 1 + 3) / 4 <= CR_MAX_STEPS;
    const bool staged = positions && dmma_rows && args.n_species <= STG_MAX_SPECIES && stg.bytes <= 200 * 1024;
    const size_t cr_bytes = sizeof(double) * ((size_t)args.n_species * 32 * stg_steps(args.lmax) + 2 * (args.lmax + 1));
    const int gradient_kinds = (staged ? CR_SELF : 0) | (strain ? CR_STRAIN : 0) | (cell ? CR_CELL : 0);
    const bool centre_rows = dmma_rows && cr_bytes <= 200 * 1024 && gradient_kinds != 0 && (staged || !positions);
    const int kinds = gradient_kinds | (values ? CR_VALUES : 0);
    if (values && !centre_rows) {
        ps_values_kernel<MAXN><<<(unsigned)args.n_centres, threads, coef_bytes, side>>>(args);
        CUDA_CHECK(cudaGetLastError());
    }
    if (events.after_values) CUDA_CHECK(cudaEventRecord(events.after_values, side));
    if (centre_rows) {
        ps_centre_rows_kernel<<<(unsigned)(CR_SPLIT * args.n_centres), 128, cr_bytes, side>>>(args, kinds);
        CUDA_CHECK(cudaGetLastError());
    } else {
        if (staged) throw std::logic_error("the centres' own rows need ps_centre_rows_kernel");
        if (strain) {
            ps_strain_cell_kernel<MAXN><<<(unsigned)args.n_centres, threads, coef_bytes, side>>>(args, 0);
            CUDA_CHECK(cudaGetLastError());
        }
        if (cell) {
            ps_strain_cell_kernel<MAXN><<<(unsigned)args.n_centres, threads, coef_bytes, side>>>(args, 1);
            CUDA_CHECK(cudaGetLastError());
        }
    }
    if (events.after_strain_cell) CUDA_CHECK(cudaEventRecord(events.after_strain_cell, side));
    CUDA_CHECK(cudaEventRecord(join, side));

    // caller's stream: positions
    if (events.before_positions) CUDA_CHECK(cudaEventRecord(events.before_positions, stream));
    if (positions) {
        if (staged) {
            const unsigned grid = (unsigned)(args.n_centres * STG_SPLIT);
            if (args.nmax == 8) ps_positions_staged_kernel<true><<<grid, STG_WARPS * 32, stg.bytes, stream>>>(args);
            else ps_positions_staged_kernel<false><<<grid, STG_WARPS * 32, stg.bytes, stream>>>(args);
        } else {
            ps_positions_kernel<MAXN><<<(unsigned)(args.n_centres * POS_SPLIT), POS_WARPS * 32, pos_bytes, stream>>>(args);
        }
        CUDA_CHECK(cudaGetLastError());
    }
    if (events.after_positions) CUDA_CHECK(cudaEventRecord(events.after_positions, stream));
    CUDA_CHECK(cudaStreamWaitEvent(stream, join, 0));
    // released once the recorded work has completed
    CUDA_CHECK(cudaEventDestroy(fork));
    CUDA_CHECK(cudaEventDestroy(join));
}

// One centre's S-way merge of its (centre, species) segments of directions,
// by the other atom's index (plan.cpp build_neighborhoods): writes its unique
// neighbours and itself with their prefix counts, one thread
constexpr int NB_MAX_SPECIES = 64;

__device__ void neighborhoods_merge(int64_t c, const int32_t* __restrict__ first, const int32_t* __restrict__ second,
                                    const int32_t* __restrict__ atom_species, const int32_t* __restrict__ dir,
                                    const int64_t* __restrict__ seg, int S, const int64_t* __restrict__ offsets,
                                    PsEntry* __restrict__ entries, int32_t* __restrict__ entry_cum) {
    int64_t pos[NB_MAX_SPECIES], end[NB_MAX_SPECIES];
    int32_t head[NB_MAX_SPECIES], cum[NB_MAX_SPECIES + 1];
    const int sc = atom_species[c];
    auto other = [&](int64_t d) -> int32_t {
        const int32_t code = dir[d];
        return (code & 1) ? first[code >> 1] : second[code >> 1];
    };
    // head[t]: the other atom at the front of segment t, INT32_MAX once it
    // is exhausted (atoms of different species differ, so heads never tie)
    for (int t = 0; t < S; t++) {
        pos[t] = seg[c * S + t];
        end[t] = seg[c * S + t + 1];
        head[t] = pos[t] < end[t] ? other(pos[t]) : INT32_MAX;
        cum[t] = 0;
    }
    cum[S] = 0;
    const int64_t base = offsets[c];
    int64_t n = 0;
    auto emit = [&](int32_t atom, int32_t species, int32_t d0, int32_t d1) {
        entries[base + n] = PsEntry{atom, species, d0, d1};
        int32_t* w = entry_cum + (base + n) * (S + 1);
        for (int t = 0; t <= S; t++) w[t] = cum[t];
        n++;
    };
    bool self_done = false;
    while (true) {
        int best = 0;
        int32_t best_atom = head[0];
        for (int t = 1; t < S; t++) {
            if (head[t] < best_atom) {
                best = t;
                best_atom = head[t];
            }
        }
        if (best_atom == INT32_MAX) best = -1;
        if (!self_done && (best < 0 || best_atom >= (int32_t)c)) {
            emit((int32_t)c, sc, -1, -1);
            cum[S] = 1;
            self_done = true;
        }
        if (best < 0) break;
        const int64_t d0 = pos[best];
        int64_t d = d0 + 1;
        int32_t next = INT32_MAX;
        while (d < end[best]) {
            next = other(d);
            if (next != best_atom) break;
            next = INT32_MAX;
            d++;
        }
        pos[best] = d;
        head[best] = next;
        if (best_atom == (int32_t)c) continue;  // periodic images of the centre itself
        emit(best_atom, best, (int32_t)d0, (int32_t)d);
        cum[best]++;
    }
}

// The filling half, a warp per centre: the centre's directions (other atom
// per direction) in shared memory; a direction that starts a run of one
// neighbour (its periodic images are adjacent) and is not the centre is an
// entry, whose place in the centre's list is the number of such entries with
// a smaller atom index (plus the centre's own entry when that comes first),
// and whose prefix count of species t the number of them in segment t.  The
// same entries and prefix counts as neighborhoods_merge, which takes
// the centres with more than NB_WARP_DIRS directions.
constexpr int NB_WARP_DIRS = 256;
constexpr int NB_FILL_WARPS = 4;

__global__ void __launch_bounds__(NB_FILL_WARPS * 32)
    neighborhoods_fill_kernel(const int32_t* __restrict__ first, const int32_t* __restrict__ second,
                              const int32_t* __restrict__ atom_species, const int32_t* __restrict__ dir,
                              const int64_t* __restrict__ seg, int S, int64_t n_atoms,
                              const int64_t* __restrict__ offsets, PsEntry* __restrict__ entries,
                              int32_t* __restrict__ entry_cum) {
    __shared__ int32_t other_s[NB_FILL_WARPS][NB_WARP_DIRS];
    __shared__ int32_t seg_s[NB_FILL_WARPS][NB_MAX_SPECIES + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t c = (int64_t)blockIdx.x * NB_FILL_WARPS + warp;
    if (c >= n_atoms) return;
    const int64_t b = seg[c * S], n = seg[c * S + S] - b;
    if (n > NB_WARP_DIRS) {
        if (lane == 0)
            neighborhoods_merge(c, first, second, atom_species, dir, seg, S, offsets, entries, entry_cum);
        return;
    }
    int32_t* other = other_s[warp];
    int32_t* sb = seg_s[warp];
    for (int64_t i = lane; i < n; i += 32) {
        const int32_t code = dir[b + i];
        other[i] = (code & 1) ? first[code >> 1] : second[code >> 1];
    }
    for (int t = lane; t <= S; t += 32) sb[t] = (int32_t)(seg[c * S + t] - b);
    __syncwarp();
    const int32_t ci = (int32_t)c;
    auto is_entry = [&](int i) { return other[i] != ci && (i == 0 || other[i - 1] != other[i]); };
    const int64_t base = offsets[c];
    // the centre's own entry: entries of smaller atoms come first
    int32_t before = 0;
    for (int t = lane; t < S; t += 32) {
        int32_t k = 0;
        for (int i = sb[t]; i < sb[t + 1]; i++) k += (is_entry(i) && other[i] < ci) ? 1 : 0;
        before += k;
    }
    for (int off = 16; off > 0; off >>= 1) before += __shfl_xor_sync(0xffffffffu, before, off);
    if (lane == 0) entries[base + before] = PsEntry{ci, atom_species[c], -1, -1};
    for (int t = lane; t <= S; t += 32) {
        int32_t k = 0;
        if (t < S)
            for (int i = sb[t]; i < sb[t + 1]; i++) k += (is_entry(i) && other[i] < ci) ? 1 : 0;
        entry_cum[(base + before) * (S + 1) + t] = k;
    }
    // the neighbours' entries
    for (int i = lane; i < n; i += 32) {
        if (!is_entry(i)) continue;
        const int32_t o = other[i];
        int t = 0;
        while (i >= sb[t + 1]) t++;
        int run = i + 1;
        while (run < sb[t + 1] && other[run] == o) run++;
        const int64_t slot_c = o > ci ? 1 : 0;
        int64_t rank = slot_c;
        int32_t* cum = nullptr;
        // first pass: the rank; second pass: the prefix counts at that rank
        for (int u = 0; u < S; u++) {
            int32_t k = 0;
            for (int j = sb[u]; j < sb[u + 1]; j++) k += (is_entry(j) && other[j] < o) ? 1 : 0;
            rank += k;
        }
        entries[base + rank] = PsEntry{o, t, (int32_t)(b + i), (int32_t)(b + run)};
        cum = entry_cum + (base + rank) * (S + 1);
        for (int u = 0; u < S; u++) {
            int32_t k = 0;
            for (int j = sb[u]; j < sb[u + 1]; j++) k += (is_entry(j) && other[j] < o) ? 1 : 0;
            cum[u] = k;
        }
        cum[S] = (int32_t)slot_c;
    }
}

// The counting half, a warp per centre: within a
// (centre, species) segment the other atoms come in increasing order with the
// periodic images of one atom adjacent, so the unique neighbours of that
// species are the directions whose other atom differs from the previous
// direction's and is not the centre.  Writes the same counts, species counts
// and species masks as the merge would (one unique neighbour per run of
// adjacent images, the centre's own images excluded).
__global__ void neighborhoods_count_kernel(const int32_t* __restrict__ first, const int32_t* __restrict__ second,
                                           const int32_t* __restrict__ atom_species, const int32_t* __restrict__ dir,
                                           const int64_t* __restrict__ seg, int S, int64_t n_atoms,
                                           int64_t* __restrict__ counts, int32_t* __restrict__ species_count,
                                           uint8_t* __restrict__ species_mask) {
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c == n_atoms && lane == 0) counts[n_atoms] = 0;  // the scan's last element
    if (c >= n_atoms) return;
    auto other = [&](int64_t d) -> int32_t {
        const int32_t code = dir[d];
        return (code & 1) ? first[code >> 1] : second[code >> 1];
    };
    const int sc = atom_species[c];
    int64_t total = 1;  // the centre itself
    for (int t = 0; t < S; t++) {
        const int64_t b = seg[c * S + t], e = seg[c * S + t + 1];
        int32_t n = 0;
        for (int64_t base = b; base < e; base += 32) {
            const int64_t d = base + lane;
            bool unique = false;
            if (d < e) {
                const int32_t o = other(d);
                unique = o != (int32_t)c && (d == b || other(d - 1) != o);
            }
            n += __popc(__ballot_sync(0xffffffffu, unique));
        }
        if (lane == 0) {
            species_count[c * S + t] = n;
            species_mask[c * S + t] = (e > b || t == sc) ? 1 : 0;
        }
        total += n;
    }
    if (lane == 0) counts[c] = total;
}

}  // namespace

DeviceNeighborhoods launch_neighborhoods(const DevicePairs& pairs, const int32_t* atom_species, const int32_t* dir_code,
                                         const int64_t* seg_offset, int n_species, int64_t n_atoms, DeviceArena& arena,
                                         cudaStream_t stream, int32_t* host_count, uint8_t* host_mask,
                                         cudaEvent_t counted) {
    if (n_species > NB_MAX_SPECIES) throw invalid_parameter("more than 64 atomic types are not supported");
    if (2 * pairs.count + n_atoms >= (int64_t)INT32_MAX) throw invalid_parameter("too many pairs");
    DeviceNeighborhoods nb;
    const int S = n_species;
    const int64_t capacity = 2 * pairs.count + n_atoms;  // every direction and every centre at most once
    int64_t* counts = arena.alloc<int64_t>("nb.counts", n_atoms + 1);
    nb.entry_offset = arena.alloc<int64_t>("nb.entry_offset", n_atoms + 1);
    nb.entries = arena.alloc<PsEntry>("nb.entries", capacity);
    nb.entry_cum = arena.alloc<int32_t>("nb.entry_cum", capacity * (S + 1));
    nb.species_count = arena.alloc<int32_t>("nb.species_count", n_atoms * S);
    nb.species_mask = arena.alloc<uint8_t>("nb.species_mask", n_atoms * S);
    const unsigned count_blocks = (unsigned)(((n_atoms + 1) * 32 + 255) / 256);
    neighborhoods_count_kernel<<<count_blocks, 256, 0, stream>>>(pairs.first, pairs.second, atom_species, dir_code,
                                                                seg_offset, S, n_atoms, counts, nb.species_count,
                                                                nb.species_mask);
    CUDA_CHECK(cudaGetLastError());
    if (host_count && host_mask) {
        CUDA_CHECK(cudaMemcpyAsync(host_count, nb.species_count, sizeof(int32_t) * n_atoms * S, cudaMemcpyDeviceToHost,
                                   stream));
        CUDA_CHECK(cudaMemcpyAsync(host_mask, nb.species_mask, n_atoms * S, cudaMemcpyDeviceToHost, stream));
        if (counted) CUDA_CHECK(cudaEventRecord(counted, stream));
    }
    size_t temp = 0;
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, temp, counts, nb.entry_offset, (int)(n_atoms + 1), stream));
    void* scan_temp = arena.alloc_bytes("nb.scan_temp", temp);  // its own: this may run beside other scans
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(scan_temp, temp, counts, nb.entry_offset, (int)(n_atoms + 1), stream));
    neighborhoods_fill_kernel<<<(unsigned)((n_atoms + NB_FILL_WARPS - 1) / NB_FILL_WARPS), NB_FILL_WARPS * 32, 0,
                                stream>>>(pairs.first, pairs.second, atom_species, dir_code, seg_offset, S, n_atoms,
                                          nb.entry_offset, nb.entries, nb.entry_cum);
    CUDA_CHECK(cudaGetLastError());
    return nb;
}

void launch_power_spectrum(const PsArgs& args, bool positions, bool strain, bool cell, cudaStream_t stream,
                           const PsEvents& events) {
    if (args.n_centres == 0) return;
    launch_all<0>(args, true, positions, strain, cell, stream, events);
}

}  // namespace fb200

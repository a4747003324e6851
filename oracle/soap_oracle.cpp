// ===========================================================================
// TEST INFRASTRUCTURE -- NOT PART OF THE PRODUCT.
//
// CPU FP64 restatement of featomic's SOAP hot path (neighbour list, GTO radial
// integral + Hermite spline, real spherical harmonics, spherical expansion,
// power spectrum and their positions / strain / cell gradients, plus the
// keys / samples / gradient-samples builders).  It is the parity oracle: only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
// load it, always as the checker or the timed CPU baseline, never as the thing
// measured or shipped.
//
// Every function cites the featomic file:line it follows (paths relative to
// the featomic checkout).  The restatement keeps the reference's arithmetic
// order (compile with -ffp-contract=off, no -ffast-math) so that neighbour
// lists are bit-identical and values agree to the last few ulps.
//
// Pinned by: tests/golden/*.npz (featomic/tests/data/generated, 10 significant
// digits) and tests/golden/known_answers.json (inline unit-test values).
// ===========================================================================
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

static const double EPS = std::numeric_limits<double>::epsilon();
static const double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// types/matrix.rs, types/vectors.rs
// ---------------------------------------------------------------------------
struct Vec3 {
    double v[3];
    double operator[](int i) const { return v[i]; }
    double& operator[](int i) { return v[i]; }
};

// vectors.rs:212-216 -- dot product, left-to-right
static inline double dot(const Vec3& a, const Vec3& b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// vectors.rs:220-225 -- cross product
static inline Vec3 cross(const Vec3& a, const Vec3& b) {
    Vec3 r;
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
    return r;
}

static inline Vec3 normalized(const Vec3& a) {
    double n = std::sqrt(dot(a, a));
    Vec3 r = {{a[0] / n, a[1] / n, a[2] / n}};
    return r;
}

struct Mat3 {
    double m[3][3];
};

// matrix.rs:243-247
static double determinant(const Mat3& a) {
    const double (*s)[3] = a.m;
    return s[0][0] * (s[1][1] * s[2][2] - s[2][1] * s[1][2])
         - s[0][1] * (s[1][0] * s[2][2] - s[1][2] * s[2][0])
         + s[0][2] * (s[1][0] * s[2][1] - s[1][1] * s[2][0]);
}

// matrix.rs:210-225
static Mat3 inverse(const Mat3& a) {
    const double (*s)[3] = a.m;
    double det = determinant(a);
    if (!(std::fabs(det) > 1e-30)) throw std::runtime_error("The matrix is not invertible!");
    double id = 1.0 / det;
    Mat3 r;
    r.m[0][0] = (s[1][1] * s[2][2] - s[2][1] * s[1][2]) * id;
    r.m[0][1] = (s[0][2] * s[2][1] - s[0][1] * s[2][2]) * id;
    r.m[0][2] = (s[0][1] * s[1][2] - s[0][2] * s[1][1]) * id;
    r.m[1][0] = (s[1][2] * s[2][0] - s[1][0] * s[2][2]) * id;
    r.m[1][1] = (s[0][0] * s[2][2] - s[0][2] * s[2][0]) * id;
    r.m[1][2] = (s[1][0] * s[0][2] - s[0][0] * s[1][2]) * id;
    r.m[2][0] = (s[1][0] * s[2][1] - s[2][0] * s[1][1]) * id;
    r.m[2][1] = (s[2][0] * s[0][1] - s[0][0] * s[2][1]) * id;
    r.m[2][2] = (s[0][0] * s[1][1] - s[1][0] * s[0][1]) * id;
    return r;
}

// matrix.rs:399-407 -- row vector times matrix
static inline Vec3 vec_mat(const Vec3& v, const Mat3& m) {
    Vec3 r;
    r[0] = v[0] * m.m[0][0] + v[1] * m.m[1][0] + v[2] * m.m[2][0];
    r[1] = v[0] * m.m[0][1] + v[1] * m.m[1][1] + v[2] * m.m[2][1];
    r[2] = v[0] * m.m[0][2] + v[1] * m.m[1][2] + v[2] * m.m[2][2];
    return r;
}

// ---------------------------------------------------------------------------
// systems/cell.rs
// ---------------------------------------------------------------------------
enum CellShape { INFINITE = 0, ORTHORHOMBIC = 1, TRICLINIC = 2 };

struct UnitCell {
    Mat3 matrix;
    Mat3 inv;
    CellShape shape;
};

// cell.rs:34-66
static UnitCell make_cell(const double* m9) {
    UnitCell c;
    bool zero = true;
    for (int i = 0; i < 9; i++) {
        c.matrix.m[i / 3][i % 3] = m9[i];
        if (m9[i] != 0.0) zero = false;
    }
    if (zero) {
        std::memset(&c.inv, 0, sizeof(c.inv));
        c.shape = INFINITE;
        return c;
    }
    if (!(std::fabs(determinant(c.matrix)) > 1e-6)) throw std::runtime_error("matrix is not invertible");
    auto z = [](double v) { return std::fabs(v) < 1e-6; };
    const double (*s)[3] = c.matrix.m;
    bool diag = z(s[0][1]) && z(s[0][2]) && z(s[1][0]) && z(s[1][2]) && z(s[2][0]) && z(s[2][1]);
    c.shape = diag ? ORTHORHOMBIC : TRICLINIC;
    c.inv = inverse(c.matrix);
    return c;
}

// cell.rs:154-169
static Vec3 distances_between_faces(const UnitCell& c) {
    Vec3 a = {{c.matrix.m[0][0], c.matrix.m[0][1], c.matrix.m[0][2]}};
    Vec3 b = {{c.matrix.m[1][0], c.matrix.m[1][1], c.matrix.m[1][2]}};
    Vec3 cc = {{c.matrix.m[2][0], c.matrix.m[2][1], c.matrix.m[2][2]}};
    Vec3 na = normalized(cross(b, cc));
    Vec3 nb = normalized(cross(cc, a));
    Vec3 nc = normalized(cross(a, b));
    Vec3 r = {{std::fabs(dot(na, a)), std::fabs(dot(nb, b)), std::fabs(dot(nc, cc))}};
    return r;
}

// ---------------------------------------------------------------------------
// systems/neighbors.rs
// ---------------------------------------------------------------------------
struct Pair {
    size_t first;
    size_t second;
    double distance;
    double vector[3];
    int32_t shift[3];
};

// neighbors.rs:316-326 -- Python-style divmod
static inline void divmod(int32_t a, size_t b, int32_t* q, size_t* r) {
    int32_t bi = (int32_t)b;
    int32_t quotient = a / bi;
    int32_t remainder = a % bi;
    if (remainder < 0) {
        remainder += bi;
        quotient -= 1;
    }
    *q = quotient;
    *r = (size_t)remainder;
}

struct CellAtom {
    size_t index;
    int32_t shift[3];
};

struct NeighborsList {
    double cutoff;
    std::vector<Pair> pairs;
    std::vector<std::vector<Pair>> pairs_by_atom;
};

static bool pair_less(const Pair& a, const Pair& b) {
    if (a.first != b.first) return a.first < b.first;
    if (a.second != b.second) return a.second < b.second;
    // the reference uses an unstable sort on (first, second): ties between
    // periodic images of one pair have no defined order.  Break them by shift
    // so that the oracle output is canonical.
    for (int k = 0; k < 3; k++)
        if (a.shift[k] != b.shift[k]) return a.shift[k] < b.shift[k];
    return false;
}

// neighbors.rs:101-163 (CellList::new), :167-201 (add_atom), :217-309 (pairs),
// :349-403 (NeighborsList::new)
static NeighborsList build_neighbors(const double* positions, size_t n_atoms, const UnitCell& cell, double cutoff) {
    const double MAX_NUMBER_OF_CELLS = 1e5;
    bool infinite = cell.shape == INFINITE;
    Vec3 dbf;
    if (infinite) {
        dbf[0] = dbf[1] = dbf[2] = 1.0;
    } else {
        dbf = distances_between_faces(cell);
    }
    double n_cells_f[3];
    for (int k = 0; k < 3; k++) {
        double v = std::trunc(dbf[k] / cutoff);
        n_cells_f[k] = v < 1.0 ? 1.0 : v;  // f64::clamp(v, 1.0, INFINITY)
    }
    double total = n_cells_f[0] * n_cells_f[1] * n_cells_f[2];
    if (total > MAX_NUMBER_OF_CELLS) {
        double rxy = n_cells_f[0] / n_cells_f[1];
        double ryz = n_cells_f[1] / n_cells_f[2];
        n_cells_f[2] = std::trunc(std::cbrt(MAX_NUMBER_OF_CELLS / (rxy * ryz * ryz)));
        n_cells_f[1] = std::trunc(ryz * n_cells_f[2]);
        n_cells_f[0] = std::trunc(rxy * n_cells_f[1]);
    }
    int32_t n_search[3];
    size_t n_cells[3];
    for (int k = 0; k < 3; k++) {
        n_search[k] = (int32_t)std::ceil(cutoff * n_cells_f[k] / dbf[k]);
        n_cells[k] = (size_t)n_cells_f[k];
    }
    for (int k = 0; k < 3; k++) {
        if (n_search[k] < 1) n_search[k] = 1;
        if (n_cells[k] == 1 && infinite) n_search[k] = 0;
    }

    std::vector<std::vector<CellAtom>> cells(n_cells[0] * n_cells[1] * n_cells[2]);
    auto cell_id = [&](size_t x, size_t y, size_t z) { return (x * n_cells[1] + y) * n_cells[2] + z; };

    for (size_t index = 0; index < n_atoms; index++) {
        Vec3 p = {{positions[3 * index], positions[3 * index + 1], positions[3 * index + 2]}};
        Vec3 frac = infinite ? p : vec_mat(p, cell.inv);
        int32_t ci[3];
        for (int k = 0; k < 3; k++) ci[k] = (int32_t)std::floor(frac[k] * (double)n_cells[k]);
        CellAtom atom;
        atom.index = index;
        size_t idx[3];
        if (infinite) {
            for (int k = 0; k < 3; k++) {
                // `cell_index as usize` wraps negative values to huge numbers,
                // which `usize::clamp` then maps onto the last cell
                uint64_t u = (uint64_t)(int64_t)ci[k];
                uint64_t hi = (uint64_t)(n_cells[k] - 1);
                idx[k] = (size_t)(u > hi ? hi : u);
                atom.shift[k] = 0;
            }
        } else {
            for (int k = 0; k < 3; k++) {
                int32_t q;
                divmod(ci[k], n_cells[k], &q, &idx[k]);
                atom.shift[k] = q;
            }
        }
        cells[cell_id(idx[0], idx[1], idx[2])].push_back(atom);
    }

    NeighborsList nl;
    nl.cutoff = cutoff;
    nl.pairs_by_atom.assign(n_atoms, {});
    double cutoff2 = cutoff * cutoff;
    const double (*H)[3] = cell.matrix.m;

    for (size_t cx = 0; cx < n_cells[0]; cx++)
    for (size_t cy = 0; cy < n_cells[1]; cy++)
    for (size_t cz = 0; cz < n_cells[2]; cz++) {
        const auto& current = cells[cell_id(cx, cy, cz)];
        for (int32_t dx = -n_search[0]; dx <= n_search[0]; dx++)
        for (int32_t dy = -n_search[1]; dy <= n_search[1]; dy++)
        for (int32_t dz = -n_search[2]; dz <= n_search[2]; dz++) {
            int32_t c_i[3] = {(int32_t)cx + dx, (int32_t)cy + dy, (int32_t)cz + dz};
            int32_t cshift[3];
            size_t nidx[3];
            for (int k = 0; k < 3; k++) divmod(c_i[k], n_cells[k], &cshift[k], &nidx[k]);
            const auto& neigh = cells[cell_id(nidx[0], nidx[1], nidx[2])];
            for (const auto& ai : current) {
                for (const auto& aj : neigh) {
                    if (ai.index > aj.index) continue;
                    int32_t s[3];
                    for (int k = 0; k < 3; k++) s[k] = cshift[k] + ai.shift[k] - aj.shift[k];
                    bool zero = s[0] == 0 && s[1] == 0 && s[2] == 0;
                    if (ai.index == aj.index) {
                        if (zero) continue;
                        if (s[0] + s[1] + s[2] < 0) continue;
                        if ((s[0] + s[1] + s[2] == 0) && (s[2] < 0 || (s[2] == 0 && s[1] < 0))) continue;
                    }
                    if (infinite && !zero) continue;

                    // neighbors.rs:364-389 -- filter the candidate pair
                    size_t i = ai.index, j = aj.index;
                    double v[3];
                    for (int k = 0; k < 3; k++) v[k] = positions[3 * j + k] - positions[3 * i + k];
                    double sx = H[0][0] * (double)s[0] + H[1][0] * (double)s[1] + H[2][0] * (double)s[2];
                    double sy = H[0][1] * (double)s[0] + H[1][1] * (double)s[1] + H[2][1] * (double)s[2];
                    double sz = H[0][2] * (double)s[0] + H[1][2] * (double)s[1] + H[2][2] * (double)s[2];
                    v[0] += sx;
                    v[1] += sy;
                    v[2] += sz;
                    double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                    if (d2 < cutoff2) {
                        Pair p;
                        p.first = i;
                        p.second = j;
                        p.distance = std::sqrt(d2);
                        for (int k = 0; k < 3; k++) {
                            p.vector[k] = v[k];
                            p.shift[k] = s[k];
                        }
                        nl.pairs.push_back(p);
                        nl.pairs_by_atom[i].push_back(p);
                        nl.pairs_by_atom[j].push_back(p);
                    }
                }
            }
        }
    }
    std::sort(nl.pairs.begin(), nl.pairs.end(), pair_less);
    for (auto& v : nl.pairs_by_atom) std::sort(v.begin(), v.end(), pair_less);
    return nl;
}

// ---------------------------------------------------------------------------
// math/gamma.rs -- Lanczos approximation (Pugh 2004, g = 10.900511, n = 11),
// the published coefficient table that statrs uses.
// ---------------------------------------------------------------------------
static const double LN_PI = 1.1447298858494002;
static const double TWO_SQRT_E_OVER_PI = 1.8603827342052657;
static const double LN_2_SQRT_E_OVER_PI = 0.6207822376352452;
static const double GAMMA_R = 10.900511;
static const double GAMMA_DK[11] = {
    2.4857408913875355e-5, 1.0514237858172197, -3.4568709722201625, 4.512277094668948,
    -2.9828522532357664, 1.056397115771267, -1.9542877319164587e-1, 1.709705434044412e-2,
    -5.719261174043057e-4, 4.633994733599057e-6, -2.7199490848860772e-9,
};
static const double E = 2.718281828459045;

// gamma.rs:41-63
static double gamma(double x) {
    if (x < 0.5) {
        double s = GAMMA_DK[0];
        for (int t = 1; t < 11; t++) s = s + GAMMA_DK[t] / ((double)t - x);
        return PI / (std::sin(PI * x) * s * TWO_SQRT_E_OVER_PI * std::pow((0.5 - x + GAMMA_R) / E, 0.5 - x));
    } else {
        double s = GAMMA_DK[0];
        for (int t = 1; t < 11; t++) s = s + GAMMA_DK[t] / (x + (double)t - 1.0);
        return s * TWO_SQRT_E_OVER_PI * std::pow((x - 0.5 + GAMMA_R) / E, x - 0.5);
    }
}

// gamma.rs:68-92
static double ln_gamma(double x) {
    if (x < 0.5) {
        double s = GAMMA_DK[0];
        for (int t = 1; t < 11; t++) s = s + GAMMA_DK[t] / ((double)t - x);
        return LN_PI - std::log(std::sin(PI * x)) - std::log(s) - LN_2_SQRT_E_OVER_PI
             - (0.5 - x) * std::log((0.5 - x + GAMMA_R) / E);
    } else {
        double s = GAMMA_DK[0];
        for (int t = 1; t < 11; t++) s = s + GAMMA_DK[t] / (x + (double)t - 1.0);
        return std::log(s) + LN_2_SQRT_E_OVER_PI + (x - 0.5) * std::log((x - 0.5 + GAMMA_R) / E);
    }
}

// f64::powi lowers to binary exponentiation (compiler-rt __powidf2)
static double powi(double a, int b) {
    bool recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// ---------------------------------------------------------------------------
// math/hyp1f1.rs -- scipy's CHGM with the 30-term asymptotic sum
// ---------------------------------------------------------------------------
static const double ACCEPTABLE_RTOL = 1e-9;

// hyp1f1.rs:53-98
static double hyp1f1_series_track_convergence(double a, double b, double x) {
    bool converged = false;
    double n_steps = 0.0;
    double term = 1.0, result = 1.0, abssum = result;
    for (int ki = 0; ki < 1000; ki++) {
        double k = (double)ki;
        double apk = a + k, bpk = b + k;
        if (bpk != 0.0) {
            term *= apk * x / bpk / (k + 1.0);
        } else if (apk == 0.0) {
            term = 0.0;
        } else {
            return NAN;
        }
        abssum += std::fabs(term);
        result += term;
        if (std::fabs(term) <= EPS * std::fabs(result)) {
            n_steps = k;
            converged = true;
            break;
        }
    }
    if (!converged) return NAN;
    if (n_steps * EPS * abssum <= ACCEPTABLE_RTOL * std::fabs(result)) return result;
    return NAN;
}

// hyp1f1.rs:101-120
static double hyp1f1_series(double a, double b, double x) {
    double term = 1.0, result = 1.0;
    bool converged = false;
    for (int ki = 0; ki < 1000; ki++) {
        double k = (double)ki;
        term *= (a + k) * x / (b + k) / (k + 1.0);
        result += term;
        if (std::fabs(term) <= EPS * std::fabs(result)) {
            converged = true;
            break;
        }
    }
    if (!converged) return NAN;
    return result;
}

// hyp1f1.rs:129-255
static double chgm(double a, double b, double x) {
    double a0 = a;
    double x0 = x;
    double result = 0.0;
    if (x < 0.0) {
        a = b - a;
        a0 = a;
        x = std::fabs(x);
    }
    int nl = 0, la = 0;
    if (a >= 2.0) {
        nl = 1;
        la = (int)a;
        a = a - (double)la - 1.0;
    }
    double y0 = 0.0, y1 = 0.0;
    for (int n = 0; n <= nl; n++) {
        if (a0 >= 2.0) a += 1.0;
        if (x <= std::fabs(b) + 30.0 || a < 0.0) {
            result = 1.0;
            double term = 1.0;
            if (x < 500.0) {
                for (int ji = 1; ji <= 500; ji++) {
                    double j = (double)ji;
                    term *= (a + j - 1.0) / (j * (b + j - 1.0)) * x;
                    result += term;
                    if (result != 0.0 && std::fabs(term / result) < 1e-15) break;
                }
                if (x0 < 0.0) result *= std::exp(x0);
            } else {
                for (int ji = 1; ji <= 50; ji++) {
                    double j = (double)ji;
                    term *= (j - a) * (b - a + j - 1.0) / (j * x);
                    result += term;
                    if (result != 0.0 && std::fabs(term / result) < 1e-15) break;
                }
                result *= std::pow(x, a - b) * gamma(b) / gamma(a);
                if (x0 > 0.0) result *= std::exp(x);
            }
        } else {
            double lga = ln_gamma(a);
            double lgb = ln_gamma(b);
            double lgba = ln_gamma(b - a);
            double sum1 = 1.0, sum2 = 1.0, term1 = 1.0, term2 = 1.0;
            for (int ii = 1; ii <= 30; ii++) {
                double i = (double)ii;
                term1 = -term1 * (a + i - 1.0) * (a - b + i) / (x * i);
                term2 = -term2 * (b - a + i - 1.0) * (a - i) / (x * i);
                sum1 += term1;
                sum2 += term2;
            }
            double hg1, hg2;
            if (x0 >= 0.0) {
                hg1 = std::exp(lgb - lgba) * std::pow(x, -a) * std::cos(PI * a) * sum1;
                hg2 = std::exp(lgb - lga + x) * std::pow(x, a - b) * sum2;
            } else {
                hg1 = std::exp(lgb - lgba + x0) * std::pow(x, -a) * std::cos(PI * a) * sum1;
                hg2 = std::exp(lgb - lga) * std::pow(x, a - b) * sum2;
            }
            result = hg1 + hg2;
        }
        if (n == 0) y0 = result;
        if (n == 1) y1 = result;
    }
    if (a0 >= 2.0) {
        for (int i = 1; i < la; i++) {
            result = ((a * 2.0 - b + x) * y1 + (b - a) * y0) / a;
            y0 = y1;
            y1 = result;
            a += 1.0;
        }
    }
    return result;
}

// hyp1f1.rs:17-50
static double hyp1f1(double a, double b, double x) {
    if (!(std::isfinite(a) && std::isfinite(b) && std::isfinite(x))) throw std::runtime_error("hyp1f1: non finite input");
    if (!(b > 0.0)) throw std::runtime_error("b must be positive");
    if (a == 0.0 || x == 0.0) return 1.0;
    if (a == -1.0) return 1.0 - x / b;
    if (a == b) return std::exp(x);
    if (a - b == 1.0) return (1.0 + x / b) * std::exp(x);
    if (a <= 0.0 && a == std::floor(a)) return hyp1f1_series_track_convergence(a, b, x);
    if (b > 0.0 && (std::fabs(a) + 1.0) * std::fabs(x) < 0.9 * b) return hyp1f1_series(a, b, x);
    return chgm(a, b, x);
}

// ---------------------------------------------------------------------------
// math/eigen.rs -- JAMA tred2 + tql2 (EISPACK) symmetric eigensolver
// ---------------------------------------------------------------------------
struct Matrix {
    size_t n = 0;
    std::vector<double> d;
    explicit Matrix(size_t n_ = 0) : n(n_), d(n_ * n_, 0.0) {}
    double& operator()(size_t i, size_t j) { return d[i * n + j]; }
    double operator()(size_t i, size_t j) const { return d[i * n + j]; }
};

// eigen.rs:23-130
static void tred2(std::vector<double>& eval, Matrix& evec, std::vector<double>& work) {
    size_t n = eval.size();
    for (size_t j = 0; j < n; j++) eval[j] = evec(n - 1, j);
    for (size_t i = n - 1; i >= 1; i--) {
        double scale = 0.0, h = 0.0;
        for (size_t k = 0; k < i; k++) scale += std::fabs(eval[k]);
        if (scale == 0.0) {
            work[i] = eval[i - 1];
            for (size_t j = 0; j < i; j++) {
                eval[j] = evec(i - 1, j);
                evec(i, j) = 0.0;
                evec(j, i) = 0.0;
            }
        } else {
            for (size_t k = 0; k < i; k++) {
                eval[k] /= scale;
                h += eval[k] * eval[k];
            }
            double f = eval[i - 1];
            double g = std::sqrt(h);
            if (f > 0.0) g = -g;
            work[i] = scale * g;
            h -= f * g;
            eval[i - 1] = f - g;
            for (size_t j = 0; j < i; j++) work[j] = 0.0;
            for (size_t j = 0; j < i; j++) {
                f = eval[j];
                evec(j, i) = f;
                g = work[j] + evec(j, j) * f;
                for (size_t k = j + 1; k < i; k++) {
                    g += evec(k, j) * eval[k];
                    work[k] += evec(k, j) * f;
                }
                work[j] = g;
            }
            f = 0.0;
            for (size_t j = 0; j < i; j++) {
                work[j] /= h;
                f += work[j] * eval[j];
            }
            double hh = f / (h + h);
            for (size_t j = 0; j < i; j++) work[j] -= hh * eval[j];
            for (size_t j = 0; j < i; j++) {
                f = eval[j];
                g = work[j];
                for (size_t k = j; k < i; k++) {
                    double orig = evec(k, j);
                    evec(k, j) = orig - (f * work[k] + g * eval[k]);
                }
                eval[j] = evec(i - 1, j);
                evec(i, j) = 0.0;
            }
        }
        eval[i] = h;
    }
    for (size_t i = 0; i + 1 < n; i++) {
        double orig = evec(i, i);
        evec(n - 1, i) = orig;
        evec(i, i) = 1.0;
        double h = eval[i + 1];
        if (h != 0.0) {
            for (size_t k = 0; k < i + 1; k++) eval[k] = evec(k, i + 1) / h;
            for (size_t j = 0; j < i + 1; j++) {
                double g = 0.0;
                for (size_t k = 0; k < i + 1; k++) g += evec(k, i + 1) * evec(k, j);
                for (size_t k = 0; k < i + 1; k++) {
                    double o = evec(k, j);
                    evec(k, j) = o - g * eval[k];
                }
            }
        }
        for (size_t k = 0; k < i + 1; k++) evec(k, i + 1) = 0.0;
    }
    for (size_t j = 0; j < n; j++) {
        eval[j] = evec(n - 1, j);
        evec(n - 1, j) = 0.0;
    }
    evec(n - 1, n - 1) = 1.0;
    work[0] = 0.0;
}

// eigen.rs:138-244
static void tql2(std::vector<double>& eval, Matrix& evec, std::vector<double>& work) {
    size_t n = eval.size();
    for (size_t i = 1; i < n; i++) work[i - 1] = work[i];
    work[n - 1] = 0.0;
    double f = 0.0, tst1 = 0.0;
    for (size_t l = 0; l < n; l++) {
        tst1 = std::max(tst1, std::fabs(eval[l]) + std::fabs(work[l]));
        size_t m = l;
        while (m < n) {
            if (std::fabs(work[m]) <= EPS * tst1) break;
            m += 1;
        }
        if (m > l) {
            for (;;) {
                double g = eval[l];
                double p = (eval[l + 1] - g) / (2.0 * work[l]);
                double r = std::hypot(p, 1.0);
                if (p < 0.0) r = -r;
                eval[l] = work[l] / (p + r);
                eval[l + 1] = work[l] * (p + r);
                double eval_lp1 = eval[l + 1];
                double h = g - eval[l];
                for (size_t i = l + 2; i < n; i++) eval[i] -= h;
                f += h;
                p = eval[m];
                double c = 1.0, c2 = c, c3 = c;
                double work_lp1 = work[l + 1];
                double s = 0.0, s2 = 0.0;
                for (size_t ii = m; ii-- > l;) {
                    size_t i = ii;
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * work[i];
                    h = c * p;
                    r = std::hypot(p, work[i]);
                    work[i + 1] = s * r;
                    s = work[i] / r;
                    c = p / r;
                    p = c * eval[i] - s * g;
                    eval[i + 1] = h + s * (c * g + s * eval[i]);
                    for (size_t k = 0; k < n; k++) {
                        h = evec(k, i + 1);
                        evec(k, i + 1) = s * evec(k, i) + c * h;
                        evec(k, i) = c * evec(k, i) - s * h;
                    }
                }
                p = -s * s2 * c3 * work_lp1 * work[l] / eval_lp1;
                work[l] = s * p;
                eval[l] = c * p;
                if (std::fabs(work[l]) <= EPS * tst1) break;
            }
        }
        eval[l] += f;
        work[l] = 0.0;
    }
    for (size_t i = 0; i + 1 < n; i++) {
        size_t k = i;
        double p = eval[i];
        for (size_t j = i + 1; j < n; j++) {
            if (eval[j] < p) {
                k = j;
                p = eval[j];
            }
        }
        if (k != i) {
            eval[k] = eval[i];
            eval[i] = p;
            for (size_t j = 0; j < n; j++) {
                p = evec(j, i);
                evec(j, i) = evec(j, k);
                evec(j, k) = p;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// calculators/shared/basis/radial/gto.rs
// ---------------------------------------------------------------------------
// gto.rs:44-50
static std::vector<double> gto_widths(size_t size, double radius) {
    std::vector<double> w(size);
    for (size_t n = 0; n < size; n++) {
        double nf = (double)n;
        w[n] = radius * std::max(std::sqrt(nf), 1.0) / (double)size;
    }
    return w;
}

// gto.rs:17-42
static Matrix gto_overlap(size_t size, double radius) {
    auto w = gto_widths(size, radius);
    Matrix S(size);
    for (size_t n1 = 0; n1 < size; n1++) {
        double s1 = w[n1], s1sq = s1 * s1;
        for (size_t n2 = n1; n2 < size; n2++) {
            double s2 = w[n2], s2sq = s2 * s2;
            double e = 0.5 * (3.0 + (double)n1 + (double)n2);
            double value = std::pow(0.5 / s1sq + 0.5 / s2sq, -e) / (powi(s1, (int)n1) * powi(s2, (int)n2)) * gamma(e)
                         / (std::pow(s1 * s2, 1.5) * std::sqrt(gamma((double)n1 + 1.5) * gamma((double)n2 + 1.5)));
            S(n2, n1) = value;
            S(n1, n2) = value;
        }
    }
    return S;
}

// gto.rs:53-75 -- returns M = S^{-1/2} diag(norm)
static Matrix gto_orthonormalization(size_t size, double radius) {
    auto w = gto_widths(size, radius);
    std::vector<double> norm(size);
    for (size_t n = 0; n < size; n++)
        norm[n] = std::sqrt(2.0 / (powi(w[n], 2 * (int)n + 3) * gamma((double)n + 1.5)));
    Matrix evec = gto_overlap(size, radius);
    std::vector<double> eval(size, 0.0), work(size, 0.0);
    tred2(eval, evec, work);
    tql2(eval, evec, work);
    for (size_t n = 0; n < size; n++) {
        if (eval[n] <= EPS) throw std::runtime_error("radial overlap matrix is singular");
        eval[n] = 1.0 / std::sqrt(eval[n]);
    }
    // eigen.rs:273-276 recompose = (V diag(eval)) V^T
    Matrix vd(size), rec(size), M(size);
    for (size_t i = 0; i < size; i++)
        for (size_t j = 0; j < size; j++) vd(i, j) = evec(i, j) * eval[j];
    for (size_t i = 0; i < size; i++)
        for (size_t j = 0; j < size; j++) {
            double s = 0.0;
            for (size_t k = 0; k < size; k++) s += vd(i, k) * evec(j, k);
            rec(i, j) = s;
        }
    for (size_t i = 0; i < size; i++)
        for (size_t j = 0; j < size; j++) M(i, j) = rec(i, j) * norm[j];
    return M;
}

// ---------------------------------------------------------------------------
// calculators/soap/radial_integral/gto.rs
// ---------------------------------------------------------------------------
struct GtoRadialIntegral {
    size_t l;
    double width2;           // σ²
    double c;                // 1/(2σ²)
    std::vector<double> bn;  // 1/(2σ_n²)
    Matrix M;                // orthonormalization (values · Mᵀ)

    GtoRadialIntegral(double cutoff, double width, size_t max_radial, size_t l_) : l(l_) {
        size_t size = max_radial + 1;
        auto w = gto_widths(size, cutoff);
        for (double s : w) bn.push_back(1.0 / (2.0 * s * s));
        M = gto_orthonormalization(size, cutoff);
        width2 = width * width;
        c = 1.0 / (2.0 * width2);
    }

    size_t size() const { return bn.size(); }

    // gto.rs:115-205
    void compute(double r, double* values, double* gradients) const {
        size_t N = size();
        std::vector<double> v(N), g(N);
        double global = std::pow(PI / width2, 0.75);
        double c_rij = c * r;
        double c_rij_l = powi(c_rij, (int)l);
        double exp_c = std::exp(-r * c_rij);
        double factor = global * exp_c * c_rij_l;
        for (size_t n = 0; n < N; n++) {
            double z = c_rij * c_rij / (c + bn[n]);
            double a = 0.5 * (double)(n + l + 3), b = (double)l + 1.5;
            double ratio = gamma(a) / gamma(b);
            v[n] = ratio * hyp1f1(a, b, z);
            if (gradients) g[n] = ratio * (a / b * hyp1f1(a + 1.0, b + 1.0, z));
            if (!std::isfinite(v[n])) throw std::runtime_error("Failed to compute radial integral with GTO basis");
            double e = 0.5 * (double)(n + l) + 1.5;
            double c_dn = std::pow(c + bn[n], -e);
            v[n] *= c_dn * factor;
            if (gradients) {
                g[n] *= c_dn * factor * 2.0 * z / r;
                g[n] += v[n] * ((double)l / r - 2.0 * c_rij);
            }
        }
        if (r == 0.0 && gradients) {
            if (l == 1) {
                for (size_t n = 0; n < N; n++) {
                    double a = 0.5 * (double)(n + l) + 1.5;
                    double b = 2.5;
                    double c_dn = std::pow(c + bn[n], -a);
                    double f = global * c * c_dn;
                    g[n] = gamma(a) / gamma(b) * f;
                }
            } else {
                std::fill(g.begin(), g.end(), 0.0);
            }
        }
        for (size_t k = 0; k < N; k++) {
            double s = 0.0, sg = 0.0;
            for (size_t n = 0; n < N; n++) {
                s += v[n] * M(k, n);
                if (gradients) sg += g[n] * M(k, n);
            }
            values[k] = s;
            if (gradients) gradients[k] = sg;
        }
    }
};

// ---------------------------------------------------------------------------
// math/splines.rs -- adaptive Hermite cubic spline
// ---------------------------------------------------------------------------
struct Spline {
    size_t size = 0;
    std::vector<double> positions;
    std::vector<std::vector<double>> values, derivs;

    // splines.rs:225-289
    void compute(double x, double* out, double* grad) const {
        // largest k with positions[k] <= x (binary search semantics), clamped
        size_t lo = 0, hi = positions.size();
        while (lo < hi) {
            size_t mid = lo + (hi - lo) / 2;
            if (positions[mid] <= x) lo = mid + 1; else hi = mid;
        }
        size_t k = lo == 0 ? 0 : lo - 1;
        if (k == positions.size() - 1) k -= 1;
        double xk = positions[k], xk1 = positions[k + 1];
        double delta = xk1 - xk;
        double t = (x - xk) / delta;
        double t2 = t * t, t3 = t2 * t;
        double h00 = 2.0 * t3 - 3.0 * t2 + 1.0;
        double h10 = t3 - 2.0 * t2 + t;
        double h01 = -2.0 * t3 + 3.0 * t2;
        double h11 = t3 - t2;
        const auto& pk = values[k]; const auto& pk1 = values[k + 1];
        const auto& mk = derivs[k]; const auto& mk1 = derivs[k + 1];
        for (size_t i = 0; i < size; i++)
            out[i] = h00 * pk[i] + h10 * delta * mk[i] + h01 * pk1[i] + h11 * delta * mk1[i];
        if (grad) {
            double dh00 = 6.0 * (t2 - t);
            double dh10 = 3.0 * t2 - 4.0 * t + 1.0;
            double dh01 = -dh00;
            double dh11 = 3.0 * t2 - 2.0 * t;
            double dxdt = 1.0 / delta;
            for (size_t i = 0; i < size; i++)
                grad[i] = dh00 * pk[i] * dxdt + dh10 * mk[i] + dh01 * pk1[i] * dxdt + dh11 * mk1[i];
        }
    }
};

// splines.rs:79-193 + radial_integral/spline.rs:28-52
static Spline build_spline(const GtoRadialIntegral& gto, double stop, double accuracy) {
    if (accuracy < 0.0) throw std::runtime_error("got invalid accuracy in spline");
    Spline sp;
    sp.size = gto.size();
    size_t N = sp.size;
    const size_t initial = 11;
    double start = 0.0;
    double step = (stop - start) / (double)(initial - 1);
    auto eval = [&](double x, std::vector<double>& v, std::vector<double>& d) {
        v.assign(N, 0.0);
        d.assign(N, 0.0);
        gto.compute(x, v.data(), d.data());
    };
    for (size_t k = 0; k < initial - 1; k++) {
        double x = start + (double)k * step;
        std::vector<double> v, d;
        eval(x, v, d);
        sp.positions.push_back(x);
        sp.values.push_back(v);
        sp.derivs.push_back(d);
    }
    {
        std::vector<double> v, d;
        eval(stop, v, d);
        sp.positions.push_back(stop);
        sp.values.push_back(v);
        sp.derivs.push_back(d);
    }
    std::vector<double> interp(N);
    for (;;) {
        double mean_abs = 0.0, mean_rel = 0.0;
        size_t count = 0;
        std::vector<std::tuple<double, std::vector<double>, std::vector<double>>> added;
        for (size_t k = 0; k + 1 < sp.positions.size(); k++) {
            double x = (sp.positions[k] + sp.positions[k + 1]) / 2.0;
            std::vector<double> v, d;
            eval(x, v, d);
            sp.compute(x, interp.data(), nullptr);
            for (size_t i = 0; i < N; i++) {
                double ae = std::fabs(interp[i] - v[i]);
                mean_abs += ae;
                mean_rel += std::fabs((interp[i] - v[i]) / v[i]);
                count += 1;
            }
            added.emplace_back(x, v, d);
        }
        mean_abs /= (double)count;
        mean_rel /= (double)count;
        if (mean_abs < accuracy || mean_rel < accuracy) break;
        if (sp.positions.size() + added.size() > 10000) throw std::runtime_error("failed to reach requested accuracy in spline interpolation");
        // the midpoints interleave with the existing knots
        Spline next;
        next.size = N;
        for (size_t k = 0; k < sp.positions.size(); k++) {
            next.positions.push_back(sp.positions[k]);
            next.values.push_back(sp.values[k]);
            next.derivs.push_back(sp.derivs[k]);
            if (k < added.size()) {
                next.positions.push_back(std::get<0>(added[k]));
                next.values.push_back(std::get<1>(added[k]));
                next.derivs.push_back(std::get<2>(added[k]));
            }
        }
        sp = std::move(next);
    }
    return sp;
}

// ---------------------------------------------------------------------------
// math/spherical_harmonics.rs (arXiv:1410.1748 recursion)
// ---------------------------------------------------------------------------
static const double SQRT_1_OVER_2PI = 0.3989422804014327;
static const double SQRT_3 = 1.7320508075688772;
static const double SQRT_3_OVER_2 = 1.224744871391589;
static const double SQRT_2 = 1.4142135623730951;

struct SphericalHarmonics {
    int lmax;
    std::vector<double> A, B, P, dP, Pot;  // LegendreArray, index m + l(l+1)/2

    static size_t li(int l, int m) { return (size_t)(m + l * (l + 1) / 2); }

    // spherical_harmonics.rs:203-224
    explicit SphericalHarmonics(int lmax_) : lmax(lmax_) {
        size_t n = (size_t)((lmax + 1) * (lmax + 2) / 2);
        A.assign(n, 0.0); B.assign(n, 0.0); P.assign(n, 0.0); dP.assign(n, 0.0); Pot.assign(n, 0.0);
        for (int l = 2; l <= lmax; l++) {
            double ls = (double)(l * l);
            double lm1s = (double)((l - 1) * (l - 1));
            for (int m = 0; m < l - 1; m++) {
                double ms = (double)(m * m);
                A[li(l, m)] = std::sqrt((4.0 * ls - 1.0) / (ls - ms));
                B[li(l, m)] = -std::sqrt((lm1s - ms) / (4.0 * lm1s - 1.0));
            }
        }
    }

    // spherical_harmonics.rs:228-251
    void legendre(double ct, double st) {
        double value = SQRT_1_OVER_2PI;
        P[li(0, 0)] = value;
        if (lmax > 0) {
            P[li(1, 0)] = ct * SQRT_3 * value;
            value *= -SQRT_3_OVER_2 * st;
            P[li(1, 1)] = value;
            for (int l = 2; l <= lmax; l++) {
                for (int m = 0; m < l - 1; m++)
                    P[li(l, m)] = A[li(l, m)] * (ct * P[li(l - 1, m)] + B[li(l, m)] * P[li(l - 2, m)]);
                P[li(l, l - 1)] = ct * std::sqrt(2.0 * (double)l + 1.0) * value;
                value *= -std::sqrt(1.0 + 0.5 / (double)l) * st;
                P[li(l, l)] = value;
            }
        }
    }

    // spherical_harmonics.rs:256-298
    void derivative_factors(double ct, double st) {
        auto delta = [](int l, int m, double pm1, double pp1) {
            return std::sqrt((double)((l + m) * (l - m + 1))) * pm1 - std::sqrt((double)((l - m) * (l + m + 1))) * pp1;
        };
        dP[li(0, 0)] = 0.0;
        for (int l = 1; l <= lmax; l++) {
            double pm1 = -1.0 / (double)(l * l + l) * P[li(l, 1)];
            double pp1 = P[li(l, 1)];
            dP[li(l, 0)] = delta(l, 0, pm1, pp1);
            for (int m = 1; m < l; m++) dP[li(l, m)] = delta(l, m, P[li(l, m - 1)], P[li(l, m + 1)]);
            dP[li(l, l)] = delta(l, l, P[li(l, l - 1)], 0.0);
        }
        if (st > 0.1) {
            for (int l = 0; l <= lmax; l++)
                for (int m = 0; m <= l; m++) Pot[li(l, m)] = (double)m / st * P[li(l, m)];
        } else {
            for (int l = 0; l <= lmax; l++)
                for (int m = 0; m <= l; m++) Pot[li(l, m)] = -0.5 / ct * dP[li(l, m)];
        }
    }

    // spherical_harmonics.rs:304-424.  values / gradients use index l*l + l + m.
    void compute(const double* d, double* values, double* gx, double* gy, double* gz) {
        double n2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (!(std::fabs(n2 - 1.0) < 1e-9)) throw std::runtime_error("expected the direction vector to be normalized");
        double sxy = std::hypot(d[0], d[1]);
        double ct = d[2], st = sxy;
        double cp, sp;
        if (sxy > EPS) { cp = d[0] / sxy; sp = d[1] / sxy; } else { cp = 1.0; sp = 0.0; }
        legendre(ct, st);
        bool grad = gx != nullptr;
        if (grad) derivative_factors(ct, st);
        auto si = [](int l, int m) { return (size_t)(l * l + l + m); };
        for (int l = 0; l <= lmax; l++) values[si(l, 0)] = P[li(l, 0)] / SQRT_2;
        if (grad) {
            gx[0] = gy[0] = gz[0] = 0.0;
            for (int l = 1; l <= lmax; l++) {
                double lf = std::sqrt(0.5 * (double)(l * (l + 1))) * P[li(l, 1)];
                gx[si(l, 0)] = cp * ct * lf;
                gy[si(l, 0)] = sp * ct * lf;
                gz[si(l, 0)] = -st * lf;
            }
        }
        double cos1 = 1.0, sin1 = 0.0;
        double cos2 = -cp, sin2 = sp;
        double m2c = -2.0 * cp;
        for (int m = 1; m <= lmax; m++) {
            double smp = m2c * sin1 - sin2;
            double cmp = m2c * cos1 - cos2;
            sin2 = sin1; sin1 = smp;
            cos2 = cos1; cos1 = cmp;
            for (int l = m; l <= lmax; l++) {
                double p = P[li(l, m)];
                values[si(l, m)] = p * cmp;
                values[si(l, -m)] = p * smp;
            }
            if (grad) {
                for (int l = m; l <= lmax; l++) {
                    double dp = dP[li(l, m)];
                    double sdp = smp * dp, cdp = cmp * dp;
                    double pot = Pot[li(l, m)];
                    gx[si(l, m)] = sp * pot * smp - 0.5 * ct * cp * cdp;
                    gx[si(l, -m)] = -sp * pot * cmp - 0.5 * ct * cp * sdp;
                    gy[si(l, m)] = -cp * pot * smp - 0.5 * ct * sp * cdp;
                    gy[si(l, -m)] = cp * pot * cmp - 0.5 * ct * sp * sdp;
                    gz[si(l, m)] = 0.5 * st * cdp;
                    gz[si(l, -m)] = 0.5 * st * sdp;
                }
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Hyper-parameters (PowerSpectrumParameters / SphericalExpansionParameters)
// ---------------------------------------------------------------------------
}  // namespace oracle

extern "C" {
typedef struct oracle_hypers {
    double cutoff;
    int32_t smoothing;       // 0 = ShiftedCosine, 1 = Step
    double smoothing_width;
    double density_width;    // Gaussian width
    double center_atom_weight;
    int32_t scaling;         // 0 = none, 1 = Willatt2018
    double scaling_scale, scaling_rate, scaling_exponent;
    int32_t max_angular;
    int32_t max_radial;
    double spline_accuracy;  // < 0 means "null" (analytic GTO)
} oracle_hypers;

typedef struct oracle_system {
    uint64_t n_atoms;
    const int32_t* types;
    const double* positions;  // n_atoms x 3
    double cell[9];           // row-major, all zero = infinite
} oracle_system;
}

namespace oracle {

// calculators/soap/cutoff.rs:48-79
static double smoothing(const oracle_hypers& h, double r) {
    if (h.smoothing == 1) return r >= h.cutoff ? 0.0 : 1.0;
    double w = h.smoothing_width;
    if (r <= h.cutoff - w) return 1.0;
    if (r >= h.cutoff) return 0.0;
    double s = PI * (r - h.cutoff + w) / w;
    return 0.5 * (1. + std::cos(s));
}

static double smoothing_gradient(const oracle_hypers& h, double r) {
    if (h.smoothing == 1) return 0.0;
    double w = h.smoothing_width;
    if (r <= h.cutoff - w || r >= h.cutoff) return 0.0;
    double s = PI * (r - h.cutoff + w) / w;
    return -0.5 * PI * std::sin(s) / w;
}

// calculators/shared/density.rs:108-128
static double scaling_value(const oracle_hypers& h, double r) {
    return h.scaling_rate / (h.scaling_rate + std::pow(r / h.scaling_scale, h.scaling_exponent));
}
static double scaling_gradient(const oracle_hypers& h, double r) {
    double rs = r / h.scaling_scale;
    double rs_m1 = std::pow(rs, h.scaling_exponent - 1.0);
    double rs_m = rs * rs_m1;
    double factor = -h.scaling_rate * h.scaling_exponent / h.scaling_scale;
    return factor * rs_m1 / ((h.scaling_rate + rs_m) * (h.scaling_rate + rs_m));
}

// spherical_expansion_pair.rs:189-210
static double scaling_functions(const oracle_hypers& h, double r) {
    double s = 1.0;
    if (h.scaling) s = scaling_value(h, r);
    return s * smoothing(h, r);
}
static double scaling_functions_gradient(const oracle_hypers& h, double r) {
    double s = 1.0, sg = 0.0;
    if (h.scaling) { s = scaling_value(h, r); sg = scaling_gradient(h, r); }
    return smoothing_gradient(h, r) * s + smoothing(h, r) * sg;
}

// radial_integral/mod.rs:139-199 -- one radial integral per angular channel
struct RadialIntegrals {
    std::vector<GtoRadialIntegral> gto;
    std::vector<Spline> splines;
    bool splined;
    size_t nmax;

    RadialIntegrals(const oracle_hypers& h) {
        nmax = (size_t)h.max_radial + 1;
        splined = h.spline_accuracy >= 0.0;
        for (int l = 0; l <= h.max_angular; l++) {
            gto.emplace_back(h.cutoff, h.density_width, (size_t)h.max_radial, (size_t)l);
            if (splined) splines.push_back(build_spline(gto.back(), h.cutoff, h.spline_accuracy));
        }
    }
    void compute(int l, double r, double* v, double* g) const {
        if (splined) splines[l].compute(r, v, g);
        else gto[l].compute(r, v, g);
    }
};

// ---------------------------------------------------------------------------
// Minimal TensorMap (metatensor layout: keys + blocks with samples,
// components, properties, values and gradient blocks)
// ---------------------------------------------------------------------------
struct Labels {
    size_t width = 0;
    std::vector<int32_t> values;
    size_t count() const { return width == 0 ? 0 : values.size() / width; }
    void add(std::initializer_list<int32_t> row) { values.insert(values.end(), row.begin(), row.end()); }
};

struct Block {
    Labels samples;
    std::vector<size_t> components;  // sizes of the component axes
    Labels properties;
    std::vector<double> values;
    std::vector<size_t> shape;
    std::map<std::string, Block> gradients;
};

struct TensorMap {
    Labels keys;
    std::vector<Block> blocks;
};

struct System {
    size_t n;
    const int32_t* types;
    const double* positions;
    UnitCell cell;
    NeighborsList nl;
};

// Options of a compute call
struct Options {
    bool positions = false, strain = false, cell = false;
    int threads = 1;
    bool se_over_centres = false;  // project variant, not the reference's decomposition
};

// Per-system accumulation, spherical_expansion.rs:101-358.  Arrays are kept
// for every l with the layouts documented at spherical_expansion.rs:607-647.
struct PairAccumulation {
    std::map<int32_t, size_t> types_mapping;  // type -> first-appearance index
    std::vector<long> center_mapping;          // atom -> mapped centre or -1
    size_t n_types = 0, n_centers = 0, n_pairs = 0;
    // l -> arrays
    std::vector<std::vector<double>> values;    // [nt][center][2l+1][n]
    std::vector<std::vector<double>> pair_grad; // [pair][3][2l+1][n]
    std::vector<std::vector<double>> self_grad; // [nt][center][3][2l+1][n]
    std::vector<std::vector<double>> cell_grad; // [nt][center][3][3][2l+1][n]
    std::vector<std::vector<double>> strain_grad;
    std::map<std::pair<size_t, size_t>, std::vector<size_t>> pairs_for_grad;
    std::vector<const Pair*> pairs;             // contributing pairs, by pair_id
};

struct Calculator {
    oracle_hypers h;
    RadialIntegrals ri;
    int lmax;
    size_t nmax;
    Calculator(const oracle_hypers& hh) : h(hh), ri(hh), lmax(hh.max_angular), nmax((size_t)hh.max_radial + 1) {}

    // spherical_expansion_pair.rs:323-422: contribution of one pair.
    // vals[l] : [2l+1][n], grads[l]: [3][2l+1][n]
    void compute_for_pair(SphericalHarmonics& sph, double distance, double dir[3], bool do_grad,
                          std::vector<std::vector<double>>& vals, std::vector<std::vector<double>>& grads,
                          std::vector<double>& Y, std::vector<double>& GX, std::vector<double>& GY, std::vector<double>& GZ,
                          std::vector<double>& R, std::vector<double>& dR) const {
        if (distance < 1e-6) { dir[0] = 0.0; dir[1] = 0.0; dir[2] = 1.0; }
        for (int l = 0; l <= lmax; l++) ri.compute(l, distance, &R[l * nmax], do_grad ? &dR[l * nmax] : nullptr);
        sph.compute(dir, Y.data(), do_grad ? GX.data() : nullptr, GY.data(), GZ.data());
        double f = scaling_functions(h, distance);
        double fg = scaling_functions_gradient(h, distance);
        for (int l = 0; l <= lmax; l++) {
            size_t nm = 2 * l + 1;
            for (size_t m = 0; m < nm; m++) {
                double y = Y[l * l + m];
                for (size_t n = 0; n < nmax; n++) vals[l][m * nmax + n] = f * y * R[l * nmax + n];
            }
            if (do_grad) {
                for (size_t m = 0; m < nm; m++) {
                    double y = Y[l * l + m];
                    double yx = GX[l * l + m], yy = GY[l * l + m], yz = GZ[l * l + m];
                    for (size_t n = 0; n < nmax; n++) {
                        double ri_v = R[l * nmax + n], ri_g = dR[l * nmax + n];
                        grads[l][(0 * nm + m) * nmax + n] = fg * dir[0] * ri_v * y + f * ri_g * dir[0] * y + f * ri_v * yx / distance;
                        grads[l][(1 * nm + m) * nmax + n] = fg * dir[1] * ri_v * y + f * ri_g * dir[1] * y + f * ri_v * yy / distance;
                        grads[l][(2 * nm + m) * nmax + n] = fg * dir[2] * ri_v * y + f * ri_g * dir[2] * y + f * ri_v * yz / distance;
                    }
                }
            }
        }
    }

    // spherical_expansion_pair.rs:222-252
    std::vector<double> self_contribution() const {
        std::vector<double> R(nmax);
        ri.compute(0, 0.0, R.data(), nullptr);
        SphericalHarmonics sph(lmax);
        std::vector<double> Y((size_t)((lmax + 1) * (lmax + 1)));
        double d[3] = {0.0, 0.0, 1.0};
        sph.compute(d, Y.data(), nullptr, nullptr, nullptr);
        double f = scaling_functions(h, 0.0);
        double factor = h.center_atom_weight * f * Y[0];
        for (auto& v : R) v = factor * v;
        return R;
    }

    // spherical_expansion.rs:101-358
    PairAccumulation accumulate_all_pairs(const System& sys, const Options& opt, const std::set<size_t>& requested, int threads) const {
        PairAccumulation res;
        for (size_t i = 0; i < sys.n; i++) {
            int32_t t = sys.types[i];
            if (!res.types_mapping.count(t)) {
                size_t next = res.types_mapping.size();
                res.types_mapping[t] = next;
            }
        }
        res.n_types = res.types_mapping.size();
        res.center_mapping.assign(sys.n, -1);
        {
            size_t k = 0;
            for (size_t a : requested) res.center_mapping[a] = (long)(k++);
        }
        res.n_centers = requested.size();
        for (const auto& p : sys.nl.pairs)
            if (requested.count(p.first) || requested.count(p.second)) res.pairs.push_back(&p);
        res.n_pairs = res.pairs.size();
        bool do_grad = opt.positions || opt.strain || opt.cell;
        size_t NT = res.n_types, NC = res.n_centers;
        res.values.resize(lmax + 1);
        if (opt.positions) { res.pair_grad.resize(lmax + 1); res.self_grad.resize(lmax + 1); }
        if (opt.cell) res.cell_grad.resize(lmax + 1);
        if (opt.strain) res.strain_grad.resize(lmax + 1);
        for (int l = 0; l <= lmax; l++) {
            size_t blk = (2 * l + 1) * nmax;
            res.values[l].assign(NT * NC * blk, 0.0);
            if (opt.positions) {
                res.pair_grad[l].assign(res.n_pairs * 3 * blk, 0.0);
                res.self_grad[l].assign(NT * NC * 3 * blk, 0.0);
            }
            if (opt.cell) res.cell_grad[l].assign(NT * NC * 9 * blk, 0.0);
            if (opt.strain) res.strain_grad[l].assign(NT * NC * 9 * blk, 0.0);
        }

        // pairs_for_positions_gradient bookkeeping (spherical_expansion.rs:200, :281)
        for (size_t pid = 0; pid < res.n_pairs; pid++) {
            const Pair& p = *res.pairs[pid];
            if (res.center_mapping[p.first] >= 0) res.pairs_for_grad[{p.first, p.second}].push_back(pid);
            if (res.center_mapping[p.second] >= 0) res.pairs_for_grad[{p.second, p.first}].push_back(pid);
        }

        // Project variant: parallel over centres.  Each thread owns a subset
        // of centres and walks every pair, keeping per-centre sums in pair
        // order, so the result is identical to the serial loop.
        int nthreads = (opt.se_over_centres && threads > 1) ? threads : 1;
#pragma omp parallel num_threads(nthreads)
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            SphericalHarmonics sph(lmax);
            size_t L2 = (size_t)((lmax + 1) * (lmax + 1));
            std::vector<double> Y(L2), GX(L2), GY(L2), GZ(L2), R((lmax + 1) * nmax), dR((lmax + 1) * nmax);
            std::vector<std::vector<double>> vals(lmax + 1), grads(lmax + 1);
            for (int l = 0; l <= lmax; l++) {
                vals[l].assign((2 * l + 1) * nmax, 0.0);
                grads[l].assign(3 * (2 * l + 1) * nmax, 0.0);
            }
            auto owns = [&](long mc) { return mc >= 0 && (nthreads == 1 || (mc % nthreads) == tid); };
            for (size_t pid = 0; pid < res.n_pairs; pid++) {
                const Pair& p = *res.pairs[pid];
                long mc1 = res.center_mapping[p.first], mc2 = res.center_mapping[p.second];
                bool own1 = owns(mc1), own2 = owns(mc2);
                bool store_pair = opt.positions && mc1 >= 0 && (nthreads == 1 || (pid % (size_t)nthreads) == (size_t)tid);
                if (!own1 && !own2 && !store_pair) continue;
                double dir[3] = {p.vector[0] / p.distance, p.vector[1] / p.distance, p.vector[2] / p.distance};
                compute_for_pair(sph, p.distance, dir, do_grad, vals, grads, Y, GX, GY, GZ, R, dR);
                if (mc1 >= 0) {
                    size_t nt = res.types_mapping.at(sys.types[p.second]);
                    for (int l = 0; l <= lmax; l++) {
                        size_t blk = (2 * l + 1) * nmax;
                        if (own1) {
                            double* out = &res.values[l][(nt * NC + mc1) * blk];
                            for (size_t k = 0; k < blk; k++) out[k] += vals[l][k];
                        }
                        if (!do_grad) continue;
                        const double* g = grads[l].data();
                        if (store_pair) std::copy(g, g + 3 * blk, &res.pair_grad[l][pid * 3 * blk]);
                        if (!own1) continue;
                        if (opt.positions && p.first != p.second) {
                            double* sg = &res.self_grad[l][(nt * NC + mc1) * 3 * blk];
                            for (size_t k = 0; k < 3 * blk; k++) sg[k] -= g[k];
                        }
                        if (opt.cell) {
                            double* cg = &res.cell_grad[l][(nt * NC + mc1) * 9 * blk];
                            for (int abc = 0; abc < 3; abc++) {
                                double s = (double)p.shift[abc];
                                for (int xyz = 0; xyz < 3; xyz++)
                                    for (size_t k = 0; k < blk; k++) cg[(abc * 3 + xyz) * blk + k] += s * g[xyz * blk + k];
                            }
                        }
                        if (opt.strain) {
                            double* st = &res.strain_grad[l][(nt * NC + mc1) * 9 * blk];
                            for (int a = 0; a < 3; a++)
                                for (int b = 0; b < 3; b++)
                                    for (size_t k = 0; k < blk; k++) st[(a * 3 + b) * blk + k] += p.vector[a] * g[b * blk + k];
                        }
                    }
                }
                if (mc2 >= 0) {
                    // inverse_pair, spherical_expansion_pair.rs:130-163
                    for (int l = 0; l <= lmax; l++) {
                        double fv = (l % 2 == 0) ? 1.0 : -1.0;
                        double fg = -fv;
                        for (auto& v : vals[l]) v *= fv;
                        if (do_grad) for (auto& v : grads[l]) v *= fg;
                    }
                    if (!own2) continue;
                    size_t nt = res.types_mapping.at(sys.types[p.first]);
                    for (int l = 0; l <= lmax; l++) {
                        size_t blk = (2 * l + 1) * nmax;
                        double* out = &res.values[l][(nt * NC + mc2) * blk];
                        for (size_t k = 0; k < blk; k++) out[k] += vals[l][k];
                        if (!do_grad) continue;
                        const double* g = grads[l].data();
                        if (opt.positions && p.first != p.second) {
                            double* sg = &res.self_grad[l][(nt * NC + mc2) * 3 * blk];
                            for (size_t k = 0; k < 3 * blk; k++) sg[k] -= g[k];
                        }
                        if (opt.cell) {
                            double* cg = &res.cell_grad[l][(nt * NC + mc2) * 9 * blk];
                            for (int abc = 0; abc < 3; abc++) {
                                double s = (double)p.shift[abc];
                                for (int xyz = 0; xyz < 3; xyz++)
                                    for (size_t k = 0; k < blk; k++) cg[(abc * 3 + xyz) * blk + k] += -s * g[xyz * blk + k];
                            }
                        }
                        if (opt.strain) {
                            double* st = &res.strain_grad[l][(nt * NC + mc2) * 9 * blk];
                            for (int a = 0; a < 3; a++)
                                for (int b = 0; b < 3; b++)
                                    for (size_t k = 0; k < blk; k++) st[(a * 3 + b) * blk + k] += -p.vector[a] * g[b * blk + k];
                        }
                    }
                }
            }
        }
        return res;
    }
};

// ---------------------------------------------------------------------------
// labels/keys.rs and labels/samples/atom_centered.rs
// ---------------------------------------------------------------------------
static int32_t neighbor_of(const Pair& p, size_t atom) { return (int32_t)(p.first == atom ? p.second : p.first); }

// atom_centered.rs:31-101, "selection" branch (Single / OneOf filters)
static std::vector<size_t> samples_single(const System& s, int32_t ct, const std::vector<int32_t>& nts) {
    auto matches = [&](int32_t t) { return std::find(nts.begin(), nts.end(), t) != nts.end(); };
    std::set<size_t> out;
    for (size_t i = 0; i < s.n; i++) {
        if (s.types[i] != ct) continue;
        if (matches(s.types[i])) out.insert(i);
        for (const auto& p : s.nl.pairs_by_atom[i])
            if (matches(s.types[neighbor_of(p, i)])) out.insert(i);
    }
    return std::vector<size_t>(out.begin(), out.end());
}

static std::set<int32_t> neighbor_types(const System& s, size_t i) {
    std::set<int32_t> t;
    for (const auto& p : s.nl.pairs_by_atom[i]) t.insert(s.types[neighbor_of(p, i)]);
    t.insert(s.types[i]);
    return t;
}

// atom_centered.rs:103-147 -- gradient samples of one sample
static std::vector<size_t> gradient_atoms(const System& s, size_t i, const std::vector<int32_t>& nts) {
    auto matches = [&](int32_t t) { return std::find(nts.begin(), nts.end(), t) != nts.end(); };
    std::set<size_t> out;
    if (matches(s.types[i])) out.insert(i);
    for (const auto& p : s.nl.pairs_by_atom[i]) {
        size_t j = (size_t)neighbor_of(p, i);
        if (matches(s.types[j])) {
            out.insert(j);
            out.insert(i);
        }
    }
    return std::vector<size_t>(out.begin(), out.end());
}

struct SampleRef { size_t system, atom; };

// Build value / gradient blocks (calculator.rs:414-495)
static void add_gradient_blocks(Block& b, const Options& opt, const std::vector<int32_t>& grad_rows, size_t n_grad_rows,
                                const std::vector<size_t>& comp, size_t n_props) {
    size_t per = n_props;
    for (size_t c : comp) per *= c;
    size_t ns = b.samples.count();
    if (opt.positions) {
        Block g;
        g.samples.width = 3;
        g.samples.values = grad_rows;
        g.components = {3};
        g.components.insert(g.components.end(), comp.begin(), comp.end());
        g.properties = b.properties;
        g.shape = {n_grad_rows, 3};
        g.shape.insert(g.shape.end(), comp.begin(), comp.end());
        g.shape.push_back(n_props);
        g.values.assign(n_grad_rows * 3 * per, 0.0);
        b.gradients["positions"] = std::move(g);
    }
    for (const char* name : {"cell", "strain"}) {
        bool want = std::string(name) == "cell" ? opt.cell : opt.strain;
        if (!want) continue;
        Block g;
        g.samples.width = 1;
        for (size_t k = 0; k < ns; k++) g.samples.add({(int32_t)k});
        g.components = {3, 3};
        g.components.insert(g.components.end(), comp.begin(), comp.end());
        g.properties = b.properties;
        g.shape = {ns, 3, 3};
        g.shape.insert(g.shape.end(), comp.begin(), comp.end());
        g.shape.push_back(n_props);
        g.values.assign(ns * 9 * per, 0.0);
        b.gradients[name] = std::move(g);
    }
}

// ---------------------------------------------------------------------------
// Spherical expansion calculator: spherical_expansion.rs:649-849
// ---------------------------------------------------------------------------
static TensorMap spherical_expansion(const Calculator& calc, std::vector<System>& systems, const Options& opt) {
    int lmax = calc.lmax;
    size_t nmax = calc.nmax;
    // keys.rs:68-95 + spherical_expansion.rs:662-677
    std::set<std::pair<int32_t, int32_t>> tp;
    for (auto& s : systems) {
        for (const auto& p : s.nl.pairs) {
            tp.insert({s.types[p.first], s.types[p.second]});
            tp.insert({s.types[p.second], s.types[p.first]});
        }
        for (size_t i = 0; i < s.n; i++) tp.insert({s.types[i], s.types[i]});
    }
    TensorMap tm;
    tm.keys.width = 4;
    std::vector<std::tuple<int, int32_t, int32_t>> key_list;
    for (auto& ctnt : tp)
        for (int l = 0; l <= lmax; l++) {
            tm.keys.add({l, 1, ctnt.first, ctnt.second});
            key_list.emplace_back(l, ctnt.first, ctnt.second);
        }

    // samples + gradient samples per key
    std::vector<std::vector<SampleRef>> key_samples;
    std::vector<std::vector<std::vector<size_t>>> key_grad_atoms;
    for (auto& k : key_list) {
        int l; int32_t ct, nt;
        std::tie(l, ct, nt) = k;
        Block b;
        b.samples.width = 2;
        std::vector<SampleRef> refs;
        std::vector<std::vector<size_t>> gatoms;
        std::vector<int32_t> grows;
        size_t n_grows = 0;
        for (size_t si = 0; si < systems.size(); si++) {
            for (size_t a : samples_single(systems[si], ct, {nt})) {
                b.samples.add({(int32_t)si, (int32_t)a});
                refs.push_back({si, a});
            }
        }
        for (size_t r = 0; r < refs.size(); r++) {
            auto atoms = gradient_atoms(systems[refs[r].system], refs[r].atom, {nt});
            for (size_t j : atoms) {
                grows.push_back((int32_t)r);
                grows.push_back((int32_t)refs[r].system);
                grows.push_back((int32_t)j);
                n_grows++;
            }
            gatoms.push_back(atoms);
        }
        size_t nm = 2 * l + 1;
        b.components = {nm};
        b.properties.width = 1;
        for (size_t n = 0; n < nmax; n++) b.properties.add({(int32_t)n});
        b.shape = {refs.size(), nm, nmax};
        b.values.assign(refs.size() * nm * nmax, 0.0);
        add_gradient_blocks(b, opt, grows, n_grows, {nm}, nmax);
        tm.blocks.push_back(std::move(b));
        key_samples.push_back(refs);
        key_grad_atoms.push_back(gatoms);
    }

    // do_self_contributions, spherical_expansion.rs:48-96
    if (true) {
        auto self = calc.self_contribution();
        for (size_t k = 0; k < key_list.size(); k++) {
            int l; int32_t ct, nt;
            std::tie(l, ct, nt) = key_list[k];
            if (l != 0 || ct != nt) continue;
            for (size_t r = 0; r < key_samples[k].size(); r++)
                for (size_t n = 0; n < nmax; n++) tm.blocks[k].values[r * nmax + n] += self[n];
        }
    }

    // per system (rayon over systems, spherical_expansion.rs:818)
    int nthreads = opt.se_over_centres ? 1 : opt.threads;
    std::vector<int> errors(systems.size(), 0);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
    for (long si = 0; si < (long)systems.size(); si++) {
        const System& sys = systems[si];
        std::set<size_t> requested;
        for (size_t k = 0; k < key_list.size(); k++)
            for (auto& r : key_samples[k]) if (r.system == (size_t)si) requested.insert(r.atom);
        PairAccumulation acc = calc.accumulate_all_pairs(sys, opt, requested, opt.threads);
        for (size_t k = 0; k < key_list.size(); k++) {
            int l; int32_t ct, nt;
            std::tie(l, ct, nt) = key_list[k];
            auto it = acc.types_mapping.find(nt);
            if (it == acc.types_mapping.end()) continue;
            size_t nti = it->second;
            size_t nm = 2 * l + 1, blk = nm * nmax, NC = acc.n_centers;
            Block& b = tm.blocks[k];
            // values_to_metatensor
            for (size_t r = 0; r < key_samples[k].size(); r++) {
                if (key_samples[k][r].system != (size_t)si) continue;
                size_t a = key_samples[k][r].atom;
                long mc = acc.center_mapping[a];
                for (size_t x = 0; x < blk; x++) b.values[r * blk + x] += acc.values[l][(nti * NC + mc) * blk + x];
            }
            // position_gradients_to_metatensor (:426-525)
            if (opt.positions) {
                Block& g = b.gradients["positions"];
                size_t row = 0;
                double m1l = (l % 2 == 0) ? 1.0 : -1.0;
                for (size_t r = 0; r < key_samples[k].size(); r++) {
                    for (size_t j : key_grad_atoms[k][r]) {
                        if (key_samples[k][r].system == (size_t)si) {
                            size_t ci = key_samples[k][r].atom;
                            double* out = &g.values[row * 3 * blk];
                            if (ci == j) {
                                long mc = acc.center_mapping[ci];
                                const double* src = &acc.self_grad[l][(nti * NC + mc) * 3 * blk];
                                for (size_t x = 0; x < 3 * blk; x++) out[x] = src[x];
                            } else {
                                for (size_t pid : acc.pairs_for_grad.at({ci, j})) {
                                    const Pair& p = *acc.pairs[pid];
                                    double factor = (p.first == ci) ? 1.0 : -m1l;
                                    const double* src = &acc.pair_grad[l][pid * 3 * blk];
                                    for (size_t x = 0; x < 3 * blk; x++) out[x] += factor * src[x];
                                }
                            }
                        }
                        row++;
                    }
                }
            }
            // cell_strain_gradients_to_metatensor (:530-604)
            for (const char* name : {"cell", "strain"}) {
                bool want = std::string(name) == "cell" ? opt.cell : opt.strain;
                if (!want) continue;
                Block& g = b.gradients[name];
                const auto& src_all = std::string(name) == "cell" ? acc.cell_grad[l] : acc.strain_grad[l];
                for (size_t r = 0; r < key_samples[k].size(); r++) {
                    if (key_samples[k][r].system != (size_t)si) continue;
                    long mc = acc.center_mapping[key_samples[k][r].atom];
                    const double* src = &src_all[(nti * NC + mc) * 9 * blk];
                    double* out = &g.values[r * 9 * blk];
                    for (size_t x = 0; x < 9 * blk; x++) out[x] += src[x];
                }
            }
        }
    }
    return tm;
}

// ---------------------------------------------------------------------------
// Power spectrum calculator: power_spectrum.rs:410-780
// ---------------------------------------------------------------------------
static TensorMap power_spectrum(const Calculator& calc, std::vector<System>& systems, const Options& opt) {
    int lmax = calc.lmax;
    size_t nmax = calc.nmax;
    // keys.rs:110-157
    std::set<std::tuple<int32_t, int32_t, int32_t>> keyset;
    for (auto& s : systems) {
        for (size_t i = 0; i < s.n; i++) {
            auto nts = neighbor_types(s, i);
            for (int32_t a : nts)
                for (int32_t b : nts)
                    if (!(b < a)) keyset.insert({s.types[i], a, b});
        }
    }
    TensorMap tm;
    tm.keys.width = 3;
    std::vector<std::tuple<int32_t, int32_t, int32_t>> keys(keyset.begin(), keyset.end());
    for (auto& k : keys) tm.keys.add({std::get<0>(k), std::get<1>(k), std::get<2>(k)});

    size_t n_props = (size_t)(lmax + 1) * nmax * nmax;
    std::vector<std::vector<SampleRef>> key_samples(keys.size());
    std::vector<std::vector<std::pair<size_t, size_t>>> key_grad_rows(keys.size());  // (sample row, atom)
    for (size_t k = 0; k < keys.size(); k++) {
        int32_t ct, a, b;
        std::tie(ct, a, b) = keys[k];
        Block blk;
        blk.samples.width = 2;
        // AllOf{a, b}, atom_centered.rs:53-77
        for (size_t si = 0; si < systems.size(); si++) {
            auto& s = systems[si];
            for (size_t i = 0; i < s.n; i++) {
                if (s.types[i] != ct) continue;
                auto nts = neighbor_types(s, i);
                if (nts.count(a) && nts.count(b)) {
                    blk.samples.add({(int32_t)si, (int32_t)i});
                    key_samples[k].push_back({si, i});
                }
            }
        }
        std::vector<int32_t> grows;
        for (size_t r = 0; r < key_samples[k].size(); r++) {
            auto& ref = key_samples[k][r];
            for (size_t j : gradient_atoms(systems[ref.system], ref.atom, {a, b})) {
                grows.push_back((int32_t)r);
                grows.push_back((int32_t)ref.system);
                grows.push_back((int32_t)j);
                key_grad_rows[k].push_back({r, j});
            }
        }
        blk.properties.width = 3;
        for (int l = 0; l <= lmax; l++)
            for (size_t n1 = 0; n1 < nmax; n1++)
                for (size_t n2 = 0; n2 < nmax; n2++) blk.properties.add({l, (int32_t)n1, (int32_t)n2});
        blk.shape = {key_samples[k].size(), n_props};
        blk.values.assign(key_samples[k].size() * n_props, 0.0);
        add_gradient_blocks(blk, opt, grows, key_grad_rows[k].size(), {}, n_props);
        tm.blocks.push_back(std::move(blk));
    }

    // The spherical expansion restricted to the needed samples (selected_spx_labels,
    // :82-193).  Its samples for (ct, nt) are the union of the PS samples of
    // keys (ct, n1, n2) with nt in {n1, n2}; per system, the requested centres
    // are all the atoms of those samples.  Values, self / pair / strain / cell
    // gradients are accumulated exactly as spherical_expansion.rs does.
    auto self = calc.self_contribution();
    int nthreads = opt.se_over_centres ? 1 : opt.threads;
    std::vector<PairAccumulation> accs(systems.size());
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
    for (long si = 0; si < (long)systems.size(); si++) {
        std::set<size_t> requested;
        for (size_t k = 0; k < keys.size(); k++)
            for (auto& r : key_samples[k]) if (r.system == (size_t)si) requested.insert(r.atom);
        accs[si] = calc.accumulate_all_pairs(systems[si], opt, requested, opt.threads);
    }

    // SE value of (system, atom, type nt, l) into `out` [2l+1][n]; self term first
    auto spx_value = [&](size_t si, size_t atom, int32_t nt, int l, double* out) {
        size_t blk = (2 * l + 1) * nmax;
        const auto& acc = accs[si];
        auto it = acc.types_mapping.find(nt);
        long mc = acc.center_mapping[atom];
        for (size_t x = 0; x < blk; x++) out[x] = 0.0;
        if (l == 0 && systems[si].types[atom] == nt)
            for (size_t n = 0; n < nmax; n++) out[n] += self[n];
        if (it == acc.types_mapping.end()) return;
        const double* src = &acc.values[l][(it->second * acc.n_centers + mc) * blk];
        for (size_t x = 0; x < blk; x++) out[x] += src[x];
    };

    for (size_t k = 0; k < keys.size(); k++) {
        int32_t ct, a, b;
        std::tie(ct, a, b) = keys[k];
        (void)ct;
        Block& blk = tm.blocks[k];
        size_t NS = key_samples[k].size();
        // values, :584-618 (rayon over samples)
#pragma omp parallel for num_threads(opt.threads) schedule(static)
        for (long r = 0; r < (long)NS; r++) {
            auto ref = key_samples[k][r];
            std::vector<double> c1((2 * lmax + 1) * nmax), c2((2 * lmax + 1) * nmax);
            size_t p = 0;
            for (int l = 0; l <= lmax; l++) {
                spx_value(ref.system, ref.atom, a, l, c1.data());
                spx_value(ref.system, ref.atom, b, l, c2.data());
                double norm = (l % 2 == 0) ? std::sqrt((double)(2 * l + 1)) : -std::sqrt((double)(2 * l + 1));
                for (size_t n1 = 0; n1 < nmax; n1++)
                    for (size_t n2 = 0; n2 < nmax; n2++, p++) {
                        double sum = 0.0;
                        for (int m = 0; m < 2 * l + 1; m++) sum += c1[m * nmax + n1] * c2[m * nmax + n2];
                        if (a != b) sum *= SQRT_2;
                        blk.values[r * n_props + p] = sum / norm;
                    }
            }
        }

        // positions gradients, :621-678
        if (opt.positions) {
            Block& g = blk.gradients["positions"];
            const auto& rows = key_grad_rows[k];
#pragma omp parallel for num_threads(opt.threads) schedule(static)
            for (long row = 0; row < (long)rows.size(); row++) {
                size_t r = rows[row].first, j = rows[row].second;
                auto ref = key_samples[k][r];
                const auto& acc = accs[ref.system];
                const System& sys = systems[ref.system];
                size_t i = ref.atom;
                long mc = acc.center_mapping[i];
                int32_t tj = sys.types[j];
                // which spx gradient samples exist (samples_mapping, :266-298)
                bool has1 = (j == i) || tj == a;
                bool has2 = (j == i) || tj == b;
                std::vector<double> c1((2 * lmax + 1) * nmax), c2((2 * lmax + 1) * nmax);
                std::vector<double> d1(3 * (2 * lmax + 1) * nmax), d2(3 * (2 * lmax + 1) * nmax);
                // SE positions gradient of (i wrt j) for neighbour type t
                auto spx_grad = [&](int32_t t, int l, double* out) {
                    size_t blk3 = 3 * (2 * l + 1) * nmax;
                    for (size_t x = 0; x < blk3; x++) out[x] = 0.0;
                    auto it = acc.types_mapping.find(t);
                    if (it == acc.types_mapping.end()) return;
                    if (i == j) {
                        const double* src = &acc.self_grad[l][(it->second * acc.n_centers + mc) * blk3];
                        for (size_t x = 0; x < blk3; x++) out[x] = src[x];
                    } else {
                        double m1l = (l % 2 == 0) ? 1.0 : -1.0;
                        for (size_t pid : acc.pairs_for_grad.at({i, j})) {
                            const Pair& p = *acc.pairs[pid];
                            double factor = (p.first == i) ? 1.0 : -m1l;
                            const double* src = &acc.pair_grad[l][pid * blk3];
                            for (size_t x = 0; x < blk3; x++) out[x] += factor * src[x];
                        }
                    }
                };
                size_t p = 0;
                double* outrow = &g.values[row * 3 * n_props];
                for (int l = 0; l <= lmax; l++) {
                    size_t nm = 2 * l + 1;
                    spx_value(ref.system, i, a, l, c1.data());
                    spx_value(ref.system, i, b, l, c2.data());
                    if (has1) spx_grad(a, l, d1.data());
                    if (has2) spx_grad(b, l, d2.data());
                    double norm = (l % 2 == 0) ? std::sqrt((double)nm) : -std::sqrt((double)nm);
                    for (size_t n1 = 0; n1 < nmax; n1++)
                        for (size_t n2 = 0; n2 < nmax; n2++, p++) {
                            double sum[3] = {0.0, 0.0, 0.0};
                            if (has1)
                                for (size_t m = 0; m < nm; m++) {
                                    double v2 = c2[m * nmax + n2];
                                    for (int d = 0; d < 3; d++) sum[d] += v2 * d1[(d * nm + m) * nmax + n1];
                                }
                            if (has2)
                                for (size_t m = 0; m < nm; m++) {
                                    double v1 = c1[m * nmax + n1];
                                    for (int d = 0; d < 3; d++) sum[d] += v1 * d2[(d * nm + m) * nmax + n2];
                                }
                            if (a != b) for (int d = 0; d < 3; d++) sum[d] *= SQRT_2;
                            for (int d = 0; d < 3; d++) outrow[d * n_props + p] = sum[d] / norm;
                        }
                }
            }
        }

        // cell / strain gradients, :681-760
        for (const char* name : {"cell", "strain"}) {
            bool want = std::string(name) == "cell" ? opt.cell : opt.strain;
            if (!want) continue;
            Block& g = blk.gradients[name];
            bool is_cell = std::string(name) == "cell";
#pragma omp parallel for num_threads(opt.threads) schedule(static)
            for (long r = 0; r < (long)NS; r++) {
                auto ref = key_samples[k][r];
                const auto& acc = accs[ref.system];
                long mc = acc.center_mapping[ref.atom];
                std::vector<double> c1((2 * lmax + 1) * nmax), c2((2 * lmax + 1) * nmax);
                std::vector<double> zero(9 * (2 * lmax + 1) * nmax, 0.0);
                size_t p = 0;
                double* outrow = &g.values[r * 9 * n_props];
                for (int l = 0; l <= lmax; l++) {
                    size_t nm = 2 * l + 1, blk9 = 9 * nm * nmax;
                    spx_value(ref.system, ref.atom, a, l, c1.data());
                    spx_value(ref.system, ref.atom, b, l, c2.data());
                    auto src_of = [&](int32_t t) -> const double* {
                        auto it = acc.types_mapping.find(t);
                        if (it == acc.types_mapping.end()) return zero.data();
                        const auto& all = is_cell ? acc.cell_grad[l] : acc.strain_grad[l];
                        return &all[(it->second * acc.n_centers + mc) * blk9];
                    };
                    const double* g1 = src_of(a);
                    const double* g2 = src_of(b);
                    double norm = (l % 2 == 0) ? std::sqrt((double)nm) : -std::sqrt((double)nm);
                    for (size_t n1 = 0; n1 < nmax; n1++)
                        for (size_t n2 = 0; n2 < nmax; n2++, p++) {
                            double sum[9] = {0};
                            for (size_t m = 0; m < nm; m++) {
                                double v2 = c2[m * nmax + n2];
                                for (int x = 0; x < 9; x++) sum[x] += v2 * g1[(x * nm + m) * nmax + n1];
                            }
                            for (size_t m = 0; m < nm; m++) {
                                double v1 = c1[m * nmax + n1];
                                for (int x = 0; x < 9; x++) sum[x] += v1 * g2[(x * nm + m) * nmax + n2];
                            }
                            if (a != b) for (int x = 0; x < 9; x++) sum[x] *= SQRT_2;
                            for (int x = 0; x < 9; x++) outrow[x * n_props + p] = sum[x] / norm;
                        }
                }
            }
        }
    }
    return tm;
}

}  // namespace oracle

// ===========================================================================
// C API used by the Python test harness (ctypes)
// ===========================================================================
using namespace oracle;

// ---------------------------------------------------------------------------
// Spherical expansion by pair: spherical_expansion_pair.rs:547-822 with the
// samples of FullNeighborList (calculators/neighbor_list.rs:372-490)
// ---------------------------------------------------------------------------
static TensorMap spherical_expansion_by_pair(const Calculator& calc, std::vector<System>& systems, const Options& opt) {
    const int lmax = calc.lmax;
    const size_t nmax = calc.nmax;
    // keys: every (first type, second type) of a pair in both orders, and
    // (t, t) for every type present (neighbor_list.rs:374-400); l inner
    std::set<std::pair<int32_t, int32_t>> tp;
    for (auto& s : systems) {
        for (const auto& p : s.nl.pairs) {
            tp.insert({s.types[p.first], s.types[p.second]});
            tp.insert({s.types[p.second], s.types[p.first]});
        }
        for (size_t i = 0; i < s.n; i++) tp.insert({s.types[i], s.types[i]});
    }
    TensorMap tm;
    tm.keys.width = 4;
    std::map<std::pair<int32_t, int32_t>, size_t> first_block;
    for (auto& t : tp) {
        first_block[t] = tm.blocks.size();
        for (int l = 0; l <= lmax; l++) {
            tm.keys.add({l, 1, t.first, t.second});
            tm.blocks.emplace_back();
        }
    }
    // samples (neighbor_list.rs:403-490): pairs of each system in pair order
    // (both directions when the types are equal), then that system's self
    // pairs; l = 0 keeps the self pairs, l > 0 does not
    using Sample = std::array<int32_t, 6>;
    std::map<std::pair<int32_t, int32_t>, std::vector<Sample>> samples0, samples1;
    for (size_t si = 0; si < systems.size(); si++) {
        const System& s = systems[si];
        for (auto& t : tp) {
            auto& s0 = samples0[t];
            auto& s1 = samples1[t];
            for (const auto& p : s.nl.pairs) {
                const int32_t a = s.types[p.first], b = s.types[p.second];
                const Sample fwd = {(int32_t)si, (int32_t)p.first, (int32_t)p.second, p.shift[0], p.shift[1], p.shift[2]};
                const Sample inv = {(int32_t)si, (int32_t)p.second, (int32_t)p.first, -p.shift[0], -p.shift[1], -p.shift[2]};
                if (t.first == t.second) {
                    if (a == t.first && b == t.second) {
                        s0.push_back(fwd);
                        s1.push_back(fwd);
                        s0.push_back(inv);
                        s1.push_back(inv);
                    }
                } else if (a == t.first && b == t.second) {
                    s0.push_back(fwd);
                    s1.push_back(fwd);
                } else if (b == t.first && a == t.second) {
                    s0.push_back(inv);
                    s1.push_back(inv);
                }
            }
            if (t.first == t.second)
                for (size_t i = 0; i < s.n; i++)
                    if (s.types[i] == t.first) s0.push_back({(int32_t)si, (int32_t)i, (int32_t)i, 0, 0, 0});
        }
    }
    // blocks, with the positions gradient samples of
    // spherical_expansion_pair.rs:647-667 (self pairs have none; i == j
    // images have one row)
    std::vector<std::map<Sample, size_t>> row_of(tm.blocks.size());
    std::vector<std::vector<size_t>> grad_row_of(tm.blocks.size());  // first positions row of each sample
    for (auto& t : tp) {
        for (int l = 0; l <= lmax; l++) {
            const size_t bi = first_block[t] + l;
            Block& b = tm.blocks[bi];
            const auto& list = l == 0 ? samples0[t] : samples1[t];
            b.samples.width = 6;
            for (size_t k = 0; k < list.size(); k++) {
                const Sample& x = list[k];
                b.samples.add({x[0], x[1], x[2], x[3], x[4], x[5]});
                row_of[bi][x] = k;
            }
            b.properties.width = 1;
            for (size_t n = 0; n < nmax; n++) b.properties.add({(int32_t)n});
            const size_t nm = 2 * l + 1;
            b.components = {nm};
            b.shape = {list.size(), nm, nmax};
            b.values.assign(list.size() * nm * nmax, 0.0);
            std::vector<int32_t> grad_rows;
            size_t n_grad = 0;
            grad_row_of[bi].assign(list.size(), SIZE_MAX);
            for (size_t k = 0; k < list.size(); k++) {
                const Sample& x = list[k];
                if (x[1] == x[2] && x[3] == 0 && x[4] == 0 && x[5] == 0) continue;
                grad_row_of[bi][k] = n_grad;
                grad_rows.insert(grad_rows.end(), {(int32_t)k, x[0], x[1]});
                n_grad++;
                if (x[1] != x[2]) {
                    grad_rows.insert(grad_rows.end(), {(int32_t)k, x[0], x[2]});
                    n_grad++;
                }
            }
            add_gradient_blocks(b, opt, grad_rows, n_grad, {nm}, nmax);
        }
    }
    // self contributions on l = 0 (spherical_expansion_pair.rs:259-313)
    const std::vector<double> self = calc.self_contribution();
    for (auto& t : tp) {
        if (t.first != t.second) continue;
        Block& b = tm.blocks[first_block[t]];
        for (size_t k = 0; k < b.samples.count(); k++) {
            const int32_t* x = &b.samples.values[6 * k];
            if (x[1] == x[2] && x[3] == 0 && x[4] == 0 && x[5] == 0)
                for (size_t n = 0; n < nmax; n++) b.values[k * nmax + n] = self[n];
        }
    }
    // pair contributions (spherical_expansion_pair.rs:731-822,
    // accumulate_in_block :424-540)
    const bool do_grad = opt.positions || opt.strain || opt.cell;
    SphericalHarmonics sph(lmax);
    const size_t L2 = (size_t)((lmax + 1) * (lmax + 1));
    std::vector<double> Y(L2), GX(L2), GY(L2), GZ(L2), R((lmax + 1) * nmax), dR((lmax + 1) * nmax);
    std::vector<std::vector<double>> vals(lmax + 1), grads(lmax + 1);
    for (int l = 0; l <= lmax; l++) {
        vals[l].assign((2 * l + 1) * nmax, 0.0);
        grads[l].assign(3 * (2 * l + 1) * nmax, 0.0);
    }
    auto accumulate = [&](int l, size_t bi, const Sample& sample, const double* v, const double* g,
                          const double vector[3]) {
        Block& b = tm.blocks[bi];
        const size_t k = row_of[bi].at(sample);
        const size_t blk = (2 * l + 1) * nmax;
        for (size_t q = 0; q < blk; q++) b.values[k * blk + q] += v[q];
        if (!do_grad) return;
        if (opt.positions) {
            Block& gb = b.gradients.at("positions");
            // rows (k, system, first) and (k, system, second): the same row
            // when first == second
            const size_t first_row = grad_row_of[bi][k];
            const size_t second_row = sample[1] == sample[2] ? first_row : first_row + 1;
            for (size_t q = 0; q < 3 * blk; q++) gb.values[first_row * 3 * blk + q] -= g[q];
            for (size_t q = 0; q < 3 * blk; q++) gb.values[second_row * 3 * blk + q] += g[q];
        }
        if (opt.strain) {
            Block& gb = b.gradients.at("strain");
            for (int x1 = 0; x1 < 3; x1++)
                for (int x2 = 0; x2 < 3; x2++)
                    for (size_t q = 0; q < blk; q++)
                        gb.values[((k * 3 + x1) * 3 + x2) * blk + q] += vector[x1] * g[x2 * blk + q];
        }
        if (opt.cell) {
            Block& gb = b.gradients.at("cell");
            const double shifts[3] = {(double)sample[3], (double)sample[4], (double)sample[5]};
            for (int abc = 0; abc < 3; abc++)
                for (int xyz = 0; xyz < 3; xyz++)
                    for (size_t q = 0; q < blk; q++)
                        gb.values[((k * 3 + abc) * 3 + xyz) * blk + q] += shifts[abc] * g[xyz * blk + q];
        }
    };
    for (size_t si = 0; si < systems.size(); si++) {
        const System& s = systems[si];
        for (const auto& p : s.nl.pairs) {
            double dir[3] = {p.vector[0] / p.distance, p.vector[1] / p.distance, p.vector[2] / p.distance};
            calc.compute_for_pair(sph, p.distance, dir, do_grad, vals, grads, Y, GX, GY, GZ, R, dR);
            const int32_t a = s.types[p.first], b = s.types[p.second];
            const Sample fwd = {(int32_t)si, (int32_t)p.first, (int32_t)p.second, p.shift[0], p.shift[1], p.shift[2]};
            const Sample inv = {(int32_t)si, (int32_t)p.second, (int32_t)p.first, -p.shift[0], -p.shift[1], -p.shift[2]};
            const double vfwd[3] = {p.vector[0], p.vector[1], p.vector[2]};
            const double vinv[3] = {-p.vector[0], -p.vector[1], -p.vector[2]};
            for (int l = 0; l <= lmax; l++)
                accumulate(l, first_block[{a, b}] + l, fwd, vals[l].data(), grads[l].data(), vfwd);
            // PairContribution::inverse_pair (:130-163): values x (-1)^l,
            // gradients x -(-1)^l
            for (int l = 0; l <= lmax; l++) {
                const double m1 = (l % 2 == 0) ? 1.0 : -1.0;
                for (auto& v : vals[l]) v *= m1;
                for (auto& g : grads[l]) g *= -m1;
                accumulate(l, first_block[{b, a}] + l, inv, vals[l].data(), grads[l].data(), vinv);
            }
        }
    }
    return tm;
}

static thread_local std::string LAST_ERROR;

struct oracle_result {
    TensorMap tm;
};

struct oracle_nl {
    std::vector<Pair> pairs;
};

extern "C" {

const char* oracle_last_error(void) { return LAST_ERROR.c_str(); }

double oracle_gamma(double x) { return oracle::gamma(x); }
double oracle_ln_gamma(double x) { return oracle::ln_gamma(x); }

int oracle_hyp1f1(double a, double b, double x, double* out) {
    try { *out = oracle::hyp1f1(a, b, x); return 0; }
    catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

int oracle_cutoff(const oracle_hypers* h, double r, double* value, double* gradient) {
    *value = smoothing(*h, r);
    *gradient = smoothing_gradient(*h, r);
    return 0;
}

// values / gradients: (lmax+1)^2 each, index l*l + l + m
int oracle_spherical_harmonics(int32_t lmax, const double* direction, double* values, double* gx, double* gy, double* gz) {
    try {
        SphericalHarmonics sph(lmax);
        sph.compute(direction, values, gx, gy, gz);
        return 0;
    } catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

// radial integral for all l at one distance: values / grads [(lmax+1) * (nmax+1)]
int oracle_radial_integral(const oracle_hypers* h, int32_t n_r, const double* r, double* values, double* grads) {
    try {
        RadialIntegrals ri(*h);
        size_t N = (size_t)h->max_radial + 1;
        for (int k = 0; k < n_r; k++)
            for (int l = 0; l <= h->max_angular; l++)
                ri.compute(l, r[k], &values[((size_t)k * (h->max_angular + 1) + l) * N],
                           grads ? &grads[((size_t)k * (h->max_angular + 1) + l) * N] : nullptr);
        return 0;
    } catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

// number of spline knots per l (0 when analytic)
int oracle_spline_sizes(const oracle_hypers* h, int32_t* sizes) {
    try {
        RadialIntegrals ri(*h);
        for (int l = 0; l <= h->max_angular; l++) sizes[l] = ri.splined ? (int32_t)ri.splines[l].positions.size() : 0;
        return 0;
    } catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

// orthonormalization matrix M[k][n] of the GTO basis
int oracle_gto_orthonormalization(int32_t size, double radius, double* out) {
    try {
        Matrix M = gto_orthonormalization((size_t)size, radius);
        std::copy(M.d.begin(), M.d.end(), out);
        return 0;
    } catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

int oracle_neighbors(const double* positions, uint64_t n_atoms, const double* cell, double cutoff, oracle_nl** out, uint64_t* n_pairs) {
    try {
        UnitCell c = make_cell(cell);
        auto nl = build_neighbors(positions, n_atoms, c, cutoff);
        *out = new oracle_nl{nl.pairs};
        *n_pairs = nl.pairs.size();
        return 0;
    } catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

// first/second as int64, distance, vector[3], shift[3]
void oracle_neighbors_get(const oracle_nl* nl, int64_t* pairs, double* distances, double* vectors, int32_t* shifts) {
    for (size_t k = 0; k < nl->pairs.size(); k++) {
        const Pair& p = nl->pairs[k];
        pairs[2 * k] = (int64_t)p.first;
        pairs[2 * k + 1] = (int64_t)p.second;
        distances[k] = p.distance;
        for (int x = 0; x < 3; x++) {
            vectors[3 * k + x] = p.vector[x];
            shifts[3 * k + x] = p.shift[x];
        }
    }
}

void oracle_neighbors_free(oracle_nl* nl) { delete nl; }

// calculator: 0 = spherical_expansion, 1 = soap_power_spectrum
int oracle_compute(int32_t calculator, const oracle_hypers* h, const oracle_system* systems, uint64_t n_systems,
                   int32_t grad_positions, int32_t grad_strain, int32_t grad_cell, int32_t threads,
                   int32_t se_over_centres, oracle_result** out) {
    try {
        Calculator calc(*h);
        std::vector<System> sys(n_systems);
        for (size_t s = 0; s < n_systems; s++) {
            sys[s].n = systems[s].n_atoms;
            sys[s].types = systems[s].types;
            sys[s].positions = systems[s].positions;
            sys[s].cell = make_cell(systems[s].cell);
            sys[s].nl = build_neighbors(sys[s].positions, sys[s].n, sys[s].cell, h->cutoff);
        }
        Options opt;
        opt.positions = grad_positions != 0;
        opt.strain = grad_strain != 0;
        opt.cell = grad_cell != 0;
        opt.threads = threads < 1 ? 1 : threads;
        opt.se_over_centres = se_over_centres != 0;
        auto* r = new oracle_result;
        if (calculator == 0) r->tm = spherical_expansion(calc, sys, opt);
        else if (calculator == 1) r->tm = power_spectrum(calc, sys, opt);
        else r->tm = spherical_expansion_by_pair(calc, sys, opt);
        *out = r;
        return 0;
    } catch (std::exception& e) { LAST_ERROR = e.what(); return 1; }
}

void oracle_result_free(oracle_result* r) { delete r; }

uint64_t oracle_result_n_blocks(const oracle_result* r) { return r->tm.blocks.size(); }

void oracle_result_keys(const oracle_result* r, const int32_t** values, uint64_t* count, uint64_t* width) {
    *values = r->tm.keys.values.data();
    *count = r->tm.keys.count();
    *width = r->tm.keys.width;
}

static const Block* select_block(const oracle_result* r, uint64_t b, const char* gradient) {
    const Block* blk = &r->tm.blocks[b];
    if (gradient && gradient[0]) {
        auto it = blk->gradients.find(gradient);
        if (it == blk->gradients.end()) return nullptr;
        blk = &it->second;
    }
    return blk;
}

// axis 0 = samples, 1 = properties
int oracle_block_labels(const oracle_result* r, uint64_t b, const char* gradient, int32_t axis,
                        const int32_t** values, uint64_t* count, uint64_t* width) {
    const Block* blk = select_block(r, b, gradient);
    if (!blk) return 1;
    const Labels& l = axis == 0 ? blk->samples : blk->properties;
    *values = l.values.data();
    *count = l.count();
    *width = l.width;
    return 0;
}

int oracle_block_values(const oracle_result* r, uint64_t b, const char* gradient, const double** data,
                        const uint64_t** shape, uint64_t* ndim) {
    const Block* blk = select_block(r, b, gradient);
    if (!blk) return 1;
    *data = blk->values.data();
    static thread_local std::vector<uint64_t> sh;
    sh.assign(blk->shape.begin(), blk->shape.end());
    *shape = sh.data();
    *ndim = sh.size();
    return 0;
}

}  // extern "C"

// Scalar math of the SOAP path, compiled for both the host (spline knot
// construction) and the device (analytic radial integral, per-pair
// features).  Everything is FP64.
//
// * confluent hypergeometric 1F1 and the GTO radial integral follow
//   featomic/src/math/hyp1f1.rs:17-255 and
//   featomic/src/calculators/soap/radial_integral/gto.rs:82-205 (scipy's CHGM
//   with a 30-term asymptotic sum);
// * the Hermite spline evaluation follows featomic/src/math/splines.rs:225-289;
// * the cutoff functions follow featomic/src/calculators/soap/cutoff.rs:48-79;
// * the Willatt2018 radial scaling follows
//   featomic/src/calculators/shared/density.rs:108-128.
//
// Gamma functions use the Lanczos approximation below (host and device).
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define SOAP_HD __host__ __device__ __forceinline__
#else
#define SOAP_HD inline
#endif

namespace soap {

#ifndef __CUDA_ARCH__
using std::isfinite;
#endif

constexpr double PI = 3.14159265358979323846;
constexpr double DBL_EPS = 2.220446049250313e-16;

// Gamma and log-Gamma by the Lanczos approximation with g = 10.900511 and the
// 11-term coefficient table of G. R. Pugh, "An Analysis of the Lanczos Gamma
// Approximation" (2004), p. 116 -- the approximation featomic uses
// (featomic/src/math/gamma.rs:20-92).  The GTO overlap matrix is
// ill-conditioned (condition number 3e4 at 8 radial functions, 4e7 at 12), so
// its inverse square root, and every radial integral after it, moves by
// cond * (relative change of the Gamma values): the same Gamma is needed to
// agree with featomic to 1e-10.
SOAP_HD double lanczos_series(double x, bool reflected) {
    const double dk[11] = {
        2.4857408913875355e-5, 1.0514237858172197, -3.4568709722201625, 4.512277094668948,
        -2.9828522532357664, 1.056397115771267, -1.9542877319164587e-1, 1.709705434044412e-2,
        -5.719261174043057e-4, 4.633994733599057e-6, -2.7199490848860772e-9,
    };
    double s = dk[0];
    for (int t = 1; t < 11; t++) s = s + dk[t] / (reflected ? ((double)t - x) : (x + (double)t - 1.0));
    return s;
}

SOAP_HD double gamma_fn(double x) {
    const double two_sqrt_e_over_pi = 1.8603827342052657;
    const double r = 10.900511;
    const double e = 2.718281828459045;
    if (x < 0.5) {
        double s = lanczos_series(x, true);
        return PI / (sin(PI * x) * s * two_sqrt_e_over_pi * pow((0.5 - x + r) / e, 0.5 - x));
    }
    double s = lanczos_series(x, false);
    return s * two_sqrt_e_over_pi * pow((x - 0.5 + r) / e, x - 0.5);
}

SOAP_HD double ln_gamma_fn(double x) {
    const double ln_pi = 1.1447298858494002;
    const double ln_2_sqrt_e_over_pi = 0.6207822376352452;
    const double r = 10.900511;
    const double e = 2.718281828459045;
    if (x < 0.5) {
        double s = lanczos_series(x, true);
        return ln_pi - log(sin(PI * x)) - log(s) - ln_2_sqrt_e_over_pi - (0.5 - x) * log((0.5 - x + r) / e);
    }
    double s = lanczos_series(x, false);
    return log(s) + ln_2_sqrt_e_over_pi + (x - 0.5) * log((x - 0.5 + r) / e);
}

// b^n by repeated squaring (the lowering of f64::powi)
SOAP_HD double powi(double a, int b) {
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

// plain power series, converging geometrically when (|a|+1)|x| < 0.9 b
SOAP_HD double hyp1f1_series(double a, double b, double x) {
    double term = 1.0, result = 1.0;
    for (int k = 0; k < 1000; k++) {
        double kf = (double)k;
        term *= (a + kf) * x / (b + kf) / (kf + 1.0);
        result += term;
        if (fabs(term) <= DBL_EPS * fabs(result)) return result;
    }
    return NAN;
}

// series for a non-positive integer a, monitoring cancellation
SOAP_HD double hyp1f1_series_tracked(double a, double b, double x) {
    double term = 1.0, result = 1.0, abssum = 1.0, steps = -1.0;
    for (int k = 0; k < 1000; k++) {
        double kf = (double)k;
        double apk = a + kf, bpk = b + kf;
        if (bpk != 0.0) term *= apk * x / bpk / (kf + 1.0);
        else if (apk == 0.0) term = 0.0;
        else return NAN;
        abssum += fabs(term);
        result += term;
        if (fabs(term) <= DBL_EPS * fabs(result)) {
            steps = kf;
            break;
        }
    }
    if (steps < 0.0) return NAN;
    if (steps * DBL_EPS * abssum <= 1e-9 * fabs(result)) return result;
    return NAN;
}

// Kummer transformation + recurrence in a (DLMF 13.2.39, 13.3.1), with the
// series (13.2.2) for moderate x, the large-x expansion (13.7.1) and the
// two-sided asymptotic sums (13.7.2) truncated at 30 terms.
SOAP_HD double hyp1f1_chgm(double a, double b, double x) {
    double a0 = a, x0 = x, result = 0.0;
    if (x < 0.0) {
        a = b - a;
        a0 = a;
        x = fabs(x);
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
        if (x <= fabs(b) + 30.0 || a < 0.0) {
            result = 1.0;
            double term = 1.0;
            if (x < 500.0) {
                for (int j = 1; j <= 500; j++) {
                    double jf = (double)j;
                    term *= (a + jf - 1.0) / (jf * (b + jf - 1.0)) * x;
                    result += term;
                    if (result != 0.0 && fabs(term / result) < 1e-15) break;
                }
                if (x0 < 0.0) result *= exp(x0);
            } else {
                for (int j = 1; j <= 50; j++) {
                    double jf = (double)j;
                    term *= (jf - a) * (b - a + jf - 1.0) / (jf * x);
                    result += term;
                    if (result != 0.0 && fabs(term / result) < 1e-15) break;
                }
                result *= pow(x, a - b) * gamma_fn(b) / gamma_fn(a);
                if (x0 > 0.0) result *= exp(x);
            }
        } else {
            double lga = ln_gamma_fn(a), lgb = ln_gamma_fn(b), lgba = ln_gamma_fn(b - a);
            double s1 = 1.0, s2 = 1.0, t1 = 1.0, t2 = 1.0;
            for (int i = 1; i <= 30; i++) {
                double fi = (double)i;
                t1 = -t1 * (a + fi - 1.0) * (a - b + fi) / (x * fi);
                t2 = -t2 * (b - a + fi - 1.0) * (a - fi) / (x * fi);
                s1 += t1;
                s2 += t2;
            }
            double h1, h2;
            if (x0 >= 0.0) {
                h1 = exp(lgb - lgba) * pow(x, -a) * cos(PI * a) * s1;
                h2 = exp(lgb - lga + x) * pow(x, a - b) * s2;
            } else {
                h1 = exp(lgb - lgba + x0) * pow(x, -a) * cos(PI * a) * s1;
                h2 = exp(lgb - lga) * pow(x, a - b) * s2;
            }
            result = h1 + h2;
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

SOAP_HD double hyp1f1(double a, double b, double x) {
    if (a == 0.0 || x == 0.0) return 1.0;
    if (a == -1.0) return 1.0 - x / b;
    if (a == b) return exp(x);
    if (a - b == 1.0) return (1.0 + x / b) * exp(x);
    if (a <= 0.0 && a == floor(a)) return hyp1f1_series_tracked(a, b, x);
    if (b > 0.0 && (fabs(a) + 1.0) * fabs(x) < 0.9 * b) return hyp1f1_series(a, b, x);
    return hyp1f1_chgm(a, b, x);
}

// Raw (non-orthonormalised) GTO radial integral for one l and all n at
// distance r.  `bn[n]` = 1/(2 sigma_n^2), `c` = 1/(2 sigma^2),
// `width2` = sigma^2.  Writes values (and derivatives when `grad` != null).
// Returns false when a value is not finite.
SOAP_HD bool gto_radial_raw(int l, int nmax, double r, double c, double width2, const double* bn,
                            double* val, double* grad) {
    double global = pow(PI / width2, 0.75);
    double c_rij = c * r;
    double factor = global * exp(-r * c_rij) * powi(c_rij, l);
    bool ok = true;
    for (int n = 0; n < nmax; n++) {
        double z = c_rij * c_rij / (c + bn[n]);
        double a = 0.5 * (double)(n + l + 3), b = (double)l + 1.5;
        double ratio = gamma_fn(a) / gamma_fn(b);
        double v = ratio * hyp1f1(a, b, z);
        if (!isfinite(v)) ok = false;
        double c_dn = pow(c + bn[n], -(0.5 * (double)(n + l) + 1.5));
        v *= c_dn * factor;
        val[n] = v;
        if (grad) {
            double g = ratio * (a / b * hyp1f1(a + 1.0, b + 1.0, z));
            g *= c_dn * factor * 2.0 * z / r;
            g += v * ((double)l / r - 2.0 * c_rij);
            grad[n] = g;
        }
    }
    if (r == 0.0 && grad) {
        // analytic limit at r = 0: only l = 1 has a non-zero slope
        for (int n = 0; n < nmax; n++) {
            if (l == 1) {
                double a = 0.5 * (double)(n + l) + 1.5;
                double c_dn = pow(c + bn[n], -a);
                grad[n] = gamma_fn(a) / gamma_fn(2.5) * (global * c * c_dn);
            } else {
                grad[n] = 0.0;
            }
        }
    }
    return ok;
}

// ShiftedCosine (type 0) or Step (type 1) smoothing and its derivative
SOAP_HD void cutoff_function(int type, double rc, double width, double r, double* f, double* df) {
    if (type == 1) {
        *f = r >= rc ? 0.0 : 1.0;
        *df = 0.0;
        return;
    }
    if (r <= rc - width) {
        *f = 1.0;
        *df = 0.0;
    } else if (r >= rc) {
        *f = 0.0;
        *df = 0.0;
    } else {
        double s = PI * (r - rc + width) / width;
        *f = 0.5 * (1. + cos(s));
        *df = -0.5 * PI * sin(s) / width;
    }
}

// rate / (rate + (r/scale)^exponent) and its derivative
SOAP_HD void willatt2018(double scale, double rate, double exponent, double r, double* s, double* ds) {
    *s = rate / (rate + pow(r / scale, exponent));
    double rs = r / scale;
    double rs_m1 = pow(rs, exponent - 1.0);
    double rs_m = rs * rs_m1;
    double factor = -rate * exponent / scale;
    *ds = factor * rs_m1 / ((rate + rs_m) * (rate + rs_m));
}

// index of the spline interval containing x: largest k with pos[k] <= x,
// capped at count - 2 (evaluating at the last knot uses the last interval)
SOAP_HD int spline_interval(const double* pos, int count, double x) {
    int lo = 0, hi = count;
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (pos[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    int k = lo == 0 ? 0 : lo - 1;
    if (k >= count - 1) k = count - 2;
    return k;
}

struct HermiteWeights {
    double delta, h00, h10, h01, h11, d00, d10, d01, d11, dxdt;
};

SOAP_HD HermiteWeights hermite_weights(double xk, double xk1, double x) {
    HermiteWeights w;
    w.delta = xk1 - xk;
    double t = (x - xk) / w.delta;
    double t2 = t * t, t3 = t2 * t;
    w.h00 = 2.0 * t3 - 3.0 * t2 + 1.0;
    w.h10 = t3 - 2.0 * t2 + t;
    w.h01 = -2.0 * t3 + 3.0 * t2;
    w.h11 = t3 - t2;
    w.d00 = 6.0 * (t2 - t);
    w.d10 = 3.0 * t2 - 4.0 * t + 1.0;
    w.d01 = -w.d00;
    w.d11 = 3.0 * t2 - 2.0 * t;
    w.dxdt = 1.0 / w.delta;
    return w;
}

SOAP_HD double hermite_value(const HermiteWeights& w, double pk, double mk, double pk1, double mk1) {
    return w.h00 * pk + w.h10 * w.delta * mk + w.h01 * pk1 + w.h11 * w.delta * mk1;
}

SOAP_HD double hermite_derivative(const HermiteWeights& w, double pk, double mk, double pk1, double mk1) {
    return w.d00 * pk * w.dxdt + w.d10 * mk + w.d01 * pk1 * w.dxdt + w.d11 * mk1;
}

}  // namespace soap

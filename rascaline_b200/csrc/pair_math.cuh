// Per-pair device math shared by the FP64 drop-in kernels and the dense
// (values + adjoint) kernels: real spherical harmonics and their gradients,
// and the radial integral from the spline tables or analytically.
#pragma once

#include "engine.hpp"
#include "soap_math.cuh"

namespace fb200 {

template <typename T, int LCAP>
struct LegendreScratch {
    static constexpr int N = (LCAP + 1) * (LCAP + 2) / 2;
    T P[N], dP[N], Pot[N];
};

__device__ __forceinline__ int lidx(int l, int m) { return m + l * (l + 1) / 2; }

// Real spherical harmonics without the Condon-Shortley phase, and their
// gradients w.r.t. the unit direction (featomic/src/math/
// spherical_harmonics.rs:228-424), evaluated in T.  Y, GX, GY, GZ hold
// (lmax + 1)^2 entries indexed l^2 + l + m; GX == nullptr skips gradients.
template <typename T, int LCAP>
__device__ void ylm_compute(const DeviceYlmT<T>& tab, T ux, T uy, T uz, T* __restrict__ Y, T* __restrict__ GX,
                            T* __restrict__ GY, T* __restrict__ GZ) {
    LegendreScratch<T, LCAP> s;
    const int lmax = tab.lmax;
    const T SQRT_1_OVER_2PI = T(0.3989422804014327);
    const T SQRT_3 = T(1.7320508075688772);
    const T SQRT_3_OVER_2 = T(1.224744871391589);
    const T SQRT_2 = T(1.4142135623730951);

    T sxy = hypot(ux, uy);
    T ct = uz, st = sxy;
    T cp, sp;
    if (sxy > T(soap::DBL_EPS)) {
        cp = ux / sxy;
        sp = uy / sxy;
    } else {
        cp = T(1);
        sp = T(0);
    }
    // associated Legendre polynomials (:228-251)
    T value = SQRT_1_OVER_2PI;
    s.P[0] = value;
    if (lmax > 0) {
        s.P[lidx(1, 0)] = ct * SQRT_3 * value;
        value *= -SQRT_3_OVER_2 * st;
        s.P[lidx(1, 1)] = value;
        for (int l = 2; l <= lmax; l++) {
            for (int m = 0; m < l - 1; m++)
                s.P[lidx(l, m)] =
                    tab.A[lidx(l, m)] * (ct * s.P[lidx(l - 1, m)] + tab.B[lidx(l, m)] * s.P[lidx(l - 2, m)]);
            s.P[lidx(l, l - 1)] = ct * tab.sq_2l1[l] * value;
            value *= -tab.sq_half[l] * st;
            s.P[lidx(l, l)] = value;
        }
    }
    const bool grad = GX != nullptr;
    if (grad) {
        // derivative factors (:256-298)
        s.dP[0] = T(0);
        for (int l = 1; l <= lmax; l++) {
            T pm1 = tab.inv_ll[l] * s.P[lidx(l, 1)];
            T pp1 = s.P[lidx(l, 1)];
            s.dP[lidx(l, 0)] = tab.sq_plus[lidx(l, 0)] * pm1 - tab.sq_minus[lidx(l, 0)] * pp1;
            for (int m = 1; m < l; m++)
                s.dP[lidx(l, m)] =
                    tab.sq_plus[lidx(l, m)] * s.P[lidx(l, m - 1)] - tab.sq_minus[lidx(l, m)] * s.P[lidx(l, m + 1)];
            s.dP[lidx(l, l)] = tab.sq_plus[lidx(l, l)] * s.P[lidx(l, l - 1)] - tab.sq_minus[lidx(l, l)] * T(0);
        }
        if (st > T(0.1)) {
            for (int l = 0; l <= lmax; l++)
                for (int m = 0; m <= l; m++) s.Pot[lidx(l, m)] = (T)m / st * s.P[lidx(l, m)];
        } else {
            for (int l = 0; l <= lmax; l++)
                for (int m = 0; m <= l; m++) s.Pot[lidx(l, m)] = T(-0.5) / ct * s.dP[lidx(l, m)];
        }
    }
    for (int l = 0; l <= lmax; l++) Y[l * l + l] = s.P[lidx(l, 0)] / SQRT_2;
    if (grad) {
        GX[0] = T(0);
        GY[0] = T(0);
        GZ[0] = T(0);
        for (int l = 1; l <= lmax; l++) {
            T lf = tab.sq_ll1[l] * s.P[lidx(l, 1)];
            GX[l * l + l] = cp * ct * lf;
            GY[l * l + l] = sp * ct * lf;
            GZ[l * l + l] = -st * lf;
        }
    }
    T cos1 = T(1), sin1 = T(0), cos2 = -cp, sin2 = sp;
    T m2c = T(-2) * cp;
    for (int m = 1; m <= lmax; m++) {
        T smp = m2c * sin1 - sin2;
        T cmp = m2c * cos1 - cos2;
        sin2 = sin1;
        sin1 = smp;
        cos2 = cos1;
        cos1 = cmp;
        for (int l = m; l <= lmax; l++) {
            T p = s.P[lidx(l, m)];
            Y[l * l + l + m] = p * cmp;
            Y[l * l + l - m] = p * smp;
        }
        if (grad) {
            for (int l = m; l <= lmax; l++) {
                T dp = s.dP[lidx(l, m)];
                T sdp = smp * dp, cdp = cmp * dp;
                T pot = s.Pot[lidx(l, m)];
                GX[l * l + l + m] = sp * pot * smp - T(0.5) * ct * cp * cdp;
                GX[l * l + l - m] = -sp * pot * cmp - T(0.5) * ct * cp * sdp;
                GY[l * l + l + m] = -cp * pot * smp - T(0.5) * ct * sp * cdp;
                GY[l * l + l - m] = cp * pot * cmp - T(0.5) * ct * sp * sdp;
                GZ[l * l + l + m] = T(0.5) * st * cdp;
                GZ[l * l + l - m] = T(0.5) * st * sdp;
            }
        }
    }
}

// The same harmonics row by row: begin(l) is called before row l and
// visit(l, m, y+, y-, g+, g-) for m = 0..l with Y_l^{+m}, Y_l^{-m} (y- unused
// for m = 0) and their gradients w.r.t. the unit direction (g+/g- all zero
// when GRAD is false).  Same operations in the same order as ylm_compute, so
// the results are identical, but in l-outer order: three rows of Legendre
// polynomials live in registers instead of a local-memory table.  For
// LCAP <= 8 (the register arrays are unrolled).
template <typename T, int LCAP, bool GRAD, typename Begin, typename Visit>
__device__ __forceinline__ void ylm_rows(const DeviceYlmT<T>& tab, T ux, T uy, T uz, Begin begin, Visit visit) {
    static_assert(LCAP <= 8, "ylm_rows keeps (LCAP + 1) x 4 Legendre values in registers");
    const int lmax = tab.lmax;
    const T SQRT_1_OVER_2PI = T(0.3989422804014327);
    const T SQRT_3 = T(1.7320508075688772);
    const T SQRT_3_OVER_2 = T(1.224744871391589);
    const T SQRT_2 = T(1.4142135623730951);
    const T sxy = hypot(ux, uy);
    const T ct = uz, st = sxy;
    T cp, sp;
    if (sxy > T(soap::DBL_EPS)) {
        cp = ux / sxy;
        sp = uy / sxy;
    } else {
        cp = T(1);
        sp = T(0);
    }
    // cos(m phi), sin(m phi) by the recursion of :300-306
    T cm[LCAP + 1], sm[LCAP + 1];
    {
        T cos1 = T(1), sin1 = T(0), cos2 = -cp, sin2 = sp;
        const T m2c = T(-2) * cp;
        cm[0] = T(1);
        sm[0] = T(0);
#pragma unroll
        for (int m = 1; m <= LCAP; m++) {
            const T smp = m2c * sin1 - sin2;
            const T cmp = m2c * cos1 - cos2;
            sin2 = sin1;
            sin1 = smp;
            cos2 = cos1;
            cos1 = cmp;
            cm[m] = cmp;
            sm[m] = smp;
        }
    }
    T p2[LCAP + 1], p1[LCAP + 1], p0[LCAP + 1], dp[LCAP + 1];
    T value = SQRT_1_OVER_2PI;
#pragma unroll
    for (int l = 0; l <= LCAP; l++) {
        if (l > lmax) break;
        // associated Legendre row l (:228-251)
        if (l == 0) {
            p0[0] = value;
        } else if (l == 1) {
            p0[0] = ct * SQRT_3 * value;
            value *= -SQRT_3_OVER_2 * st;
            p0[1] = value;
        } else {
#pragma unroll
            for (int m = 0; m < l - 1; m++) p0[m] = tab.A[lidx(l, m)] * (ct * p1[m] + tab.B[lidx(l, m)] * p2[m]);
            p0[l - 1] = ct * tab.sq_2l1[l] * value;
            value *= -tab.sq_half[l] * st;
            p0[l] = value;
        }
        // derivative factors (:256-298)
        if (GRAD) {
            if (l == 0) {
                dp[0] = T(0);
            } else {
                const T pm1 = tab.inv_ll[l] * p0[1];
                dp[0] = tab.sq_plus[lidx(l, 0)] * pm1 - tab.sq_minus[lidx(l, 0)] * p0[1];
#pragma unroll
                for (int m = 1; m < l; m++)
                    dp[m] = tab.sq_plus[lidx(l, m)] * p0[m - 1] - tab.sq_minus[lidx(l, m)] * p0[m + 1];
                dp[l] = tab.sq_plus[lidx(l, l)] * p0[l - 1] - tab.sq_minus[lidx(l, l)] * T(0);
            }
        }
        begin(l);
        {
            T g0[3] = {T(0), T(0), T(0)};
            if (GRAD && l > 0) {
                const T lf = tab.sq_ll1[l] * p0[1];
                g0[0] = cp * ct * lf;
                g0[1] = sp * ct * lf;
                g0[2] = -st * lf;
            }
            visit(l, 0, p0[0] / SQRT_2, T(0), g0, g0);
        }
#pragma unroll
        for (int m = 1; m <= l; m++) {
            const T yp = p0[m] * cm[m];
            const T ym = p0[m] * sm[m];
            T gp[3] = {T(0), T(0), T(0)}, gm[3] = {T(0), T(0), T(0)};
            if (GRAD) {
                const T pot = st > T(0.1) ? (T)m / st * p0[m] : T(-0.5) / ct * dp[m];
                const T sdp = sm[m] * dp[m], cdp = cm[m] * dp[m];
                gp[0] = sp * pot * sm[m] - T(0.5) * ct * cp * cdp;
                gm[0] = -sp * pot * cm[m] - T(0.5) * ct * cp * sdp;
                gp[1] = -cp * pot * sm[m] - T(0.5) * ct * sp * cdp;
                gm[1] = cp * pot * cm[m] - T(0.5) * ct * sp * sdp;
                gp[2] = T(0.5) * st * cdp;
                gm[2] = T(0.5) * st * sdp;
            }
            visit(l, m, yp, ym, gp, gm);
        }
#pragma unroll
        for (int m = 0; m <= LCAP; m++) {
            p2[m] = p1[m];
            p1[m] = p0[m];
        }
    }
}

// The same harmonics split by column m, for one thread per (direction, m).
// The direction's angles, as ylm_compute derives them:
template <typename T>
struct YlmAngles {
    T ct, st, cp, sp;
};

template <typename T>
__device__ __forceinline__ YlmAngles<T> ylm_angles(T ux, T uy, T uz) {
    YlmAngles<T> a;
    const T sxy = hypot(ux, uy);
    a.ct = uz;
    a.st = sxy;
    if (sxy > T(soap::DBL_EPS)) {
        a.cp = ux / sxy;
        a.sp = uy / sxy;
    } else {
        a.cp = T(1);
        a.sp = T(0);
    }
    return a;
}

// Column m of the associated Legendre table, P(l, m) for l = m..lmax, written
// to P[lidx(l, m)].  The recursions of ylm_compute restricted to one column
// (every P(l, m) depends on P(l - 1, m), P(l - 2, m) and the diagonal chain
// only), with the same operations in the same order.
template <typename T>
__device__ __forceinline__ void ylm_legendre_column(const DeviceYlmT<T>& tab, const YlmAngles<T>& a, int m,
                                                    T* __restrict__ P) {
    const int lmax = tab.lmax;
    const T SQRT_1_OVER_2PI = T(0.3989422804014327);
    const T SQRT_3 = T(1.7320508075688772);
    const T SQRT_3_OVER_2 = T(1.224744871391589);
    T value = SQRT_1_OVER_2PI;  // P(m, m) after m steps of the diagonal chain
    if (m >= 1) value *= -SQRT_3_OVER_2 * a.st;
    for (int l = 2; l <= m; l++) value *= -tab.sq_half[l] * a.st;
    P[lidx(m, m)] = value;
    if (m + 1 > lmax) return;
    T pm2 = value;
    T pm1 = m == 0 ? a.ct * SQRT_3 * value : a.ct * tab.sq_2l1[m + 1] * value;
    P[lidx(m + 1, m)] = pm1;
    for (int l = m + 2; l <= lmax; l++) {
        const T p = tab.A[lidx(l, m)] * (a.ct * pm1 + tab.B[lidx(l, m)] * pm2);
        P[lidx(l, m)] = p;
        pm2 = pm1;
        pm1 = p;
    }
}

// Y_l^{+-m} (and gradients when GX != nullptr) of column m for l = m..lmax,
// from the complete Legendre table P (all columns), indexed l^2 + l + m as in
// ylm_compute; the same operations in the same order.
template <typename T>
__device__ __forceinline__ void ylm_column_outputs(const DeviceYlmT<T>& tab, const YlmAngles<T>& a, int m,
                                                   const T* __restrict__ P, T* __restrict__ Y, T* __restrict__ GX,
                                                   T* __restrict__ GY, T* __restrict__ GZ) {
    const int lmax = tab.lmax;
    const T SQRT_2 = T(1.4142135623730951);
    const T ct = a.ct, st = a.st, cp = a.cp, sp = a.sp;
    const bool grad = GX != nullptr;
    if (m == 0) {
        for (int l = 0; l <= lmax; l++) Y[l * l + l] = P[lidx(l, 0)] / SQRT_2;
        if (grad) {
            GX[0] = T(0);
            GY[0] = T(0);
            GZ[0] = T(0);
            for (int l = 1; l <= lmax; l++) {
                T lf = tab.sq_ll1[l] * P[lidx(l, 1)];
                GX[l * l + l] = cp * ct * lf;
                GY[l * l + l] = sp * ct * lf;
                GZ[l * l + l] = -st * lf;
            }
        }
        return;
    }
    T cos1 = T(1), sin1 = T(0), cos2 = -cp, sin2 = sp;
    T m2c = T(-2) * cp;
    T smp = T(0), cmp = T(0);
    for (int k = 1; k <= m; k++) {
        smp = m2c * sin1 - sin2;
        cmp = m2c * cos1 - cos2;
        sin2 = sin1;
        sin1 = smp;
        cos2 = cos1;
        cos1 = cmp;
    }
    for (int l = m; l <= lmax; l++) {
        T p = P[lidx(l, m)];
        Y[l * l + l + m] = p * cmp;
        Y[l * l + l - m] = p * smp;
    }
    if (!grad) return;
    for (int l = m; l <= lmax; l++) {
        // derivative factor (:256-298) and P / sin(theta) or its pole form
        T dp;
        if (m < l) dp = tab.sq_plus[lidx(l, m)] * P[lidx(l, m - 1)] - tab.sq_minus[lidx(l, m)] * P[lidx(l, m + 1)];
        else dp = tab.sq_plus[lidx(l, l)] * P[lidx(l, l - 1)] - tab.sq_minus[lidx(l, l)] * T(0);
        T pot = st > T(0.1) ? (T)m / st * P[lidx(l, m)] : T(-0.5) / ct * dp;
        T sdp = smp * dp, cdp = cmp * dp;
        GX[l * l + l + m] = sp * pot * smp - T(0.5) * ct * cp * cdp;
        GX[l * l + l - m] = -sp * pot * cmp - T(0.5) * ct * cp * sdp;
        GY[l * l + l + m] = -cp * pot * smp - T(0.5) * ct * sp * cdp;
        GY[l * l + l - m] = cp * pot * cmp - T(0.5) * ct * sp * sdp;
        GZ[l * l + l + m] = T(0.5) * st * cdp;
        GZ[l * l + l - m] = T(0.5) * st * sdp;
    }
}

// Radial integral of one angular channel in FP64: Hermite spline
// (featomic/src/math/splines.rs:225-289) or the analytic GTO integral times
// the orthonormalisation matrix (radial_integral/gto.rs:115-205).  Returns
// false when the analytic integral did not converge.
__device__ inline void radial_spline_compute(const DeviceRadial& R, int l, double r, double* __restrict__ val,
                                             double* __restrict__ grad) {
    const int N = R.nmax;
    const double* pos = R.positions + R.knot_offset[l];
    int count = R.knot_count[l];
    int k = soap::spline_interval(pos, count, r);
    soap::HermiteWeights w = soap::hermite_weights(pos[k], pos[k + 1], r);
    const double* pv = R.values + ((size_t)R.knot_offset[l] + k) * N;
    const double* pd = R.derivs + ((size_t)R.knot_offset[l] + k) * N;
    for (int n = 0; n < N; n++) {
        val[n] = soap::hermite_value(w, pv[n], pd[n], pv[N + n], pd[N + n]);
        if (grad) grad[n] = soap::hermite_derivative(w, pv[n], pd[n], pv[N + n], pd[N + n]);
    }
}

__device__ inline bool radial_compute(const DeviceRadial& R, int l, double r, double* __restrict__ val,
                                      double* __restrict__ grad) {
    const int N = R.nmax;
    if (R.splined) {
        radial_spline_compute(R, l, r, val, grad);
        return true;
    }
    double raw[64], graw[64];
    bool ok = soap::gto_radial_raw(l, N, r, R.c, R.width2, R.bn, raw, grad ? graw : nullptr);
    for (int k = 0; k < N; k++) {
        double s = 0.0, sg = 0.0;
        for (int n = 0; n < N; n++) {
            s += raw[n] * R.ortho[k * N + n];
            if (grad) sg += graw[n] * R.ortho[k * N + n];
        }
        val[k] = s;
        if (grad) grad[k] = sg;
    }
    return ok;
}

// The same in T: the knot search and Hermite weights in FP64, the spline
// values and derivatives (tables in T) combined in T.  Without spline the FP64
// analytic integral is rounded to T.
template <typename T>
__device__ inline bool radial_eval(const DeviceRadial& exact, const DeviceSplineT<T>& S, int l, double r,
                                   T* __restrict__ val, T* __restrict__ grad) {
    const int N = S.nmax;
    if (S.splined) {
        const double* pos = S.positions + S.knot_offset[l];
        const int count = S.knot_count[l];
        const int k = soap::spline_interval(pos, count, r);
        const soap::HermiteWeights w = soap::hermite_weights(pos[k], pos[k + 1], r);
        const T* pv = S.values + ((size_t)S.knot_offset[l] + k) * N;
        const T* pd = S.derivs + ((size_t)S.knot_offset[l] + k) * N;
        const T h00 = (T)w.h00, h10 = (T)(w.h10 * w.delta), h01 = (T)w.h01, h11 = (T)(w.h11 * w.delta);
        const T d00 = (T)(w.d00 * w.dxdt), d10 = (T)w.d10, d01 = (T)(w.d01 * w.dxdt), d11 = (T)w.d11;
        for (int n = 0; n < N; n++) {
            const T p0 = pv[n], m0 = pd[n], p1 = pv[N + n], m1 = pd[N + n];
            val[n] = h00 * p0 + h10 * m0 + h01 * p1 + h11 * m1;
            if (grad) grad[n] = d00 * p0 + d10 * m0 + d01 * p1 + d11 * m1;
        }
        return true;
    }
    double v[64], g[64];
    const bool ok = radial_compute(exact, l, r, v, grad ? g : nullptr);
    for (int n = 0; n < N; n++) {
        val[n] = (T)v[n];
        if (grad) grad[n] = (T)g[n];
    }
    return ok;
}

}  // namespace fb200

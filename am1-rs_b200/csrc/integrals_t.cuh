// The two-centre formulas of the NDDO model as templates over the scalar type: double for the
// integrals, overlap and core-core energy the SCF uses (k_integrals.cu), D3 (dual3.cuh) for their
// exact derivatives with respect to the pair displacement (k_gradient.cu).  Both instantiations
// run the same expressions in the same order; the double one is what the SCF has always used.
//
// Formulas follow am1-rs:
//   local integrals        src/integrals.rs:309-484 (Dewar-Sabelli-Klopman multipoles)
//   frame-free rotation    src/integrals.rs:487-569 (axis n = -x_ab and projector I - n n^T)
//   electron-core terms    src/integrals.rs:232-276 (e1b / e2a = -Z * row/column 0 of w)
//   Slater overlap         src/overlap.rs:16-40, 120-322, 357-500 (n <= 3 shells)
//   numerical overlap      src/overlap_numeric.rs:22-123 (shells with n >= 4)
//   core-core pair energy  src/repulsion.rs:144-188
#pragma once

#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dual3.cuh"
#include "params/gauss_legendre.h"

namespace am1 {

template <class T>
__device__ __forceinline__ T zero();
template <>
__device__ __forceinline__ double zero<double>() { return 0.0; }
template <>
__device__ __forceinline__ D3 zero<D3>() { return d3c(0.0); }
template <class T>
__device__ __forceinline__ T one();
template <>
__device__ __forceinline__ double one<double>() { return 1.0; }
template <>
__device__ __forceinline__ D3 one<D3>() { return d3c(1.0); }

template <class T>
__device__ __forceinline__ T rinv(const T& x) { return 1.0 / sqrt(x); }

template <class T>
__device__ __forceinline__ T dpow_i(T x, int k) {
    T acc = one<T>();
    while (k) {
        if (k & 1) acc *= x;
        k >>= 1;
        if (k) x *= x;
    }
    return acc;
}

// A_k(x), k = 0..6 (the overlap never reads above index 6).
template <class T>
__device__ void aint7(const T& x, T a[7]) {
    if (fabs(val(x)) < 1.0e-12) {
#pragma unroll
        for (int i = 0; i < 7; ++i) a[i] = zero<T>();
        return;
    }
    const T inv = 1.0 / x;
    a[0] = exp(-x) * inv;
#pragma unroll
    for (int i = 1; i < 7; ++i) a[i] = a[0] + a[i - 1] * inv * (double)i;
}

// B_k(x), k = 0..6: closed form above |x| = 5, the everywhere-convergent series below.
template <class T>
__device__ void bint7(const T& x, T b[7]) {
    if (fabs(val(x)) > 5.0) {
        const T inv = 1.0 / x;
        const T tx = exp(x) * inv;
        const T tmx = -(exp(-x) * inv);
        b[0] = tx + tmx;
#pragma unroll
        for (int i = 1; i < 7; ++i) b[i] = ((i & 1) ? -tx : tx) + tmx + b[i - 1] * inv * (double)i;
        return;
    }
#pragma unroll
    for (int i = 0; i < 7; ++i) b[i] = zero<T>();
    T term = one<T>();
    double mag = 1.0;
    const double ax = fabs(val(x));
    for (int n = 0; n < 64; ++n) {
        for (int k = n & 1; k < 7; k += 2) b[k] += term * (2.0 / (double)(k + n + 1));
        term = term * x * (-1.0 / (double)(n + 1));
        mag *= ax / (double)(n + 1);
        if (n >= 4 && mag < 1.0e-18) break;
    }
}

// Overlap of two Slater orbitals in the local diatomic frame (b at +z, distance r),
// <n_a l_a m; z_a | n_b l_b m; z_b> with m = 0 (sigma) or 1 (pi), by Gauss-Legendre quadrature in
// prolate-spheroidal coordinates: xi in [1, xi_max] (48 nodes), eta in [-1, 1] (40 nodes).  The
// domain and the angular factors depend on r's value only; the radial factor carries r, so a D3
// r gives the exact derivative of this quadrature (the boundary term at xi_max is negligible:
// the integrand has decayed by e^-60 there).
template <class T>
__device__ T overlap_sto(int na, double za, int la, int m, int nb, double zb, int lb, const T& r) {
    double c;
    if (la == 0 && lb == 0) c = 0.5;
    else if (la + lb == 1 && m == 0) c = 1.7320508075688772 / 2.0;
    else if (la == 1 && lb == 1) c = m == 0 ? 1.5 : 0.75;
    else return zero<T>();
    auto norm = [](int n, double zeta) {
        double f = 1.0;
        for (int k = 2; k <= 2 * n; ++k) f *= (double)k;
        return ::pow(2.0 * zeta, (double)n + 0.5) / ::sqrt(f);
    };
    const double nab = norm(na, za) * norm(nb, zb) * c;
    const double hr = 0.5 * val(r);
    const T half_r = r * 0.5;
    const double p = (za + zb) * hr;
    const double xi_max = 1.0 + 60.0 / fmax(p, 0.05);
    const double xi_mid = 0.5 * (1.0 + xi_max), xi_half = 0.5 * (xi_max - 1.0);
    T sum = zero<T>();
    for (int i = 0; i < kGlXiN; ++i) {
        const double xi = xi_mid + xi_half * kGlXiX[i];
        for (int j = 0; j < kGlEtaN; ++j) {
            const double eta = kGlEtaX[j];
            if (hr * (xi + eta) <= 0.0 || hr * (xi - eta) <= 0.0) continue;
            const double cos_a = (1.0 + xi * eta) / (xi + eta), cos_b = (xi * eta - 1.0) / (xi - eta);
            const double ang_a = la == 0 ? 1.0 : m == 0 ? cos_a : ::sqrt(fmax(1.0 - cos_a * cos_a, 0.0));
            const double ang_b = lb == 0 ? 1.0 : m == 0 ? cos_b : ::sqrt(fmax(1.0 - cos_b * cos_b, 0.0));
            const T ra = half_r * (xi + eta), rb = half_r * (xi - eta);
            const T radial = dpow_i(ra, na - 1) * dpow_i(rb, nb - 1) * exp(ra * (-za) - rb * zb);
            sum += radial * (xi_half * kGlXiW[i] * kGlEtaW[j] * ang_a * ang_b * (xi * xi - eta * eta));
        }
    }
    return dpow_i(half_r, 3) * sum * nab;
}

// The five local overlaps of overlap_local by quadrature (any n; used for n >= 4), with the
// analytic kernel's sign convention (src/overlap_numeric.rs:22-42).
template <class T>
__device__ void overlap_local_numeric(const DevElem& ea, const DevElem& eb, const T& r, T s[5]) {
    s[0] = overlap_sto(ea.n, ea.zeta_s, 0, 0, eb.n, eb.zeta_s, 0, r);
    s[1] = overlap_sto(ea.n, ea.zeta_p, 1, 0, eb.n, eb.zeta_s, 0, r);
    s[2] = -overlap_sto(ea.n, ea.zeta_s, 0, 0, eb.n, eb.zeta_p, 1, r);
    s[3] = -overlap_sto(ea.n, ea.zeta_p, 1, 0, eb.n, eb.zeta_p, 1, r);
    s[4] = overlap_sto(ea.n, ea.zeta_p, 1, 1, eb.n, eb.zeta_p, 1, r);
}

// Local overlaps (s111, s211, s121, s221, s222) for ea.n >= eb.n: the closed forms for n <= 3,
// the quadrature above.
template <class T>
__device__ bool overlap_local(const DevElem& ea, const DevElem& eb, const T& r, T s[5]) {
    const double za0 = ea.zeta_s, za1 = ea.zeta_p, zb0 = eb.zeta_s, zb1 = eb.zeta_p;
    T a[7], b[7];
    s[0] = s[1] = s[2] = s[3] = s[4] = zero<T>();
    const int na = ea.n, nb = eb.n;
    if (na > 3) {
        overlap_local_numeric(ea, eb, r, s);
        return true;
    }
    const double sq3 = 1.7320508075688772, sq10 = 3.1622776601683795, sq30 = 5.477225575051661;
    // (s_a | s_b)
    aint7(r * (0.5 * (za0 + zb0)), a);
    bint7(r * (0.5 * (za0 - zb0)), b);
    if (na == 1 && nb == 1) {
        s[0] = pow(r * r * (za0 * zb0), 1.5) * (a[2] * b[0] - b[2] * a[0]) / 4.0;
        return true;
    }
    if (na == 2 && nb == 1) {
        s[0] = dpow_i(r, 4) * (pow(zb0, 1.5) * pow(za0, 2.5)) * (a[3] * b[0] - b[3] * a[0] + a[2] * b[1] - b[2] * a[1]) / (sq3 * 8.0);
    } else if (na == 2 && nb == 2) {
        s[0] = dpow_i(r, 5) * pow(zb0 * za0, 2.5) * (a[4] * b[0] + b[4] * a[0] - a[2] * b[2] * 2.0) / 48.0;
    } else if (na == 3 && nb == 1) {
        s[0] = dpow_i(r, 5) * (pow(zb0, 1.5) * pow(za0, 3.5)) * (a[4] * b[0] + b[1] * a[3] * 2.0 - a[1] * b[3] * 2.0 - b[4] * a[0]) / (sq10 * 24.0);
    } else if (na == 3 && nb == 2) {
        s[0] = dpow_i(r, 6) * (pow(zb0, 2.5) * pow(za0, 3.5)) *
               (a[5] * b[0] + b[1] * a[4] - b[2] * a[3] * 2.0 - a[2] * b[3] * 2.0 + b[4] * a[1] + b[5] * a[0]) / (sq30 * 48.0);
    } else {  // 3,3
        s[0] = dpow_i(r, 7) * pow(zb0 * za0, 3.5) * (a[6] * b[0] - b[2] * a[4] * 3.0 + a[2] * b[4] * 3.0 - a[0] * b[6]) / 1440.0;
    }
    // (p_a | s_b)
    aint7(r * (0.5 * (za1 + zb0)), a);
    bint7(r * (0.5 * (za1 - zb0)), b);
    if (na == 2 && nb == 1) {
        s[1] = dpow_i(r, 4) * (pow(zb0, 1.5) * pow(za1, 2.5)) * (a[2] * b[0] - b[2] * a[0] + a[3] * b[1] - b[3] * a[1]) / 8.0;
    } else if (na == 2 && nb == 2) {
        s[1] = dpow_i(r, 5) * pow(zb0 * za1, 2.5) *
               (a[3] * (b[0] - b[2]) - a[1] * (b[2] - b[4]) + b[3] * (a[0] - a[2]) - b[1] * (a[2] - a[4])) / (16.0 * sq3);
    } else if (na == 3 && nb == 1) {
        s[1] = dpow_i(r, 5) * (pow(zb0, 1.5) * pow(za1, 3.5)) *
               (a[3] * (b[0] + b[2]) - a[1] * (b[4] + b[2]) + b[1] * (a[2] + a[4]) - b[3] * (a[2] + a[0])) / (8.0 * sq30);
    } else if (na == 3 && nb == 2) {
        s[1] = dpow_i(r, 6) * (pow(zb0, 2.5) * pow(za1, 3.5)) *
               (a[4] * b[0] + b[1] * a[5] - b[3] * a[3] * 2.0 - a[2] * b[2] * 2.0 + a[1] * b[5] + a[0] * b[4]) / (48.0 * sq10);
    } else if (na == 3 && nb == 3) {
        s[1] = dpow_i(r, 7) * pow(zb0 * za1, 3.5) *
               ((a[5] * b[0] + a[6] * b[1]) + (-a[4] * b[1] - a[5] * b[2]) - (a[3] * b[2] + a[4] * b[3]) * 2.0 -
                (-a[2] * b[3] - a[3] * b[4]) * 2.0 + (a[1] * b[4] + a[2] * b[5]) + (-a[0] * b[5] - a[1] * b[6])) / (480.0 * sq3);
    }
    if (nb == 1) return true;
    // (s_a | p_b)
    aint7(r * (0.5 * (za0 + zb1)), a);
    bint7(r * (0.5 * (za0 - zb1)), b);
    if (na == 2) {
        s[2] = dpow_i(r, 5) * pow(zb1 * za0, 2.5) *
               (a[3] * (b[0] - b[2]) - a[1] * (b[2] - b[4]) - b[3] * (a[0] - a[2]) + b[1] * (a[2] - a[4])) / (16.0 * sq3);
    } else if (nb == 2) {
        s[2] = dpow_i(r, 6) * (pow(zb1, 2.5) * pow(za0, 3.5)) *
               ((a[4] * b[0] - a[5] * b[1]) + (a[3] * b[1] - a[4] * b[2]) * 2.0 - (a[1] * b[3] - a[2] * b[4]) * 2.0 -
                (a[0] * b[4] - a[1] * b[5])) / (48.0 * sq10);
    } else {
        s[2] = dpow_i(r, 7) * pow(zb1 * za0, 3.5) *
               ((a[5] * b[0] - a[6] * b[1]) + (a[4] * b[1] - a[5] * b[2]) - (a[3] * b[2] - a[4] * b[3]) * 2.0 -
                (a[2] * b[3] - a[3] * b[4]) * 2.0 + (a[1] * b[4] - a[2] * b[5]) + (a[0] * b[5] - a[1] * b[6])) / (480.0 * sq3);
    }
    // (p_a | p_b): sigma (s221) and pi (s222)
    aint7(r * (0.5 * (za1 + zb1)), a);
    bint7(r * (0.5 * (za1 - zb1)), b);
    if (na == 2) {
        const T w = dpow_i(r, 5) * pow(zb1 * za1, 2.5) / 16.0;
        s[3] = -(w * (b[2] * (a[4] + a[0]) - a[2] * (b[4] + b[0])));
        s[4] = w * (a[4] * (b[0] - b[2]) - b[4] * (a[0] - a[2]) - a[2] * b[0] + b[2] * a[0]) * 0.5;
    } else if (nb == 2) {
        const T pre = dpow_i(r, 6) * (pow(zb1, 2.5) * pow(za1, 3.5));
        s[3] = pre * ((a[3] * b[0] - a[5] * b[2]) + (a[2] * b[1] - a[4] * b[3]) - (a[1] * b[2] - a[3] * b[4]) - (a[0] * b[3] - a[2] * b[5])) /
               (16.0 * sq30);
        s[4] = pre *
               ((a[5] - a[3]) * (b[0] - b[2]) + (a[4] - a[2]) * (b[1] - b[3]) - (a[3] - a[1]) * (b[2] - b[4]) - (a[2] - a[0]) * (b[3] - b[5])) /
               (32.0 * sq30);
    } else {
        const T pre = dpow_i(r, 7) * (pow(zb1, 3.5) * pow(za1, 3.5));
        s[3] = pre * ((a[4] * b[0] - a[6] * b[2]) - (a[2] * b[2] - a[4] * b[4]) * 2.0 + (a[0] * b[4] - a[2] * b[6])) / 480.0;
        s[4] = pre * ((a[6] - a[4]) * (b[0] - b[2]) - (a[4] - a[2]) * (b[2] - b[4]) * 2.0 + (a[2] - a[0]) * (b[4] - b[6])) / 960.0;
    }
    return true;
}

// Global-frame 4x4 overlap S[i-orbital][j-orbital]; dir = unit vector i -> j.
template <class T>
__device__ bool overlap_block(const DevElem& ei, const DevElem& ej, const T& r, const T dir[3], T S[4][4]) {
    T s[5];
    const bool swap = ei.n < ej.n;
    if (!overlap_local(swap ? ej : ei, swap ? ei : ej, r, s)) return false;
    const double sg = swap ? -1.0 : 1.0;
    const T d[3] = {dir[0] * sg, dir[1] * sg, dir[2] * sg};
    T di[4][4];
    di[0][0] = s[0];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        di[1 + a][0] = s[1] * d[a];
        di[0][1 + a] = -s[2] * d[a];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const T nn = d[a] * d[b];
            const T p = (a == b ? 1.0 : 0.0) - nn;
            di[1 + a][1 + b] = -s[3] * nn + s[4] * p;
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) S[a][b] = swap ? di[b][a] : di[a][b];
    return true;
}

// The 22 local-frame heavy-heavy integrals (eV).
template <class T>
__device__ void local_xx(const DevElem& ei, const DevElem& ej, const T& r, T ri[22]) {
    const double ev1 = AM1_EV / 2.0, ev2 = AM1_EV / 4.0, ev3 = AM1_EV / 8.0, ev4 = AM1_EV / 16.0;
    const double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0, qa1 = ei.qq, qb1 = ej.qq;
    const double aee = (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0);
    const double ade = (ei.rho1 + ej.rho0) * (ei.rho1 + ej.rho0);
    const double aqe = (ei.rho2 + ej.rho0) * (ei.rho2 + ej.rho0);
    const double aed = (ei.rho0 + ej.rho1) * (ei.rho0 + ej.rho1);
    const double aeq = (ei.rho0 + ej.rho2) * (ei.rho0 + ej.rho2);
    const double axx = (ei.rho1 + ej.rho1) * (ei.rho1 + ej.rho1);
    const double adq = (ei.rho1 + ej.rho2) * (ei.rho1 + ej.rho2);
    const double aqd = (ei.rho2 + ej.rho1) * (ei.rho2 + ej.rho1);
    const double aqq = (ei.rho2 + ej.rho2) * (ei.rho2 + ej.rho2);
    // 1/sqrt(x^2 + c)
#define SQ2(x, c) rinv((x) * (x) + (c))
    const T r2 = r * r;
    const T ee = rinv(r2 + aee) * AM1_EV;
    const T dze = SQ2(r - da, ade) * ev1 - SQ2(r + da, ade) * ev1;
    const T ev1dsqr6 = rinv(r2 + aqe) * ev1;
    const T qzze = SQ2(r - qa, aqe) * ev2 + SQ2(r + qa, aqe) * ev2 - ev1dsqr6;
    const T qxxe = rinv(r2 + qa * qa + aqe) * ev1 - ev1dsqr6;
    const T edz = SQ2(r + db, aed) * ev1 - SQ2(r - db, aed) * ev1;
    const T ev1dsqr12 = rinv(r2 + aeq) * ev1;
    const T eqzz = SQ2(r - qb, aeq) * ev2 + SQ2(r + qb, aeq) * ev2 - ev1dsqr12;
    const T eqxx = rinv(r2 + qb * qb + aeq) * ev1 - ev1dsqr12;
    const T ev2dsqr20 = SQ2(r + da, adq) * ev2;
    const T ev2dsqr22 = SQ2(r - da, adq) * ev2;
    const T ev2dsqr24 = SQ2(r - db, aqd) * ev2;
    const T ev2dsqr26 = SQ2(r + db, aqd) * ev2;
    const T ev2dsqr36 = rinv(r2 + aqq) * ev2;
    const T ev2dsqr39 = rinv(r2 + qa * qa + aqq) * ev2;
    const T ev2dsqr40 = rinv(r2 + qb * qb + aqq) * ev2;
    const T ev3dsqr42 = SQ2(r - qb, aqq) * ev3;
    const T ev3dsqr44 = SQ2(r + qb, aqq) * ev3;
    const T ev3dsqr46 = SQ2(r + qa, aqq) * ev3;
    const T ev3dsqr48 = SQ2(r - qa, aqq) * ev3;
    ri[0] = ee;
    ri[1] = -dze;
    ri[2] = ee + qzze;
    ri[3] = ee + qxxe;
    ri[4] = -edz;
    ri[5] = SQ2(r + da - db, axx) * ev2 + SQ2(r - da + db, axx) * ev2 - SQ2(r - da - db, axx) * ev2 - SQ2(r + da + db, axx) * ev2;
    ri[6] = rinv(r2 + (da - db) * (da - db) + axx) * ev1 - rinv(r2 + (da + db) * (da + db) + axx) * ev1;
    ri[7] = -edz + SQ2(r + qa - db, aqd) * ev3 - SQ2(r + qa + db, aqd) * ev3 + SQ2(r - qa - db, aqd) * ev3 -
            SQ2(r - qa + db, aqd) * ev3 - ev2dsqr24 + ev2dsqr26;
    ri[8] = -edz - ev2dsqr24 + rinv((r - db) * (r - db) + qa * qa + aqd) * ev2 + ev2dsqr26 -
            rinv((r + db) * (r + db) + qa * qa + aqd) * ev2;
    ri[9] = rinv((qa1 - db) * (qa1 - db) + (r + qa1) * (r + qa1) + aqd) * ev2 -
            rinv((qa1 - db) * (qa1 - db) + (r - qa1) * (r - qa1) + aqd) * ev2 -
            rinv((qa1 + db) * (qa1 + db) + (r + qa1) * (r + qa1) + aqd) * ev2 +
            rinv((qa1 + db) * (qa1 + db) + (r - qa1) * (r - qa1) + aqd) * ev2;
    ri[10] = ee + eqzz;
    ri[11] = ee + eqxx;
    ri[12] = -dze + SQ2(r + da - qb, adq) * ev3 - SQ2(r - da - qb, adq) * ev3 + SQ2(r + da + qb, adq) * ev3 -
             SQ2(r - da + qb, adq) * ev3 + ev2dsqr22 - ev2dsqr20;
    ri[13] = -dze - ev2dsqr20 + rinv((r + da) * (r + da) + qb * qb + adq) * ev2 + ev2dsqr22 -
             rinv((r - da) * (r - da) + qb * qb + adq) * ev2;
    ri[14] = rinv((da - qb1) * (da - qb1) + (r - qb1) * (r - qb1) + adq) * ev2 -
             rinv((da - qb1) * (da - qb1) + (r + qb1) * (r + qb1) + adq) * ev2 -
             rinv((da + qb1) * (da + qb1) + (r - qb1) * (r - qb1) + adq) * ev2 +
             rinv((da + qb1) * (da + qb1) + (r + qb1) * (r + qb1) + adq) * ev2;
    ri[15] = ee + eqzz + qzze + SQ2(r + qa - qb, aqq) * ev4 + SQ2(r + qa + qb, aqq) * ev4 + SQ2(r - qa - qb, aqq) * ev4 +
             SQ2(r - qa + qb, aqq) * ev4 - ev3dsqr48 - ev3dsqr46 - ev3dsqr42 - ev3dsqr44 + ev2dsqr36;
    ri[16] = ee + eqzz + qxxe + rinv((r - qb) * (r - qb) + qa * qa + aqq) * ev3 + rinv((r + qb) * (r + qb) + qa * qa + aqq) * ev3 -
             ev3dsqr42 - ev3dsqr44 - ev2dsqr39 + ev2dsqr36;
    ri[17] = ee + eqxx + qzze + rinv((r + qa) * (r + qa) + qb * qb + aqq) * ev3 + rinv((r - qa) * (r - qa) + qb * qb + aqq) * ev3 -
             ev3dsqr46 - ev3dsqr48 - ev2dsqr40 + ev2dsqr36;
    const T qxxqxx = rinv(r2 + (qa - qb) * (qa - qb) + aqq) * ev3 + rinv(r2 + (qa + qb) * (qa + qb) + aqq) * ev3 - ev2dsqr39 -
                          ev2dsqr40 + ev2dsqr36;
    ri[18] = ee + eqxx + qxxe + qxxqxx;
    const double dm = (qa1 - qb1) * (qa1 - qb1), dp = (qa1 + qb1) * (qa1 + qb1);
    ri[19] = rinv((r + qa1 - qb1) * (r + qa1 - qb1) + dm + aqq) * ev3 - rinv((r + qa1 + qb1) * (r + qa1 + qb1) + dm + aqq) * ev3 -
             rinv((r - qa1 - qb1) * (r - qa1 - qb1) + dm + aqq) * ev3 + rinv((r - qa1 + qb1) * (r - qa1 + qb1) + dm + aqq) * ev3 -
             rinv((r + qa1 - qb1) * (r + qa1 - qb1) + dp + aqq) * ev3 + rinv((r + qa1 + qb1) * (r + qa1 + qb1) + dp + aqq) * ev3 +
             rinv((r - qa1 - qb1) * (r - qa1 - qb1) + dp + aqq) * ev3 - rinv((r - qa1 + qb1) * (r - qa1 + qb1) + dp + aqq) * ev3;
    const T qxxqyy = rinv(r2 + qa * qa + qb * qb + aqq) * ev2 - ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
    ri[20] = ee + eqxx + qxxe + qxxqyy;
    ri[21] = (qxxqxx - qxxqyy) * 0.5;
#undef SQ2
}

// Integrals of one pair (i = heavy or lower index, j), each handed to sink(kk, ll, mm, nn, value)
// as it is formed: (kk ll | mm nn) with kk >= ll the orbitals on i and mm >= nn those on j
// (0 = s, 1-3 = p), in the store's order (row pack(kk, ll), column pack(mm, nn)).
template <class T, class Sink>
__device__ void pair_integrals_each(const DevElem& ei, const DevElem& ej, const T dv[3], const T& r, Sink&& sink) {
    const T inv = 1.0 / r;
    const T n[3] = {-(dv[0] * inv), -(dv[1] * inv), -(dv[2] * inv)};  // frame axis, = -x_ij
    const bool hi = ei.norb == 4, hj = ej.norb == 4;
    if (!hi && !hj) {
        sink(0, 0, 0, 0, rinv(r * r + (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0)) * AM1_EV);
        return;
    }
    // p = I - n n^T
    T p[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) p[a][b] = (a == b ? 1.0 : 0.0) - n[a] * n[b];
    if (hi && !hj) {
        const double ev1 = AM1_EV / 2.0, ev2 = AM1_EV / 4.0;
        const double da = ei.dd, qa = ei.qq * 2.0;
        const double aee = (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0);
        const double ade = (ei.rho1 + ej.rho0) * (ei.rho1 + ej.rho0);
        const double aqe = (ei.rho2 + ej.rho0) * (ei.rho2 + ej.rho0);
        const T ee = rinv(r * r + aee) * AM1_EV;
        const T q6 = rinv(r * r + aqe) * ev1;
        const T r1 = rinv((r + da) * (r + da) + ade) * ev1 - rinv((r - da) * (r - da) + ade) * ev1;
        const T r2 = ee + rinv((r + qa) * (r + qa) + aqe) * ev2 + rinv((r - qa) * (r - qa) + aqe) * ev2 - q6;
        const T r3 = ee + rinv(r * r + qa * qa + aqe) * ev1 - q6;
        sink(0, 0, 0, 0, ee);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            sink(k + 1, 0, 0, 0, r1 * n[k]);
#pragma unroll
            for (int l = 0; l <= k; ++l) sink(k + 1, l + 1, 0, 0, r2 * (n[k] * n[l]) + r3 * p[k][l]);
        }
        return;
    }
    T ri[22];
    local_xx(ei, ej, r, ri);
#pragma unroll 1
    for (int kk = 0; kk < 4; ++kk)
        for (int ll = 0; ll <= kk; ++ll)
#pragma unroll
            for (int mm = 0; mm < 4; ++mm)
#pragma unroll
                for (int nn = 0; nn <= mm; ++nn) {
                    const int k = kk - 1, l = ll - 1, m = mm - 1, q = nn - 1;
                    T v;
                    if (kk == 0) {
                        if (mm == 0) v = ri[0];
                        else if (nn == 0) v = ri[4] * n[m];
                        else v = ri[10] * (n[m] * n[q]) + ri[11] * p[m][q];
                    } else if (ll == 0) {
                        if (mm == 0) v = ri[1] * n[k];
                        else if (nn == 0) v = ri[5] * (n[k] * n[m]) + ri[6] * p[k][m];
                        else v = ri[12] * (n[k] * n[m] * n[q]) + ri[13] * (p[m][q] * n[k]) + ri[14] * (p[k][q] * n[m] + p[k][m] * n[q]);
                    } else if (mm == 0) {
                        v = ri[2] * (n[k] * n[l]) + ri[3] * p[k][l];
                    } else if (nn == 0) {
                        v = ri[7] * (n[k] * n[l] * n[m]) + ri[8] * (p[k][l] * n[m]) + ri[9] * (p[l][m] * n[k] + p[k][m] * n[l]);
                    } else {
                        v = ri[15] * (n[k] * n[l] * n[m] * n[q]) + ri[16] * (p[k][l] * n[m] * n[q]) + ri[17] * (p[m][q] * n[k] * n[l]) +
                            ri[19] * (n[k] * (p[l][q] * n[m] + p[l][m] * n[q]) + n[l] * (p[k][q] * n[m] + p[k][m] * n[q])) +
                            ri[20] * (p[k][l] * p[m][q]) + ri[21] * (p[k][m] * p[l][q] + p[k][q] * p[l][m]);
                    }
                    sink(kk, ll, mm, nn, v);
                }
}

// pair_integrals_each written to the store: XX 10 x 10 row-major, XH 10, HH 1.
template <class T>
__device__ void pair_integrals(const DevElem& ei, const DevElem& ej, const T dv[3], const T& r, T* __restrict__ w) {
    const int nwb = ej.norb == 4 ? 10 : 1;
    pair_integrals_each(ei, ej, dv, r, [&](int kk, int ll, int mm, int nn, const T& v) {
        w[(kk * (kk + 1) / 2 + ll) * nwb + mm * (mm + 1) / 2 + nn] = v;
    });
}

template <class T>
__device__ T pair_core_energy(const DevElem& ei, const DevElem& ej, int zi, int zj, const T& r) {
    const T s = r * AM1_A0;
    const double rho = ei.rho0 + ej.rho0;
    const T gam = rinv(r * r + rho * rho) * AM1_EV;
    const double zz = ei.core_charge * ej.core_charge;
    const bool spi = (zi == 7 || zi == 8) && zj == 1;
    const bool spj = (zj == 7 || zj == 8) && zi == 1;
    T fi = exp(s * (-ei.alpha));
    T fj = exp(s * (-ej.alpha));
    if (spi) fi = s * fi;
    if (spj) fj = s * fj;
    T gi = zero<T>(), gj = zero<T>();
    for (int k = 0; k < ei.ngauss; ++k) {
        const T d = s - ei.gm[k];
        gi += exp(d * d * (-ei.gl[k])) * ei.gk[k];
    }
    for (int k = 0; k < ej.ngauss; ++k) {
        const T d = s - ej.gm[k];
        gj += exp(d * d * (-ej.gl[k])) * ej.gk[k];
    }
    return gam * (fi + fj + 1.0) * zz + (gi + gj) * zz / s;
}

}  // namespace am1

// Two-centre integrals, overlap, core Hamiltonian and core-core energy kernels.
//
// One thread per atom pair: each pair's work is a fixed, branch-uniform sequence of FP64
// transcendental evaluations (about 70 reciprocal square roots for a heavy-heavy pair plus the
// Slater overlap's exponentials), so a thread per pair keeps all 32 lanes of a warp on the FP64
// pipe; the warp's pairs are consecutive pairs of one molecule, so their coordinates and
// parameters are read from the same few cache lines.
//
// Formulas follow am1-rs:
//   local integrals        src/integrals.rs:309-484 (Dewar-Sabelli-Klopman multipoles)
//   frame-free rotation    src/integrals.rs:487-569 (axis n = -x_ab and projector I - n n^T)
//   electron-core terms    src/integrals.rs:232-276 (e1b / e2a = -Z * row/column 0 of w)
//   Slater overlap         src/overlap.rs:16-40, 120-322, 357-500 (n <= 3 shells)
//   resonance              src/hamiltonian.rs:340-352  H_ab = (beta_a + beta_b)/2 * S_ab
//   core-core pair energy  src/repulsion.rs:144-188
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

__device__ __forceinline__ double rinv(double x) { return 1.0 / sqrt(x); }

__device__ __forceinline__ double dpow_i(double x, int k) {
    double acc = 1.0;
    while (k) {
        if (k & 1) acc *= x;
        k >>= 1;
        if (k) x *= x;
    }
    return acc;
}

// A_k(x), k = 0..6 (the overlap never reads above index 6).
__device__ void aint7(double x, double a[7]) {
    if (fabs(x) < 1.0e-12) {
#pragma unroll
        for (int i = 0; i < 7; ++i) a[i] = 0.0;
        return;
    }
    const double inv = 1.0 / x;
    a[0] = exp(-x) * inv;
#pragma unroll
    for (int i = 1; i < 7; ++i) a[i] = a[0] + a[i - 1] * inv * (double)i;
}

// B_k(x), k = 0..6: closed form above |x| = 5, the everywhere-convergent series below.
__device__ void bint7(double x, double b[7]) {
    if (fabs(x) > 5.0) {
        const double inv = 1.0 / x;
        const double tx = exp(x) * inv;
        const double tmx = -(exp(-x) * inv);
        b[0] = tx + tmx;
#pragma unroll
        for (int i = 1; i < 7; ++i) b[i] = ((i & 1) ? -tx : tx) + tmx + b[i - 1] * inv * (double)i;
        return;
    }
#pragma unroll
    for (int i = 0; i < 7; ++i) b[i] = 0.0;
    double term = 1.0, mag = 1.0;
    const double ax = fabs(x);
    for (int n = 0; n < 64; ++n) {
        for (int k = n & 1; k < 7; k += 2) b[k] += term * (2.0 / (double)(k + n + 1));
        term = term * x * (-1.0 / (double)(n + 1));
        mag *= ax / (double)(n + 1);
        if (n >= 4 && mag < 1.0e-18) break;
    }
}

// Local overlaps (s111, s211, s121, s221, s222) for ea.n >= eb.n; returns false for n >= 4.
__device__ bool overlap_local(const DevElem& ea, const DevElem& eb, double r, double s[5]) {
    const double za0 = ea.zeta_s, za1 = ea.zeta_p, zb0 = eb.zeta_s, zb1 = eb.zeta_p;
    double a[7], b[7];
    s[0] = s[1] = s[2] = s[3] = s[4] = 0.0;
    const int na = ea.n, nb = eb.n;
    if (na > 3) return false;
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
        const double w = dpow_i(r, 5) * pow(zb1 * za1, 2.5) / 16.0;
        s[3] = -(w * (b[2] * (a[4] + a[0]) - a[2] * (b[4] + b[0])));
        s[4] = w * (a[4] * (b[0] - b[2]) - b[4] * (a[0] - a[2]) - a[2] * b[0] + b[2] * a[0]) * 0.5;
    } else if (nb == 2) {
        const double pre = dpow_i(r, 6) * (pow(zb1, 2.5) * pow(za1, 3.5));
        s[3] = pre * ((a[3] * b[0] - a[5] * b[2]) + (a[2] * b[1] - a[4] * b[3]) - (a[1] * b[2] - a[3] * b[4]) - (a[0] * b[3] - a[2] * b[5])) /
               (16.0 * sq30);
        s[4] = pre *
               ((a[5] - a[3]) * (b[0] - b[2]) + (a[4] - a[2]) * (b[1] - b[3]) - (a[3] - a[1]) * (b[2] - b[4]) - (a[2] - a[0]) * (b[3] - b[5])) /
               (32.0 * sq30);
    } else {
        const double pre = dpow_i(r, 7) * (pow(zb1, 3.5) * pow(za1, 3.5));
        s[3] = pre * ((a[4] * b[0] - a[6] * b[2]) - (a[2] * b[2] - a[4] * b[4]) * 2.0 + (a[0] * b[4] - a[2] * b[6])) / 480.0;
        s[4] = pre * ((a[6] - a[4]) * (b[0] - b[2]) - (a[4] - a[2]) * (b[2] - b[4]) * 2.0 + (a[2] - a[0]) * (b[4] - b[6])) / 960.0;
    }
    return true;
}

// Global-frame 4x4 overlap S[i-orbital][j-orbital]; dir = unit vector i -> j.
__device__ bool overlap_block(const DevElem& ei, const DevElem& ej, double r, const double dir[3], double S[4][4]) {
    double s[5];
    const bool swap = ei.n < ej.n;
    if (!overlap_local(swap ? ej : ei, swap ? ei : ej, r, s)) return false;
    const double sg = swap ? -1.0 : 1.0;
    const double d[3] = {dir[0] * sg, dir[1] * sg, dir[2] * sg};
    double di[4][4];
    di[0][0] = s[0];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        di[1 + a][0] = s[1] * d[a];
        di[0][1 + a] = -s[2] * d[a];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const double nn = d[a] * d[b];
            const double p = (a == b ? 1.0 : 0.0) - nn;
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
__device__ void local_xx(const DevElem& ei, const DevElem& ej, double r, double ri[22]) {
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
    const double r2 = r * r;
    const double ee = rinv(r2 + aee) * AM1_EV;
    const double dze = SQ2(r - da, ade) * ev1 - SQ2(r + da, ade) * ev1;
    const double ev1dsqr6 = rinv(r2 + aqe) * ev1;
    const double qzze = SQ2(r - qa, aqe) * ev2 + SQ2(r + qa, aqe) * ev2 - ev1dsqr6;
    const double qxxe = rinv(r2 + qa * qa + aqe) * ev1 - ev1dsqr6;
    const double edz = SQ2(r + db, aed) * ev1 - SQ2(r - db, aed) * ev1;
    const double ev1dsqr12 = rinv(r2 + aeq) * ev1;
    const double eqzz = SQ2(r - qb, aeq) * ev2 + SQ2(r + qb, aeq) * ev2 - ev1dsqr12;
    const double eqxx = rinv(r2 + qb * qb + aeq) * ev1 - ev1dsqr12;
    const double ev2dsqr20 = SQ2(r + da, adq) * ev2;
    const double ev2dsqr22 = SQ2(r - da, adq) * ev2;
    const double ev2dsqr24 = SQ2(r - db, aqd) * ev2;
    const double ev2dsqr26 = SQ2(r + db, aqd) * ev2;
    const double ev2dsqr36 = rinv(r2 + aqq) * ev2;
    const double ev2dsqr39 = rinv(r2 + qa * qa + aqq) * ev2;
    const double ev2dsqr40 = rinv(r2 + qb * qb + aqq) * ev2;
    const double ev3dsqr42 = SQ2(r - qb, aqq) * ev3;
    const double ev3dsqr44 = SQ2(r + qb, aqq) * ev3;
    const double ev3dsqr46 = SQ2(r + qa, aqq) * ev3;
    const double ev3dsqr48 = SQ2(r - qa, aqq) * ev3;
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
    const double qxxqxx = rinv(r2 + (qa - qb) * (qa - qb) + aqq) * ev3 + rinv(r2 + (qa + qb) * (qa + qb) + aqq) * ev3 - ev2dsqr39 -
                          ev2dsqr40 + ev2dsqr36;
    ri[18] = ee + eqxx + qxxe + qxxqxx;
    const double dm = (qa1 - qb1) * (qa1 - qb1), dp = (qa1 + qb1) * (qa1 + qb1);
    ri[19] = rinv((r + qa1 - qb1) * (r + qa1 - qb1) + dm + aqq) * ev3 - rinv((r + qa1 + qb1) * (r + qa1 + qb1) + dm + aqq) * ev3 -
             rinv((r - qa1 - qb1) * (r - qa1 - qb1) + dm + aqq) * ev3 + rinv((r - qa1 + qb1) * (r - qa1 + qb1) + dm + aqq) * ev3 -
             rinv((r + qa1 - qb1) * (r + qa1 - qb1) + dp + aqq) * ev3 + rinv((r + qa1 + qb1) * (r + qa1 + qb1) + dp + aqq) * ev3 +
             rinv((r - qa1 - qb1) * (r - qa1 - qb1) + dp + aqq) * ev3 - rinv((r - qa1 + qb1) * (r - qa1 + qb1) + dp + aqq) * ev3;
    const double qxxqyy = rinv(r2 + qa * qa + qb * qb + aqq) * ev2 - ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
    ri[20] = ee + eqxx + qxxe + qxxqyy;
    ri[21] = (qxxqxx - qxxqyy) * 0.5;
#undef SQ2
}

// Integrals of one pair (i = heavy or lower index, j), written to the store; returns its size.
__device__ void pair_integrals(const DevElem& ei, const DevElem& ej, const double dv[3], double r, double* __restrict__ w) {
    const double inv = 1.0 / r;
    const double n[3] = {-(dv[0] * inv), -(dv[1] * inv), -(dv[2] * inv)};  // frame axis, = -x_ij
    const bool hi = ei.norb == 4, hj = ej.norb == 4;
    if (!hi && !hj) {
        w[0] = rinv(r * r + (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0)) * AM1_EV;
        return;
    }
    // p = I - n n^T
    double p[3][3];
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
        const double ee = rinv(r * r + aee) * AM1_EV;
        const double q6 = rinv(r * r + aqe) * ev1;
        const double r1 = rinv((r + da) * (r + da) + ade) * ev1 - rinv((r - da) * (r - da) + ade) * ev1;
        const double r2 = ee + rinv((r + qa) * (r + qa) + aqe) * ev2 + rinv((r - qa) * (r - qa) + aqe) * ev2 - q6;
        const double r3 = ee + rinv(r * r + qa * qa + aqe) * ev1 - q6;
        w[0] = ee;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            w[(k + 1) * (k + 2) / 2] = r1 * n[k];
#pragma unroll
            for (int l = 0; l <= k; ++l) w[(k + 1) * (k + 2) / 2 + l + 1] = r2 * (n[k] * n[l]) + r3 * p[k][l];
        }
        return;
    }
    double ri[22];
    local_xx(ei, ej, r, ri);
    int idx = 0;
#pragma unroll 1
    for (int kk = 0; kk < 4; ++kk)
        for (int ll = 0; ll <= kk; ++ll)
#pragma unroll
            for (int mm = 0; mm < 4; ++mm)
#pragma unroll
                for (int nn = 0; nn <= mm; ++nn) {
                    const int k = kk - 1, l = ll - 1, m = mm - 1, q = nn - 1;
                    double v;
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
                    w[idx++] = v;
                }
}

__device__ double pair_core_energy(const DevElem& ei, const DevElem& ej, int zi, int zj, double r) {
    const double s = r * AM1_A0;
    const double rho = ei.rho0 + ej.rho0;
    const double gam = rinv(r * r + rho * rho) * AM1_EV;
    const double zz = ei.core_charge * ej.core_charge;
    const bool spi = (zi == 7 || zi == 8) && zj == 1;
    const bool spj = (zj == 7 || zj == 8) && zi == 1;
    double fi = exp(s * (-ei.alpha));
    double fj = exp(s * (-ej.alpha));
    if (spi) fi = s * fi;
    if (spj) fj = s * fj;
    double gi = 0.0, gj = 0.0;
    for (int k = 0; k < ei.ngauss; ++k) {
        const double d = s - ei.gm[k];
        gi += exp(d * d * (-ei.gl[k])) * ei.gk[k];
    }
    for (int k = 0; k < ej.ngauss; ++k) {
        const double d = s - ej.gm[k];
        gj += exp(d * d * (-ej.gl[k])) * ej.gk[k];
    }
    return gam * (fi + fj + 1.0) * zz + (gi + gj) * zz / s;
}

// Locate the molecule and the (i, j) pair of a flat pair index.
__device__ __forceinline__ int find_mol(const long long* __restrict__ prefix, int nmol, long long g) {
    int lo = 0, hi = nmol - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void pair_ij(long long p, int n, int& i, int& j) {
    // rows i hold n-1-i pairs; S(i) = i*n - i(i+1)/2 pairs precede row i
    const double nn = n - 0.5;
    int ii = (int)floor(nn - sqrt(fmax(nn * nn - 2.0 * (double)p, 0.0)));
    ii = max(0, min(ii, n - 2));
    while (ii > 0 && (long long)ii * n - (long long)ii * (ii + 1) / 2 > p) --ii;
    while ((long long)(ii + 1) * n - (long long)(ii + 1) * (ii + 2) / 2 <= p) ++ii;
    i = ii;
    j = (int)(p - ((long long)ii * n - (long long)ii * (ii + 1) / 2)) + ii + 1;
}

__global__ void k_pair_integrals(const MolDesc* __restrict__ mols, int nmol, const long long* __restrict__ pair_prefix,
                                 long long npairs, const DevElem* __restrict__ params, const int* __restrict__ atom_z,
                                 const double* __restrict__ atom_xyz, double* __restrict__ wstore, double* __restrict__ hmat,
                                 double* __restrict__ ecc, int* __restrict__ mol_status) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npairs) return;
    const int m = find_mol(pair_prefix, nmol, g);
    const MolDesc md = mols[m];
    const long long p = g - pair_prefix[m];
    int i, j;
    pair_ij(p, md.natoms, i, j);
    const int ai = md.atom_base + i, aj = md.atom_base + j;
    const int zi = atom_z[ai], zj = atom_z[aj];
    const DevElem& ei = params[md.method * (MAX_Z + 1) + zi];
    const DevElem& ej = params[md.method * (MAX_Z + 1) + zj];
    const double d0 = atom_xyz[3 * aj] - atom_xyz[3 * ai];
    const double d1 = atom_xyz[3 * aj + 1] - atom_xyz[3 * ai + 1];
    const double d2 = atom_xyz[3 * aj + 2] - atom_xyz[3 * ai + 2];
    const double r0 = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    // core-core uses the plain distance (src/repulsion.rs:38-56)
    ecc[md.pair_base + p] = pair_core_energy(ei, ej, zi, zj, r0);
    // integrals see delta/r * r (src/hamiltonian.rs:296-298 -> src/integrals.rs:196-200)
    const double x0 = d0 / r0, x1 = d1 / r0, x2 = d2 / r0;
    const double dv[3] = {x0 * r0, x1 * r0, x2 * r0};
    const double r = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    const int h = md.nheavy, H = md.natoms - md.nheavy;
    long long off;
    if (j < h) {
        off = 100LL * ((long long)i * h - (long long)i * (i + 1) / 2 + (j - i - 1));
    } else if (i < h) {
        off = 100LL * h * (h - 1) / 2 + 10LL * ((long long)i * H + (j - h));
    } else {
        const int i2 = i - h, j2 = j - h;
        off = 100LL * h * (h - 1) / 2 + 10LL * h * H + ((long long)i2 * H - (long long)i2 * (i2 + 1) / 2 + (j2 - i2 - 1));
    }
    pair_integrals(ei, ej, dv, r, wstore + md.w_base + off);
    // resonance block: overlap between the positions pos_i and pos_i + delta
    double S[4][4];
    const double pb0 = atom_xyz[3 * ai] + d0, pb1 = atom_xyz[3 * ai + 1] + d1, pb2 = atom_xyz[3 * ai + 2] + d2;
    const double e0 = pb0 - atom_xyz[3 * ai], e1 = pb1 - atom_xyz[3 * ai + 1], e2 = pb2 - atom_xyz[3 * ai + 2];
    const double rs = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
    if (rs < 1.0e-8) {
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) S[a][b] = a == b ? 1.0 : 0.0;
    } else {
        const double dir[3] = {e0 / rs, e1 / rs, e2 / rs};
        if (!overlap_block(ei, ej, rs, dir, S)) {
            atomicExch(&mol_status[m], 6);  // AM1GPU_UNSUPPORTED
            return;
        }
    }
    const int na = ei.norb, nb = ej.norb, n = md.nao;
    const int oa = i < h ? 4 * i : 4 * h + (i - h);
    const int ob = j < h ? 4 * j : 4 * h + (j - h);
    double* H0 = hmat + md.h_base;
    for (int a = 0; a < na; ++a) {
        const double ba = a == 0 ? ei.beta_s : ei.beta_p;
        for (int b = 0; b < nb; ++b) {
            const double bb = b == 0 ? ej.beta_s : ej.beta_p;
            const double v = 0.5 * (ba + bb) * S[a][b];
            H0[(long long)(oa + a) * n + ob + b] = v;
            H0[(long long)(ob + b) * n + oa + a] = v;
        }
    }
}

// H_core diagonal blocks: U_ss/U_pp plus the electron-core attraction of every other atom,
// -Z_B (mu nu | s_B s_B), gathered per atom in partner order (deterministic).
__global__ void k_core_diag(const MolDesc* __restrict__ mols, const int* __restrict__ atom_mol, int natoms_total,
                            const DevElem* __restrict__ params, const int* __restrict__ atom_z, const double* __restrict__ wstore,
                            double* __restrict__ hmat) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= natoms_total) return;
    const int m = atom_mol[a];
    const MolDesc md = mols[m];
    const int A = a - md.atom_base, N = md.natoms, h = md.nheavy, H = N - h;
    const DevElem& eA = params[md.method * (MAX_Z + 1) + atom_z[a]];
    const double* w = wstore + md.w_base;
    const long long xxsz = 100LL * h * (h - 1) / 2, xhsz = 10LL * h * H;
    double acc[10];
    for (int k = 0; k < 10; ++k) acc[k] = 0.0;
    const bool heavy = A < h;
    for (int B = 0; B < N; ++B) {
        if (B == A) continue;
        const double zb = -params[md.method * (MAX_Z + 1) + atom_z[md.atom_base + B]].core_charge;
        const bool bheavy = B < h;
        if (heavy && bheavy) {
            const int i = min(A, B), j = max(A, B);
            const double* blk = w + 100LL * ((long long)i * h - (long long)i * (i + 1) / 2 + (j - i - 1));
            if (A == i)
                for (int k = 0; k < 10; ++k) acc[k] += zb * blk[k * 10];  // column 0: (A A| s_B s_B)
            else
                for (int k = 0; k < 10; ++k) acc[k] += zb * blk[k];       // row 0
        } else if (heavy) {  // A heavy, B hydrogen
            const double* blk = w + xxsz + 10LL * ((long long)A * H + (B - h));
            for (int k = 0; k < 10; ++k) acc[k] += zb * blk[k];
        } else if (bheavy) {  // A hydrogen, B heavy
            acc[0] += zb * w[xxsz + 10LL * ((long long)B * H + (A - h))];
        } else {
            const int i2 = min(A, B) - h, j2 = max(A, B) - h;
            acc[0] += zb * w[xxsz + xhsz + ((long long)i2 * H - (long long)i2 * (i2 + 1) / 2 + (j2 - i2 - 1))];
        }
    }
    const int n = md.nao;
    double* H0 = hmat + md.h_base;
    if (heavy) {
        const int o = 4 * A;
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = 0; nu < 4; ++nu) {
                const int hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
                double v = acc[hi * (hi + 1) / 2 + lo];
                if (mu == nu) v += mu == 0 ? eA.u_ss : eA.u_pp;
                H0[(long long)(o + mu) * n + o + nu] = v;
            }
    } else {
        const int o = 4 * h + (A - h);
        H0[(long long)o * n + o] = eA.u_ss + acc[0];
    }
}

// Per-molecule sum of the core-core pair energies, in pair order (one block per molecule).
__global__ void k_core_energy(const MolDesc* __restrict__ mols, const double* __restrict__ ecc, MolState* __restrict__ st) {
    const int m = blockIdx.x;
    const MolDesc md = mols[m];
    const long long np = (long long)md.natoms * (md.natoms - 1) / 2;
    __shared__ double part[256];
    double s = 0.0;
    for (long long p = threadIdx.x; p < np; p += blockDim.x) s += ecc[md.pair_base + p];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) st[m].core_ev = part[0];
}

}  // namespace am1

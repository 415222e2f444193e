// am1_oracle.cpp -- CPU FP64 restatement of am1-rs 0.2.3's molecular NDDO SCF single point.
//
// TEST INFRASTRUCTURE ONLY.  This is the oracle the B200 library is checked against; it is
// loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and by
// nothing that ships.  The reference (Rust) cannot be built in this environment (no cargo, no
// crates.io), so this file restates its algorithm step by step, citing the reference file and
// line each function follows, and keeps the reference's constants and summation orders where
// that is cheap.  It is pinned against the reference's own recorded values (heats of
// formation, MOPAC CO2 spectra, parameter values) in tests/test_oracle_golden.py.
//
// Third-party arithmetic the reference delegates, restated here from the published methods:
//   * faer 0.24.4 self_adjoint_eigen (src/linalg.rs:305-306): replaced by Householder
//     tridiagonalisation + implicit-shift QR; parity is on P and eigenvalues, not on the
//     sign or degenerate-subspace rotation of eigenvectors;
//   * faer/gemm matmul (src/linalg.rs:203-224): a plain triple loop.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../include/am1gpu.h"
#include "../am1-rs_b200/csrc/params/nddo_param_table.h"

namespace {

// MOPAC7 model constants, src/constants.rs:13-25.
constexpr double AM1_EV = 27.21;
constexpr double AM1_A0 = 0.529167;
constexpr double EV_TO_KCAL = 23.061;
constexpr double AU_DIPOLE_TO_DEBYE = 2.541746473;

thread_local std::string g_err;

// Threads for the O(n^3) loops inside one molecule (oracle_set_threads; 1 by default).  The
// split is over independent output rows or columns only, so every element is summed in the
// same order as the serial loop and results do not depend on the thread count.  Threads of
// oracle_scf_batch, which already run molecules in parallel, keep these loops serial.
std::atomic<int> g_inner_threads{1};
thread_local bool t_serial = false;

// f(lo, hi) over [0, n) in contiguous chunks; `work` is the loop's operation count, below
// which threads are not worth starting.
template <class F>
void par_for(int n, double work, F&& f) {
    // each thread takes at least ~2e5 operations and 16 rows, so that starting it costs little
    // next to its share (a host with hundreds of threads would otherwise spend its time starting them)
    int nt = std::min(g_inner_threads.load(), (int)std::min(work / 2.0e5, (double)n / 16.0));
    if (nt <= 1 || t_serial) {
        f(0, n);
        return;
    }
    auto chunk = [&](int t) {
        const int lo = (int)((long long)n * t / nt), hi = (int)((long long)n * (t + 1) / nt);
        t_serial = true;
        f(lo, hi);
        t_serial = false;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(chunk, t);
    chunk(0);
    for (auto& t : pool) t.join();
}

// ----------------------------------------------------------------------------------------
// Parameters: src/params.rs:139-330, src/data_tables.rs:53-224
// ----------------------------------------------------------------------------------------
struct Elem {
    int z = 0, n = 0, norb = 0, ngauss = 0;
    double u_ss, u_pp, zeta_s, zeta_p, beta_s, beta_p, g_ss, g_sp, g_pp, g_p2, h_sp, alpha;
    double gk[4], gl[4], gm[4];
    double core_charge, eheat_ev, e_isol, dd, qq, rho0, rho1, rho2;
    bool has_p() const { return norb >= 4; }
};

// f64::powi as LLVM lowers it for small constant exponents (repeated squaring).
inline double powi(double x, int n) {
    double r = 1.0, b = x;
    while (n > 0) {
        if (n & 1) r = r * b;
        n >>= 1;
        if (n) b = b * b;
    }
    return r;
}

// src/params.rs:266-271
double dd_charge_sep(int n, double zs, double zp) {
    double nf = n;
    return (2.0 * nf + 1.0) * std::pow(4.0 * zs * zp, nf + 0.5) / std::pow(zs + zp, 2.0 * nf + 2.0) /
           std::sqrt(3.0);
}
// src/params.rs:274-277
double qq_charge_sep(int n, double zp) {
    double nf = n;
    return std::sqrt((4.0 * nf * nf + 6.0 * nf + 2.0) / 20.0) / zp;
}
// src/params.rs:283-305 (secant solve, 30 steps)
double additive_rho1(double hsp_ev, double d1) {
    double hsp = hsp_ev / AM1_EV;
    auto g = [&](double d) { return 0.5 * d - 0.5 / std::sqrt(4.0 * d1 * d1 + 1.0 / (d * d)); };
    double a = std::pow(std::fabs(hsp) / (d1 * d1), 1.0 / 3.0);
    if (hsp < 0.0) a = -a;
    double b = a + 0.04;
    for (int i = 0; i < 30; ++i) {
        double ga = g(a), gb = g(b);
        double c = std::fabs(gb - ga) > 1.0e-16 ? a + (b - a) * (hsp - ga) / (gb - ga) : b;
        a = b;
        b = c;
    }
    return 0.5 / b;
}
// src/params.rs:308-330
double additive_rho2(double hpp_ev, double d2) {
    double hpp = hpp_ev / AM1_EV;
    auto g = [&](double q) {
        return 0.25 * q - 0.5 / std::sqrt(4.0 * d2 * d2 + 1.0 / (q * q)) +
               0.25 / std::sqrt(8.0 * d2 * d2 + 1.0 / (q * q));
    };
    double a = std::pow(std::fabs(hpp) / (3.0 * powi(d2, 4)), 0.2);
    if (hpp < 0.0) a = -a;
    double b = a + 0.04;
    for (int i = 0; i < 30; ++i) {
        double ga = g(a), gb = g(b);
        double c = std::fabs(gb - ga) > 1.0e-16 ? a + (b - a) * (hpp - ga) / (gb - ga) : b;
        a = b;
        b = c;
    }
    return 0.5 / b;
}

// Average-of-configuration coefficients, src/data_tables.rs:166-216
double gssc(int z) { double n = NDDO_NS[z]; return n * (n - 1.0) / 2.0; }
double gspc(int z) { return NDDO_NS[z] * NDDO_NP[z]; }
double hspc(int z) { int n = (int)NDDO_NP[z]; return n == 6 ? 0.0 : -(double)n; }
double gp2c(int z) {
    switch ((int)NDDO_NP[z]) { case 2: return 1.5; case 3: return 4.5; case 4: return 6.5; case 5: return 10.0; default: return 0.0; }
}
double gppc(int z) {
    switch ((int)NDDO_NP[z]) { case 2: return -0.5; case 3: return -1.5; case 4: return -0.5; default: return 0.0; }
}

struct ParamSet {
    Elem by_z[NDDO_MAX_Z + 1];
    bool present[NDDO_MAX_Z + 1] = {};
    const char* name = "AM1";
};

// src/params.rs:139-263 (one row of the table -> Am1Element)
Elem derive(const nddo_raw_element& r) {
    Elem e;
    e.z = r.z;
    e.u_ss = r.raw[0]; e.u_pp = r.raw[1]; e.zeta_s = r.raw[2]; e.zeta_p = r.raw[3];
    e.beta_s = r.raw[4]; e.beta_p = r.raw[5]; e.g_ss = r.raw[6]; e.g_sp = r.raw[7];
    e.g_pp = r.raw[8]; e.g_p2 = r.raw[9]; e.h_sp = r.raw[10]; e.alpha = r.raw[11];
    e.norb = e.zeta_p > 0.0 ? 4 : 1;
    e.ngauss = 0;
    for (int k = 0; k < 4; ++k) {
        double K = r.gauss[3 * k], L = r.gauss[3 * k + 1], M = r.gauss[3 * k + 2];
        if (K != 0.0 || L != 0.0) {
            e.gk[e.ngauss] = K; e.gl[e.ngauss] = L; e.gm[e.ngauss] = M; ++e.ngauss;
        }
    }
    e.n = NDDO_QN[e.z];
    if (e.norb == 4) {
        e.dd = dd_charge_sep(e.n, e.zeta_s, e.zeta_p);
        e.qq = qq_charge_sep(e.n, e.zeta_p);
        double hpp = std::max(0.5 * (e.g_pp - e.g_p2), 0.1);
        e.rho1 = additive_rho1(e.h_sp, e.dd);
        e.rho2 = additive_rho2(hpp, e.qq);
    } else {
        e.dd = e.qq = e.rho1 = e.rho2 = 0.0;
    }
    e.rho0 = 0.5 * AM1_EV / e.g_ss;
    int z = e.z;
    e.e_isol = e.u_ss * NDDO_NS[z] + e.u_pp * NDDO_NP[z] + e.g_ss * gssc(z) + e.g_pp * gppc(z) +
               e.g_sp * gspc(z) + e.g_p2 * gp2c(z) + e.h_sp * hspc(z);
    e.core_charge = NDDO_NS[z] + NDDO_NP[z];
    e.eheat_ev = NDDO_EHEAT_KCAL[z] / EV_TO_KCAL;
    return e;
}

const ParamSet& params_for(int method) {
    static ParamSet sets[2];
    static bool once = [] {
        const nddo_raw_element* tabs[2] = {NDDO_AM1_RAW, NDDO_RM1_RAW};
        size_t counts[2] = {sizeof(NDDO_AM1_RAW) / sizeof(NDDO_AM1_RAW[0]),
                            sizeof(NDDO_RM1_RAW) / sizeof(NDDO_RM1_RAW[0])};
        for (int m = 0; m < 2; ++m) {
            sets[m].name = m == 0 ? "AM1" : "RM1";
            for (size_t i = 0; i < counts[m]; ++i) {
                Elem e = derive(tabs[m][i]);
                sets[m].by_z[e.z] = e;
                sets[m].present[e.z] = true;
            }
        }
        return true;
    }();
    (void)once;
    return sets[method == AM1GPU_METHOD_RM1 ? 1 : 0];
}

// ----------------------------------------------------------------------------------------
// Dense row-major matrix helpers
// ----------------------------------------------------------------------------------------
using Mat = std::vector<double>;

// src/linalg.rs:237-255: eight independent partial sums, then the lane total, then the tail.
double frobenius_dot(const Mat& a, const Mat& b) {
    const size_t n = std::min(a.size(), b.size());
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t chunks = n / 8;
    for (size_t c = 0; c < chunks; ++c)
        for (int l = 0; l < 8; ++l) acc[l] += a[c * 8 + l] * b[c * 8 + l];
    double total = 0.0;
    for (int l = 0; l < 8; ++l) total += acc[l];
    for (size_t k = chunks * 8; k < n; ++k) total += a[k] * b[k];
    return total;
}

// ----------------------------------------------------------------------------------------
// STO diatomic overlap, src/overlap.rs
// ----------------------------------------------------------------------------------------
// A_k(x) = int_1^inf t^k e^{-xt} dt, k = 0..12  (src/overlap.rs:357-368)
void aintgs(double x, double a[13]) {
    for (int i = 0; i < 13; ++i) a[i] = 0.0;
    if (std::fabs(x) < 1.0e-12) return;
    double inv = 1.0 / x;
    a[0] = std::exp(-x) * inv;
    for (int i = 1; i < 13; ++i) a[i] = a[0] + a[i - 1] * inv * (double)i;
}

// B_k(x) = int_{-1}^{1} t^k e^{-xt} dt, k = 0..12 (src/overlap.rs:455-500): closed form
// above |x| = 5, otherwise the everywhere-convergent Taylor series.
void bintgs(double x, double b[13]) {
    if (std::fabs(x) > 5.0) {
        double inv = 1.0 / x;
        double tx = std::exp(x) * inv;
        double tmx = std::exp(-x) * inv * (-1.0);
        b[0] = tx + tmx;
        for (int i = 1; i < 13; ++i) {
            double sign = (i % 2 == 0) ? 1.0 : -1.0;
            b[i] = tx * sign + tmx + b[i - 1] * inv * (double)i;
        }
        return;
    }
    for (int i = 0; i < 13; ++i) b[i] = 0.0;
    double term = 1.0, magnitude = 1.0, absx = std::fabs(x);
    for (int n = 0; n < 64; ++n) {
        for (int k = n % 2; k < 13; k += 2) b[k] = b[k] + term * (2.0 / (double)(k + n + 1));
        term = term * x * (-1.0 / (double)(n + 1));
        magnitude *= absx / (double)(n + 1);
        if (n >= 4 && magnitude < 1.0e-18) break;
    }
}

// src/overlap_numeric.rs:172-213: Legendre P_n and P_n' by the three-term recurrence, and the
// Gauss-Legendre rule on [-1, 1] by Newton iteration from the Chebyshev guess.
void legendre_p_dp(int n, double x, double& p, double& dp) {
    double p0 = 1.0, p1 = x;
    if (n == 0) {
        p = 1.0;
        dp = 0.0;
        return;
    }
    for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
    }
    p = p1;
    dp = n * (x * p1 - p0) / (x * x - 1.0);
}

struct GaussRule {
    std::vector<double> x, w;
};

GaussRule gauss_legendre(int n) {
    GaussRule g{std::vector<double>(n), std::vector<double>(n)};
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5)), p, dp;
        for (int it = 0; it < 100; ++it) {
            legendre_p_dp(n, x, p, dp);
            const double dx = -p / dp;
            x += dx;
            if (std::fabs(dx) < 1.0e-15) break;
        }
        legendre_p_dp(n, x, p, dp);
        const double w = 2.0 / ((1.0 - x * x) * dp * dp);
        g.x[i] = -x;
        g.x[n - 1 - i] = x;
        g.w[i] = w;
        g.w[n - 1 - i] = w;
    }
    return g;
}

// src/overlap_numeric.rs:50-123: <n_a l_a m; z_a | n_b l_b m; z_b> in the local frame (b at +z),
// prolate-spheroidal quadrature with 48 (xi) x 40 (eta) Gauss-Legendre nodes.
double overlap_sto(int na, double za, int la, int m, int nb, double zb, int lb, double r) {
    double c;
    if (la == 0 && lb == 0) c = 0.5;
    else if ((la == 1 && lb == 0 && m == 0) || (la == 0 && lb == 1 && m == 0)) c = std::sqrt(3.0) / 2.0;
    else if (la == 1 && lb == 1 && m == 0) c = 1.5;
    else if (la == 1 && lb == 1 && m == 1) c = 0.75;
    else return 0.0;
    auto norm = [](int n, double zeta) {
        double f = 1.0;
        for (int k = 2; k <= 2 * n; ++k) f *= k;
        return std::pow(2.0 * zeta, n + 0.5) / std::sqrt(std::max(f, 1.0));
    };
    static const GaussRule xr = gauss_legendre(48), er = gauss_legendre(40);
    const double hr = 0.5 * r, p = (za + zb) * hr;
    const double xi_max = 1.0 + 60.0 / std::max(p, 0.05);
    const double xi_mid = 0.5 * (1.0 + xi_max), xi_half = 0.5 * (xi_max - 1.0);
    double sum = 0.0;
    for (int i = 0; i < 48; ++i) {
        const double xi = xi_mid + xi_half * xr.x[i];
        for (int j = 0; j < 40; ++j) {
            const double eta = er.x[j];
            const double ra = hr * (xi + eta), rb = hr * (xi - eta);
            if (ra <= 0.0 || rb <= 0.0) continue;
            const double cos_a = (1.0 + xi * eta) / (xi + eta), cos_b = (xi * eta - 1.0) / (xi - eta);
            const double ang_a = la == 0 ? 1.0 : (m == 0 ? cos_a : std::sqrt(std::max(1.0 - cos_a * cos_a, 0.0)));
            const double ang_b = lb == 0 ? 1.0 : (m == 0 ? cos_b : std::sqrt(std::max(1.0 - cos_b * cos_b, 0.0)));
            const double radial = std::pow(ra, na - 1) * std::pow(rb, nb - 1) * std::exp(ra * (-za) - rb * zb);
            sum += radial * (xi_half * xr.w[i] * er.w[j] * ang_a * ang_b * (xi * xi - eta * eta));
        }
    }
    return hr * hr * hr * sum * (norm(na, za) * norm(nb, zb) * c);
}

// src/overlap_numeric.rs:22-42: the five local overlaps, in the analytic kernel's signs.
void overlap_locals_numeric(const Elem& ea, const Elem& eb, double r, double s[5]) {
    s[0] = overlap_sto(ea.n, ea.zeta_s, 0, 0, eb.n, eb.zeta_s, 0, r);
    s[1] = overlap_sto(ea.n, ea.zeta_p, 1, 0, eb.n, eb.zeta_s, 0, r);
    s[2] = -overlap_sto(ea.n, ea.zeta_s, 0, 0, eb.n, eb.zeta_p, 1, r);
    s[3] = -overlap_sto(ea.n, ea.zeta_p, 1, 0, eb.n, eb.zeta_p, 1, r);
    s[4] = overlap_sto(ea.n, ea.zeta_p, 1, 1, eb.n, eb.zeta_p, 1, r);
}

// src/overlap.rs:120-296, local-frame overlaps (s111, s211, s121, s221, s222); ea.n >= eb.n.
bool overlap_locals(const Elem& ea, const Elem& eb, double r, double s[5]) {
    int jcall;
    if (ea.n == 1 && eb.n == 1) jcall = 2;
    else if (ea.n == 2 && eb.n == 1) jcall = 3;
    else if (ea.n == 2 && eb.n == 2) jcall = 4;
    else if (ea.n == 3 && eb.n == 1) jcall = 431;
    else if (ea.n == 3 && eb.n == 2) jcall = 5;
    else if (ea.n == 3 && eb.n == 3) jcall = 6;
    else {  // n >= 4: the numerical quadrature (src/overlap.rs:128-165)
        overlap_locals_numeric(ea, eb, r, s);
        return true;
    }
    const double za[2] = {ea.zeta_s, ea.zeta_p}, zb[2] = {eb.zeta_s, eb.zeta_p};
    double a111[13], b111[13], a211[13], b211[13], a121[13], b121[13], a22[13], b22[13];
    aintgs(r * (0.5 * (za[0] + zb[0])), a111);
    bintgs(r * (0.5 * (za[0] - zb[0])), b111);
    aintgs(r * (0.5 * (za[1] + zb[0])), a211);
    bintgs(r * (0.5 * (za[1] - zb[0])), b211);
    aintgs(r * (0.5 * (za[0] + zb[1])), a121);
    bintgs(r * (0.5 * (za[0] - zb[1])), b121);
    aintgs(r * (0.5 * (za[1] + zb[1])), a22);
    bintgs(r * (0.5 * (za[1] - zb[1])), b22);
    double s111 = 0, s211 = 0, s121 = 0, s221 = 0, s222 = 0;
    const double sq3 = std::sqrt(3.0);
    switch (jcall) {
    case 2:
        s111 = std::pow(r * r * (za[0] * zb[0]), 1.5) * (a111[2] * b111[0] - b111[2] * a111[0]) / 4.0;
        break;
    case 3:
        s111 = powi(r, 4) * (std::pow(zb[0], 1.5) * std::pow(za[0], 2.5)) *
               (a111[3] * b111[0] - b111[3] * a111[0] + a111[2] * b111[1] - b111[2] * a111[1]) / (sq3 * 8.0);
        s211 = powi(r, 4) * (std::pow(zb[0], 1.5) * std::pow(za[1], 2.5)) *
               (a211[2] * b211[0] - b211[2] * a211[0] + a211[3] * b211[1] - b211[3] * a211[1]) / 8.0;
        break;
    case 4: {
        s111 = powi(r, 5) * std::pow(zb[0] * za[0], 2.5) *
               (a111[4] * b111[0] + b111[4] * a111[0] - a111[2] * b111[2] * 2.0) / 48.0;
        s211 = powi(r, 5) * std::pow(zb[0] * za[1], 2.5) *
               (a211[3] * (b211[0] - b211[2]) - a211[1] * (b211[2] - b211[4]) + b211[3] * (a211[0] - a211[2]) -
                b211[1] * (a211[2] - a211[4])) / (16.0 * sq3);
        s121 = powi(r, 5) * std::pow(zb[1] * za[0], 2.5) *
               (a121[3] * (b121[0] - b121[2]) - a121[1] * (b121[2] - b121[4]) - b121[3] * (a121[0] - a121[2]) +
                b121[1] * (a121[2] - a121[4])) / (16.0 * sq3);
        double w = powi(r, 5) * std::pow(zb[1] * za[1], 2.5) / 16.0;
        s221 = -(w * (b22[2] * (a22[4] + a22[0]) - a22[2] * (b22[4] + b22[0])));
        s222 = w * (a22[4] * (b22[0] - b22[2]) - b22[4] * (a22[0] - a22[2]) - a22[2] * b22[0] + b22[2] * a22[0]) * 0.5;
        break;
    }
    case 431:
        s111 = powi(r, 5) * (std::pow(zb[0], 1.5) * std::pow(za[0], 3.5)) *
               (a111[4] * b111[0] + b111[1] * a111[3] * 2.0 - a111[1] * b111[3] * 2.0 - b111[4] * a111[0]) /
               (std::sqrt(10.0) * 24.0);
        s211 = powi(r, 5) * (std::pow(zb[0], 1.5) * std::pow(za[1], 3.5)) *
               (a211[3] * (b211[0] + b211[2]) - a211[1] * (b211[4] + b211[2]) + b211[1] * (a211[2] + a211[4]) -
                b211[3] * (a211[2] + a211[0])) / (8.0 * std::sqrt(30.0));
        break;
    case 5:
        s111 = powi(r, 6) * (std::pow(zb[0], 2.5) * std::pow(za[0], 3.5)) *
               (a111[5] * b111[0] + b111[1] * a111[4] - b111[2] * a111[3] * 2.0 - a111[2] * b111[3] * 2.0 +
                b111[4] * a111[1] + b111[5] * a111[0]) / (std::sqrt(30.0) * 48.0);
        s211 = powi(r, 6) * (std::pow(zb[0], 2.5) * std::pow(za[1], 3.5)) *
               (a211[4] * b211[0] + b211[1] * a211[5] - b211[3] * a211[3] * 2.0 - a211[2] * b211[2] * 2.0 +
                a211[1] * b211[5] + a211[0] * b211[4]) / (48.0 * std::sqrt(10.0));
        s121 = powi(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[0], 3.5)) *
               ((a121[4] * b121[0] - a121[5] * b121[1]) + (a121[3] * b121[1] - a121[4] * b121[2]) * 2.0 -
                (a121[1] * b121[3] - a121[2] * b121[4]) * 2.0 - (a121[0] * b121[4] - a121[1] * b121[5])) /
               (48.0 * std::sqrt(10.0));
        s221 = powi(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[1], 3.5)) *
               ((a22[3] * b22[0] - a22[5] * b22[2]) + (a22[2] * b22[1] - a22[4] * b22[3]) -
                (a22[1] * b22[2] - a22[3] * b22[4]) - (a22[0] * b22[3] - a22[2] * b22[5])) / (16.0 * std::sqrt(30.0));
        s222 = powi(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[1], 3.5)) *
               ((a22[5] - a22[3]) * (b22[0] - b22[2]) + (a22[4] - a22[2]) * (b22[1] - b22[3]) -
                (a22[3] - a22[1]) * (b22[2] - b22[4]) - (a22[2] - a22[0]) * (b22[3] - b22[5])) /
               (32.0 * std::sqrt(30.0));
        break;
    case 6:
        s111 = powi(r, 7) * std::pow(zb[0] * za[0], 3.5) *
               (a111[6] * b111[0] - b111[2] * a111[4] * 3.0 + a111[2] * b111[4] * 3.0 - a111[0] * b111[6]) / 1440.0;
        s211 = powi(r, 7) * std::pow(zb[0] * za[1], 3.5) *
               ((a211[5] * b211[0] + a211[6] * b211[1]) + (-a211[4] * b211[1] - a211[5] * b211[2]) -
                (a211[3] * b211[2] + a211[4] * b211[3]) * 2.0 - (-a211[2] * b211[3] - a211[3] * b211[4]) * 2.0 +
                (a211[1] * b211[4] + a211[2] * b211[5]) + (-a211[0] * b211[5] - a211[1] * b211[6])) / (480.0 * sq3);
        s121 = powi(r, 7) * std::pow(zb[1] * za[0], 3.5) *
               ((a121[5] * b121[0] - a121[6] * b121[1]) + (a121[4] * b121[1] - a121[5] * b121[2]) -
                (a121[3] * b121[2] - a121[4] * b121[3]) * 2.0 - (a121[2] * b121[3] - a121[3] * b121[4]) * 2.0 +
                (a121[1] * b121[4] - a121[2] * b121[5]) + (a121[0] * b121[5] - a121[1] * b121[6])) / (480.0 * sq3);
        s221 = powi(r, 7) * (std::pow(zb[1], 3.5) * std::pow(za[1], 3.5)) *
               ((a22[4] * b22[0] - a22[6] * b22[2]) - (a22[2] * b22[2] - a22[4] * b22[4]) * 2.0 +
                (a22[0] * b22[4] - a22[2] * b22[6])) / 480.0;
        s222 = powi(r, 7) * (std::pow(zb[1], 3.5) * std::pow(za[1], 3.5)) *
               ((a22[6] - a22[4]) * (b22[0] - b22[2]) - (a22[4] - a22[2]) * (b22[2] - b22[4]) * 2.0 +
                (a22[2] - a22[0]) * (b22[4] - b22[6])) / 960.0;
        break;
    }
    s[0] = s111; s[1] = s211; s[2] = s121; s[3] = s221; s[4] = s222;
    return true;
}

// Transverse projector p = I - n n^T (src/integrals.rs:116-125).
void transverse_projector(const double n[3], double p[3][3]) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double nn = -(n[a] * n[b]);
            p[a][b] = (a == b) ? nn + 1.0 : nn;
        }
}

// src/overlap.rs:301-322
void build_di(const double s[5], const double dir[3], double di[4][4]) {
    double p[3][3];
    transverse_projector(dir, p);
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) di[i][j] = 0.0;
    di[0][0] = s[0];
    for (int a = 0; a < 3; ++a) {
        di[1 + a][0] = s[1] * dir[a];
        di[0][1 + a] = -s[2] * dir[a];
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) di[1 + a][1 + b] = -s[3] * (dir[a] * dir[b]) + s[4] * p[a][b];
}

// src/overlap.rs:16-40: block S[i-orbital][j-orbital] in the global frame.
bool diatom_overlap(const Elem& ei, const double pi[3], const Elem& ej, const double pj[3], double out[4][4]) {
    double d[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
    double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (r < 1.0e-8) {
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) out[i][j] = (i == j) ? 1.0 : 0.0;
        return true;
    }
    double x[3] = {d[0] / r, d[1] / r, d[2] / r};
    double s[5];
    double di[4][4];
    if (ei.n >= ej.n) {
        if (!overlap_locals(ei, ej, r, s)) return false;
        build_di(s, x, di);
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) out[i][j] = di[i][j];
    } else {
        if (!overlap_locals(ej, ei, r, s)) return false;
        double nx[3] = {x[0] * -1.0, x[1] * -1.0, x[2] * -1.0};
        build_di(s, nx, di);
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) out[i][j] = di[j][i];
    }
    return true;
}

// ----------------------------------------------------------------------------------------
// Two-centre two-electron integrals, src/integrals.rs
// ----------------------------------------------------------------------------------------
const int PACK[4][4] = {{0, 1, 3, 6}, {1, 2, 4, 7}, {3, 4, 5, 8}, {6, 7, 8, 9}};  // integrals.rs:23

struct PairTE {
    int na = 1, nb = 1, wcols = 1;
    double w[100];
    double e1b[4][4], e2a[4][4];
};

inline double rs(double x) { return 1.0 / std::sqrt(x); }  // (x).sqrt().recip()

// src/integrals.rs:309-329
void local_xh(const Elem& ei, const Elem& ej, double r, double ri[4]) {
    const double ev1 = AM1_EV / 2.0, ev2 = AM1_EV / 4.0;
    double da = ei.dd, qa = ei.qq * 2.0;
    double aee = powi(ei.rho0 + ej.rho0, 2), ade = powi(ei.rho1 + ej.rho0, 2), aqe = powi(ei.rho2 + ej.rho0, 2);
    double ee = rs(r * r + aee) * AM1_EV;
    double ev1dsqr6 = rs(r * r + aqe) * ev1;
    ri[0] = ee;
    ri[1] = rs((r + da) * (r + da) + ade) * ev1 - rs((r - da) * (r - da) + ade) * ev1;
    ri[2] = ee + rs((r + qa) * (r + qa) + aqe) * ev2 + rs((r - qa) * (r - qa) + aqe) * ev2 - ev1dsqr6;
    ri[3] = ee + rs(r * r + qa * qa + aqe) * ev1 - ev1dsqr6;
}

// src/integrals.rs:331-484 (the 22 local-frame heavy-heavy integrals)
void local_xx(const Elem& ei, const Elem& ej, double r, double ri[22]) {
    const double ev1 = AM1_EV / 2.0, ev2 = AM1_EV / 4.0, ev3 = AM1_EV / 8.0, ev4 = AM1_EV / 16.0;
    double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0, qa1 = ei.qq, qb1 = ej.qq;
    double aee = powi(ei.rho0 + ej.rho0, 2), ade = powi(ei.rho1 + ej.rho0, 2), aqe = powi(ei.rho2 + ej.rho0, 2);
    double aed = powi(ei.rho0 + ej.rho1, 2), aeq = powi(ei.rho0 + ej.rho2, 2), axx = powi(ei.rho1 + ej.rho1, 2);
    double adq = powi(ei.rho1 + ej.rho2, 2), aqd = powi(ei.rho2 + ej.rho1, 2), aqq = powi(ei.rho2 + ej.rho2, 2);
    auto g = [](double x, double c) { return rs(x + c); };
    auto sq2 = [](double a, double c) { return rs(a * a + c); };
    double ee = rs(r * r + aee) * AM1_EV;
    double dze = sq2(r - da, ade) * ev1 - sq2(r + da, ade) * ev1;
    double ev1dsqr6 = rs(r * r + aqe) * ev1;
    double qzze = sq2(r - qa, aqe) * ev2 + sq2(r + qa, aqe) * ev2 - ev1dsqr6;
    double qxxe = g(r * r + qa * qa, aqe) * ev1 - ev1dsqr6;
    double edz = sq2(r + db, aed) * ev1 - sq2(r - db, aed) * ev1;
    double ev1dsqr12 = rs(r * r + aeq) * ev1;
    double eqzz = sq2(r - qb, aeq) * ev2 + sq2(r + qb, aeq) * ev2 - ev1dsqr12;
    double eqxx = g(r * r + qb * qb, aeq) * ev1 - ev1dsqr12;
    double ev2dsqr20 = sq2(r + da, adq) * ev2;
    double ev2dsqr22 = sq2(r - da, adq) * ev2;
    double ev2dsqr24 = sq2(r - db, aqd) * ev2;
    double ev2dsqr26 = sq2(r + db, aqd) * ev2;
    double ev2dsqr36 = rs(r * r + aqq) * ev2;
    double ev2dsqr39 = g(r * r + qa * qa, aqq) * ev2;
    double ev2dsqr40 = g(r * r + qb * qb, aqq) * ev2;
    double ev3dsqr42 = sq2(r - qb, aqq) * ev3;
    double ev3dsqr44 = sq2(r + qb, aqq) * ev3;
    double ev3dsqr46 = sq2(r + qa, aqq) * ev3;
    double ev3dsqr48 = sq2(r - qa, aqq) * ev3;
    ri[0] = ee;
    ri[1] = -dze;
    ri[2] = ee + qzze;
    ri[3] = ee + qxxe;
    ri[4] = -edz;
    ri[5] = sq2(r + da - db, axx) * ev2 + sq2(r - da + db, axx) * ev2 - sq2(r - da - db, axx) * ev2 -
            sq2(r + da + db, axx) * ev2;
    ri[6] = g(r * r + (da - db) * (da - db), axx) * ev1 - g(r * r + (da + db) * (da + db), axx) * ev1;
    ri[7] = -edz + sq2(r + qa - db, aqd) * ev3 - sq2(r + qa + db, aqd) * ev3 + sq2(r - qa - db, aqd) * ev3 -
            sq2(r - qa + db, aqd) * ev3 - ev2dsqr24 + ev2dsqr26;
    ri[8] = -edz - ev2dsqr24 + g((r - db) * (r - db) + qa * qa, aqd) * ev2 + ev2dsqr26 -
            g((r + db) * (r + db) + qa * qa, aqd) * ev2;
    ri[9] = g((qa1 - db) * (qa1 - db) + (r + qa1) * (r + qa1), aqd) * ev2 -
            g((qa1 - db) * (qa1 - db) + (r - qa1) * (r - qa1), aqd) * ev2 -
            g((qa1 + db) * (qa1 + db) + (r + qa1) * (r + qa1), aqd) * ev2 +
            g((qa1 + db) * (qa1 + db) + (r - qa1) * (r - qa1), aqd) * ev2;
    ri[10] = ee + eqzz;
    ri[11] = ee + eqxx;
    ri[12] = -dze + sq2(r + da - qb, adq) * ev3 - sq2(r - da - qb, adq) * ev3 + sq2(r + da + qb, adq) * ev3 -
             sq2(r - da + qb, adq) * ev3 + ev2dsqr22 - ev2dsqr20;
    ri[13] = -dze - ev2dsqr20 + g((r + da) * (r + da) + qb * qb, adq) * ev2 + ev2dsqr22 -
             g((r - da) * (r - da) + qb * qb, adq) * ev2;
    ri[14] = g((da - qb1) * (da - qb1) + (r - qb1) * (r - qb1), adq) * ev2 -
             g((da - qb1) * (da - qb1) + (r + qb1) * (r + qb1), adq) * ev2 -
             g((da + qb1) * (da + qb1) + (r - qb1) * (r - qb1), adq) * ev2 +
             g((da + qb1) * (da + qb1) + (r + qb1) * (r + qb1), adq) * ev2;
    ri[15] = ee + eqzz + qzze + sq2(r + qa - qb, aqq) * ev4 + sq2(r + qa + qb, aqq) * ev4 +
             sq2(r - qa - qb, aqq) * ev4 + sq2(r - qa + qb, aqq) * ev4 - ev3dsqr48 - ev3dsqr46 - ev3dsqr42 -
             ev3dsqr44 + ev2dsqr36;
    ri[16] = ee + eqzz + qxxe + g((r - qb) * (r - qb) + qa * qa, aqq) * ev3 +
             g((r + qb) * (r + qb) + qa * qa, aqq) * ev3 - ev3dsqr42 - ev3dsqr44 - ev2dsqr39 + ev2dsqr36;
    ri[17] = ee + eqxx + qzze + g((r + qa) * (r + qa) + qb * qb, aqq) * ev3 +
             g((r - qa) * (r - qa) + qb * qb, aqq) * ev3 - ev3dsqr46 - ev3dsqr48 - ev2dsqr40 + ev2dsqr36;
    double qxxqxx = g(r * r + (qa - qb) * (qa - qb), aqq) * ev3 + g(r * r + (qa + qb) * (qa + qb), aqq) * ev3 -
                    ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
    ri[18] = ee + eqxx + qxxe + qxxqxx;
    double d1 = (qa1 - qb1) * (qa1 - qb1), d2 = (qa1 + qb1) * (qa1 + qb1);
    ri[19] = g((r + qa1 - qb1) * (r + qa1 - qb1) + d1, aqq) * ev3 -
             g((r + qa1 + qb1) * (r + qa1 + qb1) + d1, aqq) * ev3 -
             g((r - qa1 - qb1) * (r - qa1 - qb1) + d1, aqq) * ev3 +
             g((r - qa1 + qb1) * (r - qa1 + qb1) + d1, aqq) * ev3 -
             g((r + qa1 - qb1) * (r + qa1 - qb1) + d2, aqq) * ev3 +
             g((r + qa1 + qb1) * (r + qa1 + qb1) + d2, aqq) * ev3 +
             g((r - qa1 - qb1) * (r - qa1 - qb1) + d2, aqq) * ev3 -
             g((r - qa1 + qb1) * (r - qa1 + qb1) + d2, aqq) * ev3;
    double qxxqyy = g(r * r + qa * qa + qb * qb, aqq) * ev2 - ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
    ri[20] = ee + eqxx + qxxe + qxxqyy;
    ri[21] = (qxxqxx - qxxqyy) * 0.5;
}

// src/integrals.rs:487-497
void build_wxh(const double ri[4], const double n[3], double p[3][3], double w[10]) {
    w[PACK[0][0]] = ri[0];
    for (int k = 0; k < 3; ++k) w[PACK[k + 1][0]] = ri[1] * n[k];
    for (int k = 0; k < 3; ++k)
        for (int l = 0; l <= k; ++l) w[PACK[k + 1][l + 1]] = ri[2] * (n[k] * n[l]) + ri[3] * p[k][l];
}

// src/integrals.rs:515-569 (frame-free rotation of the 22 local integrals)
void rotate_xx(const double ri[22], const double n[3], double p[3][3], double w[100]) {
    int idx = 0;
    for (int kk = 0; kk < 4; ++kk)
        for (int ll = 0; ll <= kk; ++ll)
            for (int mm = 0; mm < 4; ++mm)
                for (int nn = 0; nn <= mm; ++nn) {
                    int k = kk - 1, l = ll - 1, m = mm - 1, q = nn - 1;
                    double val;
                    if (kk == 0) {
                        if (mm == 0) val = ri[0];
                        else if (nn == 0) val = ri[4] * n[m];
                        else val = ri[10] * (n[m] * n[q]) + ri[11] * p[m][q];
                    } else if (ll == 0) {
                        if (mm == 0) val = ri[1] * n[k];
                        else if (nn == 0) val = ri[5] * (n[k] * n[m]) + ri[6] * p[k][m];
                        else
                            val = ri[12] * (n[k] * n[m] * n[q]) + ri[13] * (p[m][q] * n[k]) +
                                  ri[14] * (p[k][q] * n[m] + p[k][m] * n[q]);
                    } else if (mm == 0) {
                        val = ri[2] * (n[k] * n[l]) + ri[3] * p[k][l];
                    } else if (nn == 0) {
                        val = ri[7] * (n[k] * n[l] * n[m]) + ri[8] * (p[k][l] * n[m]) +
                              ri[9] * (p[l][m] * n[k] + p[k][m] * n[l]);
                    } else {
                        val = ri[15] * (n[k] * n[l] * n[m] * n[q]) + ri[16] * (p[k][l] * n[m] * n[q]) +
                              ri[17] * (p[m][q] * n[k] * n[l]) +
                              ri[19] * (n[k] * (p[l][q] * n[m] + p[l][m] * n[q]) + n[l] * (p[k][q] * n[m] + p[k][m] * n[q])) +
                              ri[20] * (p[k][l] * p[m][q]) + ri[21] * (p[k][m] * p[l][q] + p[k][q] * p[l][m]);
                    }
                    w[idx++] = val;
                }
}

// src/integrals.rs:207-277; dvec = R_j - R_i (Bohr).
void pair_two_electron(const Elem& ei, const Elem& ej, const double dvec[3], PairTE& te) {
    double r = std::sqrt(dvec[0] * dvec[0] + dvec[1] * dvec[1] + dvec[2] * dvec[2]);
    double inv = 1.0 / r;
    double xij[3] = {dvec[0] * inv, dvec[1] * inv, dvec[2] * inv};
    for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) te.e1b[a][b] = te.e2a[a][b] = 0.0;
    double axis[3] = {-xij[0], -xij[1], -xij[2]};
    double proj[3][3];
    transverse_projector(axis, proj);
    if (!ei.has_p() && !ej.has_p()) {
        double aee = powi(ei.rho0 + ej.rho0, 2);
        double ee = rs(r * r + aee) * AM1_EV;
        te.na = te.nb = 1; te.wcols = 1;
        te.w[0] = ee;
        te.e1b[0][0] = ee * (-ej.core_charge);
        te.e2a[0][0] = ee * (-ei.core_charge);
        return;
    }
    if (ei.has_p() && !ej.has_p()) {
        double ri[4];
        local_xh(ei, ej, r, ri);
        double wxh[10];
        build_wxh(ri, axis, proj, wxh);
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) te.e1b[a][b] = wxh[PACK[a][b]] * (-ej.core_charge);
        te.e2a[0][0] = wxh[0] * (-ei.core_charge);
        te.na = 4; te.nb = 1; te.wcols = 1;
        for (int k = 0; k < 10; ++k) te.w[k] = wxh[k];
        return;
    }
    double ri[22];
    local_xx(ei, ej, r, ri);
    rotate_xx(ri, axis, proj, te.w);
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
            te.e1b[a][b] = te.w[PACK[a][b] * 10] * (-ej.core_charge);
            te.e2a[a][b] = te.w[PACK[a][b]] * (-ei.core_charge);
        }
    te.na = 4; te.nb = 4; te.wcols = 10;
}

// ----------------------------------------------------------------------------------------
// Molecule, basis, pair list, core Hamiltonian
// ----------------------------------------------------------------------------------------
struct Molecule {
    int natoms = 0;
    std::vector<int> z;
    std::vector<double> pos;  // Bohr, natoms*3
};

struct Basis {
    std::vector<int> offset, norb, ao_orb;
    int nao = 0;
};

struct Pair {
    int a, b;
    PairTE te;
};

struct Core {
    Mat h;
    std::vector<Pair> pairs;
};

int set_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int check_elements(const Molecule& mol, const ParamSet& ps) {
    for (int i = 0; i < mol.natoms; ++i) {
        int z = mol.z[i];
        if (z < 0 || z > NDDO_MAX_Z || !ps.present[z]) {
            std::string sup;
            for (int k = 0; k <= NDDO_MAX_Z; ++k)
                if (ps.present[k]) sup += (sup.empty() ? "" : ", ") + std::to_string(k);
            return set_error(AM1GPU_ELEMENT_NOT_PARAMETERIZED,
                             std::string(ps.name) + " has no parameters for element Z=" + std::to_string(z) +
                                 "; " + ps.name + " covers Z in {" + sup + "}");
        }
    }
    return AM1GPU_OK;
}

// src/basis.rs:37-60
Basis build_basis(const Molecule& mol, const ParamSet& ps) {
    Basis b;
    for (int i = 0; i < mol.natoms; ++i) {
        const Elem& e = ps.by_z[mol.z[i]];
        b.offset.push_back(b.nao);
        b.norb.push_back(e.norb);
        for (int k = 0; k < e.norb; ++k) b.ao_orb.push_back(k);
        b.nao += e.norb;
    }
    return b;
}

// src/hamiltonian.rs:211-366 (molecular case: NeighborList::molecular, neighbors.rs:110-130)
int build_core(const Molecule& mol, const Basis& basis, const ParamSet& ps, Core& core) {
    const int n = basis.nao;
    core.h.assign((size_t)n * n, 0.0);
    core.pairs.clear();
    for (int mu = 0; mu < n; ++mu) {
        (void)0;
    }
    for (int ia = 0; ia < mol.natoms; ++ia) {
        const Elem& e = ps.by_z[mol.z[ia]];
        for (int k = 0; k < basis.norb[ia]; ++k) {
            int mu = basis.offset[ia] + k;
            core.h[(size_t)mu * n + mu] = (k == 0) ? e.u_ss : e.u_pp;
        }
    }
    core.pairs.reserve((size_t)mol.natoms * (mol.natoms - 1) / 2);
    for (int i = 0; i < mol.natoms; ++i)
        for (int j = i + 1; j < mol.natoms; ++j) {
            const double* pi = &mol.pos[3 * i];
            const double* pj = &mol.pos[3 * j];
            double delta[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
            const Elem& eu = ps.by_z[mol.z[i]];
            const Elem& ev = ps.by_z[mol.z[j]];
            bool heavy_first = eu.has_p() || !ev.has_p();
            int a = i, b = j;
            if (!heavy_first) {
                a = j; b = i;
                for (int k = 0; k < 3; ++k) delta[k] = delta[k] * -1.0;
            }
            const Elem& ea = ps.by_z[mol.z[a]];
            const Elem& eb = ps.by_z[mol.z[b]];
            double r = std::sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]);
            // pair_two_electron(ea, eb, delta / r, r) -> pair_two_electron_g(ea, eb, xij * r)
            double x[3] = {delta[0] / r, delta[1] / r, delta[2] / r};
            double dv[3] = {x[0] * r, x[1] * r, x[2] * r};
            Pair pr;
            pr.a = a; pr.b = b;
            pair_two_electron(ea, eb, dv, pr.te);
            const double* pa = &mol.pos[3 * a];
            double pb[3] = {pa[0] + delta[0], pa[1] + delta[1], pa[2] + delta[2]};
            double s[4][4];
            if (!diatom_overlap(ea, pa, eb, pb, s)) return set_error(AM1GPU_UNSUPPORTED, "overlap not covered");
            int oa = basis.offset[a], ob = basis.offset[b], na = basis.norb[a], nb = basis.norb[b];
            for (int ii = 0; ii < na; ++ii)
                for (int jj = 0; jj < na; ++jj) core.h[(size_t)(oa + ii) * n + oa + jj] += pr.te.e1b[ii][jj];
            for (int ii = 0; ii < nb; ++ii)
                for (int jj = 0; jj < nb; ++jj) core.h[(size_t)(ob + ii) * n + ob + jj] += pr.te.e2a[ii][jj];
            for (int ii = 0; ii < na; ++ii) {
                double bi = ii == 0 ? ea.beta_s : ea.beta_p;
                for (int jj = 0; jj < nb; ++jj) {
                    double bj = jj == 0 ? eb.beta_s : eb.beta_p;
                    double value = 0.5 * (bi + bj) * s[ii][jj];
                    core.h[(size_t)(oa + ii) * n + ob + jj] += value;
                    core.h[(size_t)(ob + jj) * n + oa + ii] += value;
                }
            }
            core.pairs.push_back(pr);
        }
    return AM1GPU_OK;
}

// src/repulsion.rs:144-188
double pair_core_energy(const Elem& ei, const Elem& ej, int zi, int zj, double r) {
    double s = r * AM1_A0;
    double rho = ei.rho0 + ej.rho0;
    double gam = rs(r * r + rho * rho) * AM1_EV;
    double zz = ei.core_charge * ej.core_charge;
    bool i_special = (zi == 7 || zi == 8) && zj == 1;
    bool j_special = (zj == 7 || zj == 8) && zi == 1;
    auto expterm = [&](double alpha, bool special) {
        double e = std::exp(s * (-alpha));
        return special ? s * e : e;
    };
    double fi = expterm(ei.alpha, i_special);
    double fj = expterm(ej.alpha, j_special);
    double term1 = gam * (fi + fj + 1.0) * zz;
    auto gauss = [&](const Elem& e) {
        double g = 0.0;
        for (int k = 0; k < e.ngauss; ++k) {
            double d = s - e.gm[k];
            double ex = std::exp(d * d * (-e.gl[k]));
            g = g + ex * e.gk[k];
        }
        return g;
    };
    double gsum = gauss(ei) + gauss(ej);
    double term2 = gsum * zz / s;
    return term1 + term2;
}

// src/repulsion.rs:38-56
double core_core_energy(const Molecule& mol, const ParamSet& ps) {
    double energy = 0.0;
    for (int i = 0; i < mol.natoms; ++i)
        for (int j = i + 1; j < mol.natoms; ++j) {
            const double* pi = &mol.pos[3 * i];
            const double* pj = &mol.pos[3 * j];
            double d[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
            double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            energy += pair_core_energy(ps.by_z[mol.z[i]], ps.by_z[mol.z[j]], mol.z[i], mol.z[j], r);
        }
    return energy;
}

// ----------------------------------------------------------------------------------------
// Fock build, src/fock.rs
// ----------------------------------------------------------------------------------------
// src/fock.rs:27-65
double oc_two_electron(int a, int b, int c, int d, double gss, double gsp, double gpp, double gp2, double hsp) {
    if (a == b && c == d) {
        bool sa = a == 0, sc = c == 0;
        if (sa && sc) return gss;
        if (sa != sc) return gsp;
        return a == c ? gpp : gp2;
    }
    int ba = std::min(a, b), bb = std::max(a, b), kc = std::min(c, d), kd = std::max(c, d);
    if (ba == 0 && bb != 0 && kc == 0 && kd != 0 && bb == kd) return hsp;
    if (ba != 0 && bb != 0 && ba != bb && ba == kc && bb == kd) return 0.5 * (gpp - gp2);
    return 0.0;
}

// src/fock.rs:249-511 (FockBase::CoreHamiltonian, molecule: no long-range / far-field terms)
Mat build_fock_spin(const Molecule& mol, const Basis& basis, const ParamSet& ps, const Core& core, const Mat& ptot,
                    const Mat& pspin, double spin_scale) {
    const int n = basis.nao;
    Mat f = core.h;
    for (int ia = 0; ia < mol.natoms; ++ia) {
        const Elem& e = ps.by_z[mol.z[ia]];
        int off = basis.offset[ia], no = basis.norb[ia];
        for (int mu = 0; mu < no; ++mu)
            for (int nu = 0; nu < no; ++nu) {
                double acc = 0.0;
                for (int la = 0; la < no; ++la)
                    for (int si = 0; si < no; ++si) {
                        acc += ptot[(size_t)(off + la) * n + off + si] *
                               oc_two_electron(mu, nu, la, si, e.g_ss, e.g_sp, e.g_pp, e.g_p2, e.h_sp);
                        acc -= spin_scale * pspin[(size_t)(off + la) * n + off + si] *
                               oc_two_electron(mu, la, nu, si, e.g_ss, e.g_sp, e.g_pp, e.g_p2, e.h_sp);
                    }
                f[(size_t)(off + mu) * n + off + nu] += acc;
            }
    }
    // Pair contributions computed per pair, then scattered in pair order (fock.rs:470-507).
    for (const Pair& pr : core.pairs) {
        const PairTE& te = pr.te;
        int oa = basis.offset[pr.a], ob = basis.offset[pr.b], na = te.na, nb = te.nb, wc = te.wcols;
        double p_bb[16] = {0}, p_aa[16] = {0}, p_ab[16] = {0};
        for (int i = 0; i < nb; ++i) for (int j = 0; j < nb; ++j) p_bb[i * 4 + j] = ptot[(size_t)(ob + i) * n + ob + j];
        for (int i = 0; i < na; ++i) for (int j = 0; j < na; ++j) p_aa[i * 4 + j] = ptot[(size_t)(oa + i) * n + oa + j];
        for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j) p_ab[i * 4 + j] = spin_scale * pspin[(size_t)(oa + i) * n + ob + j];
        double ja[16] = {0}, jb[16] = {0}, kk[16] = {0};
        for (int mu = 0; mu < na; ++mu)
            for (int nu = 0; nu < na; ++nu) {
                const double* row = &te.w[PACK[mu][nu] * wc];
                double acc = 0.0;
                for (int la = 0; la < nb; ++la)
                    for (int si = 0; si < nb; ++si) acc += p_bb[la * 4 + si] * row[PACK[la][si]];
                ja[mu * 4 + nu] = acc;
            }
        for (int la = 0; la < nb; ++la)
            for (int si = 0; si < nb; ++si) {
                int ket = PACK[la][si];
                double acc = 0.0;
                for (int mu = 0; mu < na; ++mu)
                    for (int nu = 0; nu < na; ++nu) acc += p_aa[mu * 4 + nu] * te.w[PACK[mu][nu] * wc + ket];
                jb[la * 4 + si] = acc;
            }
        for (int mu = 0; mu < na; ++mu)
            for (int la = 0; la < nb; ++la) {
                double acc = 0.0;
                for (int nu = 0; nu < na; ++nu) {
                    const double* row = &te.w[PACK[mu][nu] * wc];
                    for (int si = 0; si < nb; ++si) acc += p_ab[nu * 4 + si] * row[PACK[la][si]];
                }
                kk[mu * 4 + la] = -acc * 1.0;  // exchange_scale = 1 for a molecule
            }
        for (int mu = 0; mu < na; ++mu)
            for (int nu = 0; nu < na; ++nu) f[(size_t)(oa + mu) * n + oa + nu] += ja[mu * 4 + nu];
        for (int la = 0; la < nb; ++la)
            for (int si = 0; si < nb; ++si) f[(size_t)(ob + la) * n + ob + si] += jb[la * 4 + si];
        for (int mu = 0; mu < na; ++mu)
            for (int la = 0; la < nb; ++la) {
                double v = kk[mu * 4 + la];
                f[(size_t)(oa + mu) * n + ob + la] += v;
                f[(size_t)(ob + la) * n + oa + mu] += v;
            }
    }
    return f;
}

// ----------------------------------------------------------------------------------------
// Symmetric eigensolver (stands in for faer's self_adjoint_eigen, src/linalg.rs:276-331):
// Householder reduction to tridiagonal form with Q accumulated, then implicit-shift QR sweeps
// on the tridiagonal matrix, eigenpairs sorted ascending.
// ----------------------------------------------------------------------------------------
// Householder reduction A = Q T Q^T (Golub & Van Loan, Alg. 8.3.1).  a (row-major, symmetric)
// is destroyed; q receives Q; d/e the diagonal and the subdiagonal (e[i] couples i, i+1).
void householder_tridiag(int n, std::vector<double>& a, std::vector<double>& q, std::vector<double>& d,
                         std::vector<double>& e) {
    d.assign(n, 0.0);
    e.assign(n > 0 ? n : 1, 0.0);
    std::vector<std::vector<double>> vs(n);
    std::vector<double> betas(n, 0.0), p(n), w(n);
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;  // length of the column below the diagonal
        std::vector<double>& v = vs[k];
        v.resize(m);
        double norm2 = 0.0;
        for (int i = 0; i < m; ++i) {
            v[i] = A(k + 1 + i, k);
            norm2 += v[i] * v[i];
        }
        double alpha = std::sqrt(norm2);
        if (alpha == 0.0) {
            betas[k] = 0.0;
            e[k] = 0.0;
            continue;
        }
        double sgn = v[0] >= 0.0 ? 1.0 : -1.0;
        double beta = 1.0 / (alpha * (alpha + std::fabs(v[0])));
        v[0] += sgn * alpha;
        betas[k] = beta;
        e[k] = -sgn * alpha;
        // p = beta * A_sub v, using the symmetric trailing block
        par_for(m, (double)m * m, [&](int lo, int hi) {
            for (int i = lo; i < hi; ++i) {
                double acc = 0.0;
                const double* row = &a[(size_t)(k + 1 + i) * n + k + 1];
                for (int j = 0; j < m; ++j) acc += row[j] * v[j];
                p[i] = beta * acc;
            }
        });
        double pv = 0.0;
        for (int i = 0; i < m; ++i) pv += p[i] * v[i];
        double kk = 0.5 * beta * pv;
        for (int i = 0; i < m; ++i) w[i] = p[i] - kk * v[i];
        par_for(m, (double)m * m, [&](int lo, int hi) {
            for (int i = lo; i < hi; ++i) {
                double* row = &a[(size_t)(k + 1 + i) * n + k + 1];
                for (int j = 0; j < m; ++j) row[j] -= v[i] * w[j] + w[i] * v[j];
            }
        });
    }
    for (int i = 0; i < n; ++i) d[i] = A(i, i);
    if (n >= 2) e[n - 2] = A(n - 1, n - 2);
    // Q = H_0 H_1 ... H_{n-3}, accumulated from the last reflector backwards.
    q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) q[(size_t)i * n + i] = 1.0;
    std::vector<double> t(n);
    for (int k = n - 3; k >= 0; --k) {
        if (betas[k] == 0.0) continue;
        const std::vector<double>& v = vs[k];
        const int m = n - k - 1;
        // Q_sub -= beta v (v^T Q_sub), Q_sub = rows/cols k+1..n-1 (t split by columns, the
        // update by rows: each t[j] still sums its rows in order)
        par_for(m, (double)m * m, [&](int lo, int hi) {
            for (int j = lo; j < hi; ++j) t[j] = 0.0;
            for (int i = 0; i < m; ++i) {
                const double* row = &q[(size_t)(k + 1 + i) * n + k + 1];
                for (int j = lo; j < hi; ++j) t[j] += v[i] * row[j];
            }
        });
        par_for(m, (double)m * m, [&](int lo, int hi) {
            for (int i = lo; i < hi; ++i) {
                double* row = &q[(size_t)(k + 1 + i) * n + k + 1];
                double bv = betas[k] * v[i];
                for (int j = 0; j < m; ++j) row[j] -= bv * t[j];
            }
        });
    }
}

// Implicit symmetric QR with a Wilkinson shift on the unreduced block lo..hi of a tridiagonal
// matrix (Golub & Van Loan, Alg. 8.3.2), chasing the bulge with Givens rotations that are
// also applied to the columns of z (n*n row-major).
void qr_sweep(int n, int lo, int hi, std::vector<double>& d, std::vector<double>& e, std::vector<double>& z) {
    double half = 0.5 * (d[hi - 1] - d[hi]);
    double b = e[hi - 1];
    double mu = d[hi] - b * b / (half + std::copysign(std::hypot(half, b), half));
    double x = d[lo] - mu, y = e[lo];
    // The rotations only depend on d and e: chase the bulge first, then apply the sweep's
    // rotations to z row by row (the same operations on each element, in the same order, with
    // contiguous access).
    std::vector<double> cs(hi - lo), sn(hi - lo);
    for (int k = lo; k < hi; ++k) {
        double r = std::hypot(x, y);
        double c = 1.0, s = 0.0;
        if (r != 0.0) {
            c = x / r;
            s = y / r;
        }
        cs[k - lo] = c;
        sn[k - lo] = s;
        if (k > lo) e[k - 1] = r;
        double ak = d[k], bk = e[k], an = d[k + 1];
        d[k] = ak * c * c + 2.0 * bk * c * s + an * s * s;
        d[k + 1] = ak * s * s - 2.0 * bk * c * s + an * c * c;
        e[k] = (an - ak) * c * s + bk * (c * c - s * s);
        if (k + 1 < hi) {
            double f = e[k + 1];
            y = s * f;  // bulge at (k, k+2)
            e[k + 1] = c * f;
            x = e[k];
        }
    }
    par_for(n, 6.0 * n * (hi - lo), [&](int i0, int i1) {
        for (int i = i0; i < i1; ++i) {
            double* row = &z[(size_t)i * n];
            for (int k = lo; k < hi; ++k) {
                const double c = cs[k - lo], s = sn[k - lo];
                double zk = row[k], zn = row[k + 1];
                row[k] = c * zk + s * zn;
                row[k + 1] = -s * zk + c * zn;
            }
        }
    });
}

bool tridiagonal_eigen(int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& z) {
    const double eps = std::numeric_limits<double>::epsilon();
    long budget = 40L * n + 40;
    int hi = n - 1;
    while (hi > 0) {
        if (std::fabs(e[hi - 1]) <= eps * (std::fabs(d[hi - 1]) + std::fabs(d[hi]))) {
            e[hi - 1] = 0.0;
            --hi;
            continue;
        }
        int lo = hi - 1;
        while (lo > 0 && std::fabs(e[lo - 1]) > eps * (std::fabs(d[lo - 1]) + std::fabs(d[lo]))) --lo;
        if (--budget < 0) return false;
        qr_sweep(n, lo, hi, d, e, z);
    }
    return true;
}

// symmetric_eigen: eigenvalues ascending, eigenvectors as columns of v (row-major n*n).
int symmetric_eigen(int n, const Mat& a, std::vector<double>& w, Mat& v) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (!std::isfinite(a[(size_t)i * n + j]))
                return set_error(AM1GPU_LINALG, "the matrix handed to the eigensolver is not finite at (" +
                                                    std::to_string(i) + ", " + std::to_string(j) + ")");
    if (n == 0) { w.clear(); v.clear(); return AM1GPU_OK; }
    Mat s(a.begin(), a.end());
    // Read the lower triangle, as faer's Side::Lower does.
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) s[(size_t)i * n + j] = s[(size_t)j * n + i];
    std::vector<double> d, e;
    Mat z;
    householder_tridiag(n, s, z, d, e);
    if (!tridiagonal_eigen(n, d, e, z)) return set_error(AM1GPU_LINALG, "tridiagonal QR did not converge");
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x] < d[y]; });
    w.resize(n);
    v.assign((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        w[c] = d[order[c]];
        for (int i = 0; i < n; ++i) v[(size_t)i * n + c] = z[(size_t)i * n + order[c]];
    }
    return AM1GPU_OK;
}

// ----------------------------------------------------------------------------------------
// SCF, src/scf.rs
// ----------------------------------------------------------------------------------------
// src/scf.rs:475-494
Mat sad_density(const Molecule& mol, const Basis& basis, const ParamSet& ps) {
    const int n = basis.nao;
    Mat p((size_t)n * n, 0.0);
    for (int ia = 0; ia < mol.natoms; ++ia) {
        const Elem& e = ps.by_z[mol.z[ia]];
        int off = basis.offset[ia];
        double zv = e.core_charge;
        double n_s = std::min(zv, 2.0);
        double n_p = std::max(zv - n_s, 0.0);
        p[(size_t)off * n + off] = n_s;
        if (basis.norb[ia] == 4) {
            double per_p = n_p / 3.0;
            for (int k = 1; k < 4; ++k) p[(size_t)(off + k) * n + off + k] = per_p;
        }
    }
    return p;
}

// src/scf.rs:503-524: P = w C_occ C_occ^T
Mat density_from_coeff(int n, const Mat& c, int n_occ, double weight) {
    Mat p((size_t)n * n, 0.0);
    if (n_occ == 0 || n == 0) return p;
    par_for(n, (double)n * n * n_occ, [&](int lo, int hi) {
        for (int mu = lo; mu < hi; ++mu)
            for (int nu = 0; nu < n; ++nu) {
                double acc = 0.0;
                for (int k = 0; k < n_occ; ++k) acc += c[(size_t)mu * n + k] * c[(size_t)nu * n + k];
                p[(size_t)mu * n + nu] = acc;
            }
    });
    if (weight != 1.0)
        for (double& x : p) x *= weight;
    return p;
}

// src/scf.rs:531-544: e = FP - PF using PF = (FP)^T
Mat commutator(int n, const Mat& f, const Mat& p) {
    Mat e((size_t)n * n, 0.0);
    // (FP)_ij summed over k in ascending order, as a row of accumulators (contiguous reads of P)
    par_for(n, (double)n * n * n, [&](int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            double* acc = &e[(size_t)i * n];
            for (int k = 0; k < n; ++k) {
                const double fik = f[(size_t)i * n + k];
                const double* prow = &p[(size_t)k * n];
                for (int j = 0; j < n; ++j) acc[j] += fik * prow[j];
            }
        }
    });
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            double a = e[(size_t)i * n + j], b = e[(size_t)j * n + i];
            e[(size_t)i * n + j] = a - b;
            e[(size_t)j * n + i] = b - a;
        }
        e[(size_t)i * n + i] = 0.0;
    }
    return e;
}

// src/scf.rs:546-555
double rms_diff(const Mat& a, const Mat& b) {
    size_t n = std::max<size_t>(a.size(), 1);
    double s = 0.0;
    for (size_t k = 0; k < a.size(); ++k) s += (a[k] - b[k]) * (a[k] - b[k]);
    return std::sqrt(s / (double)n);
}

double sum_sq(const Mat& a) {
    double s = 0.0;
    for (double x : a) s += x * x;
    return s;
}

// Packed triangles, src/scf.rs:877-952
std::vector<double> pack_sym(int n, const Mat& m) {
    std::vector<double> out;
    out.reserve((size_t)n * (n + 1) / 2);
    for (int i = 0; i < n; ++i) for (int j = i; j < n; ++j) out.push_back(m[(size_t)i * n + j]);
    return out;
}
std::vector<double> pack_anti(int n, const Mat& m) {
    std::vector<double> out;
    out.reserve((size_t)n * (n - 1) / 2);
    for (int i = 0; i < n; ++i) for (int j = i + 1; j < n; ++j) out.push_back(m[(size_t)i * n + j]);
    return out;
}
Mat unpack_sym(int n, const std::vector<double>& v) {
    Mat out((size_t)n * n, 0.0);
    size_t k = 0;
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) {
            double x = v[k++];
            out[(size_t)i * n + j] = x;
            if (i != j) out[(size_t)j * n + i] = x;
        }
    return out;
}
double dot_anti(const std::vector<double>& a, const std::vector<double>& b) {
    double acc = 0.0;
    for (size_t k = 0; k < a.size(); ++k) acc += a[k] * b[k];
    return 2.0 * acc;
}
double dot_sym(int n, const std::vector<double>& a, const std::vector<double>& b) {
    double acc = 0.0, diag = 0.0;
    size_t k = 0;
    for (int i = 0; i < n; ++i) {
        diag += a[k] * b[k];
        ++k;
        for (int j = i + 1; j < n; ++j) {
            acc += a[k] * b[k];
            ++k;
        }
    }
    return 2.0 * acc + diag;
}

// src/scf.rs:955-963
Mat combine_packed(int n, const std::vector<std::vector<double>>& hist, const std::vector<double>& c) {
    std::vector<double> acc((size_t)n * (n + 1) / 2, 0.0);
    for (size_t h = 0; h < hist.size() && h < c.size(); ++h)
        for (size_t k = 0; k < acc.size(); ++k) acc[k] += c[h] * hist[h][k];
    return unpack_sym(n, acc);
}

// src/scf.rs:1095-1141
bool solve_bordered_small(int n, std::vector<double> m, std::vector<double> rhs, std::vector<double>& x) {
    for (int col = 0; col < n; ++col) {
        int pivot = col;
        double best = std::fabs(m[(size_t)col * n + col]);
        for (int row = col + 1; row < n; ++row) {
            double v = std::fabs(m[(size_t)row * n + col]);
            if (v > best) { best = v; pivot = row; }
        }
        if (best < 1.0e-12) return false;
        if (pivot != col) {
            for (int j = 0; j < n; ++j) std::swap(m[(size_t)col * n + j], m[(size_t)pivot * n + j]);
            std::swap(rhs[col], rhs[pivot]);
        }
        for (int row = col + 1; row < n; ++row) {
            double factor = m[(size_t)row * n + col] / m[(size_t)col * n + col];
            if (factor == 0.0) continue;
            for (int j = col; j < n; ++j) {
                double v = m[(size_t)col * n + j];
                m[(size_t)row * n + j] -= factor * v;
            }
            rhs[row] -= factor * rhs[col];
        }
    }
    x.assign(n, 0.0);
    for (int col = n - 1; col >= 0; --col) {
        double sum = rhs[col];
        for (int j = col + 1; j < n; ++j) sum -= m[(size_t)col * n + j] * x[j];
        x[col] = sum / m[(size_t)col * n + col];
    }
    return true;
}

// src/scf.rs:966-988
bool diis_coeffs(const std::vector<std::vector<double>>& es, std::vector<double>& c) {
    int m = (int)es.size();
    if (m < 2) return false;
    int dim = m + 1;
    std::vector<double> b((size_t)dim * dim, 0.0);
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) b[(size_t)i * dim + j] = dot_anti(es[i], es[j]);
        b[(size_t)i * dim + m] = -1.0;
        b[(size_t)m * dim + i] = -1.0;
    }
    std::vector<double> rhs(dim, 0.0);
    rhs[m] = -1.0;
    return solve_bordered_small(dim, b, rhs, c);
}

// src/scf.rs:1188-1204 (Duchi et al. projection onto the probability simplex)
std::vector<double> simplex_project(const std::vector<double>& v) {
    std::vector<double> u(v);
    std::sort(u.begin(), u.end(), [](double a, double b) { return a > b; });
    double css = 0.0, theta = 0.0;
    for (size_t j = 0; j < u.size(); ++j) {
        css += u[j];
        double t = (css - 1.0) / ((double)j + 1.0);
        if (u[j] - t > 0.0) theta = t;
    }
    std::vector<double> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = std::max(v[i] - theta, 0.0);
    return out;
}

// src/scf.rs:1144-1181
std::vector<double> solve_adiis_simplex(const std::vector<double>& d, const std::vector<std::vector<double>>& s) {
    int n = (int)d.size();
    double l = 1.0e-12;
    for (int i = 0; i < n; ++i) {
        double row = 0.0;
        for (int j = 0; j < n; ++j) row += std::fabs(s[i][j] + s[j][i]);
        l = std::max(l, row);
    }
    double lr = 1.0 / l;
    std::vector<double> c(n, 0.0);
    c[n - 1] = 1.0;
    for (int it = 0; it < 400; ++it) {
        std::vector<double> g(n);
        for (int k = 0; k < n; ++k) {
            double acc = 2.0 * d[k];
            for (int j = 0; j < n; ++j) acc += (s[k][j] + s[j][k]) * c[j];
            g[k] = acc;
        }
        std::vector<double> trial(n);
        for (int i = 0; i < n; ++i) trial[i] = c[i] - lr * g[i];
        std::vector<double> proj = simplex_project(trial);
        double delta = 0.0;
        for (int i = 0; i < n; ++i) delta += std::fabs(proj[i] - c[i]);
        c = proj;
        if (delta < 1.0e-12) break;
    }
    return c;
}

// src/scf.rs:1061-1091
bool adiis_extrapolate(int n, const std::vector<std::vector<double>>& ds, const std::vector<std::vector<double>>& fs,
                       Mat& out) {
    int m = (int)ds.size();
    if (m < 2) return false;
    int last = m - 1;
    std::vector<std::vector<double>> gram(m, std::vector<double>(m));
    for (int i = 0; i < m; ++i) for (int j = 0; j < m; ++j) gram[i][j] = dot_sym(n, ds[i], fs[j]);
    std::vector<double> d(m);
    for (int i = 0; i < m; ++i) d[i] = gram[i][last] - gram[last][last];
    std::vector<std::vector<double>> s(m, std::vector<double>(m));
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) s[i][j] = gram[i][j] - gram[i][last] - gram[last][j] + gram[last][last];
    std::vector<double> c = solve_adiis_simplex(d, s);
    out = combine_packed(n, fs, c);
    return true;
}

bool all_finite(const Mat& m) {
    for (double x : m)
        if (!std::isfinite(x)) return false;
    return true;
}

struct State {
    Mat density, spin_density;
    std::vector<double> eps_a, eps_b;
    Mat c_a, c_b;
    int n_occ = 0, n_occ_b = 0;
    double electronic_ev = 0.0, residual = INFINITY;
    bool converged = false, unrestricted = false;
    int iterations = 0;
};

// src/scf.rs:557-716
int rhf_loop(const Molecule& mol, const Basis& basis, const ParamSet& ps, const Core& core, int n_occ,
             const am1gpu_options& o, State& st) {
    const int n = basis.nao;
    Mat density = sad_density(mol, basis, ps);
    double e_old = 0.0;
    std::vector<double> mo_e(n, 0.0);
    Mat mo_c((size_t)n * n, 0.0);
    std::vector<std::vector<double>> hf, he, hd;
    const size_t max_diis = 8;
    int accel = o.use_diis ? o.accelerator : AM1GPU_ACCEL_NONE;
    bool needs_d = accel == AM1GPU_ACCEL_ADIIS_CDIIS;
    bool converged = false;
    int iterations = 0;
    double residual = INFINITY;
    for (int iter = 0; iter < o.max_scf; ++iter) {
        iterations = iter + 1;
        Mat f = build_fock_spin(mol, basis, ps, core, density, density, 0.5);
        double e_elec = 0.5 * (frobenius_dot(density, core.h) + frobenius_dot(density, f));
        Mat err = commutator(n, f, density);
        double err_norm = std::sqrt(sum_sq(err));
        hf.push_back(pack_sym(n, f));
        he.push_back(pack_anti(n, err));
        if (needs_d) hd.push_back(pack_sym(n, density));
        if (hf.size() > max_diis) {
            hf.erase(hf.begin());
            he.erase(he.begin());
            if (!hd.empty()) hd.erase(hd.begin());
        }
        if (!std::isfinite(e_elec) || !std::isfinite(err_norm)) {
            st.iterations = iter + 1;
            return set_error(AM1GPU_SCF_DIVERGED, "the AM1 SCF diverged at iteration " + std::to_string(iter + 1));
        }
        Mat x;
        bool have = false;
        if (accel == AM1GPU_ACCEL_CDIIS || (accel == AM1GPU_ACCEL_ADIIS_CDIIS && !(err_norm > o.adiis_switch))) {
            std::vector<double> c;
            if (diis_coeffs(he, c)) {
                double weight = 0.0;
                for (size_t k = 0; k < hf.size(); ++k) weight += std::fabs(c[k]);
                if (std::isfinite(weight)) {
                    x = combine_packed(n, hf, c);
                    have = true;
                }
            }
        } else if (accel == AM1GPU_ACCEL_ADIIS_CDIIS) {
            have = adiis_extrapolate(n, hd, hf, x);
        }
        const Mat& f_use = (have && all_finite(x)) ? x : f;
        std::vector<double> eps;
        Mat c;
        int rc = symmetric_eigen(n, f_use, eps, c);
        if (rc != AM1GPU_OK) return rc;
        Mat p_new = density_from_coeff(n, c, n_occ, 2.0);
        double dp = rms_diff(p_new, density);
        double de = std::fabs(e_elec - e_old);
        mo_e = eps;
        mo_c = c;
        density = p_new;
        e_old = e_elec;
        residual = err_norm;
        if (iter > 0 && de < o.e_tol && (dp < o.p_tol || err_norm < 1.0e-7)) {
            converged = true;
            break;
        }
    }
    Mat f_final = build_fock_spin(mol, basis, ps, core, density, density, 0.5);
    st.electronic_ev = 0.5 * (frobenius_dot(density, core.h) + frobenius_dot(density, f_final));
    st.density = density;
    st.eps_a = mo_e;
    st.c_a = mo_c;
    st.n_occ = n_occ;
    st.converged = converged;
    st.iterations = iterations;
    st.unrestricted = false;
    st.residual = residual;
    return AM1GPU_OK;
}

// src/scf.rs:719-858
int uhf_loop(const Molecule& mol, const Basis& basis, const ParamSet& ps, const Core& core, int n_alpha, int n_beta,
             const am1gpu_options& o, State& st) {
    const int n = basis.nao;
    Mat sad = sad_density(mol, basis, ps);
    double n_tot = (double)std::max(n_alpha + n_beta, 1);
    double fa_s = (double)n_alpha / n_tot, fb_s = (double)n_beta / n_tot;
    Mat pa = sad, pb = sad;
    for (double& v : pa) v *= fa_s;
    for (double& v : pb) v *= fb_s;
    double e_old = 0.0;
    std::vector<double> eps_a(n, 0.0), eps_b(n, 0.0);
    Mat c_a((size_t)n * n, 0.0), c_b((size_t)n * n, 0.0);
    std::vector<std::vector<double>> hfa, hfb, herr;
    const size_t max_diis = 8;
    bool converged = false;
    int iterations = 0;
    double residual = INFINITY;
    for (int iter = 0; iter < o.max_scf; ++iter) {
        iterations = iter + 1;
        Mat p_tot = pa;
        for (size_t k = 0; k < p_tot.size(); ++k) p_tot[k] += pb[k];
        Mat fa = build_fock_spin(mol, basis, ps, core, p_tot, pa, 1.0);
        Mat fb = build_fock_spin(mol, basis, ps, core, p_tot, pb, 1.0);
        double e_elec = 0.5 * (frobenius_dot(p_tot, core.h) + frobenius_dot(pa, fa) + frobenius_dot(pb, fb));
        Mat ea = commutator(n, fa, pa);
        Mat eb = commutator(n, fb, pb);
        double err_norm = std::sqrt(sum_sq(ea) + sum_sq(eb));
        Mat fa_use = fa, fb_use = fb;
        if (o.use_diis) {
            std::vector<double> err = pack_anti(n, ea);
            std::vector<double> errb = pack_anti(n, eb);
            err.insert(err.end(), errb.begin(), errb.end());
            hfa.push_back(pack_sym(n, fa));
            hfb.push_back(pack_sym(n, fb));
            herr.push_back(err);
            if (hfa.size() > max_diis) {
                hfa.erase(hfa.begin());
                hfb.erase(hfb.begin());
                herr.erase(herr.begin());
            }
            std::vector<double> c;
            if (diis_coeffs(herr, c)) {
                fa_use = combine_packed(n, hfa, c);
                fb_use = combine_packed(n, hfb, c);
            }
        }
        if (!std::isfinite(e_elec) || !std::isfinite(err_norm)) {
            st.iterations = iter + 1;
            return set_error(AM1GPU_SCF_DIVERGED, "the AM1 SCF diverged at iteration " + std::to_string(iter + 1));
        }
        std::vector<double> wa, wb;
        Mat ca, cb;
        int rc = symmetric_eigen(n, fa_use, wa, ca);
        if (rc != AM1GPU_OK) return rc;
        rc = symmetric_eigen(n, fb_use, wb, cb);
        if (rc != AM1GPU_OK) return rc;
        Mat pa_new = density_from_coeff(n, ca, n_alpha, 1.0);
        Mat pb_new = density_from_coeff(n, cb, n_beta, 1.0);
        double dp = rms_diff(pa_new, pa) + rms_diff(pb_new, pb);
        double de = std::fabs(e_elec - e_old);
        eps_a = wa; c_a = ca; eps_b = wb; c_b = cb;
        pa = pa_new; pb = pb_new;
        e_old = e_elec;
        residual = err_norm;
        if (iter > 0 && de < o.e_tol && (dp < o.p_tol || err_norm < 1.0e-7)) {
            converged = true;
            break;
        }
    }
    Mat density = pa, spin = pa;
    for (size_t k = 0; k < density.size(); ++k) { density[k] += pb[k]; spin[k] -= pb[k]; }
    Mat fa = build_fock_spin(mol, basis, ps, core, density, pa, 1.0);
    Mat fb = build_fock_spin(mol, basis, ps, core, density, pb, 1.0);
    st.electronic_ev = 0.5 * (frobenius_dot(density, core.h) + frobenius_dot(pa, fa) + frobenius_dot(pb, fb));
    st.density = density;
    st.spin_density = spin;
    st.eps_a = eps_a; st.c_a = c_a; st.eps_b = eps_b; st.c_b = c_b;
    st.n_occ = n_alpha; st.n_occ_b = n_beta;
    st.converged = converged;
    st.iterations = iterations;
    st.unrestricted = true;
    st.residual = residual;
    return AM1GPU_OK;
}

Molecule to_molecule(const am1gpu_molecule* m) {
    Molecule mol;
    mol.natoms = m->natoms;
    mol.z.assign(m->z, m->z + m->natoms);
    mol.pos.assign(m->xyz_bohr, m->xyz_bohr + 3 * (size_t)m->natoms);
    return mol;
}

void copy_out(double* dst, const std::vector<double>& src) {
    if (dst) std::memcpy(dst, src.data(), src.size() * sizeof(double));
}

// src/scf.rs:294-468
// custom: a caller's parameter set (run_am1 takes any &Am1Parameters); NULL: the built-in set
// of o->method.
int run_am1(const am1gpu_molecule* m, const am1gpu_options* o, am1gpu_result* res, const ParamSet* custom = nullptr) {
    g_err.clear();
    if (!m || !o || !res || m->natoms < 0 || (m->natoms > 0 && (!m->z || !m->xyz_bohr)))
        return set_error(AM1GPU_INVALID_INPUT, "null argument");
    if (m->multiplicity < 1) return set_error(AM1GPU_INVALID_INPUT, "multiplicity must be >= 1");
    const ParamSet& ps = custom ? *custom : params_for(o->method);
    Molecule mol = to_molecule(m);
    int rc = check_elements(mol, ps);
    if (rc) return rc;
    Basis basis = build_basis(mol, ps);
    Core core;
    rc = build_core(mol, basis, ps, core);
    if (rc) return rc;
    double n_elec = 0.0;
    for (int i = 0; i < mol.natoms; ++i) n_elec += ps.by_z[mol.z[i]].core_charge;
    n_elec -= m->charge;
    long long ne = (long long)std::llround(n_elec);
    if (std::fabs(n_elec - (double)ne) > 1.0e-6 || ne < 0)
        return set_error(AM1GPU_INVALID_INPUT, "invalid electron count " + std::to_string(n_elec));
    long long unp = m->multiplicity - 1;
    if ((ne - unp) < 0 || (ne - unp) % 2 != 0)
        return set_error(AM1GPU_INVALID_INPUT, "electron count " + std::to_string(ne) +
                                                   " is incompatible with multiplicity " +
                                                   std::to_string(m->multiplicity) + " (need same parity)");
    int n_alpha = (int)((ne + unp) / 2), n_beta = (int)((ne - unp) / 2);
    bool closed = n_alpha == n_beta;
    bool use_uhf;
    if (o->reference == AM1GPU_REF_AUTO) use_uhf = !closed;
    else if (o->reference == AM1GPU_REF_UHF) use_uhf = true;
    else {
        if (!closed)
            return set_error(AM1GPU_INVALID_INPUT,
                             "restricted (RHF) reference requires a closed shell, but multiplicity " +
                                 std::to_string(m->multiplicity) + " gives " + std::to_string(n_alpha) +
                                 " alpha and " + std::to_string(n_beta) + " beta electrons");
        use_uhf = false;
    }
    State st;
    rc = use_uhf ? uhf_loop(mol, basis, ps, core, n_alpha, n_beta, *o, st)
                 : rhf_loop(mol, basis, ps, core, n_alpha, *o, st);
    if (rc) {
        res->iterations = st.iterations;
        return rc;
    }
    const int n = basis.nao;
    double core_ev = core_core_energy(mol, ps);
    double total = st.electronic_ev + core_ev;
    double e_isol = 0.0, eheat = 0.0;
    for (int i = 0; i < mol.natoms; ++i) {
        e_isol += ps.by_z[mol.z[i]].e_isol;
        eheat += ps.by_z[mol.z[i]].eheat_ev;
    }
    res->electronic_ev = st.electronic_ev;
    res->core_ev = core_ev;
    res->total_ev = total;
    res->heat_of_formation_kcal = (total - e_isol + eheat) * EV_TO_KCAL;
    res->nao = n;
    res->n_occ = st.n_occ;
    res->n_occ_beta = st.unrestricted ? st.n_occ_b : st.n_occ;
    res->iterations = st.iterations;
    res->converged = st.converged ? 1 : 0;
    res->unrestricted = st.unrestricted ? 1 : 0;
    res->residual = st.residual;
    // Mulliken charges (scf.rs:400-409) and dipole (scf.rs:412-427), written even when the SCF
    // did not converge so a caller can inspect the state it reached.
    std::vector<double> q(mol.natoms);
    for (int ia = 0; ia < mol.natoms; ++ia) {
        double pop = 0.0;
        for (int k = 0; k < basis.norb[ia]; ++k) {
            int mu = basis.offset[ia] + k;
            pop += st.density[(size_t)mu * n + mu];
        }
        q[ia] = ps.by_z[mol.z[ia]].core_charge - pop;
    }
    double dip[3] = {0, 0, 0};
    for (int ia = 0; ia < mol.natoms; ++ia) {
        for (int k = 0; k < 3; ++k) dip[k] += mol.pos[3 * ia + k] * q[ia];
        const Elem& e = ps.by_z[mol.z[ia]];
        if (e.has_p()) {
            int off = basis.offset[ia];
            double hyb = -2.0 * e.dd;
            for (int k = 0; k < 3; ++k) dip[k] += hyb * st.density[(size_t)off * n + off + 1 + k];
        }
    }
    for (int k = 0; k < 3; ++k) res->dipole_debye[k] = dip[k] * AU_DIPOLE_TO_DEBYE;
    res->dipole_magnitude = std::sqrt(res->dipole_debye[0] * res->dipole_debye[0] +
                                      res->dipole_debye[1] * res->dipole_debye[1] +
                                      res->dipole_debye[2] * res->dipole_debye[2]);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    res->homo_ev = st.n_occ >= 1 ? st.eps_a[st.n_occ - 1] : nan;
    res->lumo_ev = st.n_occ < n ? st.eps_a[st.n_occ] : nan;
    res->homo_beta_ev = res->lumo_beta_ev = nan;
    if (st.unrestricted) {
        res->homo_beta_ev = st.n_occ_b >= 1 ? st.eps_b[st.n_occ_b - 1] : nan;
        res->lumo_beta_ev = st.n_occ_b < n ? st.eps_b[st.n_occ_b] : nan;
    }
    copy_out(res->charges, q);
    copy_out(res->density, st.density);
    copy_out(res->mo_energies, st.eps_a);
    copy_out(res->mo_coeff, st.c_a);
    if (st.unrestricted) {
        copy_out(res->spin_density, st.spin_density);
        copy_out(res->beta_energies, st.eps_b);
        copy_out(res->beta_coeff, st.c_b);
    }
    if (!st.converged) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "AM1 SCF did not converge after %d iterations (error=%.3e)", st.iterations,
                      st.residual);
        return set_error(AM1GPU_SCF_NOT_CONVERGED, buf);
    }
    return AM1GPU_OK;
}

}  // namespace

// ----------------------------------------------------------------------------------------
// C ABI of the oracle (same structs as the library's public header, prefixed oracle_)
// ----------------------------------------------------------------------------------------
extern "C" {

// The five local overlaps of the pair (za, zb) at distance r (ea.n >= eb.n is arranged here):
// numeric = 1 forces the quadrature, which for n <= 3 must reproduce the closed forms
// (src/overlap.rs:718-747 checks the same).
int oracle_local_overlaps(int method, int za, int zb, double r, int numeric, double out[5]) {
    const ParamSet& ps = params_for(method);
    if (za < 0 || za > NDDO_MAX_Z || zb < 0 || zb > NDDO_MAX_Z || !ps.present[za] || !ps.present[zb]) return AM1GPU_INVALID_INPUT;
    const Elem& a = ps.by_z[za].n >= ps.by_z[zb].n ? ps.by_z[za] : ps.by_z[zb];
    const Elem& b = ps.by_z[za].n >= ps.by_z[zb].n ? ps.by_z[zb] : ps.by_z[za];
    if (numeric) overlap_locals_numeric(a, b, r, out);
    else if (!overlap_locals(a, b, r, out)) return AM1GPU_UNSUPPORTED;
    return AM1GPU_OK;
}

// Threads for the O(n^3) loops of one molecule's SCF (default 1); results do not depend on it.
void oracle_set_threads(int nthreads) { g_inner_threads.store(std::max(1, nthreads)); }

int oracle_scf(const am1gpu_molecule* mol, const am1gpu_options* opts, am1gpu_result* res) {
    return run_am1(mol, opts, res);
}

// The SCF with a caller's parameter set (the elements of an Am1Parameters, src/params.rs:24-70),
// taken as given: no field is re-derived.
int oracle_scf_params(const am1gpu_molecule* mol, const am1gpu_param_table* t, const am1gpu_options* opts,
                      am1gpu_result* res) {
    if (!t || t->count < 0 || (t->count > 0 && !t->elements)) return set_error(AM1GPU_INVALID_INPUT, "null parameter set");
    static thread_local ParamSet ps;
    ps = ParamSet{};
    ps.name = t->method == AM1GPU_METHOD_RM1 ? "RM1" : "AM1";
    for (int i = 0; i < t->count; ++i) {
        const am1gpu_element& a = t->elements[i];
        if (a.z < 1 || a.z > NDDO_MAX_Z || ps.present[a.z] || a.n_gauss < 0 || a.n_gauss > 4)
            return set_error(AM1GPU_INVALID_INPUT, "bad parameter set entry");
        Elem e;
        e.z = a.z;
        e.n = a.n;
        e.norb = a.n_orb;
        e.ngauss = a.n_gauss;
        e.u_ss = a.u_ss; e.u_pp = a.u_pp; e.zeta_s = a.zeta_s; e.zeta_p = a.zeta_p; e.beta_s = a.beta_s; e.beta_p = a.beta_p;
        e.g_ss = a.g_ss; e.g_sp = a.g_sp; e.g_pp = a.g_pp; e.g_p2 = a.g_p2; e.h_sp = a.h_sp; e.alpha = a.alpha;
        for (int k = 0; k < 4; ++k) {
            e.gk[k] = a.gauss_k[k];
            e.gl[k] = a.gauss_l[k];
            e.gm[k] = a.gauss_m[k];
        }
        e.core_charge = a.core_charge; e.eheat_ev = a.eheat_ev; e.e_isol = a.e_isol;
        e.dd = a.dd; e.qq = a.qq; e.rho0 = a.rho0; e.rho1 = a.rho1; e.rho2 = a.rho2;
        ps.by_z[a.z] = e;
        ps.present[a.z] = true;
    }
    am1gpu_options o = *opts;
    o.method = t->method;
    return run_am1(mol, &o, res, &ps);
}

// Molecules are independent; a pool of host threads takes them one at a time (CPU baseline).
int oracle_scf_batch(int nmol, const am1gpu_molecule* mols, const am1gpu_options* opts, am1gpu_result* res,
                     int* status, int nthreads) {
    int first = AM1GPU_OK;
    std::atomic<int> next{0};
    auto worker = [&]() {
        const bool was = t_serial;
        t_serial = true;  // molecules already run in parallel: keep each one's loops serial
        for (int i = next++; i < nmol; i = next++) status[i] = run_am1(&mols[i], opts, &res[i]);
        t_serial = was;
    };
    int nt = std::max(1, nthreads);
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    for (int i = 0; i < nmol; ++i)
        if (status[i] != AM1GPU_OK) { first = status[i]; break; }
    return first;
}

int oracle_build_core(const am1gpu_molecule* m, int method, double* h_core, double* core_ev) {
    const ParamSet& ps = params_for(method);
    Molecule mol = to_molecule(m);
    int rc = check_elements(mol, ps);
    if (rc) return rc;
    Basis basis = build_basis(mol, ps);
    Core core;
    rc = build_core(mol, basis, ps, core);
    if (rc) return rc;
    copy_out(h_core, core.h);
    if (core_ev) *core_ev = core_core_energy(mol, ps);
    return AM1GPU_OK;
}

int oracle_build_fock(const am1gpu_molecule* m, int method, const double* p_tot, const double* p_spin,
                      double spin_scale, double* fock) {
    const ParamSet& ps = params_for(method);
    Molecule mol = to_molecule(m);
    int rc = check_elements(mol, ps);
    if (rc) return rc;
    Basis basis = build_basis(mol, ps);
    Core core;
    rc = build_core(mol, basis, ps, core);
    if (rc) return rc;
    size_t nn = (size_t)basis.nao * basis.nao;
    Mat pt(p_tot, p_tot + nn), psn(p_spin, p_spin + nn);
    copy_out(fock, build_fock_spin(mol, basis, ps, core, pt, psn, spin_scale));
    return AM1GPU_OK;
}

int oracle_symmetric_eigen(int n, const double* a, double* w, double* v) {
    Mat am(a, a + (size_t)n * n), vm;
    std::vector<double> wv;
    int rc = symmetric_eigen(n, am, wv, vm);
    if (rc) return rc;
    copy_out(w, wv);
    copy_out(v, vm);
    return AM1GPU_OK;
}

// Derived element parameters (Am1Element, src/params.rs:24-55) for the known-answer tests:
// out[0..] = n, norb, u_ss, u_pp, zeta_s, zeta_p, beta_s, beta_p, g_ss, g_sp, g_pp, g_p2,
// h_sp, alpha, core_charge, eheat_ev, e_isol, dd, qq, rho0, rho1, rho2, ngauss.
int oracle_element(int method, int z, double out[23]) {
    const ParamSet& ps = params_for(method);
    if (z < 0 || z > NDDO_MAX_Z || !ps.present[z]) return AM1GPU_ELEMENT_NOT_PARAMETERIZED;
    const Elem& e = ps.by_z[z];
    double v[23] = {(double)e.n, (double)e.norb, e.u_ss, e.u_pp, e.zeta_s, e.zeta_p, e.beta_s, e.beta_p,
                    e.g_ss, e.g_sp, e.g_pp, e.g_p2, e.h_sp, e.alpha, e.core_charge, e.eheat_ev, e.e_isol,
                    e.dd, e.qq, e.rho0, e.rho1, e.rho2, (double)e.ngauss};
    std::memcpy(out, v, sizeof v);
    return AM1GPU_OK;
}

// One ordered pair's rotated integral block (w, row-major wcols), e1b/e2a (4x4) and the 4x4
// overlap block S[a][b]: pair_two_electron (integrals.rs:207) + diatom_overlap (overlap.rs:16).
int oracle_pair_block(int method, int za, int zb, const double dvec[3], double w[100], int* wcols, double e1b[16],
                      double e2a[16], double s[16]) {
    const ParamSet& ps = params_for(method);
    if (!ps.present[za] || !ps.present[zb]) return AM1GPU_ELEMENT_NOT_PARAMETERIZED;
    PairTE te;
    pair_two_electron(ps.by_z[za], ps.by_z[zb], dvec, te);
    int nw = (te.wcols == 10) ? 100 : (te.na == 4 ? 10 : 1);
    for (int k = 0; k < nw; ++k) w[k] = te.w[k];
    *wcols = te.wcols;
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
            e1b[a * 4 + b] = te.e1b[a][b];
            e2a[a * 4 + b] = te.e2a[a][b];
        }
    double p0[3] = {0, 0, 0};
    double so[4][4];
    if (!diatom_overlap(ps.by_z[za], p0, ps.by_z[zb], dvec, so)) return AM1GPU_UNSUPPORTED;
    for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) s[a * 4 + b] = so[a][b];
    return AM1GPU_OK;
}

// B_k(x), k = 0..12 (overlap.rs:455) for the series/closed-form continuity test.
void oracle_bintgs(double x, double out[13]) { bintgs(x, out); }

const char* oracle_last_error(void) { return g_err.c_str(); }

}  // extern "C"

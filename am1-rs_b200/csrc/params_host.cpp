// Element parameter derivation for the library (host side, once per process and method).
//
// Follows am1-rs src/params.rs:139-330 and src/data_tables.rs:166-224: the dipole/quadrupole
// charge separations dd, qq (MOPAC ddpo), the Klopman-Ohno additive terms rho0..rho2 (rho1 and
// rho2 by 30 secant steps, MOPAC calpar), the isolated-atom energy e_isol from the
// average-of-configuration coefficients, core charge = n_s + n_p and eheat in eV.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "am1gpu_internal.h"
#include "params/nddo_param_table.h"

namespace am1 {

namespace {

// x^k for small k by repeated squaring (what f64::powi lowers to).
double ipow(double x, int k) {
    double acc = 1.0;
    while (k) {
        if (k & 1) acc *= x;
        k >>= 1;
        if (k) x *= x;
    }
    return acc;
}

// 30 secant steps on target(x) = g(x) from a and a + 0.04 (src/params.rs:290-304, 315-329).
template <class G>
double secant30(double target, double a, G g) {
    double b = a + 0.04;
    for (int it = 0; it < 30; ++it) {
        const double ga = g(a), gb = g(b);
        const double next = std::fabs(gb - ga) > 1.0e-16 ? a + (b - a) * (target - ga) / (gb - ga) : b;
        a = b;
        b = next;
    }
    return b;
}

double rho1_of(double hsp_ev, double d1) {
    const double t = hsp_ev / AM1_EV;
    double start = std::pow(std::fabs(t) / (d1 * d1), 1.0 / 3.0);
    if (t < 0.0) start = -start;
    const double d = secant30(t, start, [d1](double x) { return 0.5 * x - 0.5 / std::sqrt(4.0 * d1 * d1 + 1.0 / (x * x)); });
    return 0.5 / d;
}

double rho2_of(double hpp_ev, double d2) {
    const double t = hpp_ev / AM1_EV;
    double start = std::pow(std::fabs(t) / (3.0 * ipow(d2, 4)), 0.2);
    if (t < 0.0) start = -start;
    const double q = secant30(t, start, [d2](double x) {
        return 0.25 * x - 0.5 / std::sqrt(4.0 * d2 * d2 + 1.0 / (x * x)) + 0.25 / std::sqrt(8.0 * d2 * d2 + 1.0 / (x * x));
    });
    return 0.5 / q;
}

// Average-of-configuration coefficients of the isolated-atom energy (data_tables.rs:166-216),
// in the order e_isol sums them: Gss, Gpp, Gsp, Gp2, Hsp.
void occupation_coefficients(int z, double c[5]) {
    const double ns = NDDO_NS[z], np = NDDO_NP[z];
    const int npi = (int)np;
    static const double gp2_tab[7] = {0.0, 0.0, 1.5, 4.5, 6.5, 10.0, 0.0};
    static const double gpp_tab[7] = {0.0, 0.0, -0.5, -1.5, -0.5, 0.0, 0.0};
    c[0] = ns * (ns - 1.0) / 2.0;
    c[1] = gpp_tab[npi];
    c[2] = ns * np;
    c[3] = gp2_tab[npi];
    c[4] = npi == 6 ? 0.0 : -(double)npi;
}

DevElem derive_element(const nddo_raw_element& row) {
    DevElem e{};
    const double* r = row.raw;
    e.present = 1;
    e.u_ss = r[0]; e.u_pp = r[1]; e.zeta_s = r[2]; e.zeta_p = r[3]; e.beta_s = r[4]; e.beta_p = r[5];
    e.g_ss = r[6]; e.g_sp = r[7]; e.g_pp = r[8]; e.g_p2 = r[9]; e.h_sp = r[10]; e.alpha = r[11];
    e.norb = e.zeta_p > 0.0 ? 4 : 1;
    e.ngauss = 0;
    for (int k = 0; k < 4; ++k) {
        const double K = row.gauss[3 * k], L = row.gauss[3 * k + 1], M = row.gauss[3 * k + 2];
        if (K == 0.0 && L == 0.0) continue;  // src/params.rs:194-199 keeps only nonzero triples
        e.gk[e.ngauss] = K;
        e.gl[e.ngauss] = L;
        e.gm[e.ngauss] = M;
        ++e.ngauss;
    }
    const int z = row.z;
    e.n = NDDO_QN[z];
    if (e.norb == 4) {
        const double nf = e.n;
        e.dd = (2.0 * nf + 1.0) * std::pow(4.0 * e.zeta_s * e.zeta_p, nf + 0.5) /
               std::pow(e.zeta_s + e.zeta_p, 2.0 * nf + 2.0) / std::sqrt(3.0);
        e.qq = std::sqrt((4.0 * nf * nf + 6.0 * nf + 2.0) / 20.0) / e.zeta_p;
        e.rho1 = rho1_of(e.h_sp, e.dd);
        e.rho2 = rho2_of(std::max(0.5 * (e.g_pp - e.g_p2), 0.1), e.qq);
    }
    e.rho0 = 0.5 * AM1_EV / e.g_ss;
    double c[5];
    occupation_coefficients(z, c);
    e.e_isol = e.u_ss * NDDO_NS[z] + e.u_pp * NDDO_NP[z] + e.g_ss * c[0] + e.g_pp * c[1] + e.g_sp * c[2] +
               e.g_p2 * c[3] + e.h_sp * c[4];
    e.core_charge = NDDO_NS[z] + NDDO_NP[z];
    e.eheat_ev = NDDO_EHEAT_KCAL[z] / EV_TO_KCAL;
    return e;
}

}  // namespace

// One table row (raw numbers and Gaussians in the generated table's order) to the derived
// element, as Am1Parameters::from_csv derives each CSV row (z in 0..MAX_Z).
DevElem derive_from_raw(int z, const double raw[12], const double gauss[12]) {
    nddo_raw_element row{};
    row.z = z;
    for (int k = 0; k < 12; ++k) {
        row.raw[k] = raw[k];
        row.gauss[k] = gauss[k];
    }
    return derive_element(row);
}

// Host copy of both methods' tables: [method][Z].
const DevElem* host_param_table() {
    static DevElem table[2][MAX_Z + 1];
    static std::once_flag once;
    std::call_once(once, [] {
        const nddo_raw_element* src[2] = {NDDO_AM1_RAW, NDDO_RM1_RAW};
        const size_t cnt[2] = {sizeof(NDDO_AM1_RAW) / sizeof(NDDO_AM1_RAW[0]), sizeof(NDDO_RM1_RAW) / sizeof(NDDO_RM1_RAW[0])};
        for (int m = 0; m < 2; ++m)
            for (size_t i = 0; i < cnt[m]; ++i) table[m][src[m][i].z] = derive_element(src[m][i]);
    });
    return &table[0][0];
}

}  // namespace am1

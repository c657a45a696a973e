// Host-side (FP64) construction of the ESP tables: the prolate function,
// the split polynomial, the spreading window, quadrature data for the
// influence function. Replaces the compile-time PSWF_Coeffs.h of the
// reference (generate_pswf_table.py:440-506, src/PSWF_Coeffs.h:24-27) by
// tables built at run time for any (c, r_c, P).
#pragma once

#include <vector>

namespace espb {

// psi_0^c(x) = sum_k coef[k] P_{2k}(x) (un-normalised Legendre P, even degrees).
struct Prolate {
    double c = 0.0;
    std::vector<double> coef;  // coefficient of P_{2k}
    double psi0 = 0.0;         // psi(0)
    double int01 = 0.0;        // int_0^1 psi
    void build(double c_);
    double psi(double x) const;       // accurate for |x| <= 1
    double integral(double s) const;  // int_0^s psi, |s| <= 1
};

// Short-range split S(s) = 1 - s Q(s^2); Q stored as a monomial series in
// v = 2u - 1 (u = s^2) for FP32-stable Horner evaluation on the device.
struct Split {
    double c = 0.0;
    std::vector<double> qv;  // Q(u) = sum_j qv[j] v^j, v = 2u-1
    double lambda0 = 0.0;    // Q(0): Lambda(0) = lambda0 / (4 pi r_c)
    double m2 = 0.0;         // int_0^1 psi t^2 / int_0^1 psi
    double fit_err = 0.0;
    Prolate pro;
    // Gauss-Legendre data on [0,1] with weights * psi(t)/int01, for
    // Psi(kappa) = sum_j wq[j] cos(kappa tq[j]).
    std::vector<double> tq, wq;
    void build(double c_, double tol = 1e-8);
    double Q(double u) const;
    double dQdu(double u) const;
    double fourier_ratio(double kappa) const;
};

// Window w(u) = psi_cw(2u/P)/psi_cw(0) on |u| <= P/2, P unit segments,
// degree-D monomials in t in [0,1]: coef[a*(D+1) + j].
struct Window {
    int P = 0;
    int D = 0;
    double c = 0.0;
    std::vector<double> coef;
    double fit_err = 0.0;
    void build(int P_, double c_, int D_ = 0);
    // grid-unit Fourier transform w_hat(xi) of the fitted polynomials.
    double fourier(double xi) const;
};

void gauss_legendre01(int n, std::vector<double>& t, std::vector<double>& w);
int smooth235(int n);

}  // namespace espb

// Host-side FP64 table construction (see esp_tables.h).
//
// The prolate psi_0^c is the lowest eigenvector of the prolate operator
// -((1-x^2)y')' + c^2 x^2 y in the even normalised-Legendre basis (a
// symmetric tridiagonal matrix): smallest eigenvalue by Sturm-sequence
// bisection, eigenvector by one-shift inverse iteration. The reference
// evaluates psi with scipy.special.pro_ang1 instead
// (generate_pswf_table.py:120-123).
#include "esp_tables.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace espb {

namespace {

// Legendre P_0..P_n at x.
void legendre_all(double x, int n, std::vector<double>& p) {
    p.assign(n + 1, 0.0);
    p[0] = 1.0;
    if (n >= 1) p[1] = x;
    for (int k = 1; k < n; ++k) p[k + 1] = ((2.0 * k + 1.0) * x * p[k] - k * p[k - 1]) / (k + 1.0);
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x.
int sturm_count(const std::vector<double>& d, const std::vector<double>& e, double x) {
    int cnt = 0;
    double q = d[0] - x;
    if (q < 0) ++cnt;
    for (size_t i = 1; i < d.size(); ++i) {
        double den = (q == 0.0) ? 1e-300 : q;
        q = d[i] - x - e[i - 1] * e[i - 1] / den;
        if (q < 0) ++cnt;
    }
    return cnt;
}

// Chebyshev interpolation of f on x in [-1,1] at n=deg+1 first-kind nodes,
// returned as monomial coefficients in x.
template <class F>
std::vector<double> cheb_interp_monomial(F f, int deg) {
    const int n = deg + 1;
    std::vector<double> fx(n), a(n, 0.0);
    for (int j = 0; j < n; ++j) fx[j] = f(std::cos(M_PI * (j + 0.5) / n));
    for (int m = 0; m < n; ++m) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += fx[j] * std::cos(M_PI * m * (j + 0.5) / n);
        a[m] = 2.0 * s / n;
    }
    a[0] *= 0.5;
    // T_m as monomials: T_0 = 1, T_1 = x, T_{m+1} = 2x T_m - T_{m-1}
    std::vector<double> out(n, 0.0), tm1(n, 0.0), tm(n, 0.0), tp(n, 0.0);
    tm1[0] = 1.0;
    tm[1] = n > 1 ? 1.0 : 0.0;
    for (int j = 0; j < n; ++j) out[j] += a[0] * tm1[j];
    if (n > 1)
        for (int j = 0; j < n; ++j) out[j] += a[1] * tm[j];
    for (int m = 1; m + 1 < n; ++m) {
        std::fill(tp.begin(), tp.end(), 0.0);
        for (int j = 0; j + 1 < n; ++j) tp[j + 1] += 2.0 * tm[j];
        for (int j = 0; j < n; ++j) tp[j] -= tm1[j];
        for (int j = 0; j < n; ++j) out[j] += a[m + 1] * tp[j];
        tm1 = tm;
        tm = tp;
    }
    return out;
}

double polyval(const std::vector<double>& c, double x) {
    double v = 0.0;
    for (int j = (int)c.size() - 1; j >= 0; --j) v = v * x + c[j];
    return v;
}

}  // namespace

void gauss_legendre01(int n, std::vector<double>& t, std::vector<double>& w) {
    t.resize(n);
    w.resize(n);
    for (int i = 0; i < n; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 1; k < n; ++k) {
                double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
                p0 = p1;
                p1 = p2;
            }
            dp = n * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        double p0 = 1.0, p1 = x;
        for (int k = 1; k < n; ++k) {
            double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
            p0 = p1;
            p1 = p2;
        }
        dp = n * (x * p1 - p0) / (x * x - 1.0);
        t[i] = 0.5 * (x + 1.0);
        w[i] = 1.0 / ((1.0 - x * x) * dp * dp);  // 2/((1-x^2)P'^2) scaled by 1/2
    }
}

int smooth235(int n) {
    int m = std::max(n, 1);
    for (;; ++m) {
        int k = m;
        for (int p : {2, 3, 5})
            while (k % p == 0) k /= p;
        if (k == 1) return m;
    }
}

void Prolate::build(double c_) {
    c = c_;
    const int K = (int)std::ceil(c) + 40;
    std::vector<double> d(K), e(K - 1);
    const double c2 = c * c;
    for (int k = 0; k < K; ++k) {
        const double n = 2.0 * k;
        d[k] = n * (n + 1) + c2 * (2 * n * (n + 1) - 1) / ((2 * n + 3) * (2 * n - 1));
        if (k + 1 < K) e[k] = c2 * (n + 1) * (n + 2) / ((2 * n + 3) * std::sqrt((2 * n + 1) * (2 * n + 5)));
    }
    double lo = d[0] - 2 * std::fabs(e[0]) - 1.0, hi = d[0] + 2 * std::fabs(e[0]) + 1.0;
    for (int i = 0; i < 200; ++i) {
        double mid = 0.5 * (lo + hi);
        if (sturm_count(d, e, mid) >= 1)
            hi = mid;
        else
            lo = mid;
    }
    const double lam = lo;
    // inverse iteration with a shift just below the eigenvalue: A - sigma I is SPD
    const double sigma = lam - 1e-9 * std::max(1.0, std::fabs(lam));
    std::vector<double> x(K, 1.0), cp(K), dp(K);
    for (int it = 0; it < 4; ++it) {
        // Thomas algorithm on (A - sigma I) y = x
        double b0 = d[0] - sigma;
        cp[0] = (K > 1 ? e[0] : 0.0) / b0;
        dp[0] = x[0] / b0;
        for (int k = 1; k < K; ++k) {
            double b = d[k] - sigma - e[k - 1] * cp[k - 1];
            cp[k] = (k + 1 < K ? e[k] : 0.0) / b;
            dp[k] = (x[k] - e[k - 1] * dp[k - 1]) / b;
        }
        std::vector<double> y(K);
        y[K - 1] = dp[K - 1];
        for (int k = K - 2; k >= 0; --k) y[k] = dp[k] - cp[k] * y[k + 1];
        double nrm = 0.0;
        for (double v : y) nrm += v * v;
        nrm = std::sqrt(nrm);
        for (int k = 0; k < K; ++k) x[k] = y[k] / nrm;
    }
    coef.resize(K);
    for (int k = 0; k < K; ++k) coef[k] = x[k] * std::sqrt((4.0 * k + 1.0) / 2.0);
    psi0 = psi(0.0);
    if (psi0 < 0) {
        for (double& v : coef) v = -v;
        psi0 = -psi0;
    }
    int01 = integral(1.0);
}

double Prolate::psi(double xv) const {
    std::vector<double> p;
    const int K = (int)coef.size();
    legendre_all(xv, 2 * K, p);
    double s = 0.0;
    for (int k = 0; k < K; ++k) s += coef[k] * p[2 * k];
    return s;
}

double Prolate::integral(double s) const {
    std::vector<double> p;
    const int K = (int)coef.size();
    legendre_all(s, 2 * K + 1, p);
    double acc = coef[0] * s;
    for (int k = 1; k < K; ++k) {
        const int n = 2 * k;
        acc += coef[k] * (p[n + 1] - p[n - 1]) / (2.0 * n + 1.0);
    }
    return acc;
}

void Split::build(double c_, double tol) {
    c = c_;
    pro.build(c);
    auto qfun = [this](double u) {
        double s = std::sqrt(std::max(u, 0.0));
        if (s < 1e-6) return pro.psi(s) / pro.int01;
        return pro.integral(s) / (s * pro.int01);
    };
    for (int deg = 6; deg <= 30; ++deg) {
        qv = cheb_interp_monomial([&](double v) { return qfun(0.5 * (v + 1.0)); }, deg);
        // pin Q(1) = 1 (v = 1: sum of the coefficients), i.e. S(r_c) = 0, so
        // the pair energy is continuous at the cutoff
        double s1 = 0.0;
        for (double c : qv) s1 += c;
        qv[0] += 1.0 - s1;
        double err = 0.0;
        for (int i = 0; i <= 2000; ++i) {
            double u = i / 2000.0;
            err = std::max(err, std::fabs(polyval(qv, 2 * u - 1) - qfun(u)));
        }
        fit_err = err;
        if (err < tol) break;
    }
    lambda0 = qfun(0.0);
    std::vector<double> t, w;
    gauss_legendre01(64, t, w);
    double s = 0.0;
    for (int j = 0; j < 64; ++j) s += w[j] * pro.psi(t[j]) * t[j] * t[j];
    m2 = s / pro.int01;
    gauss_legendre01(128, tq, wq);
    for (size_t j = 0; j < tq.size(); ++j) wq[j] *= pro.psi(tq[j]) / pro.int01;
}

double Split::Q(double u) const { return polyval(qv, 2 * u - 1); }

double Split::dQdu(double u) const {
    double v = 2 * u - 1, d = 0.0;
    for (int j = (int)qv.size() - 1; j >= 1; --j) d = d * v + j * qv[j];
    return 2.0 * d;
}

double Split::fourier_ratio(double kappa) const {
    double s = 0.0;
    for (size_t j = 0; j < tq.size(); ++j) s += wq[j] * std::cos(kappa * tq[j]);
    return s;
}

void Window::build(int P_, double c_, int D_) {
    P = P_;
    c = c_;
    D = D_ > 0 ? D_ : std::max(P + 2, 9);
    if (P < 2 || P > 12) throw std::invalid_argument("window support P must be in [2, 12]");
    if (D > 15) throw std::invalid_argument("window degree must be <= 15");
    Prolate pro;
    pro.build(c);
    coef.assign((size_t)P * (D + 1), 0.0);
    fit_err = 0.0;
    for (int a = 0; a < P; ++a) {
        auto f = [&](double t) {
            double u = a - 0.5 * P + t;
            double x = std::min(1.0, std::max(-1.0, 2.0 * u / P));
            return pro.psi(x) / pro.psi0;
        };
        // interpolate in x = 2t-1, then substitute x = 2t - 1
        std::vector<double> mx = cheb_interp_monomial([&](double x) { return f(0.5 * (x + 1.0)); }, D);
        std::vector<double> mt(D + 1, 0.0), pw(D + 1, 0.0), nxt(D + 1, 0.0);
        pw[0] = 1.0;  // (2t-1)^j
        for (int j = 0; j <= D; ++j) {
            for (int i = 0; i <= D; ++i) mt[i] += mx[j] * pw[i];
            std::fill(nxt.begin(), nxt.end(), 0.0);
            for (int i = 0; i < D; ++i) {
                nxt[i + 1] += 2.0 * pw[i];
                nxt[i] -= pw[i];
            }
            pw = nxt;
        }
        for (int j = 0; j <= D; ++j) coef[(size_t)a * (D + 1) + j] = mt[j];
        for (int i = 0; i <= 256; ++i) {
            double t = i / 256.0;
            fit_err = std::max(fit_err, std::fabs(polyval(mt, t) - f(t)));
        }
    }
}

double Window::fourier(double xi) const {
    static thread_local std::vector<double> t, w;
    if (t.size() != 24) gauss_legendre01(24, t, w);
    double s = 0.0;
    for (int a = 0; a < P; ++a) {
        const double* c0 = &coef[(size_t)a * (D + 1)];
        for (int q = 0; q < 24; ++q) {
            double v = 0.0;
            for (int j = D; j >= 0; --j) v = v * t[q] + c0[j];
            s += w[q] * v * std::cos(xi * (a - 0.5 * P + t[q]));
        }
    }
    return s;
}

}  // namespace espb

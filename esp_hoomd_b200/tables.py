"""PSWF tables for the ESP (Ewald Summation with Prolates) split.

This module is the runtime table generator: it replaces the compile-time
``PSWF_Coeffs.h`` of the reference plugin (generated offline by
``generate_pswf_table.py:440-506`` and baked in with ``PSWF_RCUT=1``,
``src/PSWF_Coeffs.h:24-27``) by tables built per (epsilon, r_c, P) at run
time, in reduced units ``s = r / r_c`` so one table serves any cutoff.

Mathematics (Liang, Lu, Barnett, Greengard, Jiang, "Accelerating molecular
dynamics simulations using fast Ewald summation with prolates", cited at
``src/EvaluatorPairPSWF.h:58-62``):

* ``psi(x)`` is the zeroth prolate spheroidal wave function psi_0^c on
  [-1, 1], computed here as the lowest eigenvector of the prolate
  differential operator in a normalised Legendre basis (the reference calls
  ``scipy.special.pro_ang1``, ``generate_pswf_table.py:120-123``).
* Split: ``1/(4 pi r) = L(r) + Lambda(r)`` with the screening function
  ``S(s) = 1 - int_0^s psi / int_0^1 psi`` (so ``S(0)=1``, ``S(1)=0``) and
  ``L(r) = S(r/r_c)/(4 pi r)``.  The reference uses the CDF of psi^2 on
  [-1, 1] (``generate_pswf_table.py:114-118, 159-165``), which gives
  ``S(0)=1/2`` and is not a Coulomb split; the form here has the exact
  compact support and the PSWF Fourier decay the method relies on.
* Because ``int_0^s psi`` is odd in s, ``S(s) = 1 - s Q(s^2)`` with ``Q`` a
  smooth polynomial, hence ``4 pi L(r) = 1/r - Q(r^2/r_c^2)/r_c``: the pair
  term needs no sqrt-indexed segment table on the fast path.
* Fourier side: ``Lambda_hat(k) = Psi(k r_c)/k^2`` with
  ``Psi(kappa) = int_0^1 psi(t) cos(kappa t) dt / int_0^1 psi``
  (``= psi(kappa/c)/psi(0)`` by the PSWF eigen-relation).
* Spreading window: ``w(u) = psi_{c_w}(2u/P)`` on ``|u| <= P/2`` grid
  units, stored as P per-unit-segment polynomials in ``t in [0, 1]``
  (the reference's stencil format ``PSWF_STENCIL_COEFFS[P][5]``,
  ``src/PSWF_Coeffs.h:9606-9624``, here with configurable degree because
  degree 4 limits the weights to ~1e-5).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence, Tuple

import numpy as np

INV_4PI = 0.079577471545947673  # ESP_INV_4PI, src/ESPForceCompute.cc:36

# ---------------------------------------------------------------------------
# Zeroth prolate spheroidal wave function
# ---------------------------------------------------------------------------


class Prolate:
    """psi_0^c(x) as a normalised-Legendre series sum_k beta_k Pbar_k(x).

    The prolate operator ``-((1-x^2) y')' + c^2 x^2 y`` is tridiagonal on
    the even normalised Legendre functions; its lowest eigenvector gives the
    series coefficients of psi_0^c (Bouwkamp / Xiao-Rokhlin-Yarvin method).
    The sign is fixed so that psi(0) > 0; the overall scale is irrelevant to
    every quantity derived here (all are ratios).
    """

    def __init__(self, c: float, n_terms: Optional[int] = None):
        self.c = float(c)
        n = n_terms or int(2 * self.c + 60)
        ks = np.arange(0, 2 * n, 2, dtype=np.float64)  # even degrees
        c2 = self.c * self.c
        diag = ks * (ks + 1) + c2 * (2 * ks * (ks + 1) - 1) / ((2 * ks + 3) * (2 * ks - 1))
        off = c2 * (ks[:-1] + 1) * (ks[:-1] + 2) / (
            (2 * ks[:-1] + 3) * np.sqrt((2 * ks[:-1] + 1) * (2 * ks[:-1] + 5)))
        a = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
        w, v = np.linalg.eigh(a)
        beta = v[:, 0]
        self.chi = float(w[0])
        self.degrees = ks.astype(np.int64)
        # coefficients of the un-normalised Legendre polynomials P_k
        coef = beta * np.sqrt((2 * ks + 1) / 2.0)
        if self._legendre_sum(coef, np.array([0.0]))[0] < 0:
            coef = -coef
        self._coef = coef
        self.psi0 = float(self._legendre_sum(coef, np.array([0.0]))[0])
        self.int01 = float(self.integral(np.array([1.0]))[0])

    def _legendre_sum(self, coef: np.ndarray, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        kmax = int(self.degrees[-1]) + 1
        full = np.zeros(kmax + 1)
        full[self.degrees] = coef
        return np.polynomial.legendre.legval(x, full)

    def psi(self, x) -> np.ndarray:
        """psi_0^c(x) (Legendre series; accurate for |x| <= 1)."""
        return self._legendre_sum(self._coef, x)

    def integral(self, s) -> np.ndarray:
        """int_0^s psi(t) dt for |s| <= 1."""
        s = np.asarray(s, dtype=np.float64)
        kmax = int(self.degrees[-1]) + 2
        full = np.zeros(kmax + 1)
        # int_0^s P_0 = s = P_1(s); int_0^s P_k = (P_{k+1} - P_{k-1})/(2k+1), k even >= 2
        for k, a in zip(self.degrees, self._coef):
            if k == 0:
                full[1] += a
            else:
                full[k + 1] += a / (2 * k + 1)
                full[k - 1] -= a / (2 * k + 1)
        return np.polynomial.legendre.legval(s, full)

    def fourier_ratio(self, kappa, n_quad: int = 96) -> np.ndarray:
        """Psi(kappa) = int_0^1 psi(t) cos(kappa t) dt / int_0^1 psi.

        Gauss-Legendre quadrature on [0, 1]; stable for any kappa (the
        Legendre series itself loses accuracy for |x| > 1).
        """
        kappa = np.atleast_1d(np.asarray(kappa, dtype=np.float64))
        nq = max(n_quad, int(np.max(np.abs(kappa), initial=0.0) * 0.6) + 40)
        x, w = np.polynomial.legendre.leggauss(nq)
        t = 0.5 * (x + 1.0)
        w = 0.5 * w * self.psi(t) / self.int01
        return np.cos(np.outer(kappa, t)) @ w


# ---------------------------------------------------------------------------
# Split (short-range screening) polynomial
# ---------------------------------------------------------------------------


def _cheb_interp_monomial(f, degree: int):
    """Chebyshev interpolation of f on x in [-1, 1] at degree+1 first-kind
    nodes, returned as monomial coefficients in x (increasing powers).
    Same construction as the C++ builder (csrc/esp_tables.cpp)."""
    n = degree + 1
    j = np.arange(n)
    x = np.cos(np.pi * (j + 0.5) / n)
    fx = f(x)
    m = np.arange(n)
    a = 2.0 / n * (np.cos(np.pi * np.outer(m, j + 0.5) / n) @ fx)
    a[0] *= 0.5
    return np.polynomial.chebyshev.cheb2poly(a)


@dataclasses.dataclass
class SplitTable:
    """Short-range split in reduced units s = r / r_c.

    ``qv``: monomial coefficients (increasing powers of v = 2u - 1, u = s^2)
    of Q, with ``S(s) = 1 - s Q(s^2)``; the v form keeps FP32 Horner
    evaluation at round-off level.
    ``lambda0``: r_c * Lambda(0) * 4 pi = Q(0) (the long-range kernel at the
    origin, reduced): ``Lambda(0) = Q(0) / (4 pi r_c)``.
    ``m2``: int_0^1 psi t^2 dt / int_0^1 psi, so ``int L d^3r = r_c^2 m2 / 2``.
    """

    c: float
    qv: np.ndarray
    lambda0: float
    m2: float
    fit_err: float
    prolate: Prolate

    def S(self, s):
        s = np.asarray(s, dtype=np.float64)
        out = 1.0 - self.prolate.integral(np.clip(s, 0, 1)) / self.prolate.int01
        return np.where(s >= 1.0, 0.0, out)

    def dS(self, s):
        """dS/ds."""
        s = np.asarray(s, dtype=np.float64)
        out = -self.prolate.psi(np.clip(s, 0, 1)) / self.prolate.int01
        return np.where(s >= 1.0, 0.0, out)

    def Q(self, u):
        v = 2.0 * np.asarray(u, dtype=np.float64) - 1.0
        return np.polynomial.polynomial.polyval(v, self.qv)

    def dQ(self, u):
        """dQ/du."""
        v = 2.0 * np.asarray(u, dtype=np.float64) - 1.0
        return 2.0 * np.polynomial.polynomial.polyval(v, np.polynomial.polynomial.polyder(self.qv))

    def fourier_ratio(self, kappa):
        return self.prolate.fourier_ratio(kappa)


def make_split(c: float, degree: int = 0, tol: float = 1e-8) -> SplitTable:
    pro = Prolate(c)

    def qfun(u):
        s = np.sqrt(np.maximum(u, 0.0))
        out = np.empty_like(s)
        small = s < 1e-6
        out[~small] = pro.integral(s[~small]) / (s[~small] * pro.int01)
        out[small] = pro.psi(s[small]) / pro.int01
        return out

    uu = np.linspace(0.0, 1.0, 2001)
    degs = [degree] if degree else range(6, 31)
    for d in degs:
        qv = _cheb_interp_monomial(lambda v: qfun(0.5 * (v + 1.0)), d)
        # pin Q(1) = 1, i.e. S(r_c) = 0: the pair energy is continuous at r_c
        qv[0] += 1.0 - float(np.sum(qv))
        err =float(np.max(np.abs(np.polynomial.polynomial.polyval(2 * uu - 1, qv) - qfun(uu))))
        if err < tol:
            break
    xg, wg = np.polynomial.legendre.leggauss(64)
    t = 0.5 * (xg + 1)
    m2 = float(np.sum(0.5 * wg * pro.psi(t) * t * t) / pro.int01)
    return SplitTable(c=float(c), qv=qv, lambda0=float(qfun(np.array([0.0]))[0]),
                      m2=m2, fit_err=err, prolate=pro)


# ---------------------------------------------------------------------------
# Spreading / interpolation window
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class Window:
    """Separable 1D window on |u| <= P/2 grid units, P unit segments.

    Segment ``a`` covers ``u in [a - P/2, a - P/2 + 1]`` and holds a
    polynomial in ``t in [0, 1]`` (``coef[a, j]`` = coefficient of t^j).
    For a particle at grid coordinate ``g`` the first stencil point is
    ``i0 = floor(g - P/2) + 1`` and ``t = i0 + P/2 - g in (0, 1]``; the
    weight of point ``i0 + a`` is ``p_a(t)`` -- every segment is evaluated
    at the SAME t (the reference's per-tap argument mapping is wrong,
    ``src/ESPForceComputeGPU.cu:138-152, 249-254``).
    """

    P: int
    c: float
    coef: np.ndarray  # [P, D+1]
    fit_err: float

    @property
    def degree(self) -> int:
        return self.coef.shape[1] - 1

    def weights(self, t):
        """w[a] at local coordinate t (vectorised over t)."""
        t = np.asarray(t, dtype=np.float64)
        return np.stack([np.polynomial.polynomial.polyval(t, self.coef[a]) for a in range(self.P)], -1)

    def dweights(self, t):
        """d w[a] / d t."""
        t = np.asarray(t, dtype=np.float64)
        return np.stack([np.polynomial.polynomial.polyval(
            t, np.polynomial.polynomial.polyder(self.coef[a])) for a in range(self.P)], -1)

    def value(self, u):
        """Window w(u) at offsets u (grid units) from the particle."""
        u = np.asarray(u, dtype=np.float64)
        out = np.zeros_like(u)
        x = u + self.P / 2.0
        a = np.floor(x).astype(np.int64)
        ok = (a >= 0) & (a < self.P)
        t = x - a
        for s in range(self.P):
            m = ok & (a == s)
            out[m] = np.polynomial.polynomial.polyval(t[m], self.coef[s])
        return out

    def fourier(self, xi, n_gauss: int = 24):
        """w_hat(xi) = int w(u) exp(-i xi u) du, xi in radians per grid unit.

        Computed from the FITTED polynomials (the window actually used), so
        dividing by it de-convolves exactly what spreading applied.
        """
        xi = np.atleast_1d(np.asarray(xi, dtype=np.float64))
        xg, wg = np.polynomial.legendre.leggauss(n_gauss)
        t = 0.5 * (xg + 1)
        wg = 0.5 * wg
        out = np.zeros_like(xi)
        for a in range(self.P):
            u = a - self.P / 2.0 + t
            vals = np.polynomial.polynomial.polyval(t, self.coef[a]) * wg
            out += np.cos(np.outer(xi, u)) @ vals
        return out


def make_window(P: int, c: float, degree: int = 0) -> Window:
    """Interpolate psi_c(2u/P)/psi_c(0) on each unit segment at degree+1
    Chebyshev nodes (same construction as csrc/esp_tables.cpp)."""
    pro = Prolate(c)
    D = degree or max(P + 2, 9)
    coefs = []
    errs = []
    half = np.polynomial.Polynomial([-1.0, 2.0])  # x = 2t - 1
    for a in range(P):
        def f(t, a=a):
            u = a - P / 2.0 + t
            return pro.psi(np.clip(2.0 * u / P, -1, 1)) / pro.psi0
        mx = _cheb_interp_monomial(lambda x: f(0.5 * (x + 1.0)), D)
        coef = np.polynomial.Polynomial(mx)(half).coef
        coef = np.concatenate([coef, np.zeros(D + 1 - coef.size)])
        tt = np.linspace(0, 1, 257)
        errs.append(float(np.max(np.abs(np.polynomial.polynomial.polyval(tt, coef) - f(tt)))))
        coefs.append(coef)
    return Window(P=int(P), c=float(c), coef=np.array(coefs), fit_err=max(errs))


# ---------------------------------------------------------------------------
# Parameter sets
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class ESPParams:
    """Everything the mesh + pair stages need for one system.

    mesh: (nx, ny, nz); box: (Lx, Ly, Lz) orthorhombic; rcut: real-space
    cutoff; split: SplitTable; window: Window.
    """

    mesh: Tuple[int, int, int]
    box: Tuple[float, float, float]
    rcut: float
    split: SplitTable
    window: Window

    @property
    def P(self) -> int:
        return self.window.P


def window_shape_for(P: int, sigma: float) -> float:
    """Window bandwidth c_w for P points at oversampling sigma.

    Chosen like the 'exponential of semicircle' rule (c_w ~ pi P (1 - 1/(2
    sigma)) * 0.98), the relation NUFFT kernels use between support,
    oversampling and shape; then refined by :func:`tune_window`.
    """
    sigma = max(sigma, 1.05)
    return 0.98 * math.pi * P * (1.0 - 0.5 / sigma)


def smooth235(n: int) -> int:
    """Smallest 2/3/5-smooth integer >= n."""
    m = max(int(n), 1)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


_SPLIT_CACHE: dict = {}
_WINDOW_CACHE: dict = {}


def split_cached(c: float) -> SplitTable:
    key = round(float(c), 6)
    if key not in _SPLIT_CACHE:
        _SPLIT_CACHE[key] = make_split(key)
    return _SPLIT_CACHE[key]


def window_cached(P: int, c: float, degree: int = 0) -> Window:
    key = (int(P), round(float(c), 6), int(degree))
    if key not in _WINDOW_CACHE:
        _WINDOW_CACHE[key] = make_window(int(P), key[1], degree)
    return _WINDOW_CACHE[key]


# ---------------------------------------------------------------------------
# Reference-format (PSWF_Coeffs.h) segment tables
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class SegmentTable:
    """S(r) and S'(r) as per-segment Horner polynomials in t in [0,1].

    Layout of ``src/PSWF_Coeffs.h:29-30, 4130, 8229, 8915``:
    ``screen[seg*5 + j]``, ``dscreen[seg*5 + j]``, ``r_lo[seg]``,
    ``dr_inv[seg]``, cutoff ``rcut`` (PSWF_RCUT). The lookup is
    ``detail::pswf_eval_L`` of ``src/EvaluatorPairPSWF.h:113-143``.
    """

    rcut: float
    screen: np.ndarray  # [n_segs*5] float64
    dscreen: np.ndarray
    r_lo: np.ndarray
    dr_inv: np.ndarray

    @property
    def n_segs(self) -> int:
        return int(self.r_lo.shape[0])


def parse_pswf_coeffs_header(text: str) -> SegmentTable:
    """Read a PSWF_Coeffs.h-format header (as emitted by
    ``generate_pswf_table.py:440-506``) into a SegmentTable."""
    import re

    def arr(name):
        m = re.search(r"%s\[(\d+)\]\s*=\s*\{(.*?)\};" % name, text, re.S)
        if not m:
            raise ValueError("array %s not found" % name)
        vals = np.array([float(v) for v in m.group(2).replace("\n", " ").split(",") if v.strip()])
        if vals.size != int(m.group(1)):
            raise ValueError("array %s has %d values, declared %s" % (name, vals.size, m.group(1)))
        return vals

    m = re.search(r"PSWF_RCUT\s*=\s*([0-9eE+\-.]+);", text)
    rcut = float(m.group(1)) if m else 1.0
    return SegmentTable(rcut=rcut, screen=arr("PSWF_SCREEN_COEFFS"), dscreen=arr("PSWF_DSCREEN_COEFFS"),
                        r_lo=arr("PSWF_R_LO"), dr_inv=arr("PSWF_DR_INV"))


def segment_table_from_split(split: SplitTable, rcut: float, n_segs: int = 4096) -> SegmentTable:
    """Tabulate the ESP split in the reference's segment format (degree 4,
    interpolating at Chebyshev points of each segment)."""
    seg_w = rcut / n_segs
    screen = np.zeros((n_segs, 5))
    dscreen = np.zeros((n_segs, 5))
    j = np.arange(5)
    tn = 0.5 - 0.5 * np.cos(np.pi * (j + 0.5) / 5)
    V = np.vander(tn, 5, increasing=True)
    Vinv = np.linalg.inv(V)
    for i in range(n_segs):
        r = (i + tn) * seg_w
        screen[i] = Vinv @ split.S(r / rcut)
        dscreen[i] = Vinv @ (split.dS(r / rcut) / rcut)
    return SegmentTable(rcut=rcut, screen=screen.ravel(), dscreen=dscreen.ravel(),
                        r_lo=np.arange(n_segs) * seg_w, dr_inv=np.full(n_segs, 1.0 / seg_w))


def emit_pswf_coeffs_header(tab: SegmentTable, window: Optional[Window] = None, c: float = 0.0) -> str:
    """Emit a header in the PSWF_Coeffs.h layout (names and array shapes of
    ``src/PSWF_Coeffs.h``), so a HOOMD build of the reference evaluator can
    consume tables generated here."""
    def fmt(name, vals, per=5):
        vals = np.asarray(vals, dtype=np.float64).ravel()
        lines = ["    " + ", ".join("%.17e" % v for v in vals[i:i + per]) + ","
                 for i in range(0, vals.size, per)]
        return "inline constexpr double %s[%d] = {\n%s\n};\n" % (name, vals.size, "\n".join(lines))

    out = ["// PSWF_Coeffs.h layout, generated by esp_hoomd_b200.tables", "#pragma once", "",
           "namespace hoomd\n{\nnamespace md\n{\nnamespace esp_pswf_coeffs\n{", "",
           "inline constexpr int PSWF_N_SEGS = %d;" % tab.n_segs,
           "inline constexpr int PSWF_ORDER = %d;" % (window.P if window else 0),
           "inline constexpr double PSWF_C = %.17e;" % c,
           "inline constexpr double PSWF_RCUT = %.17e;" % tab.rcut, "",
           fmt("PSWF_SCREEN_COEFFS", tab.screen), fmt("PSWF_DSCREEN_COEFFS", tab.dscreen),
           fmt("PSWF_R_LO", tab.r_lo, 6), fmt("PSWF_DR_INV", tab.dr_inv, 6)]
    if window is not None:
        out += ["inline constexpr int PSWF_STENCIL_ORDER = %d;" % window.P, "",
                fmt("PSWF_STENCIL_COEFFS", window.coef, window.coef.shape[1])]
    out += ["} // namespace esp_pswf_coeffs\n} // namespace md\n} // namespace hoomd", ""]
    return "\n".join(out)


def eval_segment_L(tab: SegmentTable, r, rcut: Optional[float] = None):
    """FP64 restatement of ``detail::pswf_eval_L`` (``src/EvaluatorPairPSWF.h:113-143``):
    returns (L, -dL/dr) with the reference's segment and t arithmetic."""
    rcut = tab.rcut if rcut is None else rcut
    r = np.atleast_1d(np.asarray(r, dtype=np.float64))
    L = np.zeros_like(r)
    D = np.zeros_like(r)
    ok = ~((r < 1e-12) | (r > rcut))
    s = np.clip(r[ok] / rcut, 0.0, 1.0 - 1e-9)
    seg = np.minimum((s * tab.n_segs).astype(np.int64), tab.n_segs - 1)
    t = (r[ok] - tab.r_lo[seg]) * tab.dr_inv[seg]
    cs = tab.screen.reshape(-1, 5)[seg]
    cd = tab.dscreen.reshape(-1, 5)[seg]

    def horner(c):
        v = c[:, 4]
        for j in (3, 2, 1, 0):
            v = c[:, j] + t * v
        return v

    S = horner(cs)
    dS = horner(cd)
    inv4pir = INV_4PI / r[ok]
    inv4pir2 = inv4pir / r[ok]
    L[ok] = S * inv4pir
    D[ok] = S * inv4pir2 - dS * inv4pir
    return L, D

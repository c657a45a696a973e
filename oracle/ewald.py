"""FP64 direct Ewald sum -- the physics oracle (test infrastructure only).

The reference's own force/energy results are unavailable (its CPU stages
are stubs, ``src/ESPForceCompute.cc:200-248``, and its GPU overrides are
never dispatched, ``src/ESPForceCompute.h:131-175``), so every ESP result is
pinned against this textbook Gaussian-split Ewald sum, written in the
reference's unit convention ``E = q_i q_j / (4 pi r)`` (``ESP_INV_4PI``,
``src/ESPForceCompute.cc:36``).

Parameters are chosen so the Ewald truncation error is < 1e-12 relative:
alpha from ``erfc(alpha r_c) < 1e-16`` with the minimum-image real-space
cutoff ``r_c = min(L)/2``, and the k-space sphere from
``exp(-k^2/4 alpha^2) < 1e-17``.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc

INV_4PI = 0.079577471545947673


def ewald(pos, q, box, tol_exp: float = 38.0, chunk: int = 2048):
    """Return (energy, forces[N,3], virial[6]) for point charges in an
    orthorhombic periodic box; virial order xx, xy, xz, yy, yz, zz with
    ``W_ab = -dE/d eps_ab`` (pair form ``sum r_ij,a F_ij,b``)."""
    pos = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    L = np.asarray(box, dtype=np.float64)
    N = pos.shape[0]
    V = float(np.prod(L))
    rc = 0.5 * float(L.min())
    alpha = math.sqrt(tol_exp) / rc
    F = np.zeros((N, 3))
    W = np.zeros((3, 3))
    E_real = 0.0
    for s in range(0, N, chunk):
        d = pos[s:s + chunk, None, :] - pos[None, :, :]
        d -= L * np.round(d / L)
        r2 = np.sum(d * d, -1)
        idx = np.arange(s, min(s + chunk, N))
        r2[np.arange(idx.size), idx] = np.inf
        m = r2 < rc * rc
        r = np.sqrt(np.where(m, r2, 1.0))
        qq = q[idx, None] * q[None, :]
        e = np.where(m, qq * erfc(alpha * r) / r, 0.0) * INV_4PI
        E_real += 0.5 * e.sum()
        fdr = np.where(m, qq * (erfc(alpha * r) / r + 2 * alpha / math.sqrt(math.pi)
                                * np.exp(-alpha * alpha * r * r)) / (r * r), 0.0) * INV_4PI
        F[idx] += np.einsum("ij,ijk->ik", fdr, d)
        W += 0.5 * np.einsum("ij,ija,ijb->ab", fdr, d, d)
    kmax = 2 * alpha * math.sqrt(tol_exp)
    nmax = [int(math.ceil(kmax * Li / (2 * math.pi))) for Li in L]
    nx = np.arange(0, nmax[0] + 1)
    ny = np.arange(-nmax[1], nmax[1] + 1)
    nz = np.arange(-nmax[2], nmax[2] + 1)
    NX, NY, NZ = np.meshgrid(nx, ny, nz, indexing="ij")
    kv = np.stack([NX.ravel() * 2 * math.pi / L[0], NY.ravel() * 2 * math.pi / L[1],
                   NZ.ravel() * 2 * math.pi / L[2]], -1)
    half = (NX.ravel() > 0) | ((NX.ravel() == 0) & (NY.ravel() > 0)) | \
           ((NX.ravel() == 0) & (NY.ravel() == 0) & (NZ.ravel() > 0))
    kv = kv[half]
    k2 = np.sum(kv * kv, -1)
    keep = k2 < kmax * kmax
    kv = kv[keep]
    k2 = k2[keep]
    g = np.exp(-k2 / (4 * alpha * alpha)) / k2  # FT of erf part of 1/(4 pi r)
    E_k = 0.0
    for s in range(0, kv.shape[0], chunk):
        kk = kv[s:s + chunk]
        ph = pos @ kk.T  # [N, K]
        c = np.cos(ph)
        sn = np.sin(ph)
        Sr = q @ c
        Si = -(q @ sn)  # S(k) = sum q exp(-i k r)
        gg = g[s:s + chunk]
        S2 = Sr * Sr + Si * Si
        # factor 2: the half space stands for +k and -k
        E_k += float(np.sum(gg * S2)) / V
        # dE/dr_i = (2 q_i / V) sum_half g k Im[exp(-i k r_i) conj(S)]
        im = (-sn) * Sr[None, :] - c * Si[None, :]  # Im[e^{-ikr} conj(S)]
        F += -(2.0 / V) * q[:, None] * ((im * gg[None, :]) @ kk)
        kk2 = k2[s:s + chunk]
        fac = (gg * S2 / V)[:, None, None] * (np.eye(3)[None] - 2.0 * kk[:, :, None] * kk[:, None, :]
                                              * ((1.0 / kk2 + 1.0 / (4 * alpha * alpha))[:, None, None]))
        W += fac.sum(0)
    Q = float(q.sum())
    E_self = -alpha / math.sqrt(math.pi) * float(np.sum(q * q)) * INV_4PI
    E_bg = -Q * Q / (8.0 * V * alpha * alpha)
    W += np.eye(3) * E_bg
    E = E_real + E_k + E_self + E_bg
    vir = np.array([W[0, 0], W[0, 1], W[0, 2], W[1, 1], W[1, 2], W[2, 2]])
    return E, F, vir

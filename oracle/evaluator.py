"""FP64 numpy restatement of the reference pair evaluator (test
infrastructure only).

``EvaluatorPairPSWF::evalForceAndEnergy`` (``src/EvaluatorPairPSWF.h:274-295``)
with ``detail::pswf_eval_L`` (``src/EvaluatorPairPSWF.h:113-143``), operation
for operation, on a PSWF_Coeffs.h-layout segment table; including the
reference's ``sqrtf`` on a double (an FP32 square root). Pinned bit-exact
against the reference compiled from its own sources (oracle/_ref) through
the committed golden fixtures.
"""
from __future__ import annotations

import numpy as np

INV_4PI = 0.079577471545947673


def pswf_eval_L(r, rcut, screen, dscreen, r_lo, dr_inv):
    """(L, -dL/dr) of ``detail::pswf_eval_L``."""
    r = np.atleast_1d(np.asarray(r, dtype=np.float64))
    n_segs = r_lo.shape[0]
    L = np.zeros_like(r)
    D = np.zeros_like(r)
    ok = ~((r < 1.0e-12) | (r > rcut))
    rr = r[ok]
    s = rr / rcut
    s = np.where(s < 0.0, 0.0, np.where(s > 1.0 - 1.0e-9, 1.0 - 1.0e-9, s))
    seg = (s * float(n_segs)).astype(np.int64)
    seg = np.where(seg >= n_segs, n_segs - 1, seg)
    t = (rr - r_lo[seg]) * dr_inv[seg]
    cs = screen.reshape(-1, 5)[seg]
    cd = dscreen.reshape(-1, 5)[seg]

    def horner(c):
        v = c[:, 4].copy()
        for j in (3, 2, 1, 0):
            v = c[:, j] + t * v
        return v

    S = horner(cs)
    dS = horner(cd)
    i4r = INV_4PI / rr
    i4r2 = i4r / rr
    L[ok] = S * i4r
    D[ok] = S * i4r2 - dS * i4r
    return L, D


def eval_force_energy(rsq, qiqj, rcut, table):
    """(force_divr, pair_eng, evaluated) of ``evalForceAndEnergy`` with
    energy_shift false; ``table`` = (screen, dscreen, r_lo, dr_inv)."""
    rsq = np.asarray(rsq, dtype=np.float64)
    qiqj = np.asarray(qiqj, dtype=np.float64)
    ok = ~((rsq >= rcut * rcut) | (qiqj == 0.0) | (rcut < 1.0e-12))
    fd = np.zeros_like(rsq)
    pe = np.zeros_like(rsq)
    r = np.sqrt(rsq[ok].astype(np.float32)).astype(np.float64)
    rinv = 1.0 / r
    L, D = pswf_eval_L(r, rcut, *table)
    pe[ok] = qiqj[ok] * L
    fd[ok] = qiqj[ok] * D * rinv
    return fd, pe, ok.astype(np.int32)

"""Rigid three-site molecules: SETTLE positions and the RATTLE velocity
constraint, FP64 (test infrastructure only: the checker of the device's
constraint kernels).

The reference plugin has no constraint code (HOOMD supplies its
integrators); the workloads' water boxes are rigid (O, H, H) molecules, and
this is the analytical constraint method of Miyamoto & Kollman, J. Comput.
Chem. 13, 952 (1992), restated from its geometry:

* positions: after an unconstrained update x0 -> x1 of a molecule whose old
  positions x0 satisfy the constraints, the constrained x3 = x1 + Delta with
  m_i Delta_i a combination of the OLD bond vectors. Those lie in the old
  molecular plane, so in a frame with z normal to that plane the z
  coordinates keep their unconstrained values; the canonical triangle
  rotated by phi (about x) and psi (about y) reproduces them, and a final
  rotation theta about z makes the constraint forces torque-free:
  A sin(theta) + B cos(theta) = C with A, B, C the sums of the old bond
  vectors against the rotated and the unconstrained positions;
* velocities: v_i += sum_k mu_k dsigma_k/dx_i / m_i with the three
  multipliers from the 3x3 system r_k . v_k = 0 (bonds ab, ac, bc).
"""
from __future__ import annotations

import numpy as np


def geometry(d_oh: float, d_hh: float, m_o: float, m_h: float):
    """(ra, rb, rc): distances of O and of the H-H line from the centre of
    mass along the bisector, and half the H-H distance."""
    mt = m_o + 2.0 * m_h
    rc = 0.5 * d_hh
    h = np.sqrt(d_oh * d_oh - rc * rc)
    ra = 2.0 * m_h / mt * h
    return ra, h - ra, rc


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def settle_positions(x0, x1, m, d_oh: float, d_hh: float):
    """x0, x1: [M, 3, 3] old (constrained) and new (unconstrained) positions
    of M molecules (rows O, H, H; one periodic image per molecule); m: the
    three masses. Returns the constrained positions [M, 3, 3]."""
    x0 = np.asarray(x0, dtype=np.float64)
    x1 = np.asarray(x1, dtype=np.float64)
    mo, mh = float(m[0]), float(m[1])
    mt = mo + 2.0 * mh
    ra, rb, rc = geometry(d_oh, d_hh, mo, mh)
    com = (mo * x1[:, 0] + mh * (x1[:, 1] + x1[:, 2])) / mt
    A1, B1, C1 = x1[:, 0] - com, x1[:, 1] - com, x1[:, 2] - com
    b0a0 = x0[:, 1] - x0[:, 0]
    c0a0 = x0[:, 2] - x0[:, 0]
    ez = _unit(np.cross(b0a0, c0a0))
    ex = _unit(np.cross(A1, ez))
    ey = np.cross(ez, ex)
    dot = lambda u, v: np.sum(u * v, -1)  # noqa: E731
    xb0, yb0 = dot(b0a0, ex), dot(b0a0, ey)
    xc0, yc0 = dot(c0a0, ex), dot(c0a0, ey)
    za1 = dot(A1, ez)
    xb1, yb1, zb1 = dot(B1, ex), dot(B1, ey), dot(B1, ez)
    xc1, yc1, zc1 = dot(C1, ex), dot(C1, ey), dot(C1, ez)
    sphi = za1 / ra
    cphi = np.sqrt(1.0 - sphi * sphi)
    spsi = (zb1 - zc1) / (2.0 * rc * cphi)
    cpsi = np.sqrt(1.0 - spsi * spsi)
    ya2 = ra * cphi
    xb2 = -rc * cpsi
    t1 = -rb * cphi
    t2 = rc * spsi * sphi
    yb2 = t1 - t2
    yc2 = t1 + t2
    A = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2
    B = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2
    C = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0
    ab2 = A * A + B * B
    sth = (A * C - B * np.sqrt(ab2 - C * C)) / ab2
    cth = np.sqrt(1.0 - sth * sth)
    xyz = np.empty_like(x1)
    loc = [(-ya2 * sth, ya2 * cth, za1),
           (xb2 * cth - yb2 * sth, xb2 * sth + yb2 * cth, zb1),
           (-xb2 * cth - yc2 * sth, -xb2 * sth + yc2 * cth, zc1)]
    for i, (x, y, z) in enumerate(loc):
        xyz[:, i] = com + x[:, None] * ex + y[:, None] * ey + z[:, None] * ez
    return xyz


def rattle_velocities(x, v, m):
    """Removes the bond-stretching relative velocities of rigid molecules:
    x, v [M, 3, 3] (constrained positions, velocities), m the three masses.
    Returns the corrected velocities."""
    x = np.asarray(x, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64).copy()
    ia, ib, ic = 1.0 / m[0], 1.0 / m[1], 1.0 / m[2]
    r0, r1, r2 = x[:, 0] - x[:, 1], x[:, 0] - x[:, 2], x[:, 1] - x[:, 2]
    v0, v1, v2 = v[:, 0] - v[:, 1], v[:, 0] - v[:, 2], v[:, 1] - v[:, 2]
    dot = lambda u, w: np.sum(u * w, -1)  # noqa: E731
    M = np.empty((x.shape[0], 3, 3))
    M[:, 0, 0] = (ia + ib) * dot(r0, r0)
    M[:, 0, 1] = ia * dot(r0, r1)
    M[:, 0, 2] = -ib * dot(r0, r2)
    M[:, 1, 0] = ia * dot(r1, r0)
    M[:, 1, 1] = (ia + ic) * dot(r1, r1)
    M[:, 1, 2] = ic * dot(r1, r2)
    M[:, 2, 0] = -ib * dot(r2, r0)
    M[:, 2, 1] = ic * dot(r2, r1)
    M[:, 2, 2] = (ib + ic) * dot(r2, r2)
    rhs = -np.stack([dot(r0, v0), dot(r1, v1), dot(r2, v2)], -1)
    mu = np.linalg.solve(M, rhs[..., None])[..., 0]
    v[:, 0] += (mu[:, 0, None] * r0 + mu[:, 1, None] * r1) * ia
    v[:, 1] += (-mu[:, 0, None] * r0 + mu[:, 2, None] * r2) * ib
    v[:, 2] += (-mu[:, 1, None] * r1 - mu[:, 2, None] * r2) * ic
    return v

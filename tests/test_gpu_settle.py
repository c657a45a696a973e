"""Rigid water in the MD harness (esp_batch_set_rigid_water): SETTLE
positions and RATTLE velocities against the FP64 restatement in
``oracle/settle.py``, and trajectories that keep the molecules rigid.

* one velocity-Verlet step of 216 molecules with arbitrary forces: device
  positions and velocities equal the oracle's SETTLE / RATTLE of the same
  FP32 inputs (positions to 2e-6 nm, velocities to 1e-5 relative);
* 10 NVE steps of a 512-molecule box with the full ESP forces (mesh + pair,
  no exclusions, r_c 0.9 nm, the library's pair list): O-H and H-H distances
  stay at their targets to 1e-6 relative in FP64 and to the FP32 storage
  limit (4 ulp of the box edge) in FP32; the total energy drift is small.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems  # noqa: E402
from esp_hoomd_b200._lib import ESP_ALL  # noqa: E402
from oracle import settle as ST  # noqa: E402

D_OH = 0.1
D_HH = 2 * 0.1 * math.sin(math.radians(109.47 / 2))


def _mol(x, L):
    """[M, 3, 3] positions, hydrogens moved to the oxygen's periodic image."""
    m = x.reshape(-1, 3, 3).copy()
    d = m[:, 1:] - m[:, :1]
    m[:, 1:] = m[:, :1] + d - L * np.round(d / L)
    return m


def _dist(m):
    return (np.linalg.norm(m[:, 0] - m[:, 1], axis=-1), np.linalg.norm(m[:, 0] - m[:, 2], axis=-1),
            np.linalg.norm(m[:, 1] - m[:, 2], axis=-1))


def test_settle_step_matches_oracle():
    w = systems.water(216, seed=31)
    L = np.asarray(w.box)
    M = 216
    rng = np.random.default_rng(5)
    masses = np.array([16.0, 1.0, 1.0])
    x0 = _mol(w.pos.astype(np.float32).astype(np.float64), L)
    v = rng.normal(0, 1, (M, 3, 3)) / np.sqrt(masses)[None, :, None]
    v = ST.rattle_velocities(x0, v, masses).astype(np.float32).astype(np.float64)
    f = rng.normal(0, 20, (M, 3, 3)).astype(np.float32).astype(np.float64)
    dt = 0.002
    b = native.Batch(native.make_params(rcut=0.9), [w.N], [w.box])
    b.set_rigid_water([0], [M], D_OH, D_HH)
    p4 = np.zeros((w.N, 4), np.float32)
    p4[:, :3] = w.pos
    v4 = np.zeros((w.N, 4), np.float32)
    v4[:, :3] = v.reshape(-1, 3)
    v4[:, 3] = np.tile(masses, M)
    f4 = np.zeros((w.N, 4), np.float32)
    f4[:, :3] = f.reshape(-1, 3)
    pos, vel, frc = (torch.tensor(a, device="cuda") for a in (p4, v4, f4))
    b.nve_step1(pos, vel, frc, dt)
    torch.cuda.synchronize()
    x1 = x0 + dt * (v + 0.5 * dt * f / masses[None, :, None])
    x3 = ST.settle_positions(x0, x1, masses, D_OH, D_HH)
    v3 = (x3 - x0) / dt
    got = pos.double().cpu().numpy()[:, :3].reshape(M, 3, 3)
    d = got - x3
    d -= L * np.round(d / L)
    assert np.abs(d).max() <= 2e-6
    gv = vel.double().cpu().numpy()[:, :3].reshape(M, 3, 3)
    assert np.abs(gv - v3).max() <= 1e-5 * np.abs(v3).max()
    # second half kick + RATTLE at the new positions
    b.nve_step2(vel, frc, dt, pos4=pos)
    torch.cuda.synchronize()
    xg = _mol(pos.double().cpu().numpy()[:, :3], L)
    v2 = ST.rattle_velocities(xg, gv + 0.5 * dt * f / masses[None, :, None], masses)
    gv2 = vel.double().cpu().numpy()[:, :3].reshape(M, 3, 3)
    assert np.abs(gv2 - v2).max() <= 1e-5 * np.abs(v2).max()


def _water_md(prec):
    w = systems.water(512, seed=33)
    N, M = w.N, 512
    L = np.asarray(w.box)
    masses = np.tile([16.0, 1.0, 1.0], M)
    dt, nsteps = 0.002, 10
    rng = np.random.default_rng(9)
    x0 = _mol(w.pos, L)
    v = ST.rattle_velocities(x0, rng.normal(0, 0.3, (M, 3, 3)) / np.sqrt(masses.reshape(M, 3))[..., None],
                             masses[:3])
    if prec == 64:
        b = native.Batch(native.make_params(order=8, rcut=0.9, precision=1), [N], [w.box])
        dtype = torch.float64
    else:
        b = native.Batch(native.make_params(order=8, rcut=0.9), [N], [w.box])
        dtype = torch.float32
    b.set_rigid_water([0], [M], D_OH, D_HH)
    p4 = np.zeros((N, 4))
    p4[:, :3] = w.pos
    v4 = np.zeros((N, 4))
    v4[:, :3] = v.reshape(-1, 3)
    v4[:, 3] = masses
    pos = torch.tensor(p4, dtype=dtype, device="cuda")
    vel = torch.tensor(v4, dtype=dtype, device="cuda")
    q = torch.tensor(w.q, dtype=dtype, device="cuda")
    force = torch.zeros((N, 4), dtype=dtype, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    if prec == 64:
        # neighbour list from the FP32 harness, rebuilt every step (FP64 steps)
        b32 = native.Batch(native.make_params(order=8, rcut=0.9), [N], [w.box])
        head = torch.zeros(N, dtype=torch.int32, device="cuda")
        nn = torch.zeros_like(head)
        nl = torch.zeros(N * 512, dtype=torch.int32, device="cuda")

        def evaluate():
            b32.build_nlist(pos.float(), 0.9, 512, head, nn, nl)
            b.compute_f64(pos, q, force, energy, None, nlist=(head, nn, nl))

        evaluate()
        e0 = energy.item() + 0.5 * float((vel[:, 3] * (vel[:, :3] ** 2).sum(1)).sum().item())
        for _ in range(nsteps):
            b.nve_step1_f64(pos, vel, force, dt)
            evaluate()
            b.nve_step2_f64(vel, force, dt, pos4=pos)
    else:
        b.build_pairlist(pos, 1.0, 512)
        b.compute(pos, q, force, energy, None, nlist=None)
        e0 = energy.item() + 0.5 * float((vel[:, 3].double() * (vel[:, :3].double() ** 2).sum(1)).sum().item())
        b.md_run(pos, vel, q, force, energy, None, None, nsteps, dt, use_graph=True)
        b.pairlist_check()
    torch.cuda.synchronize()
    e1 = energy.item() + 0.5 * float((vel[:, 3].double() * (vel[:, :3].double() ** 2).sum(1)).sum().item())
    m = _mol(pos.double().cpu().numpy()[:, :3], L)
    d_oh1, d_oh2, d_hh = _dist(m)
    res = max(np.abs(d_oh1 - D_OH).max() / D_OH, np.abs(d_oh2 - D_OH).max() / D_OH, np.abs(d_hh - D_HH).max() / D_HH)
    return res, e0, e1, L


@pytest.mark.parametrize("prec", [32, 64])
def test_settle_md_keeps_water_rigid(prec):
    res, e0, e1, L = _water_md(prec)
    if prec == 64:
        assert res <= 1e-6
    else:
        ulp = np.spacing(np.float32(L.max()))
        assert res <= 4 * ulp / D_OH
    # total energy of the rigid-body motion (no bond vibration to absorb drift)
    assert abs(e1 - e0) <= 1e-3 * abs(e0)

"""The esp.py API mirror driving the sm_100a library: Spectral + Local forces
of a rock-salt system against the FP64 Ewald oracle (<= 1e-5 relative RMS
force error, energy <= 1e-6 relative), runtime set_params, and a short NVE
run that conserves energy."""
import warnings

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import esp, systems  # noqa: E402
from oracle import esp_ref as R  # noqa: E402
from oracle.ewald import ewald  # noqa: E402


@pytest.fixture(scope="module")
def rs10():
    s = systems.rocksalt(10, seed=1000)
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    return s, ewald(s.pos, s.q, s.box)


def _sim(s, resolution=(20, 20, 20)):
    state = esp.State(s.pos, s.q, s.box, velocities=s.vel, masses=s.mass)
    nl = esp.NeighborList(buffer=0.4)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        sp, lo = esp.make_esp_forces(nl, 3.0, resolution=resolution, order=8)
    lo.params[("A", "A")] = {}
    sim = esp.Simulation(state, nl, dt=0.002)
    sim.add(sp, lo)
    return sim, sp, lo


def test_spectral_plus_local_match_ewald(rs10):
    s, (E0, F0, W0) = rs10
    sim, sp, lo = _sim(s)
    sim.compute()
    F = sp.forces + lo.forces
    assert R.rel_rms(F, F0) <= 1e-5
    E = sp.energy + lo.energy
    assert abs(E - E0) <= 1e-6 * abs(E0)
    assert np.abs(sp.virial + lo.virial - W0).max() <= 1e-5 * np.abs(W0).max()
    assert abs(sp.q_sum) < 1e-9 and sp.q2_sum == pytest.approx(s.N)
    assert sp.resolution == (20, 20, 20) and sp.kappa > 0
    assert lo.params[("A", "A")]["rcut"] == 3.0 and lo.params[("A", "A")]["V_cut"] == 0.0


def test_set_params_rebuilds(rs10):
    s, (E0, F0, W0) = rs10
    sim, sp, lo = _sim(s, resolution=(16, 16, 16))
    sim.compute()
    err16 = R.rel_rms(sp.forces + lo.forces, F0)
    sp.set_params(resolution=(24, 24, 24))
    sim.compute()
    assert sp.resolution == (24, 24, 24)
    err24 = R.rel_rms(sp.forces + lo.forces, F0)
    assert err24 <= 1e-5 and err24 < err16
    with pytest.raises(ValueError):
        sp.set_params(order=20)


def test_local_needs_attached_spectral(rs10):
    s, _ = rs10
    state = esp.State(s.pos, s.q, s.box)
    nl = esp.NeighborList()
    sp = esp.Spectral(nl, 3.0, resolution=(20, 20, 20), order=8, kappa=6.0)
    lo = esp.Local(nl, 3.0, spectral=sp)
    sim = esp.Simulation(state, nl)
    with pytest.raises(RuntimeError):
        sim.add(lo)
    sim.add(sp)
    lo2 = esp.Local(nl, 2.5, spectral=sp)
    with pytest.raises(ValueError):
        sim.add(lo2)  # one cutoff for the split


def test_nve_run_conserves_energy(rs10):
    s, _ = rs10
    sim, sp, lo = _sim(s)

    def total():
        v = sim.state.vel4.double().cpu().numpy()
        ke = 0.5 * np.sum(v[:, 3:4] * v[:, :3] ** 2)
        return ke + sp.energy + lo.energy

    sim.compute()
    e_start = total()
    sim.run(50)
    e_end = total()
    assert np.isfinite(e_end)
    assert abs(e_end - e_start) <= 2e-4 * abs(e_start)
    assert sim.timestep == 50 and sim.nlist.builds >= 1

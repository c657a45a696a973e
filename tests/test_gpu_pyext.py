"""The `_esp` module on the GPU: ESPForceComputeGPU (long-range) plus
PotentialPairPSWFGPU (short-range) over the HOOMD stand-in classes, against
the FP64 oracle on the same float32 inputs:

* total forces <= 5e-6 relative RMS;
* total energy = sum of per-particle energies + external energies of both
  computes, <= 2e-6 relative;
* total virial = sum of per-particle virials + external virials,
  <= 1e-5 of its largest component;
* the introspection table reproduces L(r) and -dL/dr of the split in use;
* parameters are validated as the reference does (ValueError).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import _esp, systems, tables  # noqa: E402
from oracle import esp_ref as R  # noqa: E402


def _system(s):
    pd = _esp.ParticleData(s.N, _esp.BoxDim(*s.box))
    p4 = np.zeros((s.N, 4), np.float32)
    p4[:, :3] = s.pos
    pd.setPositions(p4)
    pd.setCharges(s.q.astype(np.float32))
    sysdef = _esp.SystemDefinition(pd)
    return sysdef


def test_forcecompute_pair_vs_oracle():
    s = systems.rocksalt(10, seed=6001)
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    sysdef = _system(s)
    nlist = _esp.NeighborList(sysdef, 0.0)
    group = _esp.ParticleGroup(sysdef)
    lr = _esp.ESPForceComputeGPU(sysdef, nlist, group)
    lr.setParams(20, 20, 20, 8, 0.0, 3.0)
    lr.compute(0)
    kappa = lr.getKappa()
    pair = _esp.PotentialPairPSWFGPU(sysdef, nlist)
    pair.setParams("A", "A", dict(kappa=kappa, alpha=0.0, rcut=3.0))
    pair.compute(0)
    f = lr.getForces().astype(np.float64) + pair.getForces().astype(np.float64)
    E = lr.calcEnergySum() + pair.calcEnergySum()
    W = lr.getVirials().astype(np.float64).sum(1) + pair.getVirials().astype(np.float64).sum(1) + \
        np.array(lr.getExternalVirial()) + np.array(pair.getExternalVirial())
    assert abs(lr.getQSum()) < 1e-6 and abs(lr.getQ2Sum() - s.N) < 1e-3
    c = kappa * 3.0
    prm = tables.ESPParams(mesh=(20, 20, 20), box=s.box, rcut=3.0, split=tables.split_cached(c),
                           window=tables.window_cached(8, 2.2 * 8, 8))
    E0, F0, W0 = R.esp(s.pos, s.q, prm)
    assert R.rel_rms(f[:, :3], F0) <= 5e-6
    assert abs(E - E0) <= 2e-6 * abs(E0)
    assert np.abs(W - W0).max() <= 1e-5 * np.abs(W0).max()
    # introspection table: L(r) and -dL/dr of the split
    tab = lr.table
    assert len(tab) == lr.getTableSize() == 512
    sp = tables.split_cached(c)
    for k in (40, 200, 480):
        e = lr.getTableEntry(k)
        t = 0.37
        r = e.r_lo + t / e.dr_inv
        cp = list(e.potential_coeffs) + [e.potential_coeff4]
        cf = list(e.force_coeffs) + [e.force_coeff4]
        L = sum(cj * t ** j for j, cj in enumerate(cp))
        D = sum(cj * t ** j for j, cj in enumerate(cf))
        u = r * r / 9.0
        L0 = R.INV_4PI * (1.0 / r - sp.Q(u) / 3.0)
        D0 = R.INV_4PI * (1.0 / (r * r) + 2.0 * r * sp.dQ(u) / 27.0)
        # the table interpolates the C++ split fit (1e-12); the Python split here is fitted to 1e-8
        # of its scale, 1/(4 pi r_c) for L and 1/(4 pi r_c^2) for D (near r_c both values vanish)
        lsc, dsc = R.INV_4PI / 3.0, R.INV_4PI / 9.0
        assert abs(L - L0) <= 1e-8 * max(abs(L0), lsc) and abs(D - D0) <= 1e-7 * max(abs(D0), dsc)


def test_forcecompute_validation():
    s = systems.rocksalt(8, seed=6002)
    sysdef = _system(s)
    nlist = _esp.NeighborList(sysdef, 0.0)
    lr = _esp.ESPForceCompute(sysdef, nlist, _esp.ParticleGroup(sysdef))
    with pytest.raises(RuntimeError):
        lr.compute(0)  # before setParams
    with pytest.raises(ValueError):
        lr.setParams(16, 16, 16, 8, 0.0, 3.0, alpha=0.5)
    with pytest.raises(ValueError):
        lr.setParams(16, 16, 16, 13, 0.0, 3.0)
    pair = _esp.PotentialPairPSWF(sysdef, nlist)
    with pytest.raises(ValueError):
        pair.setParams("A", "A", dict(rcut=3.0, alpha=1.0))
    pair.setParams("A", "A", dict(rcut=3.0, kappa=5.0))
    assert pair.getParams("A", "A")["kappa"] == 5.0
    with pytest.raises(ValueError):
        pair.setParams("A", "B", dict(rcut=2.5, kappa=5.0))

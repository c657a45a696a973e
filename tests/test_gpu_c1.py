"""The CPU-runnable plain case (N = 1000 rock-salt ions on a 10^3 lattice,
spacing 1, jitter 0.1, L = 10; mesh 32^3, support 8, r_c 3.0, double
precision, Lennard-Jones eps 1 sigma 0.9 r_cut 2.5 core repulsion; one
evaluation and 100 NVE steps at dt = 0.002) in the FP64 mode:

* first evaluation (ESP + LJ) against the FP64 oracle: forces <= 1e-8
  relative RMS, energy <= 1e-10 relative;
* the electrostatic part against FP64 Ewald: <= 1e-5 relative RMS;
* 100 NVE steps (neighbour list rebuilt every 10 steps, skin 0.4) follow
  the FP64 oracle's trajectory: total energy within 1e-8 relative and
  positions within 1e-6 after 100 steps. (The total energy itself is not
  conserved to better than ~1% from this jittered start: the unshifted LJ
  core swings by hundreds of energy units at dt = 0.002, in the oracle
  as on the GPU.)
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems, tables  # noqa: E402
from oracle import esp_ref as R  # noqa: E402
from oracle.ewald import ewald  # noqa: E402

EPS, SIG, RLJ = 1.0, 0.9, 2.5


def _nl_dev(nl):
    return tuple(torch.as_tensor(a.astype(np.int32), device="cuda") for a in nl)


def _dev4(a, w):
    out = np.zeros((a.shape[0], 4))
    out[:, :3] = a
    out[:, 3] = w
    return torch.as_tensor(out, dtype=torch.float64, device="cuda")


def test_c1_plain_fp64_with_lj():
    s = systems.rocksalt(10, seed=1000)
    s.pos = s.pos.astype(np.float32).astype(np.float64)  # the oracle's mesh stage reads float32 positions
    b = native.Batch(native.make_params(order=8, rcut=3.0, mesh=(32, 32, 32), precision=1), [s.N], [s.box])
    pos, vel = _dev4(s.pos, 0.0), _dev4(s.vel, 1.0)
    q = torch.as_tensor(s.q, dtype=torch.float64, device="cuda")
    force = torch.zeros((s.N, 4), dtype=torch.float64, device="cuda")
    e_esp = torch.zeros(1, dtype=torch.float64, device="cuda")
    e_lj = torch.zeros(1, dtype=torch.float64, device="cuda")

    def evaluate(nl):
        e_lj.zero_()
        b.compute_f64(pos, q, force, e_esp, nlist=nl)
        b.lj(pos, nl, EPS, SIG, RLJ, force, e_lj)

    nlist = R.neighbor_list(s.pos, s.box, 3.4)
    nl = _nl_dev(nlist)
    evaluate(nl)
    torch.cuda.synchronize()
    inf = b.info(0)
    prm = tables.ESPParams(mesh=(32, 32, 32), box=s.box, rcut=3.0, split=tables.make_split(inf["c_split"], tol=1e-12),
                           window=tables.window_cached(8, inf["c_window"], inf["window_degree"]))
    E, F, _ = R.esp(s.pos, s.q, prm, nlist=nlist)
    Flj, elj = R.lj_forces(s.pos, s.box, nlist, EPS, SIG, RLJ)
    f = force.cpu().numpy()
    assert R.rel_rms(f[:, :3], F + Flj) <= 1e-8
    assert abs(e_esp.item() + e_lj.item() - (E + elj.sum())) <= 1e-10 * abs(E + elj.sum())
    E0, F0, _ = ewald(s.pos, s.q, s.box)
    f_esp = f[:, :3] - Flj
    assert R.rel_rms(f_esp, F0) <= 1e-5

    def total():
        v = vel.cpu().numpy()
        return 0.5 * np.sum(v[:, :3] ** 2) + e_esp.item() + e_lj.item()

    # the oracle's trajectory: same integrator, same list schedule
    po, vo = s.pos.copy(), s.vel.copy()
    L = np.asarray(s.box)

    def oracle_eval(p, nlo):
        Eo, Fo, _ = R.esp(p, s.q, prm, nlist=nlo)
        Fl, el = R.lj_forces(p, s.box, nlo, EPS, SIG, RLJ)
        return Eo + el.sum(), Fo + Fl

    nlo = nlist
    Uo, Fo = oracle_eval(po, nlo)
    for step in range(100):
        if step % 10 == 0 and step > 0:
            nl = _nl_dev(R.neighbor_list(pos.cpu().numpy()[:, :3], s.box, 3.4))
            nlo = R.neighbor_list(po, s.box, 3.4)
        b.nve_step1_f64(pos, vel, force, 0.002)
        evaluate(nl)
        b.nve_step2_f64(vel, force, 0.002)
        vo += 0.001 * Fo
        po = np.mod(po + 0.002 * vo, L)
        Uo, Fo = oracle_eval(po, nlo)
        vo += 0.001 * Fo
    torch.cuda.synchronize()
    e_gpu = total()
    e_oracle = Uo + 0.5 * np.sum(vo ** 2)
    assert np.isfinite(e_gpu)
    assert abs(e_gpu - e_oracle) <= 1e-8 * abs(e_oracle)
    d = pos.cpu().numpy()[:, :3] - po
    d -= L * np.round(d / L)
    assert np.abs(d).max() <= 1e-6


@pytest.mark.parametrize("use_graph", [False, True])
def test_md_run_f64_equals_the_step_loop(use_graph):
    """esp_batch_md_run_f64 (ESP + LJ, 10 steps, eager or replayed from a
    captured graph) follows the explicit loop of nve_step1_f64 / compute_f64
    / lj / nve_step2_f64 on the same list: positions to 1e-12, forces and the
    energy (ESP + LJ) to 1e-10 relative (the mesh flush's FP64 atomics may
    add in another order)."""
    s = systems.rocksalt(10, seed=1000)
    b = native.Batch(native.make_params(order=8, rcut=3.0, mesh=(32, 32, 32), precision=1), [s.N], [s.box])
    q = torch.as_tensor(s.q, dtype=torch.float64, device="cuda")
    nl = _nl_dev(R.neighbor_list(s.pos, s.box, 3.4))
    runs = []
    for fused in (False, True):
        pos, vel = _dev4(s.pos, 0.0), _dev4(s.vel, 1.0)
        force = torch.zeros((s.N, 4), dtype=torch.float64, device="cuda")
        energy = torch.zeros(1, dtype=torch.float64, device="cuda")
        b.compute_f64(pos, q, force, energy, nlist=nl)
        b.lj(pos, nl, EPS, SIG, RLJ, force, energy)
        if fused:
            b.md_run_f64(pos, vel, q, force, energy, None, nl, 10, 0.002, lj=(EPS, SIG, RLJ), use_graph=use_graph)
            if use_graph:  # a second call replays the captured steps
                b.md_run_f64(pos, vel, q, force, energy, None, nl, 5, 0.002, lj=(EPS, SIG, RLJ), use_graph=True)
        else:
            for _ in range(15 if use_graph else 10):
                b.nve_step1_f64(pos, vel, force, 0.002)
                b.compute_f64(pos, q, force, energy, nlist=nl)
                b.lj(pos, nl, EPS, SIG, RLJ, force, energy)
                b.nve_step2_f64(vel, force, 0.002)
        torch.cuda.synchronize()
        runs.append((pos.cpu().numpy(), vel.cpu().numpy(), force.cpu().numpy(), energy.item()))
    (p0, v0, f0, e0), (p1, v1, f1, e1) = runs
    assert np.abs(p1[:, :3] - p0[:, :3]).max() <= 1e-12 * 10
    assert np.abs(v1 - v0).max() <= 1e-10 * np.abs(v0).max()
    assert R.rel_rms(f1[:, :3], f0[:, :3]) <= 1e-10
    assert abs(e1 - e0) <= 1e-10 * abs(e0)


def test_md_run_f64_rejects_an_fp32_context():
    s = systems.rocksalt(8, seed=1000)
    b = native.Batch(native.make_params(order=8, rcut=3.0), [s.N], [s.box])
    t = torch.zeros((s.N, 4), dtype=torch.float64, device="cuda")
    q = torch.zeros(s.N, dtype=torch.float64, device="cuda")
    nl = _nl_dev(R.neighbor_list(s.pos, s.box, 3.4))
    with pytest.raises(RuntimeError):
        b.md_run_f64(t, t.clone(), q, t.clone(), None, None, nl, 1, 0.002)

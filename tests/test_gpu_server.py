"""The continuous-batching server (esp_server_*) on the GPU:

* evaluation-only requests (rock-salt, r_c = 3; water, r_c = 0.9 nm) meet
  the 1e-5 relative RMS force bar against the FP64 Ewald oracle;
* a request's result is the same alone and in a mix of requests that
  arrive while it runs (forces <= 1e-6 relative RMS, positions <= 1e-5
  absolute, energy <= 1e-7 relative), and equals the batch path's
  nlist + evaluation + 10 NVE steps with the same parameters;
* admission under a small HBM budget holds back requests that do not fit,
  and a request larger than the arenas fails alone.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems  # noqa: E402
from esp_hoomd_b200._lib import ESP_ALL  # noqa: E402
from oracle import esp_ref as R  # noqa: E402
from oracle.ewald import ewald  # noqa: E402


def _host(s):
    pos4 = np.zeros((s.N, 4), np.float32)
    pos4[:, :3] = s.pos
    vel4 = np.zeros((s.N, 4), np.float32)
    vel4[:, :3] = s.vel
    vel4[:, 3] = s.mass
    return pos4, vel4, s.q.astype(np.float32)


class _Req:
    def __init__(self, srv, s, rcut, skin, nsteps, arrival=0.0, rigid=None):
        self.s = s
        self.pos4, self.vel4, self.q = _host(s)
        self.out_pos = np.zeros_like(self.pos4)
        self.out_vel = np.zeros_like(self.vel4)
        self.out_force = np.zeros_like(self.pos4)
        self.out_e = np.zeros(1, np.float64)
        self.id = srv.submit(self.pos4, self.q, s.box, rcut, vel4=self.vel4, nsteps=nsteps, dt=0.002, skin=skin,
                             arrival=arrival, out_pos4=self.out_pos, out_vel4=self.out_vel,
                             out_force4=self.out_force, out_energy=self.out_e, rigid_water=rigid)


def _server(budget=2 << 30, slots=64):
    return native.Server(native.make_params(order=8, target_error=1e-5), hbm_budget=budget, max_systems=slots,
                         max_particles=262144)


def _f32(s):
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    return s


def test_server_evaluation_accuracy():
    rs = _f32(systems.rocksalt(10, seed=3001))
    wa = _f32(systems.water(512, seed=3002))
    srv = _server()
    a = _Req(srv, rs, 3.0, 0.4, 0)
    b = _Req(srv, wa, 0.9, 0.1, 0)
    srv.start()
    srv.wait_all(300)
    for r, rc in ((a, 3.0), (b, 0.9)):
        st = srv.status(r.id)
        assert st["state"] == 2
        E0, F0, _ = ewald(r.s.pos, r.s.q, r.s.box)
        assert R.rel_rms(r.out_force[:, :3].astype(np.float64), F0) <= 1e-5
        assert abs(r.out_e[0] - E0) <= 1e-6 * abs(E0)
    stt = srv.stats()
    assert stt["completed"] == 2 and stt["failed"] == 0 and stt["rounds"] >= 1
    srv.close()


def _mix_systems():
    out = []
    for i, n in enumerate([8, 14, 10, 16, 12, 20, 8, 18]):
        out.append((systems.rocksalt(n, seed=4000 + i), 3.0, 0.4))
    out.insert(3, (systems.water(600, seed=4100), 0.9, 0.1))
    out.insert(6, (systems.water(900, seed=4101), 0.9, 0.1))
    return out


def test_alone_equals_in_mix_and_batch_path():
    x = systems.rocksalt(12, seed=4242)
    srv = _server()
    alone = _Req(srv, x, 3.0, 0.4, 10)
    srv.start()
    srv.wait_all(300)
    assert srv.status(alone.id)["state"] == 2
    mesh = [srv.status(alone.id)[k] for k in ("nx", "ny", "nz")]
    srv.close()

    srv = _server()
    reqs = []
    mix = _mix_systems()
    for k, (s, rc, skin) in enumerate(mix[:5]):
        reqs.append(_Req(srv, s, rc, skin, 10, arrival=0.0))
    mixed = _Req(srv, x, 3.0, 0.4, 10, arrival=0.002)  # arrives while the first five run
    for s, rc, skin in mix[5:]:
        reqs.append(_Req(srv, s, rc, skin, 10, arrival=0.004))
    srv.start()
    srv.wait_all(300)
    for r in reqs + [mixed]:
        assert srv.status(r.id)["state"] == 2
    stt = srv.stats()
    assert stt["max_active"] >= 2
    srv.close()

    f_a, f_m = alone.out_force[:, :3].astype(np.float64), mixed.out_force[:, :3].astype(np.float64)
    assert R.rel_rms(f_m, f_a) <= 1e-6
    assert np.abs(mixed.out_pos - alone.out_pos).max() <= 1e-5
    assert abs(mixed.out_e[0] - alone.out_e[0]) <= 1e-7 * abs(alone.out_e[0])

    # the batch path with the same split (c = 17, c / r_c = kappa) and mesh
    kappa = 17.0 / 3.0
    b = native.Batch(native.make_params(order=8, rcut=3.0, kappa=kappa, mesh=mesh), [x.N], [x.box])
    pos4, vel4, q = (torch.tensor(v, device="cuda") for v in _host(x))
    N = x.N
    head = torch.zeros(N, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(N * 256, dtype=torch.int32, device="cuda")
    force = torch.zeros((N, 4), device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    b.build_nlist(pos4, 3.4, 256, head, nn, nl)
    b.compute(pos4, q, force, energy, None, nlist=(head, nn, nl), flags=ESP_ALL)
    b.md_run(pos4, vel4, q, force, energy, None, (head, nn, nl), 10, 0.002, use_graph=False)
    torch.cuda.synchronize()
    assert np.abs(pos4.cpu().numpy() - alone.out_pos).max() <= 1e-5
    assert R.rel_rms(force[:, :3].double().cpu().numpy(), f_a) <= 1e-6
    assert abs(energy.item() - alone.out_e[0]) <= 1e-7 * abs(alone.out_e[0])


def test_admission_under_budget_and_oversized_request():
    srv = _server(budget=256 << 20, slots=256)
    small = [_Req(srv, systems.rocksalt(16, seed=5000 + i), 3.0, 0.4, 2) for i in range(40)]
    big = _Req(srv, systems.rocksalt(52, seed=5100), 3.0, 0.4, 0)
    tail = _Req(srv, systems.rocksalt(8, seed=5101), 3.0, 0.4, 2)
    srv.start()
    srv.wait_all(300)
    stt = srv.stats()
    for r in small + [tail]:
        assert srv.status(r.id)["state"] == 2
    assert srv.status(big.id)["state"] < 0
    assert stt["completed"] == 41 and stt["failed"] == 1
    assert 2 <= stt["max_active"] < 40  # the neighbour-list pool holds about 30 of these systems
    assert stt["peak_bytes"] <= 256 << 20
    assert stt["influence_hits"] >= 39  # one influence table for 40 equal boxes


def test_served_rigid_water_equals_batch_path():
    """A water request served with rigid molecules (SETTLE / RATTLE) keeps
    its O-H and H-H distances (to the FP32 storage limit) and equals the
    batch path's md_run with the same rigid geometry, split and mesh."""
    import math
    d_oh, d_hh = 0.1, 2 * 0.1 * math.sin(math.radians(109.47 / 2))
    w = systems.water(729, seed=4300)
    w.vel = np.random.default_rng(3).normal(0, 0.2, w.pos.shape) / np.sqrt(w.mass)[:, None]
    from oracle import settle as ST
    L = np.asarray(w.box)
    x = w.pos.reshape(-1, 3, 3).copy()
    d = x[:, 1:] - x[:, :1]
    x[:, 1:] = x[:, :1] + d - L * np.round(d / L)
    w.vel = ST.rattle_velocities(x, w.vel.reshape(-1, 3, 3), w.mass[:3]).reshape(-1, 3)
    srv = _server()
    r = _Req(srv, w, 0.9, 0.1, 10, rigid=(d_oh, d_hh))
    srv.start()
    srv.wait_all(300)
    st = srv.status(r.id)
    assert st["state"] == 2
    mesh = [st[k] for k in ("nx", "ny", "nz")]
    srv.close()
    m = r.out_pos[:, :3].astype(np.float64).reshape(-1, 3, 3)
    dd = m[:, 1:] - m[:, :1]
    dd -= L * np.round(dd / L)
    doh = np.linalg.norm(dd, axis=-1)
    dhh = np.linalg.norm(dd[:, 0] - dd[:, 1], axis=-1)
    ulp = float(np.spacing(np.float32(L.max())))
    assert np.abs(doh - d_oh).max() <= 4 * ulp
    assert np.abs(dhh - d_hh).max() <= 4 * ulp
    # the batch path with the server's split (c = 17, kappa = c / r_c) and mesh
    b = native.Batch(native.make_params(order=8, rcut=0.9, kappa=17.0 / 0.9, mesh=mesh), [w.N], [w.box])
    b.set_rigid_water([0], [w.N // 3], d_oh, d_hh)
    pos4, vel4, q = (torch.tensor(v, device="cuda") for v in _host(w))
    N = w.N
    head = torch.zeros(N, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(N * 512, dtype=torch.int32, device="cuda")
    force = torch.zeros((N, 4), device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    b.build_nlist(pos4, 1.0, 512, head, nn, nl)
    b.compute(pos4, q, force, energy, None, nlist=(head, nn, nl), flags=ESP_ALL)
    b.md_run(pos4, vel4, q, force, energy, None, (head, nn, nl), 10, 0.002, use_graph=False)
    torch.cuda.synchronize()
    dp = pos4.cpu().numpy()[:, :3] - r.out_pos[:, :3]
    dp -= L * np.round(dp / L)
    assert np.abs(dp).max() <= 1e-5
    assert abs(energy.item() - r.out_e[0]) <= 1e-6 * abs(r.out_e[0])

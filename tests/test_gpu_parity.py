"""GPU parity: every stage of the sm_100a path, called through the C ABI,
against the FP64 oracle on the same seeded inputs.

Tolerances (FP32 bulk arithmetic, FP64 reductions):
* sort keys and permutation: bit-exact;
* charge mesh: max |d rho| <= 2e-6 max |rho|;
* potential mesh: max |d phi| <= 5e-6 max |phi|;
* forces: relative RMS difference <= 5e-6; energy relative <= 2e-6;
  virial max abs <= 1e-5 max |W|;
* physics: relative RMS force error vs FP64 Ewald <= 1e-5 at the default
  target (the accuracy bar of the headline metric).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems, tables  # noqa: E402
from esp_hoomd_b200._lib import ESP_LONG_RANGE, ESP_SHORT_RANGE, ESP_ALL, EspError  # noqa: E402
from oracle import esp_ref as R  # noqa: E402
from oracle.ewald import ewald  # noqa: E402


def _dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _upload(sysm):
    pos4 = np.zeros((sysm.N, 4), dtype=np.float32)
    pos4[:, :3] = sysm.pos
    return _dev(pos4, torch.float32), _dev(sysm.q, torch.float32)


def _oracle_params(info, box):
    return tables.ESPParams(mesh=(info["nx"], info["ny"], info["nz"]), box=tuple(box), rcut=info["rcut"],
                            split=tables.split_cached(info["c_split"]),
                            window=tables.window_cached(info["order"], info["c_window"], info["window_degree"]))


def _nlist_dev(head, cnt, lst):
    return (_dev(head.astype(np.int32), torch.int32), _dev(cnt.astype(np.int32), torch.int32),
            _dev(lst.astype(np.int32), torch.int32))


@pytest.fixture(scope="module")
def rs8():
    s = systems.rocksalt(8, seed=1001)
    s.pos = s.pos.astype(np.float32).astype(np.float64)  # the device sees float32 positions
    return s


def test_sort_bit_exact(rs8):
    ctx = native.Context(native.make_params(), rs8.box, rs8.N)
    pos4, q = _upload(rs8)
    ctx.spread(pos4, q)
    key, perm = ctx.sort_state(rs8.N)
    torch.cuda.synchronize()
    inf = ctx.info()
    k_ref, p_ref = R.bin_sort(rs8.pos, rs8.box, (inf["nx"], inf["ny"], inf["nz"]), inf["order"], inf["tile"])
    assert np.array_equal(key.cpu().numpy().astype(np.uint32), k_ref)
    assert np.array_equal(perm.cpu().numpy().astype(np.uint32), p_ref)


def test_spread_matches_oracle(rs8):
    ctx = native.Context(native.make_params(), rs8.box, rs8.N)
    pos4, q = _upload(rs8)
    rho = ctx.spread(pos4, q).cpu().numpy()
    prm = _oracle_params(ctx.info(), rs8.box)
    ref = R.spread(rs8.pos, rs8.q, prm)
    assert np.abs(rho - ref).max() <= 2e-6 * np.abs(ref).max()
    # spreading conserves charge up to the window normalisation
    assert abs(rho.sum() - ref.sum()) <= 1e-6 * np.abs(ref).sum()


def test_potential_and_forces_match_oracle(rs8):
    ctx = native.Context(native.make_params(), rs8.box, rs8.N)
    pos4, q = _upload(rs8)
    head, cnt, lst = R.neighbor_list(rs8.pos, rs8.box, ctx.info()["rcut"])
    nl = _nlist_dev(head, cnt, lst)
    force = torch.zeros((rs8.N, 4), dtype=torch.float32, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    virial = torch.zeros(6, dtype=torch.float64, device="cuda")
    ctx.compute(pos4, q, force, energy, virial, nlist=nl)
    phi = ctx.potential().cpu().numpy()
    torch.cuda.synchronize()
    prm = _oracle_params(ctx.info(), rs8.box)
    E, F, W, parts = R.esp(rs8.pos, rs8.q, prm, nlist=(head, cnt, lst), return_parts=True)
    assert np.abs(phi - parts["phi"]).max() <= 5e-6 * np.abs(parts["phi"]).max()
    f = force.cpu().numpy()
    assert R.rel_rms(f[:, :3].astype(np.float64), F) <= 5e-6
    assert abs(energy.item() - E) <= 2e-6 * abs(E)
    assert np.abs(virial.cpu().numpy() - W).max() <= 1e-5 * np.abs(W).max()
    # per-particle energies sum to the total minus the background term
    assert abs(f[:, 3].astype(np.float64).sum() - (E - parts["E_bg"])) <= 5e-6 * abs(E)


@pytest.mark.parametrize("shape", [(22, 22, 22), (90, 90, 8), (90, 8, 90), (12, 10, 14)])
def test_mesh_shapes_match_oracle(shape):
    """Odd meshes (45), xy planes (180 x 180) and xz slabs (180 x 180)
    too large for shared memory (the per-line FFT passes) and non-cubic
    boxes, against the FP64 oracle."""
    s = systems.rocksalt(0, seed=sum(shape), shape=shape)
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    ctx = native.Context(native.make_params(), s.box, s.N)
    pos4, q = _upload(s)
    head, cnt, lst = R.neighbor_list(s.pos, s.box, 3.0)
    force = torch.zeros((s.N, 4), dtype=torch.float32, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    virial = torch.zeros(6, dtype=torch.float64, device="cuda")
    ctx.compute(pos4, q, force, energy, virial, nlist=_nlist_dev(head, cnt, lst))
    torch.cuda.synchronize()
    prm = _oracle_params(ctx.info(), s.box)
    E, F, W = R.esp(s.pos, s.q, prm, nlist=(head, cnt, lst))
    f = force.cpu().numpy()[:, :3].astype(np.float64)
    assert R.rel_rms(f, F) <= 5e-6
    assert abs(energy.item() - E) <= 2e-6 * abs(E)
    assert np.abs(virial.cpu().numpy() - W).max() <= 1e-5 * np.abs(W).max()


def test_accuracy_vs_ewald(rs8):
    ctx = native.Context(native.make_params(target_error=1e-5), rs8.box, rs8.N)
    pos4, q = _upload(rs8)
    head, cnt, lst = R.neighbor_list(rs8.pos, rs8.box, 3.0)
    force = torch.zeros((rs8.N, 4), dtype=torch.float32, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.compute(pos4, q, force, energy, nlist=_nlist_dev(head, cnt, lst))
    E0, F0, _ = ewald(rs8.pos, rs8.q, rs8.box)
    f = force.cpu().numpy()[:, :3].astype(np.float64)
    assert R.rel_rms(f, F0) <= 1e-5
    assert abs(energy.item() - E0) <= 1e-5 * abs(E0)


def test_long_plus_short_equals_all(rs8):
    ctx = native.Context(native.make_params(), rs8.box, rs8.N)
    pos4, q = _upload(rs8)
    nl = _nlist_dev(*R.neighbor_list(rs8.pos, rs8.box, 3.0))
    out = {}
    for flags in (ESP_LONG_RANGE, ESP_SHORT_RANGE, ESP_ALL):
        f = torch.zeros((rs8.N, 4), dtype=torch.float32, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        ctx.compute(pos4, q, f, e, nlist=nl, flags=flags)
        out[flags] = (f.cpu().numpy().astype(np.float64), e.item())
    fl, el = out[ESP_LONG_RANGE]
    fs, es = out[ESP_SHORT_RANGE]
    fa, ea = out[ESP_ALL]
    assert np.abs(fl + fs - fa).max() <= 1e-6 * np.abs(fa).max() + 1e-7
    assert abs(el + es - ea) <= 1e-9 * abs(ea)


def test_reference_evaluator_bit_exact(golden_dir):
    g = np.load(golden_dir + "/pswf_eval_golden.npz")
    t = np.load(golden_dir + "/pswf_coeffs_shipped.npz")
    table = tuple(_dev(t[k], torch.float64) for k in ("screen", "dscreen", "r_lo", "dr_inv"))
    fd, pe, ev = native.pswf_eval_pairs(_dev(g["rsq"], torch.float64), _dev(g["qiqj"], torch.float64),
                                        float(g["rcut"]), table)
    torch.cuda.synchronize()
    assert np.array_equal(ev.cpu().numpy(), g["evaluated"])
    # r = 0 gives the reference's own NaN (0 * inf), compared as equal
    assert np.array_equal(fd.cpu().numpy(), g["force_divr"], equal_nan=True)
    assert np.array_equal(pe.cpu().numpy(), g["pair_eng"], equal_nan=True)


def test_batch_alone_equals_in_mix():
    sys_list = [systems.rocksalt(n, seed=300 + n) for n in (8, 10, 12)]
    params = native.make_params()
    N = [s.N for s in sys_list]
    boxes = [s.box for s in sys_list]
    b = native.Batch(params, N, boxes)
    pos4 = np.zeros((sum(N), 4), dtype=np.float32)
    pos4[:, :3] = np.concatenate([s.pos for s in sys_list])
    q = np.concatenate([s.q for s in sys_list])
    nls = [R.neighbor_list(s.pos.astype(np.float32).astype(np.float64), s.box, 3.0) for s in sys_list]
    heads, cnts, lsts, off = [], [], [], 0
    for h, c, l in nls:
        heads.append(h.astype(np.int64) + off)
        cnts.append(c)
        lsts.append(l)
        off += l.size
    nl = _nlist_dev(np.concatenate(heads), np.concatenate(cnts), np.concatenate(lsts))
    fb = torch.zeros((sum(N), 4), dtype=torch.float32, device="cuda")
    eb = torch.zeros(len(N), dtype=torch.float64, device="cuda")
    vb = torch.zeros(6 * len(N), dtype=torch.float64, device="cuda")
    b.compute(_dev(pos4, torch.float32), _dev(q, torch.float32), fb, eb, vb, nlist=nl)
    fb = fb.cpu().numpy()
    for i, s in enumerate(sys_list):
        ctx = native.Context(params, s.box, s.N)
        p4, qq = _upload(s)
        f = torch.zeros((s.N, 4), dtype=torch.float32, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        v = torch.zeros(6, dtype=torch.float64, device="cuda")
        ctx.compute(p4, qq, f, e, v, nlist=_nlist_dev(*nls[i]))
        a, z = b.offsets[i], b.offsets[i + 1]
        fa = f.cpu().numpy()
        assert np.abs(fa - fb[a:z]).max() <= 1e-6 * np.abs(fa).max()
        # the FP64 charge-mesh flush is atomic, so mesh sums may round in a
        # different order before the FP32 potential: energies agree to 1e-8
        # relative, virials to 1e-6 of the largest component
        assert abs(e.item() - eb[i].item()) <= 1e-8 * abs(e.item())
        va, vbi = v.cpu().numpy(), vb[6 * i:6 * i + 6].cpu().numpy()
        assert np.abs(va - vbi).max() <= 1e-6 * np.abs(va).max()


@pytest.mark.parametrize("n,rlist,cap", [
    (10, 3.4, 256),   # 2 cells per axis: minimum-image test
    (12, 3.4, 256),   # 3 cells per axis: shifted images
    (20, 3.4, 256),   # 5 cells per axis
    (16, 5.29, 768),  # 152 particles per cell: several passes and staging rounds
])
def test_gpu_nlist_matches_oracle(n, rlist, cap):
    s = systems.rocksalt(n, seed=77)
    b = native.Batch(native.make_params(), [s.N], [s.box])
    pos4 = np.zeros((s.N, 4), dtype=np.float32)
    pos4[:, :3] = s.pos
    head = torch.zeros(s.N, dtype=torch.int32, device="cuda")
    nn = torch.zeros(s.N, dtype=torch.int32, device="cuda")
    nl = torch.zeros(s.N * cap, dtype=torch.int32, device="cuda")
    b.build_nlist(_dev(pos4, torch.float32), rlist, cap, head, nn, nl)
    h, c, l = head.cpu().numpy(), nn.cpu().numpy(), nl.cpu().numpy()
    rh, rc, rl = R.neighbor_list(s.pos.astype(np.float32).astype(np.float64), s.box, rlist)
    assert np.array_equal(c, rc.astype(np.int32))
    for i in range(s.N):
        assert set(l[h[i]:h[i] + c[i]].tolist()) == set(rl[rh[i]:rh[i] + rc[i]].tolist())


def test_errors_are_reported():
    with pytest.raises(EspError):
        native.Context(native.make_params(order=13), (10, 10, 10), 10)
    with pytest.raises(EspError):
        native.Context(native.make_params(alpha=0.5), (10, 10, 10), 10)
    with pytest.raises(EspError):
        native.Context(native.make_params(mesh=(14, 14, 14)), (10, 10, 10), 10)  # 14 is not 2/3/5-smooth


def test_exclusions_match_oracle_and_ewald():
    # rigid water with every intramolecular pair excluded: GPU vs the FP64
    # oracle (same parameters), and the physics vs Ewald without those pairs
    w = systems.water(216, seed=7)
    w.pos = w.pos.astype(np.float32).astype(np.float64)
    excl = R.molecule_exclusions(216, 3)
    ctx = native.Context(native.make_params(rcut=0.9, mesh=(16, 16, 16)), w.box, w.N)
    pos4, q = _upload(w)
    nlist = R.remove_pairs(R.neighbor_list(w.pos, w.box, 0.9), *excl)
    nl = _nlist_dev(*nlist)
    n_ex = _dev(excl[0].astype(np.int32), torch.int32)
    ex = _dev(excl[1].astype(np.int32), torch.int32)
    ctx.set_exclusions(n_ex, ex, excl[2])
    force = torch.zeros((w.N, 4), dtype=torch.float32, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    virial = torch.zeros(6, dtype=torch.float64, device="cuda")
    ctx.compute(pos4, q, force, energy, virial, nlist=nl)
    torch.cuda.synchronize()
    f = force.cpu().numpy()[:, :3].astype(np.float64)
    prm = _oracle_params(ctx.info(), w.box)
    E, F, W = R.esp(w.pos, w.q, prm, nlist=nlist, exclusions=excl)
    scale = R.INV_4PI * np.sum(w.q ** 2) / 0.9  # the remaining energy nearly cancels
    assert R.rel_rms(f, F) <= 5e-6
    assert abs(energy.item() - E) <= 1e-6 * scale
    assert np.abs(virial.cpu().numpy() - W).max() <= 1e-5 * np.abs(W).max()
    # per-particle energies add up to the total
    assert abs(float(force[:, 3].double().sum().item()) - energy.item()) <= 1e-6 * scale
    # clearing the exclusions restores the unexcluded mesh result
    ctx.set_exclusions(None)
    ctx.compute(pos4, q, force, energy, None, nlist=_nlist_dev(*R.neighbor_list(w.pos, w.box, 0.9)))
    E1, F1, _ = R.esp(w.pos, w.q, prm)
    torch.cuda.synchronize()
    assert R.rel_rms(force.cpu().numpy()[:, :3].astype(np.float64), F1) <= 5e-6


@pytest.mark.parametrize("order,target", [(6, 1e-3), (8, 1e-5), (10, 1e-5)])
def test_water_accuracy_sweep(order, target):
    # the water-like accuracy sweep (three-site molecules, r_c 0.9 nm, no
    # exclusions) at the planner's mesh for each target, FP32 path vs Ewald
    w = systems.water(512, seed=9)
    w.pos = w.pos.astype(np.float32).astype(np.float64)
    ctx = native.Context(native.make_params(order=order, rcut=0.9, target_error=target), w.box, w.N)
    pos4, q = _upload(w)
    nl = _nlist_dev(*R.neighbor_list(w.pos, w.box, 0.9))
    force = torch.zeros((w.N, 4), dtype=torch.float32, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.compute(pos4, q, force, energy, None, nlist=nl)
    torch.cuda.synchronize()
    E0, F0, _ = ewald(w.pos, w.q, w.box)
    assert R.rel_rms(force.cpu().numpy()[:, :3].astype(np.float64), F0) <= target
    assert abs(energy.item() - E0) <= target * abs(E0)


def test_autotune_keeps_results():
    # the autotuner re-plans with the fastest candidate on the same meshes:
    # forces and energies are the same as before tuning, within the parity
    # tolerance, and every candidate was timed
    sl = [systems.rocksalt(n, seed=7100 + n) for n in (10, 12, 14)]
    N = [s.N for s in sl]
    b = native.Batch(native.make_params(), N, [s.box for s in sl])
    pos4 = np.zeros((sum(N), 4), np.float32)
    pos4[:, :3] = np.concatenate([s.pos for s in sl])
    pos = torch.tensor(pos4, device="cuda")
    q = torch.tensor(np.concatenate([s.q for s in sl]).astype(np.float32), device="cuda")
    tot = sum(N)
    head = torch.zeros(tot, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(tot * 256, dtype=torch.int32, device="cuda")
    b.build_nlist(pos, 3.4, 256, head, nn, nl)
    f0 = torch.zeros((tot, 4), device="cuda")
    e0 = torch.zeros(3, dtype=torch.float64, device="cuda")
    b.compute(pos, q, f0, e0, nlist=(head, nn, nl))
    res = b.autotune(pos, q, nlist=(head, nn, nl), reps=2)
    assert res["threads_per_particle"] in (4, 8, 16) and 5 <= res["tile"] <= 9 and res["fft_mode"] in (0, 1)
    assert len(res["trial_ms"]) >= 5 and min(res["trial_ms"]) > 0
    f1 = torch.zeros_like(f0)
    e1 = torch.zeros_like(e0)
    b.compute(pos, q, f1, e1, nlist=(head, nn, nl))
    torch.cuda.synchronize()
    assert R.rel_rms(f1.cpu().numpy()[:, :3].astype(np.float64), f0.cpu().numpy()[:, :3].astype(np.float64)) <= 5e-6
    assert np.allclose(e1.cpu().numpy(), e0.cpu().numpy(), rtol=2e-6, atol=0)


def test_md_graphs_follow_buffer_sets():
    """Captured MD steps are cached per set of caller pointers: alternating
    between two buffer sets replays the graph of each set, and the result
    matches the same steps run without a graph."""
    sys_list = [systems.rocksalt(n, seed=900 + n) for n in (8, 10)]
    N = [s.N for s in sys_list]
    b = native.Batch(native.make_params(), N, [s.box for s in sys_list])
    tot = sum(N)
    p4 = np.zeros((tot, 4), np.float32)
    p4[:, :3] = np.concatenate([s.pos for s in sys_list])
    v4 = np.zeros((tot, 4), np.float32)
    v4[:, :3] = np.concatenate([s.vel for s in sys_list])
    v4[:, 3] = 1.0
    q = torch.tensor(np.concatenate([s.q for s in sys_list]).astype(np.float32), device="cuda")
    head = torch.zeros(tot, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(tot * 256, dtype=torch.int32, device="cuda")

    def fresh():
        return (torch.tensor(p4, device="cuda"), torch.tensor(v4, device="cuda"),
                torch.zeros((tot, 4), device="cuda"), torch.zeros(len(N), dtype=torch.float64, device="cuda"))

    def run(bufs, use_graph):
        p, v, f, e = bufs
        b.build_nlist(p, 3.4, 256, head, nn, nl)
        b.compute(p, q, f, e, None, nlist=(head, nn, nl), flags=ESP_ALL)
        b.md_run(p, v, q, f, e, None, (head, nn, nl), 5, 0.002, use_graph=use_graph)

    ref, a, c = fresh(), fresh(), fresh()
    for _ in range(3):
        run(ref, False)
    for _ in range(3):  # A, C, A, C, A, C: two cached graphs, each replayed
        run(a, True)
        run(c, True)
    torch.cuda.synchronize()
    for got in (a, c):
        for x, y in zip(got, ref):
            xa, ya = x.double().cpu().numpy(), y.double().cpu().numpy()
            assert np.abs(xa - ya).max() <= 1e-5 * max(np.abs(ya).max(), 1.0)


@pytest.mark.parametrize("use_graph", [True, False])
def test_md_run_final_energy_is_full(use_graph):
    """MD steps before the last skip the pair energies (the next step
    overwrites them): the energy and per-particle energies that md_run leaves
    equal a full evaluation at its final positions."""
    sys_list = [systems.rocksalt(n, seed=950 + n) for n in (8, 12)]
    N = [s.N for s in sys_list]
    b = native.Batch(native.make_params(), N, [s.box for s in sys_list])
    tot = sum(N)
    p4 = np.zeros((tot, 4), np.float32)
    p4[:, :3] = np.concatenate([s.pos for s in sys_list])
    v4 = np.zeros((tot, 4), np.float32)
    v4[:, :3] = np.concatenate([s.vel for s in sys_list])
    v4[:, 3] = 1.0
    pos, vel = torch.tensor(p4, device="cuda"), torch.tensor(v4, device="cuda")
    q = torch.tensor(np.concatenate([s.q for s in sys_list]).astype(np.float32), device="cuda")
    head = torch.zeros(tot, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(tot * 256, dtype=torch.int32, device="cuda")
    f = torch.zeros((tot, 4), device="cuda")
    e = torch.zeros(len(N), dtype=torch.float64, device="cuda")
    b.build_nlist(pos, 3.4, 256, head, nn, nl)
    b.compute(pos, q, f, e, None, nlist=(head, nn, nl), flags=ESP_ALL)
    b.md_run(pos, vel, q, f, e, None, (head, nn, nl), 6, 0.002, use_graph=use_graph)
    f2 = torch.zeros_like(f)
    e2 = torch.zeros_like(e)
    b.compute(pos, q, f2, e2, None, nlist=(head, nn, nl), flags=ESP_ALL)
    torch.cuda.synchronize()
    assert np.abs(e.cpu().numpy() - e2.cpu().numpy()).max() <= 1e-8 * np.abs(e2.cpu().numpy()).max()
    a, c = f.cpu().numpy(), f2.cpu().numpy()
    assert np.abs(a[:, 3] - c[:, 3]).max() <= 1e-5 * np.abs(c[:, 3]).max()
    assert R.rel_rms(a[:, :3].astype(np.float64), c[:, :3].astype(np.float64)) <= 1e-6


def test_empty_system_in_batch():
    """A system with no particles in the middle of a batch: zero energy and
    virial, and its neighbours in the batch get the same results as alone."""
    a, c = systems.rocksalt(8, seed=971), systems.rocksalt(10, seed=972)
    N = [a.N, 0, c.N]
    boxes = [a.box, (10.0, 10.0, 10.0), c.box]
    b = native.Batch(native.make_params(), N, boxes)
    tot = a.N + c.N
    p4 = np.zeros((tot, 4), np.float32)
    p4[:, :3] = np.concatenate([a.pos, c.pos])
    pos = torch.tensor(p4, device="cuda")
    q = torch.tensor(np.concatenate([a.q, c.q]).astype(np.float32), device="cuda")
    head = torch.zeros(tot, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(tot * 256, dtype=torch.int32, device="cuda")
    b.build_nlist(pos, 3.4, 256, head, nn, nl)
    f = torch.zeros((tot, 4), device="cuda")
    e = torch.zeros(3, dtype=torch.float64, device="cuda")
    w = torch.zeros(18, dtype=torch.float64, device="cuda")
    b.compute(pos, q, f, e, w, nlist=(head, nn, nl), flags=ESP_ALL)
    torch.cuda.synchronize()
    assert e[1].item() == 0.0 and np.all(w[6:12].cpu().numpy() == 0.0)
    fb = f.cpu().numpy()
    for k, (s, lo) in enumerate(((a, 0), (c, a.N))):
        b1 = native.Batch(native.make_params(), [s.N], [s.box])
        p1 = pos[lo:lo + s.N].contiguous()
        h1 = torch.zeros(s.N, dtype=torch.int32, device="cuda")
        n1 = torch.zeros_like(h1)
        l1 = torch.zeros(s.N * 256, dtype=torch.int32, device="cuda")
        b1.build_nlist(p1, 3.4, 256, h1, n1, l1)
        f1 = torch.zeros((s.N, 4), device="cuda")
        e1 = torch.zeros(1, dtype=torch.float64, device="cuda")
        b1.compute(p1, q[lo:lo + s.N].contiguous(), f1, e1, None, nlist=(h1, n1, l1), flags=ESP_ALL)
        torch.cuda.synchronize()
        fa = f1.cpu().numpy()
        assert np.abs(fa - fb[lo:lo + s.N]).max() <= 1e-6 * np.abs(fa).max()
        assert abs(e1.item() - e[2 * k].item()) <= 1e-8 * abs(e1.item())


def test_nlist_row_overflow_is_reported():
    """Rows longer than the capacity are reported with ESP_ERR_OVERFLOW (the
    build does not synchronise: nlist_check waits for it, and the next
    evaluation over those rows fails); n_neigh then holds the counts the
    caller needs, and rows keep their first cap entries."""
    s = systems.rocksalt(12, seed=973)
    b = native.Batch(native.make_params(), [s.N], [s.box])
    p4 = np.zeros((s.N, 4), np.float32)
    p4[:, :3] = s.pos
    pos = torch.tensor(p4, device="cuda")
    cap = 64
    head = torch.zeros(s.N, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(s.N * cap, dtype=torch.int32, device="cuda")
    b.build_nlist(pos, 3.4, cap, head, nn, nl)
    with pytest.raises(EspError) as ei:
        b.nlist_check()
    assert ei.value.code == -5
    q = torch.tensor(s.q.astype(np.float32), device="cuda")
    f = torch.zeros((s.N, 4), device="cuda")
    with pytest.raises(EspError) as ei:
        b.compute(pos, q, f, None, None, nlist=(head, nn, nl))
    assert ei.value.code == -5
    rh, rc, rl = R.neighbor_list(s.pos.astype(np.float32).astype(np.float64), s.box, 3.4)
    c = nn.cpu().numpy()
    assert np.array_equal(c, rc.astype(np.int32))
    h, l = head.cpu().numpy(), nl.cpu().numpy()
    for i in range(0, s.N, 97):
        row = set(l[h[i]:h[i] + cap].tolist())
        assert row <= set(rl[rh[i]:rh[i] + rc[i]].tolist())


def test_hoomd_forcecompute_contract():
    """esp_compute_hoomd fills HOOMD's ForceCompute arrays: m_force as
    esp_compute, m_virial per particle (pair + exclusion halves) against the
    oracle's per-particle virial, and the terms no particle owns (background
    energy; k-space + background virial) in the external slots, with
    per-particle sums + external = esp_compute's totals."""
    w = systems.water(216, seed=77)
    w.pos = w.pos.astype(np.float32).astype(np.float64)
    excl = R.molecule_exclusions(216, 3)
    nlh = R.remove_pairs(R.neighbor_list(w.pos, w.box, 0.9), *excl)
    ctx = native.Context(native.make_params(rcut=0.9, mesh=(24, 24, 24)), w.box, w.N)
    n_ex = torch.as_tensor(excl[0].astype(np.int32), device="cuda")
    ex = torch.as_tensor(excl[1].astype(np.int32), device="cuda")
    ctx.set_exclusions(n_ex, ex, excl[2])
    pos4, q = _upload(w)
    nl = _nlist_dev(*nlh)
    f_tot = torch.zeros((w.N, 4), dtype=torch.float32, device="cuda")
    e_tot = torch.zeros(1, dtype=torch.float64, device="cuda")
    v_tot = torch.zeros(6, dtype=torch.float64, device="cuda")
    ctx.compute(pos4, q, f_tot, e_tot, v_tot, nlist=nl)
    pitch = w.N + 13  # HOOMD pads m_virial rows to a pitch
    f = torch.zeros((w.N, 4), dtype=torch.float32, device="cuda")
    vpp = torch.full((6, pitch), 7.0, dtype=torch.float32, device="cuda")  # must be overwritten
    ext = torch.zeros(7, dtype=torch.float64, device="cuda")
    ctx.compute_hoomd(pos4, q, f, vpp, ext, nlist=nl)
    torch.cuda.synchronize()
    fa, fb = f.double().cpu().numpy(), f_tot.double().cpu().numpy()
    assert R.rel_rms(fa[:, :3], fb[:, :3]) <= 1e-6
    W = v_tot.cpu().numpy()
    V = vpp.double().cpu().numpy()[:, :w.N]
    X = ext.cpu().numpy()
    assert np.abs(V.sum(1) + X[1:] - W).max() <= 1e-5 * np.abs(W).max()
    assert abs(fa[:, 3].sum() + X[0] - e_tot.item()) <= 1e-5 * R.INV_4PI * np.sum(w.q ** 2) / 0.9
    # against the oracle: per-particle virial of the pair and exclusion terms,
    # the background energy and the k-space + background virial
    prm = _oracle_params(ctx.info(), w.box)
    _, _, _, Wp = R.pair_forces(w.pos, w.q, w.box, prm.split, prm.rcut, *nlh, per_particle=True)
    _, _, _, Wx = R.exclusion_correction(w.pos, w.q, w.box, prm.split, prm.rcut, *excl, per_particle=True)
    Wpp = (Wp + Wx).T
    assert np.abs(V - Wpp).max() <= 1e-5 * np.abs(Wpp).max()
    E, F, Wt, parts = R.esp(w.pos, w.q, prm, nlist=nlh, exclusions=excl, return_parts=True)
    assert abs(X[0] - parts["E_bg"]) <= 1e-6 * abs(parts["E_bg"]) + 1e-12
    assert np.abs(X[1:] - parts["W_k"]).max() <= 1e-5 * np.abs(parts["W_k"]).max()

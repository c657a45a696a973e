"""CPU tests of the oracle and the table generator (no GPU needed).

* the oracle's restatement of the reference pair evaluator is bit-exact
  against the reference compiled from its own sources (golden fixtures);
* the shipped PSWF_Coeffs.h known answers (S(0) = 1/2 etc., the reference's
  defects, pinned as they are);
* the prolate solver against scipy.special.pro_ang1 and the Fourier
  eigen-relation; split and window fits;
* the Ewald oracle against finite differences and its own parameter
  independence;
* the ESP oracle: forces are the exact gradient of its energy, and it
  converges to Ewald at the default (1e-5) parameters.
"""
import math

import numpy as np
import pytest

from esp_hoomd_b200 import systems, tables
from oracle import esp_ref as R
from oracle import evaluator as EV
from oracle.ewald import ewald


@pytest.fixture(scope="module")
def shipped(golden_dir):
    t = np.load(golden_dir + "/pswf_coeffs_shipped.npz")
    return (t["screen"], t["dscreen"], t["r_lo"], t["dr_inv"]), float(t["rcut"])


def test_evaluator_restatement_bit_exact(golden_dir, shipped):
    g = np.load(golden_dir + "/pswf_eval_golden.npz")
    table, rcut = shipped
    with np.errstate(divide="ignore", invalid="ignore"):
        fd, pe, ok = EV.eval_force_energy(g["rsq"], g["qiqj"], rcut, table)
    assert np.array_equal(ok, g["evaluated"])
    assert np.array_equal(fd, g["force_divr"], equal_nan=True)
    assert np.array_equal(pe, g["pair_eng"], equal_nan=True)
    L, D = EV.pswf_eval_L(g["r"], rcut, *table)
    assert np.array_equal(L, g["L"]) and np.array_equal(D, g["negdLdr"])


def test_evaluator_known_answers(shipped):
    # values of the reference evaluator compiled from its sources (r_c = 1)
    table, rcut = shipped
    L, D = EV.pswf_eval_L(np.array([0.1, 0.25, 0.5, 0.75]), rcut, *table)
    assert L.tolist() == [0.2698302206310154, 0.04716774142484325, 0.002554122723247796, 3.573561155029599e-05]
    assert D.tolist() == [3.9099951149259775, 0.5010553234185513, 0.034535829960987245, 0.0007858715534125451]
    fd, pe, ok = EV.eval_force_energy(np.array([0.25]), np.array([-1.0]), rcut, table)
    assert fd[0] == -0.06907165992197449 and pe[0] == -0.002554122723247796 and ok[0] == 1


def test_shipped_table_is_not_a_coulomb_split(shipped):
    # the reference screening starts at S(0) = 1/2 (CDF of psi^2 on [-1, 1])
    (screen, dscreen, r_lo, dr_inv), rcut = shipped
    assert screen[0] == 5.00000000000008993e-01
    assert r_lo.size == 4096 and dr_inv[0] == 4096.0


def test_segment_table_roundtrip(shipped):
    (screen, dscreen, r_lo, dr_inv), rcut = shipped
    tab = tables.SegmentTable(rcut=rcut, screen=screen, dscreen=dscreen, r_lo=r_lo, dr_inv=dr_inv)
    text = tables.emit_pswf_coeffs_header(tab)
    back = tables.parse_pswf_coeffs_header(text)
    assert np.array_equal(back.screen, screen) and np.array_equal(back.r_lo, r_lo)
    r = np.linspace(0.0, 1.1, 777)
    L1, D1 = tables.eval_segment_L(tab, r)
    L2, D2 = EV.pswf_eval_L(r, rcut, screen, dscreen, r_lo, dr_inv)
    assert np.array_equal(L1, L2) and np.array_equal(D1, D2)


@pytest.mark.parametrize("c", [6.0, 12.0, 18.0])
def test_prolate_matches_scipy(c):
    from scipy.special import pro_ang1

    p = tables.Prolate(c)
    x = np.linspace(-0.95, 0.95, 9)
    ref, _ = pro_ang1(0, 0, c, x)
    ratio = ref / p.psi(x)
    assert np.ptp(ratio) < 1e-9 * abs(ratio.mean())
    kap = np.array([0.0, 1.0, 0.5 * c, 0.9 * c])
    assert np.allclose(p.fourier_ratio(kap), p.psi(kap / c) / p.psi0, rtol=1e-10, atol=1e-14)


def test_split_properties():
    sp = tables.make_split(17.5)
    s = np.linspace(0, 1, 101)
    assert abs(sp.S(np.array([0.0]))[0] - 1.0) < 1e-14
    assert abs(sp.S(np.array([1.0 - 1e-12]))[0]) < 1e-9
    # S(s) = 1 - s Q(s^2) with the fitted polynomial
    assert np.max(np.abs(1.0 - s * sp.Q(s * s) - sp.S(s))) < 2e-8
    # dQ/du is the derivative of Q
    u = np.linspace(0.05, 0.95, 19)
    h = 1e-6
    assert np.allclose(sp.dQ(u), (sp.Q(u + h) - sp.Q(u - h)) / (2 * h), rtol=1e-6, atol=1e-8)
    assert sp.fit_err < 1e-8


def test_window_fit_and_fourier():
    w = tables.make_window(8, 17.6)
    assert w.fit_err < 1e-9
    t = np.linspace(0.0, 1.0, 11)[:-1]  # t = 1 is the support edge (value() returns 0 there)
    W = w.weights(t)
    # weights at t and the continuous window at the stencil offsets agree
    u = np.arange(8)[None, :] - 4.0 + t[:, None]
    assert np.allclose(W, w.value(u), atol=1e-10)
    # Fourier transform at 0 equals the integral of the window
    xs = np.linspace(-4, 4, 40001)
    assert abs(w.fourier(0.0)[0] - np.trapezoid(w.value(xs), xs)) < 1e-6


def test_smooth235():
    assert [tables.smooth235(n) for n in (1, 7, 14, 28, 44, 52, 77, 97)] == [1, 8, 15, 30, 45, 54, 80, 100]


def test_ewald_forces_are_gradients():
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, 4.0, (24, 3))
    q = rng.choice([-1.0, 1.0], 24)
    E, F, W = ewald(pos, q, (4.0, 4.0, 4.0))
    h = 1e-5
    for i, a in ((0, 0), (5, 2)):
        p1, p2 = pos.copy(), pos.copy()
        p1[i, a] += h
        p2[i, a] -= h
        fd = -(ewald(p1, q, (4.0, 4.0, 4.0))[0] - ewald(p2, q, (4.0, 4.0, 4.0))[0]) / (2 * h)
        assert abs(fd - F[i, a]) < 1e-7
    E2, F2, W2 = ewald(pos, q, (4.0, 4.0, 4.0), tol_exp=30.0)
    assert abs(E - E2) < 1e-11 and np.abs(F - F2).max() < 1e-10 and np.abs(W - W2).max() < 1e-10


def test_esp_oracle_gradient_and_accuracy():
    s = systems.rocksalt(8, seed=11)
    # the mesh stage sees float32 positions (as the device does): start from
    # float32 values and step by an exactly representable h, with a fixed list
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    prm = tables.ESPParams(mesh=(16, 16, 16), box=s.box, rcut=3.0, split=tables.split_cached(17.5),
                           window=tables.window_cached(8, 17.6, 10))
    nl = R.neighbor_list(s.pos, s.box, 3.3)
    E, F, W = R.esp(s.pos, s.q, prm, nlist=nl)
    h = 2.0 ** -12
    for i, a in ((0, 0), (100, 1)):
        p1, p2 = s.pos.copy(), s.pos.copy()
        p1[i, a] += h
        p2[i, a] -= h
        fd = -(R.esp(p1, s.q, prm, nlist=nl)[0] - R.esp(p2, s.q, prm, nlist=nl)[0]) / (2 * h)
        assert abs(fd - F[i, a]) < 2e-7
    E0, F0, W0 = ewald(s.pos, s.q, s.box)
    assert R.rel_rms(F, F0) < 1e-5
    assert abs(E - E0) < 1e-6 * abs(E0)
    assert np.abs(W - W0).max() < 1e-5 * np.abs(W0).max()


def test_bin_sort_is_stable():
    # tiles in key order; inside a tile by the stencil's y origin, then index
    s = systems.rocksalt(6, seed=2)
    key, perm = R.bin_sort(s.pos, s.box, (16, 16, 16), 8, 8)
    assert np.all(np.diff(key[perm].astype(np.int64)) >= 0)
    i0, _ = R.stencil_origin(R.grid_coords(s.pos, s.box, (16, 16, 16)), 8)
    oy = np.mod(i0[:, 1], 16) % 8
    for k in np.unique(key):
        idx = perm[key[perm] == k].astype(np.int64)
        comp = oy[idx] * (1 << 26) + idx
        assert np.all(np.diff(comp) > 0)


def test_neighbor_list_matches_brute_force():
    s = systems.rocksalt(6, seed=4)
    head, cnt, lst = R.neighbor_list(s.pos, s.box, 2.5)
    L = np.asarray(s.box)
    d = s.pos[:, None, :] - s.pos[None, :, :]
    d -= L * np.round(d / L)
    r2 = np.sum(d * d, -1)
    np.fill_diagonal(r2, np.inf)
    for i in range(0, s.N, 17):
        ref = np.nonzero(r2[i] < 2.5 ** 2)[0]
        assert np.array_equal(np.sort(lst[head[i]:head[i] + cnt[i]]), ref)


def test_water_system():
    w = systems.water(27, seed=1)
    assert w.N == 81
    assert abs(w.q.sum()) < 1e-12
    L = w.box[0]
    assert abs(L - (27 / 33.4) ** (1 / 3)) < 1e-12


def test_exclusion_correction_matches_ewald_without_excluded_pairs():
    # rigid water: every atom excludes the other two of its molecule; the
    # physical answer is Ewald minus the bare Coulomb of the excluded pairs
    w = systems.water(216, seed=7)
    L = np.asarray(w.box)
    excl = R.molecule_exclusions(216, 3)
    prm = tables.ESPParams(mesh=(16, 16, 16), box=w.box, rcut=0.9, split=tables.split_cached(22.5),
                           window=tables.window_cached(8, 17.6, 10))
    E, F, W = R.esp(w.pos, w.q, prm, exclusions=excl)
    E0, F0, W0 = ewald(w.pos, w.q, w.box)
    n_ex, ex, pitch = excl
    for i in range(w.N):
        for k in range(int(n_ex[i])):
            j = int(ex[i * pitch + k])
            d = w.pos[i] - w.pos[j]
            d -= L * np.round(d / L)
            r = np.sqrt(d @ d)
            qq = w.q[i] * w.q[j]
            E0 -= 0.5 * qq * R.INV_4PI / r
            F0[i] -= qq * R.INV_4PI * d / r ** 3
            W0 -= 0.5 * qq * R.INV_4PI / r ** 3 * np.array([d[0] * d[0], d[0] * d[1], d[0] * d[2],
                                                             d[1] * d[1], d[1] * d[2], d[2] * d[2]])
    assert R.rel_rms(F, F0) < 1e-5
    # the remaining (intermolecular) energy nearly cancels: measure its error
    # against the system's energy scale sum q^2 / (4 pi r_c)
    assert abs(E - E0) < 1e-7 * R.INV_4PI * np.sum(w.q ** 2) / 0.9
    assert np.abs(W - W0).max() < 1e-5 * np.abs(W0).max()


def test_c_port_matches_numpy_oracle():
    # the compiled FP64 restatement (the timed CPU baseline) against the numpy
    # oracle on float32-representable positions (the mesh stage's input)
    from oracle import esp_port as EP
    s = systems.rocksalt(10, seed=21)
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    prm = EP.plan([s], 3.0)
    _, _, F, E = EP.run_batch([s], prm, 3.4, 0, 0.002, threads=1)
    E0, F0, _ = R.esp(s.pos, s.q, prm[0], nlist=R.neighbor_list(s.pos, s.box, 3.4))
    assert R.rel_rms(F[0], F0) < 1e-12
    assert abs(E[0] - E0) < 1e-12 * abs(E0)


def test_c_port_batch_is_independent_of_threads_and_conserves_energy():
    from oracle import esp_port as EP
    sl = [systems.rocksalt(n, seed=30 + n) for n in (8, 10, 8)] + [systems.water(216, seed=5)]
    rs, wa = sl[:3], sl[3:]
    prm_rs = EP.plan(rs, 3.0)
    p1, v1, F1, E1 = EP.run_batch(rs, prm_rs, 3.4, 20, 0.002, threads=1)
    p2, v2, F2, E2 = EP.run_batch(rs, prm_rs, 3.4, 20, 0.002, threads=3)
    assert np.array_equal(E1, E2) and all(np.array_equal(a, b) for a, b in zip(p1, p2))
    # kinetic + potential energy of the rock-salt systems over 20 NVE steps
    _, _, _, E0 = EP.run_batch(rs, prm_rs, 3.4, 0, 0.002, threads=1)
    for s, v, e0, e1 in zip(rs, v1, E0, E1):
        k0 = 0.5 * np.sum(s.mass[:, None] * s.vel ** 2)
        k1 = 0.5 * np.sum(s.mass[:, None] * v ** 2)
        assert abs((k1 + e1) - (k0 + e0)) < 1e-4 * abs(k0 + e0)
    # water (r_c 0.9 nm) against Ewald
    prm_w = EP.plan(wa, 0.9)
    _, _, Fw, Ew = EP.run_batch(wa, prm_w, 1.0, 0, 0.002, threads=1)
    E_e, F_e, _ = ewald(wa[0].pos, wa[0].q, wa[0].box)
    assert R.rel_rms(Fw[0], F_e) < 1e-5


@pytest.mark.parametrize("kind", ["rocksalt", "water", "box"])
def test_torch_ewald_matches_numpy_ewald(kind):
    # the workload-size Ewald (cell-list real space, separable structure
    # factor) against the direct numpy sum, on the CPU: energy, forces,
    # virial, and forces of a subset with the structure factor over all
    from oracle.ewald_torch import ewald_torch
    if kind == "rocksalt":
        s = systems.rocksalt(8, seed=3)
    elif kind == "water":
        s = systems.water(64, seed=5)
    else:
        s = systems.rocksalt(0, seed=2, shape=(6, 8, 10))
    E, F, W = ewald(s.pos, s.q, s.box)
    for re in (None, 2.0):
        E2, F2, W2 = ewald_torch(s.pos, s.q, s.box, device="cpu", re=re)
        assert abs(E2 - E) <= 1e-10 * abs(E)
        assert R.rel_rms(F2, F) <= 1e-9
        assert np.abs(W2 - W).max() <= 1e-9 * np.abs(W).max()
    sub = np.random.default_rng(0).choice(s.N, size=40, replace=False)
    E3, F3, W3 = ewald_torch(s.pos, s.q, s.box, targets=sub, device="cpu")
    assert E3 is None and W3 is None
    assert R.rel_rms(F3, F[sub]) <= 1e-9

"""The library's pair list (esp_batch_build_pairlist: rows in cell order,
entries cell-sorted slots, read from the slot-ordered positions) against
the HOOMD-layout neighbour list path, which is pinned to the oracle
(test_gpu_parity.py): same forces, energies and virials up to summation
order (relative RMS <= 1e-6, energy and virial <= 1e-6 relative,
per-particle energies <= 5e-6 of the largest).

Cases:
* a batch mixing cell grids of 2, 3 and >= 4 cells per axis (minimum image
  in the builder vs staged periodic images), positions given in other
  periodic images than the box;
* MD: 10 velocity-Verlet steps from the same state over both lists (the
  pair list is built once, particles cross the box faces);
* a clustered system whose dense cells' neighbourhoods exceed the builder's
  shared-memory stage (scanned in windows);
* a row capacity too small: ESP_ERR_OVERFLOW from the check and from the
  next evaluation, with the longest row reported;
* exclusions set on the batch: both builders leave the excluded pairs out.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems  # noqa: E402
from esp_hoomd_b200._lib import ESP_ALL, ESP_SHORT_RANGE, EspError  # noqa: E402
from oracle import esp_ref as R  # noqa: E402


def _inputs(sl, shift_images=False, seed=0):
    tot = sum(s.N for s in sl)
    p4 = np.zeros((tot, 4), np.float32)
    pos = np.concatenate([s.pos for s in sl])
    if shift_images:
        # some particles handed over in another periodic image
        rng = np.random.default_rng(seed)
        L = np.concatenate([np.tile(np.asarray(s.box), (s.N, 1)) for s in sl])
        pos = pos + L * rng.integers(-2, 3, size=pos.shape)
    p4[:, :3] = pos
    v4 = np.zeros((tot, 4), np.float32)
    v4[:, :3] = np.concatenate([s.vel for s in sl])
    v4[:, 3] = np.concatenate([s.mass for s in sl])
    q = np.concatenate([s.q for s in sl]).astype(np.float32)
    return (torch.tensor(p4, device="cuda"), torch.tensor(v4, device="cuda"), torch.tensor(q, device="cuda"))


def _both(b, pos, q, rlist, cap, flags=ESP_ALL):
    """(forces, energies, virials) over the HOOMD-layout list and over the pair list."""
    tot, ns = b.total, b.nsys
    head = torch.zeros(tot, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(tot * cap, dtype=torch.int32, device="cuda")
    b.build_nlist(pos, rlist, cap, head, nn, nl)
    out = []
    for nlist in ((head, nn, nl), None):
        if nlist is None:
            b.build_pairlist(pos, rlist, cap)
        f = torch.zeros((tot, 4), device="cuda")
        e = torch.zeros(ns, dtype=torch.float64, device="cuda")
        w = torch.zeros(6 * ns, dtype=torch.float64, device="cuda")
        b.compute(pos, q, f, e, w, nlist=nlist, flags=flags)
        torch.cuda.synchronize()
        out.append((f.double().cpu().numpy(), e.cpu().numpy(), w.cpu().numpy().reshape(ns, 6)))
    b.pairlist_check()
    return out


def _same(a, c, tol=1e-6):
    (fa, ea, wa), (fc, ec, wc) = a, c
    assert R.rel_rms(fc[:, :3], fa[:, :3]) <= tol
    # per-particle energies: FP32 sums of ~160 cancelling pair terms in a
    # different order
    assert np.abs(fc[:, 3] - fa[:, 3]).max() <= 5 * tol * np.abs(fa[:, 3]).max()
    assert np.all(np.abs(ec - ea) <= tol * np.abs(ea))
    assert np.abs(wc - wa).max() <= tol * np.abs(wa).max()


@pytest.mark.parametrize("flags", [ESP_SHORT_RANGE, ESP_ALL])
def test_pairlist_matches_hoomd_list(flags):
    # n = 8: 2 cells per axis, 10 and 12: 3 (minimum image per pair), 14+: staged nearest images
    sl = [systems.rocksalt(n, seed=8800 + n) for n in (8, 10, 12, 14, 20, 24)]
    sl.append(systems.rocksalt(0, seed=8899, shape=(14, 10, 22)))
    b = native.Batch(native.make_params(), [s.N for s in sl], [s.box for s in sl])
    pos, _, q = _inputs(sl, shift_images=True, seed=1)
    a, c = _both(b, pos, q, 3.4, 256, flags)
    _same(a, c)


def test_pairlist_md_matches_hoomd_list():
    sl = [systems.rocksalt(n, seed=8900 + n, T=30.0) for n in (12, 16, 22)]
    b = native.Batch(native.make_params(), [s.N for s in sl], [s.box for s in sl])
    pos0, vel0, q = _inputs(sl)
    tot = b.total
    res = []
    for use_pl in (False, True):
        pos, vel = pos0.clone(), vel0.clone()
        head = torch.zeros(tot, dtype=torch.int32, device="cuda")
        nn = torch.zeros_like(head)
        nl = torch.zeros(tot * 256, dtype=torch.int32, device="cuda")
        if use_pl:
            b.build_pairlist(pos, 3.4, 256)
            nlist = None
        else:
            b.build_nlist(pos, 3.4, 256, head, nn, nl)
            nlist = (head, nn, nl)
        f = torch.zeros((tot, 4), device="cuda")
        e = torch.zeros(len(sl), dtype=torch.float64, device="cuda")
        b.compute(pos, q, f, e, None, nlist=nlist)
        b.md_run(pos, vel, q, f, e, None, nlist, 10, 0.002, use_graph=True)
        torch.cuda.synchronize()
        res.append((pos.double().cpu().numpy(), f.double().cpu().numpy(), e.cpu().numpy()))
    (pa, fa, ea), (pc, fc, ec) = res
    L = np.concatenate([np.tile(np.asarray(s.box), (s.N, 1)) for s in sl])
    d = pc[:, :3] - pa[:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() <= 1e-5
    assert R.rel_rms(fc[:, :3], fa[:, :3]) <= 1e-5
    assert np.all(np.abs(ec - ea) <= 1e-6 * np.abs(ea))


def test_pairlist_windowed_staging_for_dense_cells():
    # 60% of the particles squeezed into one corner: those cells hold several
    # times the mean density, beyond the staging capacity sized for the mean
    rng = np.random.default_rng(4)
    L = 24.0
    n = 6000
    pos = rng.uniform(0, L, (n, 3))
    dense = rng.random(n) < 0.6
    pos[dense] = rng.uniform(0, 7.0, (int(dense.sum()), 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    s = systems.System(pos=pos, q=q, vel=np.zeros_like(pos), mass=np.ones(n), box=(L, L, L))
    b = native.Batch(native.make_params(), [n], [s.box])
    p, _, qq = _inputs([s])
    a, c = _both(b, p, qq, 2.2, 1024, ESP_SHORT_RANGE)
    _same(a, c)


def test_pairlist_overflow_is_reported():
    s = systems.rocksalt(16, seed=974)
    b = native.Batch(native.make_params(), [s.N], [s.box])
    pos, _, q = _inputs([s])
    b.build_pairlist(pos, 3.4, 64)
    with pytest.raises(EspError) as ei:
        b.pairlist_check()
    assert ei.value.code == -5
    f = torch.zeros((s.N, 4), device="cuda")
    with pytest.raises(EspError) as ei:
        b.compute(pos, q, f, None, None, nlist=None, flags=ESP_SHORT_RANGE)
    assert ei.value.code == -5
    # the longest row is reported, and a rebuild with room for it clears the error
    counts = R.neighbor_list(s.pos.astype(np.float32).astype(np.float64), s.box, 3.4)[1]
    b.build_pairlist(pos, 3.4, 64)
    with pytest.raises(EspError):
        b.pairlist_check()
    assert counts.max() > 64
    b.build_pairlist(pos, 3.4, 256)
    assert b.pairlist_check() == 0
    b.compute(pos, q, f, None, None, nlist=None, flags=ESP_SHORT_RANGE)


def test_lists_leave_exclusions_out():
    # rigid water with every intramolecular pair excluded, exclusions set on
    # the batch before the builds: the HOOMD-layout rows are the oracle's list
    # without the excluded pairs (order kept), and the pair list gives the same
    # forces, energies and virials
    w = systems.water(216, seed=71)
    w.pos = w.pos.astype(np.float32).astype(np.float64)
    excl = R.molecule_exclusions(216, 3)
    b = native.Batch(native.make_params(rcut=0.9, mesh=(16, 16, 16)), [w.N], [w.box])
    pos, _, q = _inputs([w])
    b.set_exclusions(torch.tensor(excl[0].astype(np.int32), device="cuda"),
                     torch.tensor(excl[1].astype(np.int32), device="cuda"), excl[2])
    cap = 512
    head = torch.zeros(w.N, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(w.N * cap, dtype=torch.int32, device="cuda")
    b.build_nlist(pos, 0.9, cap, head, nn, nl)
    b.nlist_check()
    rh, rc, rl = R.remove_pairs(R.neighbor_list(w.pos, w.box, 0.9), *excl)
    h, c, l = head.cpu().numpy(), nn.cpu().numpy(), nl.cpu().numpy()
    assert np.array_equal(c, rc.astype(np.int32))
    for i in range(0, w.N, 7):
        assert sorted(l[h[i]:h[i] + c[i]].tolist()) == sorted(rl[rh[i]:rh[i] + rc[i]].tolist())
    a, d = _both(b, pos, q, 0.9, cap, ESP_ALL)
    _same(a, d)

"""FP64 mode (esp_compute_f64) on the GPU:

* against the FP64 oracle with the same parameters (split fitted to 1e-12):
  forces <= 1e-8 relative RMS, energy <= 1e-10 relative, virial <= 1e-9 of
  its largest component;
* accuracy below the FP32 floor against FP64 Ewald: <= 1e-7 relative RMS
  force error at the 1e-7 target (rock-salt and water, support 10);
* other supports and tile edges (regions larger than a CTA's threads, odd
  supports, split tiles) against the oracle;
* exclusions in FP64 against the oracle;
* a context serves only the precision it was created for.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems, tables  # noqa: E402
from esp_hoomd_b200._lib import EspError  # noqa: E402
from oracle import esp_ref as R  # noqa: E402
from oracle.ewald import ewald  # noqa: E402


def _dev64(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _run(s, params, nlist, excl=None):
    ctx = native.Context(params, s.box, s.N)
    pos4 = np.zeros((s.N, 4))
    pos4[:, :3] = s.pos
    head, cnt, lst = nlist
    nl = tuple(torch.as_tensor(a.astype(np.int32), device="cuda") for a in (head, cnt, lst))
    if excl is not None:
        n_ex = torch.as_tensor(excl[0].astype(np.int32), device="cuda")
        ex = torch.as_tensor(excl[1].astype(np.int32), device="cuda")
        ctx.set_exclusions(n_ex, ex, excl[2])
    force = torch.zeros((s.N, 4), dtype=torch.float64, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    virial = torch.zeros(6, dtype=torch.float64, device="cuda")
    ctx.compute_f64(_dev64(pos4), _dev64(s.q), force, energy, virial, nlist=nl)
    torch.cuda.synchronize()
    return ctx, force.cpu().numpy(), energy.item(), virial.cpu().numpy()


def _oracle_params(info, box):
    return tables.ESPParams(mesh=(info["nx"], info["ny"], info["nz"]), box=tuple(box), rcut=info["rcut"],
                            split=tables.make_split(info["c_split"], tol=1e-12),
                            window=tables.window_cached(info["order"], info["c_window"], info["window_degree"]))


def test_fp64_matches_oracle():
    s = systems.rocksalt(8, seed=6401)
    s.pos = s.pos.astype(np.float32).astype(np.float64)  # the oracle's mesh stage reads float32 positions
    nlist = R.neighbor_list(s.pos, s.box, 3.0)
    ctx, f, e, w = _run(s, native.make_params(precision=1), nlist)
    prm = _oracle_params(ctx.info(), s.box)
    E, F, W = R.esp(s.pos, s.q, prm, nlist=nlist)
    assert R.rel_rms(f[:, :3], F) <= 1e-8
    assert abs(e - E) <= 1e-10 * abs(E)
    assert np.abs(w - W).max() <= 1e-9 * np.abs(W).max()
    assert abs(f[:, 3].sum() - e) <= 1e-10 * abs(E)


@pytest.mark.parametrize("order,tile,n", [(8, 10, 32), (4, 20, 24), (5, 0, 24), (7, 5, 24), (12, 0, 24), (4, 0, 16)])
def test_fp64_tiles_and_orders_match_oracle(order, tile, n):
    """The FP64 tile kernels at other supports and tile edges: extended
    regions of 17 and 23 (more rows than threads, two register segments per
    row), odd supports, a region of 11, support 12 (3P > 32 weights), and
    the small meshes whose few tiles are split over several CTAs."""
    s = systems.rocksalt(8, seed=6404 + order)
    s.pos = s.pos.astype(np.float32).astype(np.float64)
    nlist = R.neighbor_list(s.pos, s.box, 3.0)
    ctx, f, e, w = _run(s, native.make_params(order=order, mesh=(n, n, n), tile=tile, precision=1), nlist)
    prm = _oracle_params(ctx.info(), s.box)
    E, F, W = R.esp(s.pos, s.q, prm, nlist=nlist)
    assert R.rel_rms(f[:, :3], F) <= 1e-8
    assert abs(e - E) <= 1e-10 * abs(E)
    # the virial comes from the FFT's z pass, not from the tile kernels; the
    # oracle's virial factor takes Psi' by a finite difference (h = 1e-6),
    # which on the finer meshes here limits it to ~1e-8 (2e-9 at 32^3)
    assert np.abs(w - W).max() <= 2e-8 * np.abs(W).max()


@pytest.mark.parametrize("kind", ["rocksalt", "water"])
def test_fp64_accuracy_below_fp32_floor(kind):
    if kind == "rocksalt":
        s, rc = systems.rocksalt(10, seed=6402), 3.0
    else:
        s, rc = systems.water(512, seed=6403), 0.9
    nlist = R.neighbor_list(s.pos, s.box, rc)
    _, f, e, _ = _run(s, native.make_params(order=10, rcut=rc, target_error=1e-7, precision=1), nlist)
    E0, F0, _ = ewald(s.pos, s.q, s.box)
    assert R.rel_rms(f[:, :3], F0) <= 1e-7
    assert abs(e - E0) <= 1e-8 * abs(E0)


def test_fp64_exclusions_match_oracle():
    w = systems.water(216, seed=7)
    w.pos = w.pos.astype(np.float32).astype(np.float64)
    excl = R.molecule_exclusions(216, 3)
    nlist = R.remove_pairs(R.neighbor_list(w.pos, w.box, 0.9), *excl)
    ctx, f, e, wv = _run(w, native.make_params(rcut=0.9, mesh=(16, 16, 16), precision=1), nlist, excl)
    prm = _oracle_params(ctx.info(), w.box)
    E, F, W = R.esp(w.pos, w.q, prm, nlist=nlist, exclusions=excl)
    assert R.rel_rms(f[:, :3], F) <= 1e-8
    assert abs(e - E) <= 1e-9 * R.INV_4PI * np.sum(w.q ** 2) / 0.9
    # the oracle's virial factor takes Psi' by a finite difference (h = 1e-6);
    # with the large cancelling intramolecular terms that limits it to ~1e-8
    assert np.abs(wv - W).max() <= 5e-8 * np.abs(W).max()


def test_oversized_tile_is_refused():
    """A tile whose extended region needs more shared memory than a CTA has
    is refused at create with ESP_ERR_UNSUPPORTED (support 8, tile 20)."""
    s = systems.rocksalt(8, seed=1)
    with pytest.raises(EspError, match="tile edge 20"):
        native.Context(native.make_params(order=8, mesh=(32, 32, 32), tile=20, precision=1), s.box, s.N)


def test_precision_is_checked():
    s = systems.rocksalt(8, seed=1)
    c64 = native.Context(native.make_params(precision=1), s.box, s.N)
    pos = torch.zeros((s.N, 4), device="cuda")
    q = torch.zeros(s.N, device="cuda")
    with pytest.raises(EspError):
        c64.compute(pos, q, torch.zeros((s.N, 4), device="cuda"), flags=1)
    c32 = native.Context(native.make_params(), s.box, s.N)
    with pytest.raises(EspError):
        c32.compute_f64(pos.double(), q.double(), torch.zeros((s.N, 4), dtype=torch.float64, device="cuda"), flags=1)
    with pytest.raises(EspError):
        native.Context(native.make_params(precision=2), s.box, s.N).compute(pos, q, torch.zeros_like(pos), flags=1)

"""Interpolation with the potential tile staged by TMA (one
cp.async.bulk.tensor box of the halo-padded potential mesh per tile; one CTA
per tile, or persistent CTAs fed from a tile queue) against
the cp.async staging of the same plan: the same forces and per-particle
energies (each particle's contraction is the same arithmetic on the same
staged values), for supports 5..8, odd, non-cubic and small meshes (where
the halo is widest) and the autotuner's smaller tiles, and for a clustered
system whose empty tiles the persistent tile-queue kernel passes over; the
kernels' error word stays clear. The cp.async form itself is pinned to the
oracle by test_gpu_parity.py."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems  # noqa: E402
from esp_hoomd_b200._lib import ESP_LONG_RANGE  # noqa: E402


def _run(sl, **kw):
    N = [s.N for s in sl]
    b = native.Batch(native.make_params(**kw), N, [s.box for s in sl])
    p4 = np.zeros((sum(N), 4), np.float32)
    p4[:, :3] = np.concatenate([s.pos for s in sl])
    pos = torch.tensor(p4, device="cuda")
    q = torch.tensor(np.concatenate([s.q for s in sl]).astype(np.float32), device="cuda")
    f = torch.zeros((sum(N), 4), device="cuda")
    e = torch.zeros(len(sl), dtype=torch.float64, device="cuda")
    b.compute(pos, q, f, e, None, flags=ESP_LONG_RANGE)
    torch.cuda.synchronize()
    assert b.device_errors() == 0
    return f.double().cpu().numpy(), e.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 2])
@pytest.mark.parametrize("order,tile", [(8, 0), (6, 0), (5, 0), (8, 8), (8, 7)])
def test_tma_interp_equals_cp_async(order, tile, mode):
    sl = [systems.rocksalt(n, seed=9100 + n) for n in (8, 11, 20)]
    sl.append(systems.rocksalt(0, seed=9199, shape=(13, 22, 9)))
    kw = dict(order=order, tile=tile)
    fa, ea = _run(sl, interp_mode=1, **kw)
    fb, eb = _run(sl, interp_mode=mode, **kw)
    assert np.abs(fb - fa).max() <= 1e-6 * np.abs(fa).max()
    assert np.all(np.abs(eb - ea) <= 1e-9 * np.abs(ea))


def test_tma_interp_with_empty_tiles():
    # every particle in one corner octant: most tiles hold none
    rng = np.random.default_rng(12)
    L, n = 24.0, 3000
    pos = rng.uniform(0.0, 0.45 * L, (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    s = systems.System(pos=pos, q=q, vel=np.zeros_like(pos), mass=np.ones(n), box=(L, L, L))
    sl = [systems.rocksalt(10, seed=9201), s, systems.rocksalt(12, seed=9202)]
    fa, ea = _run(sl, interp_mode=1, order=8)
    for mode in (0, 2):
        fb, eb = _run(sl, interp_mode=mode, order=8)
        assert np.abs(fb - fa).max() <= 1e-6 * np.abs(fa).max()
        assert np.all(np.abs(eb - ea) <= 1e-9 * np.abs(ea))

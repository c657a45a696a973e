"""The scale-up case: one system of 10^6 rock-salt ions (100^3 lattice,
spacing 1, jitter 0.1, L = 100; support 8, r_c 3.0, 1e-5 target), single
evaluations in the FP32 and FP64 modes on the plain one-system path:

* against FP64 direct Ewald on a seeded subset of 10^4 ions, with the
  structure factor over all 10^6 charges (``oracle/ewald_torch.py``): both
  modes <= 1e-5 relative RMS force error;
* FP32 forces within 5e-6 relative RMS of FP64 (the parity tolerance of
  the FP32 path), energies within 1e-6;
* the k-space virial agrees to 1e-5 of its largest component;
* per-particle energies add up to the total.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import native, systems  # noqa: E402
from oracle import esp_ref as R  # noqa: E402
from oracle.ewald_torch import ewald_torch  # noqa: E402


@pytest.fixture(scope="module")
def scaleup():
    s = systems.rocksalt(100, seed=1001)
    N = s.N
    p4 = np.zeros((N, 4), np.float32)
    p4[:, :3] = s.pos
    pos32 = torch.as_tensor(p4, device="cuda")
    q32 = torch.as_tensor(s.q.astype(np.float32), device="cuda")
    # the FP64 run uses the same (float32-representable) positions
    pos64 = pos32.double()
    q64 = q32.double()
    b32 = native.Batch(native.make_params(), [N], [s.box])
    head = torch.zeros(N, dtype=torch.int32, device="cuda")
    nn = torch.zeros_like(head)
    nl = torch.zeros(N * 256, dtype=torch.int32, device="cuda")
    b32.build_nlist(pos32, 3.4, 256, head, nn, nl)
    f32 = torch.zeros((N, 4), device="cuda")
    e32 = torch.zeros(1, dtype=torch.float64, device="cuda")
    w32 = torch.zeros(6, dtype=torch.float64, device="cuda")
    b32.compute(pos32, q32, f32, e32, w32, nlist=(head, nn, nl))
    inf = b32.info(0)
    assert (inf["nx"], inf["ny"], inf["nz"]) == (200, 200, 200)
    b64 = native.Batch(native.make_params(precision=1, mesh=(200, 200, 200)), [N], [s.box])
    f64 = torch.zeros((N, 4), dtype=torch.float64, device="cuda")
    e64 = torch.zeros(1, dtype=torch.float64, device="cuda")
    w64 = torch.zeros(6, dtype=torch.float64, device="cuda")
    b64.compute_f64(pos64, q64, f64, e64, w64, nlist=(head, nn, nl))
    torch.cuda.synchronize()
    out = dict(s=s, pos=pos64[:, :3].cpu().numpy(), f32=f32.double().cpu().numpy(), e32=e32.item(),
               w32=w32.cpu().numpy(), f64=f64.cpu().numpy(), e64=e64.item(), w64=w64.cpu().numpy())
    del b32, b64, head, nn, nl
    torch.cuda.empty_cache()
    return out


def test_scaleup_fp32_matches_fp64(scaleup):
    a, c = scaleup["f32"], scaleup["f64"]
    assert R.rel_rms(a[:, :3], c[:, :3]) <= 5e-6
    assert abs(scaleup["e32"] - scaleup["e64"]) <= 1e-6 * abs(scaleup["e64"])
    w32, w64 = scaleup["w32"], scaleup["w64"]
    assert np.abs(w32 - w64).max() <= 1e-5 * np.abs(w64).max()
    assert abs(a[:, 3].sum() - scaleup["e32"]) <= 1e-5 * abs(scaleup["e32"])


def test_scaleup_subset_vs_ewald(scaleup):
    s = scaleup["s"]
    sub = np.sort(np.random.default_rng(1002).choice(s.N, size=10000, replace=False))
    _, F0, _ = ewald_torch(scaleup["pos"], s.q, s.box, targets=sub)
    for key in ("f32", "f64"):
        err = R.rel_rms(scaleup[key][sub, :3], F0)
        assert err <= 1e-5, (key, err)

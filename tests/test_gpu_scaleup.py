"""The scale-up case: one system of 10^6 rock-salt ions (100^3 lattice,
spacing 1, jitter 0.1, L = 100; support 8, r_c 3.0, 1e-5 target), single
evaluations in the FP32 (compensated) and FP64 modes on the plain
one-system path. A direct Ewald sum is out of reach at this size; the FP64
mode (pinned against Ewald at smaller sizes) is the reference here:

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


def test_scaleup_fp32_matches_fp64():
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
    a, c = f32.double().cpu().numpy(), f64.cpu().numpy()
    assert R.rel_rms(a[:, :3], c[:, :3]) <= 5e-6
    assert abs(e32.item() - e64.item()) <= 1e-6 * abs(e64.item())
    assert np.abs(w32.cpu().numpy() - w64.cpu().numpy()).max() <= 1e-5 * np.abs(w64.cpu().numpy()).max()
    assert abs(a[:, 3].sum() - e32.item()) <= 1e-5 * abs(e32.item())

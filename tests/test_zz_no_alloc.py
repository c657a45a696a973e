"""esp_spread_noalloc: charge spreading without any device allocation.

Callers such as an MD engine whose own pool allocator holds the device
memory, or a time step that must not call cudaFree (it synchronises the
device), cannot create a context, because esp_create allocates its work
arrays. esp_spread_noalloc gives them bin + sort + spreading with its work
arrays in a fixed scratch array inside the library. This test calls it
through the C ABI on two different systems in a row (so a stale scratch
from the first call would show in the second), and a third time on the
first system, and checks every mesh against esp_spread's on the same
inputs within the spreading tolerance of the parity tests,
max |d rho| <= 2e-6 max |rho|. It does so for the default plan (support 8,
the 16^3 tensor-core tile), for smaller dense tiles at supports 4 and 6
(which change the tile and chunk counts inside the scratch), and for a
context created with FP64 precision (whose window has a higher degree). The
file is named to be collected last, and it also passes alone in a fresh
process (its first call does the per-device set-up).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from esp_hoomd_b200 import _lib, native, systems  # noqa: E402

TOL = 2e-6


def _upload(s):
    pos4 = np.zeros((s.N, 4), dtype=np.float32)
    pos4[:, :3] = s.pos
    return (torch.as_tensor(pos4, device="cuda"),
            torch.as_tensor(s.q.astype(np.float32), device="cuda"))


def _case(s, order=8, tile=0, precision=0):
    """(inputs, esp_spread's mesh, the parameters that reproduce its plan;
    the window degree is left to the entry point's own default)."""
    pos4, q = _upload(s)
    ctx = native.Context(native.make_params(order=order, tile=tile, precision=precision), s.box, s.N)
    ref = ctx.spread(pos4, q)
    inf = ctx.info()
    p = native.make_params(order=inf["order"], mesh=(inf["nx"], inf["ny"], inf["nz"]), window_c=inf["c_window"],
                           tile=inf["tile"], precision=precision)
    return pos4, q, ref, p


def _noalloc(s, pos4, q, p, rho):
    lib = _lib.get_lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.esp_spread_noalloc(stream, ctypes.byref(p), *(float(b) for b in s.box),
                                ctypes.c_void_p(pos4.data_ptr()), ctypes.c_void_p(q.data_ptr()), s.N,
                                ctypes.c_void_p(rho.data_ptr()))
    _lib.check(rc, "esp_spread_noalloc")


@pytest.mark.parametrize("order,tile,precision", [(8, 0, 0), (4, 11, 0), (6, 9, 0), (8, 0, 1)])
def test_noalloc_spread_matches_esp_spread_on_consecutive_calls(order, tile, precision):
    a = systems.rocksalt(8, seed=2024)                        # 512 ions, mesh 16^3
    b = systems.rocksalt(0, seed=2025, shape=(12, 10, 14))    # 1680 ions, non-cubic mesh
    cases = [(s, _case(s, order, tile, precision)) for s in (a, b, a)]
    for s, (pos4, q, ref, p) in cases:
        rho = torch.full_like(ref, 123.0)  # the entry point must clear the mesh itself
        _noalloc(s, pos4, q, p, rho)
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), rho.cpu().numpy()
        assert np.abs(g - r).max() <= TOL * np.abs(r).max()
        assert abs(g.sum() - r.sum()) <= 1e-9 * np.abs(r).sum()


def test_noalloc_spread_rejects_sizes_beyond_its_limit():
    lib = _lib.get_lib()
    s = systems.rocksalt(4, seed=1)
    pos4, q = _upload(s)
    rho = torch.zeros((16, 16, 16), dtype=torch.float64, device="cuda")
    p = native.make_params(mesh=(16, 16, 16))
    args = (None, ctypes.byref(p), 16.0, 16.0, 16.0, ctypes.c_void_p(pos4.data_ptr()),
            ctypes.c_void_p(q.data_ptr()))
    assert lib.esp_spread_noalloc(*args, 32769, ctypes.c_void_p(rho.data_ptr())) == -4
    assert b"32768" in lib.esp_last_error()
    p_auto = native.make_params()  # no explicit mesh
    assert lib.esp_spread_noalloc(None, ctypes.byref(p_auto), 16.0, 16.0, 16.0, ctypes.c_void_p(pos4.data_ptr()),
                                  ctypes.c_void_p(q.data_ptr()), s.N, ctypes.c_void_p(rho.data_ptr())) == -1
    p_bad = native.make_params(mesh=(16, 16, 16), precision=2)  # neither ESP_FP32 nor ESP_FP64
    assert lib.esp_spread_noalloc(None, ctypes.byref(p_bad), 16.0, 16.0, 16.0, ctypes.c_void_p(pos4.data_ptr()),
                                  ctypes.c_void_p(q.data_ptr()), s.N, ctypes.c_void_p(rho.data_ptr())) == -1

"""The C ABI library loads and exports every entry point include/esp_b200.h
declares; host-side argument validation needs no GPU."""
import ctypes
import os
import re

import pytest

from esp_hoomd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "esp_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(esp_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    assert _declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.get_lib()
    for name in _declared():
        assert hasattr(lib, name), name


def test_params_default():
    lib = _lib.get_lib()
    p = _lib.EspParams()
    assert lib.esp_params_default(ctypes.byref(p)) == 0
    assert p.order == 8 and p.rcut == 3.0 and p.target_error == 1e-5 and p.alpha == 0.0
    assert lib.esp_params_default(None) == -1
    assert b"null" in lib.esp_last_error()


def test_null_handles_are_rejected():
    lib = _lib.get_lib()
    assert lib.esp_compute(None, None, None, None, 0, None, None, None, None, None, None, 3) == -1
    assert lib.esp_batch_compute(None, None, None, None, None, None, None, None, None, None, 3) == -1
    assert lib.esp_destroy(None) == 0


def test_oracle_reference_build_present_or_skipped():
    path = os.path.join(ROOT, "oracle", "_ref", "libpswf_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference evaluator not built (needs the reference sources)")
    lib = ctypes.CDLL(path)
    assert hasattr(lib, "ref_eval_pairs") and hasattr(lib, "ref_eval_L")


def _prototypes():
    """name -> parameter count of every entry point in the header."""
    text = open(os.path.join(ROOT, "include", "esp_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*(?:int|const char\*)\s+(esp_\w+)\s*\(([^;]*?)\)\s*;", text, re.M):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_argument_counts_match_the_header():
    """Every ctypes argtypes list has as many entries as the header's
    prototype has parameters (a missing or extra argument would pass the
    wrong values silently)."""
    lib = _lib.get_lib()
    protos = _prototypes()
    assert set(protos) == set(_declared())
    checked = 0
    for name, n in protos.items():
        at = getattr(lib, name).argtypes
        if at is not None:
            assert len(at) == n, (name, len(at), n)
            checked += 1
    assert checked >= 40


def test_md_run_f64_rejects_a_null_batch():
    lib = _lib.get_lib()
    assert lib.esp_batch_md_run_f64(None, None, None, None, None, None, None, None, None, None, None, 1, 0.002,
                                    0.0, 0.0, 0.0, 1) == -1
    assert b"null" in lib.esp_last_error()


@pytest.mark.parametrize("field,value,code,text", [
    ("order", 13, -4, b"order must be in [2, 12]"),
    ("order", 1, -4, b"order must be in [2, 12]"),
    ("tile", 70, -4, b"tile edge must be <= 64"),
    ("threads_per_particle", 3, -4, b"threads_per_particle must be 4, 8, 16 or 32"),
    ("precision", 2, -1, b"precision must be ESP_FP32 or ESP_FP64"),
    ("interp_mode", 3, -1, b"interp_mode must be 0, 1 or 2"),
])
def test_create_validates_parameters_before_any_device_work(field, value, code, text):
    """Parameter errors are reported by the host with their own status code
    and message (ESP_ERR_UNSUPPORTED / ESP_ERR_INVALID), before the context
    touches the device, so they need no GPU."""
    lib = _lib.get_lib()
    p = _lib.EspParams()
    assert lib.esp_params_default(ctypes.byref(p)) == 0
    setattr(p, field, value)
    h = ctypes.c_void_p()
    assert lib.esp_create(ctypes.byref(p), 8.0, 8.0, 8.0, 512, ctypes.byref(h)) == code
    assert text in lib.esp_last_error()
    assert not h.value


def test_create_rejects_a_negative_particle_count():
    lib = _lib.get_lib()
    p = _lib.EspParams()
    lib.esp_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    assert lib.esp_create(ctypes.byref(p), 8.0, 8.0, 8.0, -5, ctypes.byref(h)) == -1
    assert b"negative particle count" in lib.esp_last_error()


def test_batch_create_validates_on_the_host():
    lib = _lib.get_lib()
    p = _lib.EspParams()
    lib.esp_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    n = (ctypes.c_int * 2)(512, 512)
    boxes = (ctypes.c_double * 6)(8, 8, 8, 8, 8, 8)
    assert lib.esp_batch_create(ctypes.byref(p), 0, n, boxes, None, ctypes.byref(h)) == -1
    assert b"number of systems must be positive" in lib.esp_last_error()
    assert lib.esp_batch_create(ctypes.byref(p), 2, None, boxes, None, ctypes.byref(h)) == -1
    small = (ctypes.c_double * 6)(8, 8, 8, 1, 8, 8)  # r_c = 3 exceeds half of the second box
    assert lib.esp_batch_create(ctypes.byref(p), 2, n, small, None, ctypes.byref(h)) == -1
    assert b"rcut must not exceed half the box" in lib.esp_last_error()
    assert not h.value

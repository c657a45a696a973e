"""Regenerate the committed golden fixtures from the reference.

Run from the repository root in a checkout that has the reference sources
(the directory ``reference`` beside the repository root by default,
override with ESP_REF):

    make -C oracle ref          # builds oracle/_ref/libpswf_ref.so
    python tests/golden/make_golden.py

Writes
* ``pswf_coeffs_shipped.npz``: the shipped table src/PSWF_Coeffs.h
  (PSWF_SCREEN_COEFFS, PSWF_DSCREEN_COEFFS, PSWF_R_LO, PSWF_DR_INV,
  PSWF_RCUT) read as text;
* ``pswf_eval_golden.npz``: EvaluatorPairPSWF::evalForceAndEnergy and
  detail::pswf_eval_L outputs of the reference compiled from its own
  sources (oracle/_ref), on seeded (rsq, qiqj) samples.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from esp_hoomd_b200.tables import parse_pswf_coeffs_header  # noqa: E402

REF = os.environ.get("ESP_REF", os.path.join(os.path.dirname(ROOT), "reference"))


def main() -> None:
    with open(os.path.join(REF, "src", "PSWF_Coeffs.h")) as f:
        tab = parse_pswf_coeffs_header(f.read())
    np.savez_compressed(os.path.join(HERE, "pswf_coeffs_shipped.npz"), screen=tab.screen, dscreen=tab.dscreen,
                        r_lo=tab.r_lo, dr_inv=tab.dr_inv, rcut=np.array(tab.rcut))
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpswf_ref.so"))
    rng = np.random.default_rng(20261203)
    n = 6000
    r = np.concatenate([rng.uniform(0.0, 1.2, n - 8),
                        [0.0, 1e-13, 1e-6, 0.1, 0.25, 0.5, 0.75, 1.0]])
    rsq = r * r
    qiqj = rng.choice([-1.0, 1.0, 0.5, -0.25, 0.0], size=n)
    qiqj[-8:] = -1.0
    fdr = np.zeros(n)
    eng = np.zeros(n)
    ok = np.zeros(n, dtype=np.int32)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    lib.ref_eval_pairs(n, vp(rsq), vp(qiqj), ctypes.c_double(1.0), vp(fdr), vp(eng), vp(ok))
    L = np.zeros(n)
    D = np.zeros(n)
    lib.ref_eval_L(n, vp(r), ctypes.c_double(1.0), vp(L), vp(D))
    np.savez_compressed(os.path.join(HERE, "pswf_eval_golden.npz"), r=r, rsq=rsq, qiqj=qiqj, force_divr=fdr,
                        pair_eng=eng, evaluated=ok, L=L, negdLdr=D, rcut=np.array(1.0))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()

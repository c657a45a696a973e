"""The Python API mirror of the reference plugin's esp.py (src/esp.py):
argument validation, error types, properties before attachment, the
Spectral <-> Local link, the factory and the aliases. No GPU needed."""
import warnings

import pytest

from esp_hoomd_b200 import esp


def _nl():
    return esp.NeighborList(buffer=0.4)


def test_constants_and_aliases():
    assert esp.MAX_ORDER == 12 and esp.DEFAULT_TABLE_SEGMENTS == 512 and esp.MIN_TABLE_SEGMENTS == 16
    assert esp.Coulomb is esp.Spectral and esp.Pair is esp.Local
    for name in ("Spectral", "Local", "make_esp_forces", "Coulomb", "Pair", "MAX_ORDER",
                 "DEFAULT_TABLE_SEGMENTS", "MIN_TABLE_SEGMENTS"):
        assert name in esp.__all__


def test_spectral_defaults_and_properties_before_attach():
    s = esp.Spectral(_nl(), 3.0, resolution=(24, 24, 24), order=8, kappa=6.0)
    assert s.resolution == (24, 24, 24) and s.order == 8 and s.kappa == 6.0 and s.r_cut == 3.0
    assert s.alpha == 0.0 and s.n_table == 512
    with pytest.raises(RuntimeError):
        _ = s.q_sum
    with pytest.raises(RuntimeError):
        _ = s.q2_sum
    with pytest.raises(RuntimeError):
        s.set_params(order=6)
    with pytest.raises(RuntimeError):
        _ = s.forces
    s.invalidate()  # no-op before attachment
    assert "esp.Spectral(" in repr(s)


def test_spectral_kappa_none_warns():
    with pytest.warns(UserWarning, match="kappa"):
        s = esp.Spectral(_nl(), 3.0)
    assert s.kappa is None and s.order == 6 and s.resolution == (32, 32, 32)


@pytest.mark.parametrize("kw", [
    dict(default_r_cut=0.0), dict(default_r_cut=-1.0), dict(default_r_cut="3"),
    dict(resolution=(32, 32)), dict(resolution=(32, 0, 32)), dict(resolution=(32, 32, 2.5)),
    dict(order=1), dict(order=13), dict(order=6.0), dict(order=True),
    dict(kappa=0.0), dict(kappa=-1.0),
    dict(alpha=-0.1), dict(alpha=0.5),
    dict(n_table=15), dict(n_table=100.0),
])
def test_spectral_validation_errors(kw):
    args = dict(nlist=_nl(), default_r_cut=3.0, resolution=(32, 32, 32), order=6, kappa=5.0)
    args.update(kw)
    with pytest.raises(ValueError):
        esp.Spectral(**args)


def test_local_validation():
    s = esp.Spectral(_nl(), 3.0, kappa=6.0)
    with pytest.raises(ValueError):
        esp.Local(_nl(), 3.0)
    with pytest.raises(TypeError):
        esp.Local(_nl(), 3.0, spectral=object())
    with pytest.raises(ValueError):
        esp.Local(_nl(), 3.0, spectral=s, mode="shift")
    with pytest.warns(DeprecationWarning):
        loc = esp.Local(_nl(), 3.0, coulomb=s)
    assert loc._spectral is s and s._pair is loc


def test_local_params_accept_empty_dict_and_warn_on_keys():
    s = esp.Spectral(_nl(), 3.0, kappa=6.0)
    loc = esp.Local(_nl(), 3.0, spectral=s)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        loc.params[("A", "A")] = {}
    with pytest.warns(UserWarning, match="Ignoring keys"):
        loc.params[("A", "B")] = {"epsilon": 1.0}
    assert loc.params[("A", "B")] == {}
    with pytest.raises(TypeError):
        loc.params["A"] = {}
    assert "esp.Local(" in repr(loc)


def test_make_esp_forces_links_the_pair():
    nl = _nl()
    sp, lo = esp.make_esp_forces(nl, 3.0, resolution=(20, 20, 20), order=8, kappa=6.0)
    assert isinstance(sp, esp.Spectral) and isinstance(lo, esp.Local)
    assert lo._spectral is sp and sp._pair is lo and sp.resolution == (20, 20, 20)
    with pytest.raises(ValueError):
        esp.make_esp_forces(nl, 3.0, order=0)


def test_simulation_validation():
    with pytest.raises(ValueError):
        esp.NeighborList(buffer=-1.0)
    with pytest.raises(ValueError):
        esp.NeighborList(capacity=0)

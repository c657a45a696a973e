"""The `_esp` extension module (CPU checks, no device calls): it imports,
and exports the reference plugin's classes with their Python-facing method
names (src/module.cc:57-85, src/ESPForceCompute.cc:411-509,
src/ESPForceComputeGPU.cc:457-481)."""
import pytest

_esp = pytest.importorskip("esp_hoomd_b200._esp")


def test_module_exports_reference_classes():
    assert _esp.gpu_enabled is True
    for cls in ("ESPForceCompute", "ESPForceComputeGPU", "ESPTableEntry", "PotentialPairPSWF",
                "PotentialPairPSWFGPU"):
        assert hasattr(_esp, cls), cls
    for meth in ("setParams", "getResolution", "getOrder", "getKappa", "getRCut", "getAlpha", "getQSum",
                 "getQ2Sum", "getTableSize", "getTablePtr", "getTableEntry", "invalidate", "compute", "table"):
        assert hasattr(_esp.ESPForceCompute, meth), meth
    assert issubclass(_esp.ESPForceComputeGPU, _esp.ESPForceCompute)
    assert issubclass(_esp.PotentialPairPSWFGPU, _esp.PotentialPairPSWF)
    for attr in ("potential_coeffs", "force_coeffs", "potential_coeff4", "force_coeff4", "r_lo", "dr_inv"):
        assert hasattr(_esp.ESPTableEntry, attr), attr
    # the HOOMD stand-in classes the module is compiled against
    for cls in ("SystemDefinition", "ParticleData", "ParticleGroup", "NeighborList", "ForceCompute", "BoxDim"):
        assert hasattr(_esp, cls), cls
    assert _esp.BoxDim(1.0, 2.0, 3.0).L == (1.0, 2.0, 3.0)

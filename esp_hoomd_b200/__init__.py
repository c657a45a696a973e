"""esp_hoomd_b200: Blackwell-native ESP (Ewald Summation with Prolates)
long-range electrostatics for HOOMD-blue style simulations.

Python surface: ``esp`` (Spectral / Local / make_esp_forces, the reference
plugin's API), ``native`` (device contexts over the C ABI), ``tables`` (the
runtime PSWF table generator) and ``systems`` (synthetic inputs).
"""
__version__ = "0.9.1"

"""trhepd-opt_b200: B200-native multislice surface solve of sim-trhepd-rheed.

The directory name carries a hyphen, so the package is loaded under the module
name ``trhepd_opt_b200`` (see ``load()`` in bench.py / tests/conftest.py).
"""
__all__ = ["generator", "formats", "surface", "native"]

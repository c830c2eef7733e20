"""blade_b200: B200-native nonbonded direct space for BLaDE.

The compute path is libbnb.so (hand-written sm_100a CUDA behind the C ABI in
include/bnb.h).  This package is its Python host side: ctypes bindings
(``_lib``), the Domdec/getforce_nbdirect mirror (``nbdirect``), the MSLD
lambda maps (``msld``) and seeded synthetic systems (``systems``).
"""
__all__ = ["systems", "nbdirect", "msld"]

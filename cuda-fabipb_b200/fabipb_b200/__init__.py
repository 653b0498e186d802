"""fabipb_b200: B200-native FABIPB boundary-integral Poisson-Boltzmann hot path.

The compute lives in the CUDA shared library ``libfabipb_b200.so`` (built from
``cuda-fabipb_b200/csrc``); this package is the host side: mesh/charge input
(``meshio``), seeded synthetic cases (``meshgen``) and the ctypes binding of
the C ABI (``lib``).
"""

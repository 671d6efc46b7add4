"""B200-native dense direct solve behind PLAPACK's PLA_Obj / PLA_Template API.

The product is the C library libplapack_b200.so (include/PLA.h); this package
holds its sources (csrc/), the build step (build.py) and a ctypes binding
(pla.py) used by the tests and the benchmark.
"""

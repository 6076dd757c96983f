"""wema_b200 - B200-native (sm_100a) WEMA per-frame motion-amplification path.

The product is the C-ABI library ``lib/libwema_cuda.so`` (headers in the
repository's ``include/``); this package holds its sources (``csrc/``), the
in-tree build (``_build``), a ctypes binding used by tests and the benchmark
(``cuda``) and the seeded synthetic video generator (``synth``).
"""

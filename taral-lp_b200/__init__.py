"""B200-native PDHG engine for large continuous LPs (sm_100a CUDA behind a C ABI).

Modules: ``pdhg`` (ctypes binding of include/taral_pdhg.h), ``lpgen`` (seeded synthetic LP families),
``build`` (in-tree compile of lib/libtaral_pdhg.so and bin/pdhg). The directory name is not a Python
identifier; load it with :func:`load` from a file beside it, or put it on sys.path as ``taral_lp_b200``.
"""

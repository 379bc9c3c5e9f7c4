"""tflows_b200: B200-native replacement of T-Flows' Native_Mod Krylov path.

The product is the C ABI in ``lib/libtfkrylov.so`` (declared in
``include/tf_krylov.h``); :mod:`tflows_b200.native` binds it for Python.
:mod:`tflows_b200.grids` and :mod:`tflows_b200.systems` generate the seeded
synthetic systems the solvers are tested and measured on.
"""
from . import grids, native, systems  # noqa: F401

__all__ = ["grids", "native", "systems"]

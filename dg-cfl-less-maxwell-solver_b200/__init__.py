"""gdon3d_b200: B200 (sm_100a) implementation of Gdon3d's two data-parallel hot
paths behind the C-ABI in include/gdon3d_cuda.h.

  capi   ctypes bindings of libgdon3d_cuda.so (the product; CUDA only)
  kuhn   seeded synthetic Kuhn-cube meshes and gmsh v2.2 I/O

This directory is loaded as the Python package `gdon3d_b200` (its on-disk
name is not a Python identifier): see load_package() in tests/conftest.py and
bench.py.
"""

from . import capi, kuhn  # noqa: E402,F401

"""B200 (sm_100a) engine for the extrapolation + imaging path of Imaging2D_WLSQ.

Modules:
  interface       mirror of the reference's cpp_src/interface.py (host argument order)
  interface_cuda  mirror of the reference's cpp_src/interface_cuda.py (device argument order)
  migration       compact-table migration: host-buffer `migrate` and device-resident `Plan`
  operators       host-side WLSQ / phase-shift operator design and the compact table
  synthetic       seeded synthetic workloads of the benchmark configurations
The CUDA library libimaging2d_wlsq_b200.so is built in-tree by `python -m imaging2d_wlsq_b200.build`.
"""
from ._lib import LIB_PATH, DROPIN_DIR, LibraryError  # noqa: F401

__version__ = "1.0.0"

"""ocfd_b200 -- host side of the B200 implementation of the OpenCFD-EC per-iteration hot path.

The compute path is the CUDA library ``libocfd_b200.so`` (csrc/), reached through the C-ABI
declared in include/ocfd_ec_gpu.h; this package holds its ctypes binding (``capi``), parameter
handling (``params``), the bc3d.inp -> .inc converter (``connectivity``), analytic meshes for
the benchmark configurations (``meshgen``, ``cases``), file formats (``formats``) and the
continuous-batching request loop (``serve``).
"""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)  # opencfd-ec_b200/

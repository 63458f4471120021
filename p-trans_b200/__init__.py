"""B200 (sm_100a) Monte Carlo ray-tracing phonon transport: Python host mirror.

The product is the C ABI in include/ptrans_gpu.h, implemented by
libptrans_b200.so (CUDA kernels + C++ host code).  This package binds it with
ctypes and adds seeded input generators.  The directory name is not an
identifier; load it as a package named ``ptrans_b200`` (see ``load``).
"""
from . import abi, synth  # noqa: F401
from .abi import (GeomBuf, Handle, Model, PtgError, Spectrum, kappa_from_counts,  # noqa: F401
                  load_library, make_run)

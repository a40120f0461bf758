"""B200 density-matrix propagator (EDUS right-hand side + RK4/AB steppers).

The product is the CUDA library ``lib/libedus_gpu.so`` with the C ABI of
``include/edus_gpu.h``.  This Python package is a thin ctypes host layer over
that ABI (``edus``) plus the synthetic benchmark workloads (``workloads``).
The directory name is not a valid Python identifier; load it with
``importlib`` (see ``load_package`` in ``__graft_entry__.py``).
"""
from . import edus, h5, hhg, model, surrogate, sweep, workloads  # noqa: F401
from .edus import Solver, EdusError, Laser, load_library  # noqa: F401

"""B200-native Hamiltonian apply H.psi of the plane-wave Davidson path.

The compute path is libbaandi_b200.so (hand-written sm_100a CUDA behind the C ABI of
include/baandi_gpu.h); this package holds the ctypes binding, the host-side mirror of
the reference operator interface and the synthetic workloads.  There is no CPU
fallback: the operators raise if the library or a B200 is missing.
"""
from . import _lib  # noqa: F401

__all__ = ["hamiltonian", "operands", "systems", "build"]

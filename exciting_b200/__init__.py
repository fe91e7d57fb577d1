"""exciting_b200: B200 (sm_100a) per-k-point LAPW Hamiltonian/overlap setup.

The compute lives in libexciting_b200.so (C-ABI, include/exciting_b200.h);
this package holds the ctypes binding (``abi``), the host-side mirror of the
reference's interface (``fvsystem.Setup``) and the host-side producers of the
setup's inputs (``crystal``, ``basis``, ``system``, ``workloads``).
"""
from . import abi, basis, crystal, system, workloads  # noqa: F401

__all__ = ["abi", "basis", "crystal", "system", "workloads"]

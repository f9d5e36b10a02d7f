"""B200-native short-range Lennard-Jones hot path of MarDyn (linked cells, LJ 12-6 pair forces,
Leapfrog) behind a C ABI (include/mdgpu.h, libmdgpu.so)."""
from . import workloads  # noqa: F401

__all__ = ["workloads", "mdgpu", "build"]

"""Host-side Python mirror of the MPCD B200 solvent timestep (C ABI in
include/mpcd_gpu.h, kernels in niamh-mpcd_b200/csrc)."""
from . import abi, workloads  # noqa: F401

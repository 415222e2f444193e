"""B200-native NDDO (AM1/RM1) SCF single point, a drop-in for am1-rs's run_am1.

``native`` mirrors the reference's Python entry points; ``workloads`` generates the seeded
synthetic molecules of the benchmark configurations.  The compute path is libam1gpu.so
(CUDA, sm_100a) behind the C ABI in include/am1gpu.h.
"""

from . import _abi  # noqa: F401

"""ubolt_b200: UBOLT's fixed-source discrete-ordinates solve on B200 (sm_100a).

The compute path is libubolt_b200.so (CUDA kernels + C ABI, include/ubolt_b200.h).
`ubolt_b200.problem` builds meshes, geometry and the named workloads;
`ubolt_b200.transport` mirrors the reference's operator / preconditioner
classes over the C ABI (needs torch and a CUDA device).
"""
from . import _lib  # noqa: F401  (raises if the shared library is missing)

__all__ = ["problem", "transport"]

"""ubolt_b200: UBOLT's fixed-source discrete-ordinates solve on B200 (sm_100a).

The compute path is libubolt_b200.so (CUDA kernels + C ABI, include/ubolt_b200.h),
built in-tree by `python -m ubolt_b200.build`. `ubolt_b200.problem` builds
meshes, geometry and the named workloads; `ubolt_b200.problem_file` reads
the reference's JSON problem files and Gmsh 2.2 meshes into a problem and
solves one group by group; `ubolt_b200.transport` mirrors the
reference's operator / preconditioner / solver classes over the C ABI (needs
torch and a CUDA device). Importing either loads the library and raises if it
is missing - there is no fallback path.
"""

__all__ = ["problem", "problem_file", "transport", "build"]

"""Build libubolt_b200.so in-tree: nvcc for sm_100a, g++ for the host C++.

    python -m ubolt_b200.build            # incremental
    python -m ubolt_b200.build --clean

Objects go to ubolt_b200/_build/, the shared library to
ubolt_b200/libubolt_b200.so (both git-ignored; the .so travels with the
source tree to wherever it runs).
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libubolt_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
CU_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
            "--expt-relaxed-constexpr", "-Xptxas", "-O3"] + ARCH + INCLUDES
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function"] + INCLUDES + \
    ["-I" + os.path.join(CUDA, "include")]


def _sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def _headers_mtime():
    paths = [os.path.join(CSRC, n) for n in os.listdir(CSRC) if n.endswith((".h", ".cuh"))]
    paths.append(os.path.join(ROOT, "include", "ubolt_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + CU_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj, None


def build(verbose=False, jobs=None):
    """Compile every source for sm_100a and link libubolt_b200.so. Raises on failure."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("build failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, "-shared"] + ARCH + ["-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    if "--clean" in sys.argv:
        shutil.rmtree(BUILD, ignore_errors=True)
        if os.path.exists(LIB):
            os.remove(LIB)
    print(build(verbose="-v" in sys.argv))

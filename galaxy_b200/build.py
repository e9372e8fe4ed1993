"""Build recipe of libgalaxy_b200.so (sm_100a) -- run by ``__graft_entry__.build()``.

Every CUDA source is compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
only (the B200); objects are rebuilt when their source or a header is newer, and
linked into ``galaxy_b200/libgalaxy_b200.so`` in-tree with a static CUDA runtime.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgalaxy_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Sources whose FP64 arithmetic keeps every product and sum rounded separately, in the
# reference's operation order (no fused multiply-add contraction).
NO_FMA = {"gx_sph.cu"}


def _host_cxx() -> str:
    # The system compiler; the image's wrapper under /opt/gcc lacks libgomp specs.
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _deps_mtime() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hdrs.append(os.path.join(ROOT, "include", "galaxy_b200.h"))
    return max(os.path.getmtime(h) for h in hdrs if os.path.exists(h))


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps_mtime()):
        return obj
    cmd = [_nvcc(), "-ccbin", _host_cxx(), "-std=c++17", "-O3", "-lineinfo", "-ftz=true", *ARCH, "-Xcompiler", "-fPIC",
           "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fopenmp", "-I", os.path.join(ROOT, "include"), "-c", src,
           "-o", obj]
    if src.endswith(".cu"):
        cmd[1:1] = ["-x", "cu"]
        if os.path.basename(src) in NO_FMA:
            cmd.insert(1, "-fmad=false")
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose_ptxas and (res.stderr or res.stdout):
        sys.stderr.write(res.stdout + res.stderr)
    return obj


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs,
               "-Xcompiler", "-fopenmp", "-Xlinker", "--no-undefined"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))

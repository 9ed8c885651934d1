"""Build libfwt.so (the CUDA library behind include/fwt.h) in-tree for sm_100a.

    python -m fastweavturb_b200.build          # or __graft_entry__.build()

Objects go to fastweavturb_b200/_build/, the library to fastweavturb_b200/libfwt.so and the
command-line driver (the `tube` program's stand-in) to fastweavturb_b200/fwt_tube.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfwt.so")
DRIVER = os.path.join(HERE, "fwt_tube")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # the system g++ (the toolkit's supported host compiler); another one earlier on PATH may lack pieces
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str, verbose_ptxas: bool = False) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "fwt.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc(), "-ccbin", host_cxx(), *ARCH, *NVFLAGS, "-c", path, "-o", obj]
    if verbose_ptxas:
        cmd[cmd.index("-warn-spills")] = "-v"
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-ccbin", host_cxx(), "-x", "cu", *ARCH, *NVFLAGS, "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and ("spill" in r.stderr or "warning" in r.stderr):
        sys.stderr.write(r.stderr)
    return obj


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [s for s in sources() if s != "fwt_tube_main.cpp"]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc(), "-ccbin", host_cxx(), *ARCH, "-shared", "-o", LIB, *objs, "-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # command-line driver linked against the library
    drv_src = os.path.join(HERE, "driver", "fwt_tube_main.cpp")
    if os.path.exists(drv_src) and (not os.path.exists(DRIVER) or os.path.getmtime(drv_src) > os.path.getmtime(DRIVER)
                                    or os.path.getmtime(LIB) > os.path.getmtime(DRIVER)):
        cmd = [host_cxx(), "-O2", "-std=c++17", "-o", DRIVER, drv_src, f"-I{os.path.join(HERE, '..', 'include')}",
               f"-L{HERE}", "-lfwt", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))

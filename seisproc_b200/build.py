"""Builds libseispstm.so (sm_100a) in-tree with nvcc.

The shared library lands next to this file (``seisproc_b200/libseispstm.so``)
so that it travels with the source tree.  Object files are compiled in
parallel and only rebuilt when a source or header is newer than the library.

``build(checked=True)`` builds the checked test variant,
``libseispstm_checked.so``, from the same sources: every staged-row shared
address and every trace-list entry is bounds-checked in the kernels
(PSTM_ERR_BOUNDS instead of the access), the bounded device waits give up
after 50 ms instead of 2 s, and the test-only entry ``pstm_test_set_injection``
simulates faults (a stage copy never issued, the index clamp left out, a
corrupt list entry).  The tests load it in a separate process
(``SEISPSTM_LIBRARY=checked``); the product library contains none of it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libseispstm.so")
OBJDIR = os.path.join(HERE, "_build")
LIB_CHECKED = os.path.join(HERE, "libseispstm_checked.so")
OBJDIR_CHECKED = os.path.join(HERE, "_build", "checked")
CHECKED_FLAGS = ["-DPSTM_CHECKED_BUILD", "-DPSTM_BOUNDS_CHECK", "-DPSTM_WAIT_NS=50000000ull"]

SOURCES = [
    "pstm_plan.cu",
    "pstm_migrate.cu",
    "pstm_gather_fwd.cu",
    "pstm_gather_fwd_icpt.cu",
    "pstm_gather_fwd_taper.cu",
    "pstm_adjoint.cu",
    "pstm_gather_vgrad.cu",
    "pstm_noalloc.cu",
    "pstm_batch.cu",
    "pstm_velocity.cu",
    "pstm_time_domain.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + INCLUDE, "-I" + CSRC]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libseispstm.so")
    return cand


def _deps_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, extra: list, verbose: bool, objdir: str = OBJDIR) -> str:
    obj = os.path.join(objdir, src.replace(".cu", ".o"))
    cmd = [_nvcc(), *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False,
          checked: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link libseispstm.so (or, with
    ``checked``, libseispstm_checked.so); returns its path."""
    lib, objdir = (LIB_CHECKED, OBJDIR_CHECKED) if checked else (LIB, OBJDIR)
    if not force and os.path.exists(lib) and os.path.getmtime(lib) >= _deps_mtime():
        return lib
    os.makedirs(objdir, exist_ok=True)
    extra = (["-Xptxas", "-v"] if ptxas_info else []) + (CHECKED_FLAGS if checked else [])
    with cf.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, verbose or ptxas_info, objdir), SOURCES))
    tmp = lib + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv,
                ptxas_info="--ptxas" in sys.argv, checked="--checked" in sys.argv))

"""Build the engine's shared library in-tree with nvcc (sm_100a).

    python -m cablegen_b200.build          # -> cablegen_b200/libcablegen_b200.so

Every CUDA/C++ source under csrc/ is compiled to an object under _build/ and
linked into one shared library with the CUDA runtime linked statically, so the
library has no dependency beyond the driver.  The reference's own CLI sources
link against the same library (build_cli).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcablegen_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", f"-I{ROOT}/include",
                     "-Xcudafe", "--diag_suppress=177"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src: str, hdr_mtime: float, verbose: bool) -> str:
    obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = _sources()
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [os.path.getmtime(__file__)])
    if force:
        for o in glob.glob(os.path.join(OUT_DIR, "*.o")):
            os.remove(o)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr_mtime, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart_static", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


CL_LIB = os.path.join(HERE, "libcablegen_b200_cl.so")


def build_cl_seam(verbose: bool = False) -> str:
    """libcablegen_b200_cl.so: the reference's GPU plug-in seam (include/cablegen_cl.h) on the
    engine, without the library's own restatement of the reference API (refapi.cu), so the
    reference's own objects can link it; their get_settings_min() is resolved at load time."""
    build(verbose)
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [os.path.getmtime(__file__)])
    seam = _compile(os.path.join(CSRC, "clseam", "cl_seam.cu"), hdr_mtime, verbose)
    objs = [os.path.join(OUT_DIR, os.path.basename(s) + ".o") for s in _sources()
            if os.path.basename(s) not in ("refapi.cu",)] + [seam]
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(CL_LIB) or os.path.getmtime(CL_LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", CL_LIB + ".tmp"] + objs + ["-lcudart_static", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(CL_LIB + ".tmp", CL_LIB)
    return CL_LIB


CLI = os.path.join(OUT_DIR, "cli_b200")


def build_cli(reference: str, verbose: bool = False) -> str:
    """Link the reference's own CLI sources (frontends/cli/main.c, parse.c),
    unmodified, against this library: the drop-in check of the C API."""
    src = os.path.join(reference, "frontends", "cli")
    if not os.path.exists(os.path.join(src, "main.c")):
        raise FileNotFoundError(src)
    build()
    cc = os.environ.get("CC") or shutil.which("gcc") or "cc"
    cmd = [cc, "-std=c2x", "-O2", "-w", f"-I{ROOT}/include", os.path.join(src, "main.c"), os.path.join(src, "parse.c"),
           "-o", CLI, f"-L{HERE}", "-lcablegen_b200", "-Wl,-rpath,$ORIGIN/..", "-lm", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return CLI


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))

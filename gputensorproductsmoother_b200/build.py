"""Build recipe of the in-tree CUDA library ``libtps.so`` (sm_100a only).

Every translation unit is compiled with ``nvcc -gencode
arch=compute_100a,code=sm_100a -lineinfo -O3`` in parallel and linked into
``gputensorproductsmoother_b200/libtps.so`` (kept in the source tree so the
built library travels with the repository).  Re-running is incremental: a
unit is recompiled only when it or a header under csrc/ is newer than its
object file.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
REPO = os.path.dirname(PKG_DIR)
OBJ_DIR = os.path.join(CSRC, "_build")
LIB_PATH = os.path.join(PKG_DIR, "libtps.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include"),
                     "-I" + CSRC]


def _nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = os.path.join(cuda_home, "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _host_compiler() -> list[str]:
    # nvcc's default host compiler lookup; the system g++ carries libstdc++/libgomp
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if os.path.exists(gxx) else []


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, extra: list[str], verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    hdr = _newest_header()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else []
    cmd = [_nvcc()] + _host_compiler() + NVCC_FLAGS + extra + lang + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stderr.strip()):
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None, extra_flags: list[str] | None = None) -> str:
    """Compile and link libtps.so; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    extra = list(extra_flags or [])
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        cmd = [_nvcc()] + _host_compiler() + ARCH + ["-shared", "-o", LIB_PATH] + objs + \
            ["-lcudart", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

"""Builds libslosh_b200.so, the sm_100a CUDA library behind include/slosh_cuda.h, in the package
directory (so it ships with the source tree). Kernels compile with --fmad=false and the host code
with -ffp-contract=off: every float expression rounds in source order."""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libslosh_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["driver.cu", "kernels_grid.cu", "kernels_particles.cu", "kernels_mg.cu", "kernels_sort.cu", "sort_static.cu", "kernels_surface.cu", "kernels_unet.cu", "unet.cu"]
HEADERS = ["common.cuh", "kernels.h", "tc.cuh", "unet.h"]
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden,-O2", "-Xptxas", "-O3",
    "--extended-lambda", "-ccbin", "g++",
]


def _deps():
    hdr = [os.path.join(CSRC, h) for h in HEADERS]
    hdr.append(os.path.join(HERE, "..", "include", "slosh_cuda.h"))
    return [h for h in hdr if os.path.exists(h)]


def _compile(src, extra):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    srcp = os.path.join(CSRC, src)
    newest = max(os.path.getmtime(p) for p in [srcp] + _deps())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest and not extra:
        return obj
    cmd = [NVCC] + FLAGS + list(extra) + ["-c", srcp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), SOURCES))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs) or extra:
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])

"""Build libslimtracin_b200.so (and the benchmark's libst_peaks.so) in-tree with nvcc for sm_100a.

Usage: python -m slimtracin_b200.build [--force]
The library is compiled with --fmad=false and without fast-math: the tracing path keeps the
reference's unfused float operations and IEEE division/sqrt (see csrc/st_device.cuh).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libslimtracin_b200.so")
PEAKS_LIB = os.path.join(HERE, "libst_peaks.so")      # bench.py's L2 read-rate measurement
PEAKS_SRC = "st_peaks.cu"
SOURCES = ["st_api.cu", "st_render.cu", "st_bvh.cu", "st_sah.cu", "st_refsah.cu", "st_overlay.cu", "st_texture.cu", "st_io.cu", "st_obj.cu"]
HEADERS = ["st_device.cuh", "st_trace.cuh", "st_kernels.h"]
INCLUDES = [os.path.join(ROOT, "include"), CSRC]
NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + [PEAKS_SRC]]
    deps += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, objdir, verbose):
    inc = sum([["-I", d] for d in INCLUDES], [])
    obj = os.path.join(objdir, src.replace(".cu", ".o"))
    cmd = [_nvcc()] + NVCC_FLAGS + inc + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return obj


def _link(objs, out):
    tmp = out + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-cudart", "static"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)


def build(force=False, verbose=False):
    """Compile the library's sources in parallel and link libslimtracin_b200.so; also the benchmark's
    measurement helper libst_peaks.so."""
    from concurrent.futures import ThreadPoolExecutor
    if force or _stale() or not os.path.exists(PEAKS_LIB):
        objdir = os.path.join(HERE, "_build")
        os.makedirs(objdir, exist_ok=True)
        with ThreadPoolExecutor(max_workers=min(len(SOURCES) + 1, os.cpu_count() or 1)) as pool:
            jobs = [pool.submit(_compile, src, objdir, verbose) for src in SOURCES + [PEAKS_SRC]]
            objs = [j.result() for j in jobs]
        _link(objs[:-1], LIB)
        _link(objs[-1:], PEAKS_LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)

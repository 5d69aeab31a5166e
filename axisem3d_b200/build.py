"""Build the in-tree shared library libaxg.so (CUDA for sm_100a + C++ host).

    python -m axisem3d_b200.build          # or __graft_entry__.build()

nvcc cross-compiles for sm_100a without a GPU. The three precision engines are
separate translation units compiled in parallel; the result is linked with the
static CUDA runtime so the library only needs the driver at run time.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libaxg.so")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                   "-diag-suppress", "607"]
CU_SOURCES = ["engine_fp32.cu", "engine_fp64.cu", "engine_mixed.cu", "noalloc.cu"]
CPP_SOURCES = ["capi.cpp", "operands.cpp"]


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = _sources() + [os.path.join(HERE, "..", "include", "axg.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def build(force=False, verbose=False):
    if not force and not _stale():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    for src in CU_SOURCES:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        jobs.append([NVCC] + CU_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj])
    for src in CPP_SOURCES:
        obj = os.path.join(BUILD, src.replace(".cpp", ".o"))
        jobs.append([NVCC] + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-x", "cu"] + ARCH +
                    ["-c", os.path.join(CSRC, src), "-o", obj])
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        for r in ex.map(_run, jobs):
            if verbose and r.stderr:
                sys.stderr.write(r.stderr)
    objs = [os.path.join(BUILD, s.replace(".cu", ".o")) for s in CU_SOURCES] + \
           [os.path.join(BUILD, s.replace(".cpp", ".o")) for s in CPP_SOURCES]
    tmp = OUT + ".tmp"
    _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build recipe for libsundog.so (sm_100a) — compiled in-tree so the shared
library travels with the repository.

CUDA translation units go through nvcc with -gencode arch=compute_100a,
code=sm_100a; host C++ through g++ with FP contraction off, so host-side scene
derivation and CDF builds round exactly like a plain IEEE build. Everything
links into sundog_b200/lib/libsundog.so against the static CUDA runtime.
"""

import os
import subprocess
import sys
import hashlib

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libsundog.so")
OBJ_DIR = os.path.join(HERE, "_build")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["pt_kernel.cu", "selftest.cu", "noalloc.cu", "guide.cu", "serve.cu", "wavefront.cu",
              "cdf_build.cu", "film_out.cu", "bvh_device.cu", "denoise.cu"]
CPP_SOURCES = ["scene_api.cpp", "scene_derive.cpp", "assets.cpp", "bvh_build.cpp",
               "render.cpp", "render_api.cpp", "serve_host.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                     "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-pthread", "-fvisibility=hidden", "-ffp-contract=off",
             "-Wall", "-Wno-unused-function", "-I" + os.path.join(CUDA_HOME, "include")]


def _sources():
    return [s for s in CU_SOURCES + CPP_SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _digest(path, extra):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        h.update(f.read())
    for e in extra:
        h.update(e.encode())
    return h.hexdigest()[:16]


def _headers_digest():
    h = hashlib.sha256()
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for name in sorted(os.listdir(d)):
            if name.endswith((".h", ".cuh")):
                with open(os.path.join(d, name), "rb") as f:
                    h.update(f.read())
    return h.hexdigest()[:16]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")
    return r.stdout


def build(verbose=False, force=False, defines=(), out=None):
    """Compile every translation unit (cached by content hash, in parallel)
    and link. `defines` adds -D flags to every unit; `out` overrides the
    output library path."""
    from concurrent.futures import ThreadPoolExecutor
    lib_path = out or LIB
    os.makedirs(os.path.dirname(lib_path), exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr = _headers_digest()
    objs, jobs = [], []
    for src in _sources():
        path = os.path.join(CSRC, src)
        is_cu = src.endswith(".cu")
        flags = (NVCC_FLAGS if is_cu else CXX_FLAGS) + ["-D" + d for d in defines]
        tag = _digest(path, flags + [hdr])
        obj = os.path.join(OBJ_DIR, "%s.%s.o" % (src, tag))
        if force or not os.path.exists(obj):
            if is_cu:
                jobs.append([NVCC] + flags + ["-c", path, "-o", obj])
            else:
                jobs.append(["g++"] + flags + ["-c", path, "-o", obj])
        objs.append(obj)
    if jobs:
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            for text in ex.map(lambda c: _run(c, verbose), jobs):
                if verbose and text.strip():
                    print(text)
    link = [NVCC] + ARCH + ["-shared", "-o", lib_path] + objs + ["-cudart", "static", "-lpthread",
                                                               "-lz", "-Xlinker",
                                                               "-soname=libsundog.so"]
    _run(link, verbose)
    return lib_path


# The same sources with the compressed 8-wide BVH (8-bit outward-rounded child
# boxes, SDB_WIDE_BVH) in place of the binary one: a second in-tree library
# with the identical ABI, loaded instead of the default through the
# SUNDOG_B200_LIB environment variable.
LIB_CW8 = os.path.join(OUT_DIR, "libsundog_cw8.so")


def build_all(verbose=False, force=False):
    """Both libraries: the default (binary BVH) and the 8-wide variant."""
    build(verbose=verbose, force=force)
    build(verbose=verbose, force=force, defines=("SDB_WIDE_BVH=1",), out=LIB_CW8)
    return LIB, LIB_CW8


if __name__ == "__main__":
    print(build_all(verbose="-v" in sys.argv, force="-f" in sys.argv))

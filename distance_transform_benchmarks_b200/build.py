"""Build recipes for the native libraries of the package (run by __graft_entry__.build()).

* ``libdtb.so``        -- the CUDA kernels and the C ABI of include/dtb.h, compiled for sm_100a only.
* ``libdtb_host.so``   -- host-only C++: the seeded synthetic workload generators.

The C++ ``namespace dt`` layer (include/dt/*.hpp) is header-only over libdtb.so.

Everything is built in-tree next to this file; nothing is installed.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx():
    # The system g++ (the image's $CXX wrapper lacks OpenMP).
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: %s" % " ".join(cmd[:3]))
    return r


def _deps(*names):
    files = [os.path.join(CSRC, n) for n in names]
    files += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".hpp"))]
    files += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    files.append(os.path.abspath(__file__))
    return files


def build_dtb(force=False, verbose=False, ptxas_verbose=False):
    out = os.path.join(HERE, "libdtb.so")
    srcs = ["dtb_api.cu", "dtb_plan.cu", "dtb_host_pipeline.cu", "dtb_serve.cu", "dtb_noalloc.cu", "dtb_io.cpp",
            "dtb_jpeg.cpp"]
    srcs = [s for s in srcs if os.path.exists(os.path.join(CSRC, s))]
    if force or _stale(out, _deps(*srcs)):
        cmd = [_nvcc()] + ARCH + NVCC_FLAGS + ["-I" + INCLUDE, "-I" + CSRC, "-shared", "-o", out]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        cmd += [os.path.join(CSRC, s) for s in srcs] + ["-lz"]  # zlib: PNG files (dtb_io.cpp)
        r = _run(cmd, verbose)
        if ptxas_verbose:
            sys.stdout.write(r.stderr)
    return out


def build_host(force=False, verbose=False):
    out = os.path.join(HERE, "libdtb_host.so")
    srcs = [s for s in ("datagen.cpp",) if os.path.exists(os.path.join(CSRC, s))]
    if not srcs:
        return None
    if force or _stale(out, _deps(*srcs)):
        cmd = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
               "-fvisibility=hidden", "-I" + INCLUDE, "-I" + CSRC, "-o", out]
        cmd += [os.path.join(CSRC, s) for s in srcs]
        _run(cmd, verbose)
    return out


def build_all(force=False, verbose=False):
    return [p for p in (build_dtb(force, verbose), build_host(force, verbose)) if p]


if __name__ == "__main__":
    force = "--force" in sys.argv
    build_dtb(force=force, verbose=True, ptxas_verbose="-v" in sys.argv)
    build_host(force=force, verbose=True)

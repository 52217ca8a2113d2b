"""Build libnui_b200.so (the C-ABI library) in-tree for sm_100a.

    python -m natureuserinterfacestudio_b200.build        (or build() from Python)

Every CUDA source is compiled with nvcc for arch=compute_100a,code=sm_100a, with
--fmad=false (no contraction: the kernels reproduce the reference's float arithmetic
bit for bit) and -lineinfo; host sources with the same nvcc driver.  The tolerance-mode
kernels of the FP16 serving formats (*_fast.cu) are compiled with contraction on.  Objects go to
natureuserinterfacestudio_b200/_build/, the library next to this file.

The synthetic-input generator of the tests and the benchmark (synth/nui_synth.cpp) is a
separate host library, libnui_synth.so, so that generating input never loads the product
library.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnui_b200.so")
SYNTH_SRC = os.path.join(HERE, "synth", "nui_synth.cpp")
SYNTH_LIB = os.path.join(HERE, "libnui_synth.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-fvisibility=hidden",
          "-I", INCLUDE, "-I", CSRC]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(nvcc, src, verbose):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    deps.append(os.path.join(INCLUDE, "nui_b200.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj, ""
    flags = COMMON
    if src.endswith("_fast.cu"):  # tolerance-mode kernels: contraction allowed
        flags = [f if f != "--fmad=false" else "--fmad=true" for f in COMMON]
    cmd = [nvcc] + ARCH + flags + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc] + COMMON + ["-x", "c++", "-c", path, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj, r.stderr


def build_synth():
    """libnui_synth.so: the seeded scenes, trajectories and Kinect-like renderer."""
    deps = [SYNTH_SRC, os.path.join(HERE, "synth", "nui_synth.h")]
    if os.path.exists(SYNTH_LIB) and os.path.getmtime(SYNTH_LIB) >= max(os.path.getmtime(d) for d in deps):
        return SYNTH_LIB
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-fvisibility=hidden", "-shared", SYNTH_SRC, "-o",
           SYNTH_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("synth build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return SYNTH_LIB


def build(verbose=False):
    build_synth()
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(nvcc, s, verbose), sources()))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc] + ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-o", LIB] + objs + ["-lgomp", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

"""Build oracle/_ref/libnui_ref.so from the reference's own OpenCL kernel sources.

Test infrastructure.  The reference's hot-path kernels (src/Kernels/*.cl of
hustztz/NatureUserInterfaceStudio) are read from the read-only reference tree, rewritten
mechanically into C++ that compiles against ref_shim/clshim.hpp, and compiled together
with the launchers in ref_shim/launch_*.inc into one shared library.  The rewritten
sources go to a temporary directory and are deleted after the build; only the .so is
kept (oracle/_ref is git-ignored).  The library runs the reference kernels on the host
cores and is used to pin the oracle restatement (tests/test_oracle_*pins.py).

Rewrites (each purely syntactic):
  * `(float3)(a, b, c)` vector literals      -> `float3(a, b, c)`
  * multi-component swizzles `.xy`, `.s012`  -> `.swz<0,1>()`, `.swz<0,1,2>()`
  * `__local T name[N];` inside a kernel      -> `static thread_local T name[N];`
  * `__attribute__((reqd_work_group_size(..)))` and `#pragma OPENCL` lines removed
  * implicit-int declarations `const idx =` (extract.cl) -> `const int idx =`

Usage:  python oracle/build_ref.py [--reference TREE]
        (TREE defaults to $NUI_REFERENCE_TREE, else /root/reference)
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "ref_shim")
OUT_DIR = os.path.join(HERE, "_ref")

# kernel file -> launcher include compiled in the same translation unit
UNITS = {
    "filters.cl": "launch_filters.inc",
    "bilateralFilter.cl": "launch_bilateral.inc",
    "transformMaps.cl": "launch_transform.inc",
    # only the simple-normals kernel: the rest of the file (covariance normals, unused by
    # the hot path) needs sincos/shuffle/swizzle stores that the shim does not provide
    "normalEstimation.cl": ("launch_normals.inc", ["estimate_normals_simple_kernel"]),
    "tsdfVolume.cl": "launch_tsdf.inc",
    "raycast.cl": "launch_raycast.inc",
    "marchingCube.cl": "launch_mc.inc",
    "icp.cl": "launch_icp.inc",
    "colorIcp.cl": "launch_color_icp.inc",
    "KinfuHashScene.cl": "launch_hash_scene.inc",
    "KinfuHashRaycast.cl": "launch_hash_raycast.inc",
    "KinfuHashVisualization.cl": "launch_hash_mesh.inc",
    "extract.cl": "launch_extract.inc",
    # the global cache's kernels (the swap-in prefix-scan kernels, replaced by the host
    # compaction of the launcher, are left out)
    "KinfuHashSwapping.cl": ("launch_hash_swap.inc", ["reAllocateSwappedOutVoxelBlocks_kernel",
                                                      "integrateOldIntoActiveData_kernel", "buildSwapOutList_kernel",
                                                      "moveActiveDataToTransferBuffer_kernel",
                                                      "cleanVoxelMemory_kernel"]),
}
# The reference fixes its hash table sizes at compile time (hashing_gpu_def.h:9-20:
# 0x150000 buckets, 0x30000 excess entries, 2^20 voxel blocks = 3.2 GB of voxels).  The
# host build uses small tables of the same structure so that tests can run it; only
# these constants change.
HASH_TEST_SIZES = {"SDF_BUCKET_NUM": "0x10000", "SDF_HASH_MASK": "0xffff", "SDF_EXCESS_LIST_SIZE": "0x4000",
                   "SDF_LOCAL_BLOCK_NUM": "0x8000"}
# every file the units include
INCLUDED = ["utils.cl", "gpu_def.h", "cameraUtils.cl", "hashing_gpu_def.h", "KinfuHashUtils.cl",
            "prefixSum.cl"]

VEC_T = r"(?:u?char|u?short|u?int|u?long|float|double)(?:2|3|4|8|16)"
SWZ_XYZW = {"x": 0, "y": 1, "z": 2, "w": 3}


def swizzle_indices(name):
    if name.startswith("s") and len(name) > 2 and all(c in "0123456789" for c in name[1:]):
        return [int(c, 16) for c in name[1:]]
    if 2 <= len(name) <= 4 and all(c in SWZ_XYZW for c in name):
        return [SWZ_XYZW[c] for c in name]
    return None


def rewrite(src):
    src = re.sub(r"^\s*#pragma\s+OPENCL.*$", "", src, flags=re.M)
    src = re.sub(r"__attribute__\s*\(\(\s*reqd_work_group_size\s*\([^)]*\)\s*\)\)", "", src)
    src = re.sub(r"\(\s*(%s)\s*\)\s*\(" % VEC_T, r"\1(", src)
    src = re.sub(r"\bconst\s+idx\s*=", "const int idx =", src)

    def swz(m):
        idx = swizzle_indices(m.group(1))
        if idx is None:
            return m.group(0)
        return ".swz<%s>()" % ",".join(str(i) for i in idx)

    src = re.sub(r"\.([A-Za-z][A-Za-z0-9]*)\b(?!\s*\()", swz, src)
    # __local declarations at statement start inside function bodies (not parameters)
    src = re.sub(r"(^|[;{]\s*)__local(\s+(?:volatile\s+)?\w+\s+\w+\s*\[)", r"\1static thread_local\2",
                 src, flags=re.M)
    return src


def extract(src, names):
    """Keep the #include lines and the named top-level functions of a kernel file."""
    keep = [l for l in src.splitlines() if l.strip().startswith("#include")]
    for name in names:
        m = re.search(r"__kernel\s+void\s+%s\s*\(" % name, src)
        if not m:
            raise ValueError("kernel %s not found" % name)
        i = src.index("{", m.end())
        depth = 0
        for j in range(i, len(src)):
            if src[j] == "{":
                depth += 1
            elif src[j] == "}":
                depth -= 1
                if depth == 0:
                    break
        keep.append(src[m.start():j + 1])
    return "\n".join(keep) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("NUI_REFERENCE_TREE", "/root/reference"))
    ap.add_argument("--cxx", default="g++")
    args = ap.parse_args()
    kdir = os.path.join(args.reference, "src", "Kernels")
    mc_header_dir = os.path.join(args.reference, "src", "SLAM", "VisualOdometry", "DeviceSpecific", "OpenCL")
    if not os.path.isdir(kdir):
        print("reference kernels not found at %s; oracle/_ref not built" % kdir)
        return 1
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="nui_ref_")
    try:
        for f in list(UNITS) + INCLUDED:
            with open(os.path.join(kdir, f)) as fh:
                text = fh.read()
            spec = UNITS.get(f)
            if isinstance(spec, tuple):
                text = extract(text, spec[1])
            if f == "hashing_gpu_def.h":
                for k, v in HASH_TEST_SIZES.items():
                    text = re.sub(r"(#define\s+%s\s+)\S+" % k, r"\g<1>" + v, text)
            with open(os.path.join(tmp, f), "w") as fh:
                fh.write(rewrite(text))
        objs = []
        for cl, spec in UNITS.items():
            launcher = spec[0] if isinstance(spec, tuple) else spec
            ns = "refk_" + os.path.splitext(cl)[0]
            unit = os.path.join(tmp, ns + ".cpp")
            with open(unit, "w") as fh:
                fh.write('#include "clshim.hpp"\n#include <cstdint>\n')
                fh.write("namespace %s {\nusing namespace clshim;\n#include \"%s\"\n}  // namespace %s\n" % (ns, cl, ns))
                fh.write("#define REF_NS %s\n#include \"%s\"\n" % (ns, launcher))
            objs.append(unit)
        objs.append(os.path.join(SHIM, "clshim_rt.cpp"))
        out = os.path.join(OUT_DIR, "libnui_ref.so")
        cmd = [args.cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-fno-fast-math", "-w", "-I", tmp, "-I", SHIM, "-I", mc_header_dir, "-o", out] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr[-20000:])
            return r.returncode
        print("built", out)
        return 0
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    sys.exit(main())

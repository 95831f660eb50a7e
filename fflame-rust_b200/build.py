"""Build the C-ABI library of the B200 fractal-flame path in-tree.

    python fflame-rust_b200/build.py

Compiles csrc/ with nvcc for sm_100a into ffb200/libffb200.so.  The
chaos-game kernels themselves are compiled per flame structure at run time
by NVRTC from the device sources embedded here (ffb_device_src.inc).
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "ffb200", "libffb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["ffb_tail.cu", "ffb_diff_tail.cu", "ffb_tiles.cu", "ffb_runtime.cpp", "ffb_flame.cpp", "ffb_codegen.cpp",
           "ffb_png.cpp", "ffb_flame_xml.cpp"]
HEADERS = ["ffb_json.hpp", "ffb_flame.hpp", "ffb_codegen.hpp", "ffb_tail.cuh", "ffb_device.cuh", "ffb_kernels.cuh",
           "ffb_diff_jac.cuh", "ffb_diff.cuh", "ffb_png.hpp", "ffb_flame_xml.hpp"]


def embed():
    """Device sources as raw string literals for NVRTC."""
    parts = []
    for name, var in (("ffb_device.cuh", "kDeviceSrc"), ("ffb_kernels.cuh", "kKernelsSrc"),
                      ("ffb_diff_jac.cuh", "kDiffJacSrc"), ("ffb_diff.cuh", "kDiffSrc")):
        with open(os.path.join(CSRC, name), encoding="utf-8") as f:
            text = f.read()
        assert ")FFBSRC\"" not in text
        parts.append(f'extern const char* const {var} = R"FFBSRC(\n{text})FFBSRC";\n')
    body = ("// generated by build.py from the device sources (ffb_device.cuh, ffb_kernels.cuh, ffb_diff*.cuh)\nnamespace ffb {\n"
            + "".join(parts) + "}  // namespace ffb\n")
    path = os.path.join(CSRC, "ffb_device_src.inc")
    old = open(path, encoding="utf-8").read() if os.path.exists(path) else None
    if old != body:
        with open(path, "w", encoding="utf-8") as f:
            f.write(body)


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = SOURCES + HEADERS + ["ffb_device_src.inc", "../../include/ffb200.h", "../build.py"]
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in deps)


def build(force=False, verbose=False):
    embed()
    if not force and not stale():
        return OUT
    cmd = [NVCC, "-O3", "-std=c++17", "-shared", "-lineinfo",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
           "-I", os.path.join(HERE, "..", "include"),
           "-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lnvrtc", "-lz"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build recipe of the CUDA library: nvcc for sm_100a, output in-tree.

    python virial-engine_b200/build.py            # builds virial_lj/libvirial_lj.so
    python virial-engine_b200/build.py --verbose  # also prints ptxas register use

`build(defines=..., out=...)` compiles a variant with preprocessor overrides
(the tuning knobs in csrc/vlj_internal.cuh) into another file; tune.py uses it.
"""

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "virial_lj", "libvirial_lj.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-shared", "--cudart", "static",
    "-I", os.path.join(ROOT, "include"), "-I", CSRC,
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def needs_build(out=OUT):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(ROOT, "include", "virial_lj.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(verbose=False, force=False, defines=None, out=OUT):
    if not force and not needs_build(out):
        return out
    macros = [f"-D{k}={v}" for k, v in sorted((defines or {}).items())]
    cmd = [NVCC] + FLAGS + macros + (["-Xptxas", "-v"] if verbose else []) + sources() \
        + ["-o", out + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(OUT)

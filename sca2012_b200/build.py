"""Builds the in-tree CUDA library (sm_100a) and the CPU oracle.

    python -m sca2012_b200.build

The CUDA library is compiled by nvcc straight from csrc/ into
sca2012_b200/libsca2012_b200.so (so it travels with the source tree);
no torch extension cache is involved.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsca2012_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["sph_api.cu", "sph_config.cpp", "sph_noalloc.cu", "sph_pov.cpp"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "sph", "sph.h")]
    if not force and not _newer(LIB, deps):
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


def build_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def build_reference_oracle(ref=None):
    """Compiles the reference itself into oracle/_ref when its source tree is
    given (`ref`, else the SCA2012_REFERENCE environment variable) and the
    libraries are not built yet."""
    ref = ref or os.environ.get("SCA2012_REFERENCE", "")
    script = os.path.join(ROOT, "oracle", "build_ref.sh")
    have = all(os.path.exists(os.path.join(ROOT, "oracle", "_ref", f"libref_{v}_gpu.so"))
               for v in ("2d", "3d2", "3d4"))
    if ref and os.path.isdir(ref) and not have:
        subprocess.run(["bash", script, ref], check=True)


def main():
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_oracle()
    build_reference_oracle()


if __name__ == "__main__":
    main()

"""Build recipe for the in-tree shared library cress_b200/_lib/libcress_b200.so.

Compiles every CUDA source under cress_b200/csrc for sm_100a with nvcc and
links them into one C-ABI shared library (declared in include/cress_b200.h).
The library goes next to the package so it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libcress_b200.so")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "--compiler-options", "-fPIC -ffp-contract=off",
    "-Xptxas", "-v",
]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def newest_input_mtime():
    paths = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                         if f.endswith((".h", ".cuh"))]
    paths.append(os.path.join(os.path.dirname(HERE), "include", "cress_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it.  Returns its path."""
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_input_mtime():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    tmp = LIB + ".tmp"
    cmd = [nvcc] + NVCC_FLAGS + ["-shared", "-o", tmp] + sources()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libcress_b200.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

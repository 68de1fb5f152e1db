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


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    paths.append(os.path.join(os.path.dirname(HERE), "include", "cress_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it.  Returns its path.

    Each .cu is compiled to its own object (in parallel; an object is
    rebuilt when its source or any header is newer) and the objects are
    linked into one shared library: the same as one nvcc call over all
    sources, since no device code crosses translation units."""
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_input_mtime():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    hdr = _headers_mtime()

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        if (not force and os.path.exists(obj) and
                os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr)):
            return obj, None
        cmd = [nvcc] + NVCC_FLAGS + ["-c", "-o", obj + ".tmp", src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(obj + ".tmp", obj)
        return obj, r

    jobs = int(os.environ.get("CRESS_BUILD_JOBS", str(min(8, os.cpu_count() or 1))))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(compile_one, sources()))
    failed = False
    for obj, r in results:
        if r is None:
            continue
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        failed |= r.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed building libcress_b200.so")
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + \
        [o for o, _ in results]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed linking libcress_b200.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

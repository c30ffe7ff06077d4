"""Build libsu2g.so (CUDA C++ for sm_100a) in-tree with nvcc.

The library has a plain C ABI (include/su2g.h) and links the CUDA runtime statically, so
nothing of PyTorch is involved.  The output lands in masterarbeit_b200/_lib/, next to the
sources, so that it travels with the repository snapshot.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libsu2g.so")
DRIVERS = ("su2meas", "su2qcd")   # native drivers, driver/<name>.cpp -> _lib/<name>

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
    "-shared", "-cudart", "static", "--expt-relaxed-constexpr",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libsu2g.so")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", "su2g.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    """Compile every .cu under csrc/ into one shared library; returns its path."""
    if not force and not _stale():
        build_driver()
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [_nvcc()] + ARCH + NVCC_FLAGS + ["-I", CSRC, "-I", os.path.join(REPO, "include")]
    cmd += list(extra) + sources() + ["-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose and res.stderr:
        print(res.stderr, file=sys.stderr)
    os.replace(tmp, LIB)
    build_driver(force=True)
    return LIB


def build_driver(force=False):
    """The native drivers (host C++ over the C ABI), next to the library."""
    cxx = shutil.which("g++") or "g++"
    for name in DRIVERS:
        src, out = os.path.join(PKG, "driver", name + ".cpp"), os.path.join(LIBDIR, name)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src),
                                                                               os.path.getmtime(LIB)):
            continue
        cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(REPO, "include"), src, "-L", LIBDIR, "-lsu2g",
               "-Wl,-rpath,$ORIGIN", "-o", out + ".tmp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"building {name} failed:\n" + res.stdout + res.stderr)
        os.replace(out + ".tmp", out)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"]))

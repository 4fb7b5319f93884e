"""Build recipe of the CUDA library: every .cu in csrc/ -> cupythia_b200/libcupythia_b200.so (sm_100a).

Run as ``python -m cupythia_b200.build`` or through ``__graft_entry__.build()``.  nvcc
cross-compiles without a GPU, so the library builds on CPU-only machines too.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcupythia_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


BIN = os.path.join(HERE, "bin")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
DRIVERS = ["fused_gg2gg", "vegas", "pdf_xsec", "cub_compaction", "unweight_lhe", "generate"]


def deps():
    return sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(
        os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in deps())


def build(force=False, verbose=False, ptxas_v=False):
    if not force and up_to_date():
        return LIB
    cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_v else []) + sources() + [
        "-o", LIB, "-lcuda"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcupythia_b200.so")
    if ptxas_v or verbose:
        sys.stdout.write(r.stdout + r.stderr)
    return LIB


def build_drivers(force=False, verbose=False):
    """Stage drivers (drivers/*.cc, C++ over the C ABI) -> bin/<name>, linked to the library."""
    build(force=False)
    os.makedirs(BIN, exist_ok=True)
    hdr = [os.path.join(HERE, "drivers", "drv.h"), os.path.join(ROOT, "include", "cupythia_b200.h")]
    out = []
    for name in DRIVERS:
        src = os.path.join(HERE, "drivers", name + ".cc")
        exe = os.path.join(BIN, name)
        out.append(exe)
        if not force and os.path.exists(exe) and all(
                os.path.getmtime(f) <= os.path.getmtime(exe) for f in [src, LIB] + hdr):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", src, "-I" + os.path.join(CUDA_HOME, "include"),
               "-L" + HERE, "-lcupythia_b200", "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart",
               "-Wl,-rpath,$ORIGIN/..", "-o", exe]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"g++ failed building the stage driver {name}")
    return out


if __name__ == "__main__":
    build(force=True, verbose=True, ptxas_v="-v" in sys.argv)
    build_drivers(force=True, verbose=True)

"""Build libprovekit_b200.so in-tree with nvcc for sm_100a.

    python -m provekit_b200.build [--force] [--verbose]

The library has a plain C ABI (include/provekit_b200.h); Python binds it with
ctypes, so no torch extension machinery is involved.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libprovekit_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(CSRC, "*.h")) + [
        os.path.join(ROOT, "include", "provekit_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def _compile(src: str, obj: str, verbose: bool) -> None:
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
           "-I", os.path.join(ROOT, "include"), "-o", obj, src]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit to an object in parallel (each is
    self-contained: no device code crosses files), then link the shared
    library."""
    import concurrent.futures as cf

    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(objdir, os.path.basename(c)[:-3] + ".o") for c in srcs]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 4))) as ex:
        for f in [ex.submit(_compile, c, o, verbose) for c, o in zip(srcs, objs)]:
            f.result()
    subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))

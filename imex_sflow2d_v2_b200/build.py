"""Build libimexgpu.so (exact mode) and libimexgpu_fast.so (contracted
multiply-adds) for sm_100a (nvcc; no GPU needed)."""
import os
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(_HERE, "csrc")
LIB = os.path.join(_HERE, "libimexgpu.so")
LIB_FAST = os.path.join(_HERE, "libimexgpu_fast.so")


def sources():
    return [os.path.join(CSRC, f) for f in ("imex_gpu.cu", "imex_batch.cu", "imex_kernels.cuh",
                                             "imex_batch.cuh", "imex_batch_api.h", "imex_mlp.cuh",
                                             "imex_device.cuh", "imex_setup.cuh", "imex_output.cuh",
                                             "imex_fortran_fmt.h",
                                             "ipow_tables.h")] + [
        os.path.join(_HERE, "..", "include", "imex_gpu.h")]


def needs_build():
    for lib in (LIB, LIB_FAST):
        if not os.path.exists(lib):
            return True
        t = os.path.getmtime(lib)
        if any(os.path.getmtime(s) > t for s in sources()):
            return True
    return False


def build(force=False, verbose=False):
    if force or needs_build():
        cmd = ["make", "-j4", "-C", CSRC, "NVCC=/usr/local/cuda/bin/nvcc", "all"]
        if force:
            cmd.insert(1, "-B")
        out = subprocess.run(cmd, capture_output=not verbose, text=True)
        if out.returncode != 0:
            sys.stderr.write((out.stdout or "") + (out.stderr or ""))
            raise RuntimeError("nvcc build of libimexgpu.so failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

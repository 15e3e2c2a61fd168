"""Build the sm_100a extension in-tree: ``python -m pyclaw_b200.build``.

The CUDA sources under ``csrc/`` compile into ``lib/libclaw2.so`` (plain C ABI,
declared in ``include/claw2.h``), with the CUDA runtime linked statically so the
library only needs the driver at run time.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libclaw2.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
# the sources compile side by side, then link.  (nvcc's parallel
# split-compile of one source cut the build by half but made the headline
# kernel 1% slower, so the device code is optimised whole)
SOURCES = ["claw2.cu", "claw2_noalloc.cu", "frame_io.cpp"]
OBJDIR = os.path.join(HERE, "lib", "_build")


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pyclaw_b200")
    return exe


def _deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(d, f))
    return out


def build(force=False, verbose=False):
    """Compile lib/libclaw2.so if any source is newer (or ``force``)."""
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(f) <= t for f in _deps()):
            return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, src + ".o")
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
            ["-c", "-o", obj, os.path.join(CSRC, src)]
        jobs.append((obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    logs, failed = [], False
    for obj, proc in jobs:
        out, _ = proc.communicate()
        logs.append(out)
        failed = failed or proc.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed:\n" + "".join(logs))
    link = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB + ".tmp"] + [o for o, _ in jobs]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stdout.write("".join(logs) + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

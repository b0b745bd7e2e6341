"""Builds the sm_100a shared library libsimcraft_fluid.so in-tree with nvcc.

Usage: python -m simcraft_b200.build [--force] [-v]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsimcraft_fluid.so")
OBJDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The particle/grid transfers, the finite-volume build, the mesh SDF and the surface export restate
# the CPU arithmetic operation by operation: no fused multiply-add contraction there.
EXTRA = {"sc_flip.cu": ["--fmad=false"], "sc_fvm.cu": ["--fmad=false"], "sc_diff.cu": ["--fmad=false"],
         "sc_mesh.cu": ["--fmad=false"], "sc_surface.cu": ["--fmad=false"]}


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(os.path.dirname(HERE), "include", "simcraft_fluid_capi.h"))
    files.append(os.path.abspath(__file__))
    return [f for f in files if os.path.isfile(f)]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(force=False, verbose=False):
    if not force and os.path.exists(LIB):
        lt = os.path.getmtime(LIB)
        if all(os.path.getmtime(f) <= lt for f in _deps()):
            return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    flags = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
             "-ccbin", "g++"] + ARCH
    if verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [nvcc()] + flags + EXTRA.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            sys.stderr.write("FAILED: " + " ".join(cmd) + "\n")
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc(), "-shared", "-o", tmp] + ARCH + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

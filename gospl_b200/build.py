"""Build libgospl_b200.so in-tree with nvcc for sm_100a.

All kernels are compiled with ``--fmad=false`` so that every floating-point
expression rounds operation by operation, as the reference's x86-64 build
does (no fused multiply-add contraction), which keeps the device results
bit-comparable with the CPU oracle.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgospl_b200.so")
SOURCES = ["gs_capi.cu", "gs_plan.cu", "gs_receivers.cu", "gs_sweep.cu", "gs_pitfill.cu", "gs_flow.cu",
           "gs_spl.cu", "gs_diffusion.cu", "gs_force.cu", "gs_mesh.cu", "gs_noalloc.cu", "gs_adjoint.cu",
           "gs_sed.cu", "gs_output.cu", "gs_marine.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-I" + os.path.join(ROOT, "include")]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "gospl_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [NVCC] + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, pr in procs:
        out = pr.communicate()[0].decode()
        if pr.returncode != 0 or verbose:
            sys.stderr.write(out)
        if pr.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for %s" % failed)
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xlinker",
                           "--no-undefined", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

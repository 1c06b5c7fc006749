"""Build libchapsim_gpu.so in-tree for sm_100a (nvcc, no JIT cache)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchapsim_gpu.so")
SOURCES = ["chs_plan.cpp", "chs_kernels.cu", "chs_stencil_f64.cu", "chs_stencil_f32.cu", "chs_solver.cu",
           "chs_static.cu", "chs_mlp.cu", "chs_fused.cu"]
OBJDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _host_cxx():
    for c in ("/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(c):
            return c
    return "g++"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "chapsim_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False, extra=()):
    """Compile the sources (in parallel, one object each) and link chapsim2_b200/libchapsim_gpu.so."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJDIR, exist_ok=True)
    common = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O2", *extra]

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        cmd = [*common, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "--shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, extra=[a for a in sys.argv[1:] if a != "--force"])

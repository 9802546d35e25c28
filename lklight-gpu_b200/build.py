"""Builds liblkg.so (all CUDA sources for sm_100a, host C++) in-tree.

nvcc -gencode arch=compute_100a,code=sm_100a; the f64 exact-path kernels and
the far-field builder are compiled with --fmad=false so their f64 arithmetic
follows the reference's operation order.  The CUDA runtime is linked
statically, so the library needs only the CUDA driver at run time.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_objs")
LIB = os.path.join(HERE, "lib", "liblkg.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fopenmp", "-I" + INCLUDE]
NO_FMAD = {"lkg_kernels_exact.cu", "lkg_field.cu", "lkg_gso_dev.cu"}
HEADERS = ["lkg_internal.h", "lkg_runtime.h", "lkg_score.cuh", "lkg_score_warp.cuh", "lkg_rng.h", "lkg_gso_dev.h"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src):
    obj = os.path.join(OBJ, src + ".o")
    cmd = [_nvcc()] + ARCH + NVCC_FLAGS
    if src in NO_FMAD:
        cmd.append("--fmad=false")
    cmd += ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "lkg.h")]
    todo = [s for s in sources()
            if force or _stale(os.path.join(OBJ, s + ".o"), [os.path.join(CSRC, s)] + hdrs)]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for obj in ex.map(_compile, todo):
            if verbose:
                print("compiled", obj)
    objs = [os.path.join(OBJ, s + ".o") for s in sources()]
    if force or todo or _stale(LIB, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

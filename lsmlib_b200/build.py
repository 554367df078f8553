"""Build liblsmgpu.so (sm_100a) in-tree with nvcc.

Usage: python -m lsmlib_b200.build [--force]

Each .cu file of csrc/ compiles to an object under lsmlib_b200/_build/ with
its own floating-point flags: the drop-in toolbox kernels and the "strict"
fused stages are built with --fmad=false (reference expression order, no FMA
contraction), the "fast" fused stages with FMA enabled.  The objects link into
lsmlib_b200/liblsmgpu.so with the CUDA runtime linked statically.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblsmgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                 "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
                 "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]

# source -> extra flags
SOURCES = {
    "toolbox_kernels.cu": ["--fmad=false"],
    "toolbox_extra.cu": ["--fmad=false"],
    "capi.cu": ["--fmad=false"],
    "stage_strict.cu": ["--fmad=false"],
    "stage_fast.cu": ["--fmad=true"],
    "integrator.cu": ["--fmad=false"],
    "batched.cu": ["--fmad=true"],
    "adjoint.cu": ["--fmad=true"],
    "noalloc.cu": ["--fmad=false"],
    "distance.cu": ["--fmad=false"],
}


def _obj(src):
    return os.path.join(BUILD, src.replace(".cu", ".o"))


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(INCLUDE, "lsmgpu", "lsmgpu.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def compile_one(src, flags, force):
    obj = _obj(src)
    if not force and not _stale(obj, _deps()):
        return obj, ""
    cmd = [NVCC] + COMMON + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd),
                                                           r.stdout + r.stderr))
    return obj, r.stdout + r.stderr


def build(force=False, verbose=False):
    """Compile every CUDA source for sm_100a and link liblsmgpu.so."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = [ex.submit(compile_one, s, SOURCES[s], force) for s in srcs]
        objs = []
        for f in futs:
            obj, log = f.result()
            objs.append(obj)
            if verbose and log.strip():
                print(log)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s" % (r.stdout + r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

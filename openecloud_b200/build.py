"""Build liboec.so (all CUDA kernels + host C++ of the package) for sm_100a.

``python -m openecloud_b200.build`` compiles every ``csrc/*.cu`` and
``csrc/*.cpp`` with nvcc into ``openecloud_b200/liboec.so`` (in-tree, so the
shared object travels with the source tree).  Objects are rebuilt only when a
source or header is newer than the object.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build", "liboec")
LIB = os.path.join(PKG, "liboec.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]
CPP_FLAGS = COMMON + ["-x", "c++"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _compile(src, extra=()):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC] + CU_FLAGS + list(extra) + ["-c", src, "-o", obj]
    else:
        cmd = [NVCC] + CPP_FLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, force=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = _headers()
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    todo = [s for s in srcs if force or ptxas_info or
            _stale(os.path.join(BUILD, os.path.basename(s) + ".o"), s, deps)]
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    if todo:
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj, err in ex.map(lambda s: _compile(s, extra), todo):
                if verbose and err:
                    print(err, file=sys.stderr)
    if force or todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv))

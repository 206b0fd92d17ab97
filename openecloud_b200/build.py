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
# the bounds-checked build: every guarded grid/particle index is checked and
# an out-of-range one counted and skipped (oec_bound_violations)
BUILD_CHECKED = os.path.join(ROOT, "_build", "liboec_checked")
LIB_CHECKED = os.path.join(PKG, "liboec_checked.so")

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


def _compile(src, extra=(), build_dir=BUILD):
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC] + CU_FLAGS + list(extra) + ["-c", src, "-o", obj]
    else:
        cmd = [NVCC] + CPP_FLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, force=False, ptxas_info=False, bounds_check=False):
    """Compiles the stale objects and links the library (liboec.so, or
    liboec_checked.so with bounds_check)."""
    build_dir, lib = (BUILD_CHECKED, LIB_CHECKED) if bounds_check else (BUILD, LIB)
    os.makedirs(build_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = _headers()
    extra = (["-Xptxas", "-v"] if ptxas_info else []) + (["-DOEC_BOUNDS_CHECK"] if bounds_check else [])
    todo = [s for s in srcs if force or ptxas_info or
            _stale(os.path.join(build_dir, os.path.basename(s) + ".o"), s, deps)]
    objs = [os.path.join(build_dir, os.path.basename(s) + ".o") for s in srcs]
    if todo:
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj, err in ex.map(lambda s: _compile(s, extra, build_dir), todo):
                if verbose and err:
                    print(err, file=sys.stderr)
    if force or todo or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib + ".tmp"] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv,
                bounds_check="--bounds-check" in sys.argv))

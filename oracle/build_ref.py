"""Compile the openECLOUD reference Cython modules into ``oracle/_ref``.

TEST INFRASTRUCTURE ONLY.  The compiled reference is used (a) to generate the
golden fixtures under ``tests/golden`` and (b) as the timed CPU baseline
("reference" arm of ``bench.py``).  Nothing in ``openecloud_b200`` imports it.

Recipe (the reference's own ``setup.py`` is not used):

1. copy the reference ``*.pyx``/``*.pxd``/``beam.py`` from the read-only tree
   into ``oracle/_ref/src`` (build scratch, git-ignored);
2. apply the minimal patches the modern toolchain needs:

   * ``poissonSolver.pyx:45``: ``spsp.eye(np, np, -nx)`` with ``nx`` typed
     ``unsigned int`` wraps to a huge positive offset; current SciPy raises.
     The offset is cast to a signed int, the evident intent.
   * ``particleEmitter.pyx`` (``FurmanEmitter``): the cdef attribute ``eHat0``
     (copperMod, :139) cannot be set from Python; a setter ``setEHat0`` is
     appended so the E_max=300 eV configuration can be expressed.
   * ``grid.pyx:7`` imports matplotlib (absent): a stub package is written.

3. cythonize with ``language_level=2`` (the sources are Python-2 Cython with
   ``print`` statements) and ``cpow=True`` (C semantics of ``**``), compile
   with ``-O3`` and link ``randomGen``/``specFun`` against the project-written
   GSL stand-in ``oracle/gsl_shim/oec_gsl_shim.c``;
4. compile the project-written probe ``oracle/ref_probe.pyx`` against the
   reference's .pxd files: it exposes the reference's cdef special functions
   and random-number wrappers to Python for golden-vector generation.

Usage: ``python oracle/build_ref.py [--src /path/to/reference]``.
"""
import argparse
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM_DIR = os.path.join(HERE, "gsl_shim")
# Where this build environment mounts the reference tree (read-only); the
# OEC_REFERENCE environment variable or --src names another one.
MOUNTED_SRC = "/root/reference"


def locate():
    """The reference source tree to build from, or None when it is absent
    (the GPU hosts carry only the built modules)."""
    src = os.environ.get("OEC_REFERENCE", MOUNTED_SRC)
    return src if os.path.isdir(src) else None

MODULES = ["constants", "randomGen", "specFun", "grid", "particles", "particleBoundary",
           "kdTree", "particleManagement", "particleEmitter", "poissonSolver", "magneticField", "util",
           "ref_probe"]
GSL_MODULES = {"randomGen", "specFun"}


def _patch(path, old, new, count=1):
    with open(path) as f:
        text = f.read()
    if old not in text:
        raise RuntimeError(f"patch anchor not found in {path}: {old!r}")
    text = text.replace(old, new, count)
    with open(path, "w") as f:
        f.write(text)


def prepare_sources(src):
    dst = os.path.join(OUT, "src")
    os.makedirs(dst, exist_ok=True)
    for name in os.listdir(src):
        if name.endswith((".pyx", ".pxd")) or name == "beam.py":
            shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))
    # Q1: signed offset for the y-derivative operator.
    _patch(os.path.join(dst, "poissonSolver.pyx"),
           "pymt = spsp.identity(np)-spsp.eye(np,np,-nx)",
           "pymt = spsp.identity(np)-spsp.eye(np,np,-(<int> nx))")
    # Setter for the copper E_max parameter.
    pe = os.path.join(dst, "particleEmitter.pyx")
    _patch(pe, "    def getEmittedParticles(self):\n        return self.secondaries",
           "    def getEmittedParticles(self):\n        return self.secondaries\n\n"
           "    def setEHat0(self, double value):\n        self.eHat0 = value\n")
    # SecElecEmitter / SimpleSecEmitter size their output by a double
    # (nSecSum), which numpy >= 1.12 rejects: cast it to an integer.
    _patch(pe, "numpy.empty((nSecSum, nCoords)", "numpy.empty((<Py_ssize_t> nSecSum, nCoords)", count=2)
    # matplotlib stub (grid.pyx imports pyplot at module import time).
    mpl = os.path.join(OUT, "matplotlib")
    os.makedirs(mpl, exist_ok=True)
    with open(os.path.join(mpl, "__init__.py"), "w") as f:
        f.write('"""Headless stub: the oracle build never plots."""\n')
    with open(os.path.join(mpl, "pyplot.py"), "w") as f:
        f.write('"""Headless stub for grid.pyx\'s unused import."""\n')
    # beam.py uses long-removed scipy aliases; the compat module maps them.
    shutil.copyfile(os.path.join(dst, "beam.py"), os.path.join(OUT, "beam.py"))
    with open(os.path.join(OUT, "ref_compat.py"), "w") as f:
        f.write(
            '"""Map removed scipy aliases used by the reference beam.py onto numpy."""\n'
            "import numpy, scipy\n"
            "for _n in ('zeros', 'tile', 'reshape', 'clip', 'sum', 'mod'):\n"
            "    if not hasattr(scipy, _n):\n"
            "        setattr(scipy, _n, getattr(numpy, _n))\n")
    return dst


def build(src):
    if not os.path.isdir(src):
        raise SystemExit(f"reference sources not found at {src}")
    import numpy
    from Cython.Build import cythonize
    from setuptools import Extension
    from setuptools.dist import Distribution

    dst = prepare_sources(src)
    shutil.copyfile(os.path.join(HERE, "ref_probe.pyx"), os.path.join(dst, "ref_probe.pyx"))
    exts = []
    for m in MODULES:
        sources = [os.path.join(dst, m + ".pyx")]
        if m in GSL_MODULES:
            sources.append(os.path.join(SHIM_DIR, "oec_gsl_shim.c"))
        exts.append(Extension(m, sources, include_dirs=[numpy.get_include(), SHIM_DIR, dst],
                              extra_compile_args=["-O3", "-w"]))
    cwd = os.getcwd()
    os.chdir(dst)  # cimports resolve relative to the module directory
    try:
        mods = cythonize(exts, compiler_directives={"language_level": 2, "cpow": True},
                         include_path=[dst], quiet=True, build_dir=os.path.join(OUT, "cbuild"))
        dist = Distribution({"ext_modules": mods})
        cmd = dist.get_command_obj("build_ext")
        cmd.build_lib = OUT
        cmd.build_temp = os.path.join(OUT, "tmp")
        cmd.inplace = False
        cmd.ensure_finalized()
        cmd.run()
    finally:
        os.chdir(cwd)
    print("reference modules built into", OUT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=None, help="reference source tree (default: OEC_REFERENCE or the mount)")
    args = ap.parse_args()
    src = args.src or locate()
    if src is None:
        raise SystemExit("reference source tree not found: pass --src or set OEC_REFERENCE")
    build(src)


if __name__ == "__main__":
    sys.exit(main())

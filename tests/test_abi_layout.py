"""The ctypes structures of the Python layer have the layout of the C ABI's
structures in include/oec.h: a small C program compiled with the host
compiler prints sizeof and offsetof of every field the Python side names, and
both must agree with ctypes (a field added on one side only would shift every
field after it)."""
import ctypes
import importlib
import shutil
import subprocess

import pytest

from conftest import ROOT

# C typedef -> (module of openecloud_b200, ctypes class)
STRUCTS = {
    "oec_particles_t": ("_lib", "Particles_t"),
    "oec_grid_t": ("_lib", "Grid_t"),
    "oec_boundary_t": ("_lib", "Boundary_t"),
    "oec_cnn_t": ("cnn", "Cnn_t"),
    "oec_furman_t": ("furman", "Furman_t"),
    "oec_secelec_t": ("particleEmitter", "SecElec_t"),
    "oec_geom_in_t": ("grid_geom", "GeomIn"),
    "oec_geom_out_t": ("grid_geom", "GeomOut"),
    "oec_lu_t": ("lu_setup", "LU_t"),
    "oec_stencil_t": ("poissonSolver", "Stencil_t"),
    "oec_pcg_stats_t": ("poissonSolver", "PcgStats_t"),
    "oec_mg_level_t": ("poissonSolver", "MgLevel_t"),
    "oec_mg_t": ("poissonSolver", "Mg_t"),
    "oec_status_t": ("session", "Status_t"),
    "oec_run_desc_t": ("session", "RunDesc_t"),
}


def _classes():
    return {c: getattr(importlib.import_module("openecloud_b200." + m), k) for c, (m, k) in STRUCTS.items()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_ctypes_structures_follow_the_header(tmp_path):
    classes = _classes()
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "oec.h"', "int main(void) {"]
    for c, cls in classes.items():
        lines.append(f'printf("{c} %zu\\n", sizeof({c}));')
        for name, *_ in cls._fields_:
            lines.append(f'printf("{c}.{name} %zu\\n", offsetof({c}, {name}));')
    lines.append("return 0; }")
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    r = subprocess.run(["gcc", "-std=c11", "-I", f"{ROOT}/include", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]  # a field the header does not have
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    bad = []
    for c, cls in classes.items():
        if int(out[c]) != ctypes.sizeof(cls):
            bad.append((c, "sizeof", int(out[c]), ctypes.sizeof(cls)))
        for name, *_ in cls._fields_:
            if int(out[f"{c}.{name}"]) != getattr(cls, name).offset:
                bad.append((c, name, int(out[f"{c}.{name}"]), getattr(cls, name).offset))
    assert not bad, bad

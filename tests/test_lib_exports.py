"""liboec.so loads on the CPU host and exports every symbol include/*.h declares."""
import glob
import os
import re

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(?:int|int64_t)\s+(oec_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "oec_push_gather" in names and "oec_deposit" in names
    assert len(names) >= 10


def test_library_exports_all_declared_symbols():
    from openecloud_b200 import _lib
    L = _lib.lib()  # loads without a GPU: no CUDA call happens at load time
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    import importlib
    import openecloud_b200
    from openecloud_b200 import _lib
    for m in openecloud_b200.__all__:  # every binding module registers its entry points
        importlib.import_module("openecloud_b200." + m)
    missing = [n for n in declared_symbols() if n not in _lib.SIGNATURES and n not in _lib.OTHER_DECLARED]
    assert not missing, missing

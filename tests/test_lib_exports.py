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


def declared_parameters():
    """{entry point: its parameter count} from include/*.h."""
    out = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for name, params in re.findall(r"\b(?:int|int64_t)\s+(oec_\w+)\s*\(([^)]*)\)", text):
            params = params.strip()
            out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_argument_counts_match_header():
    """Every ctypes signature passes as many arguments as the header declares
    (an entry point whose parameters changed would otherwise read garbage):
    the common table of _lib and the ones each binding module declares."""
    import importlib
    import openecloud_b200
    from openecloud_b200 import _lib
    for m in openecloud_b200.__all__:
        mod = importlib.import_module("openecloud_b200." + m)
        if callable(getattr(mod, "_declare", None)):
            mod._declare()
    L = _lib.lib()
    declared = declared_parameters()
    unset = [n for n in declared if getattr(L, n).argtypes is None]
    assert not unset, unset
    wrong = {n: (len(getattr(L, n).argtypes), k) for n, k in declared.items() if len(getattr(L, n).argtypes) != k}
    assert not wrong, wrong


def test_status_fields_follow_header():
    """The Python names of the device status words are the header's fields,
    in order, and the struct is STATUS_WORDS int32 long."""
    from openecloud_b200 import _lib
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "oec.h")).read(), flags=re.S)
    body = re.search(r"typedef struct oec_status \{(.*?)\} oec_status_t;", text, flags=re.S).group(1)
    fields = re.findall(r"int32_t\s+(\w+)\s*(?:\[(\d+)\])?\s*;", body)
    names = [f for f, n in fields if not n]
    words = sum(int(n) if n else 1 for _, n in fields)
    assert names == _lib.STATUS_FIELDS
    assert words == _lib.STATUS_WORDS

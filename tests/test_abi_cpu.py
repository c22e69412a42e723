"""The C-ABI boundary without a GPU: both library builds (64-bit and 32-bit
idx/val) load, and every function include/*.h declares is exported.  No
call into the library is made."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
PKG = os.path.join(ROOT, "splatt-stream_b200")


def _declared():
    """Function names declared (prototypes, not typedefs or macros) in the
    public headers."""
    names = set()
    for f in sorted(os.listdir(INC)):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(INC, f)).read()
        src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)     # comments
        src = re.sub(r"//[^\n]*", " ", src)
        src = re.sub(r"^\s*#[^\n]*", " ", src, flags=re.M)    # preprocessor lines
        src = re.sub(r"typedef\s+[^;]*?\([^;]*?;", " ", src, flags=re.S)  # function-pointer typedefs
        for m in re.finditer(r"\b(splatt_\w+)\s*\(", src):
            name = m.group(1)
            prev = src[max(0, m.start() - 2):m.start()].strip()
            if prev.endswith("(*") or prev.endswith("*)"):
                continue
            names.add(name)
    return names


def test_header_declares_functions():
    names = _declared()
    for must in ("splatt_csf_convert", "splatt_mttkrp", "splatt_cpd", "splatt_cpd_stream",
                 "splatt_b200_stream_push", "splatt_b200_stream_set_prox",
                 "splatt_register_nonneg"):
        assert must in names, must


@pytest.mark.parametrize("lib", ["libsplatt_b200.so", "libsplatt_b200_w32.so"])
def test_library_exports_every_declared_function(lib):
    path = os.path.join(PKG, lib)
    assert os.path.exists(path), "build first: python splatt-stream_b200/build.py"
    L = ctypes.CDLL(path)
    missing = []
    for name in sorted(_declared()):
        try:
            getattr(L, name)
        except AttributeError:
            missing.append(name)
    assert not missing, missing

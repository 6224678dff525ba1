"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
LIB = REPO / "qws_b200" / "libqws_b200.so"


def declared_functions():
    names = set()
    for h in sorted((REPO / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("qwsg_", "qws_", "bicgstab_", "prec_", "ddd_", "jinv_",
                                "fermi_", "print_", "zero_", "get_clock", "deo_", "dee_",
                                "one_minus_", "mtilde", "clv", "assign_", "bqcd_")):
                names.add(name)
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        import qws_b200.build as b
        b.build()
    return ctypes.CDLL(str(LIB))


def test_headers_declare_functions():
    assert len(declared_functions()) > 20


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(lib, name):
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_last_error_without_gpu(lib):
    lib.qwsg_last_error.restype = ctypes.c_char_p
    lib.qwsg_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.qwsg_version()
    assert lib.qwsg_last_error() is not None

"""The C ABI library: it loads and exports every entry point include/softdft.h
declares.  No compute call is made here (no GPU in this container)."""
import os
import re

from softdft_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "softdft.h")).read()
    return sorted(set(re.findall(r"\b(sdft_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = native.lib()
    names = _declared()
    assert "sdft_solve" in names and "sdft_request_create" in names
    for n in names:
        assert hasattr(L, n), n
    assert set(native.EXPORTS) <= set(names)


def test_abi_version():
    assert native.lib().sdft_abi_version() == 2

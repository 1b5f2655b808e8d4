"""The C-ABI library loads without a GPU and exports every symbol the public header
declares; the provider table carries the expected ABI version and name."""
import os
import re

from conftest import ROOT


def declared_symbols():
    syms = []
    inc = os.path.join(ROOT, "include")
    for name in sorted(os.listdir(inc)):
        if not name.endswith(".h"):
            continue
        text = "\n".join(l for l in open(os.path.join(inc, name)).read().splitlines()
                         if not l.lstrip().startswith("#"))
        for m in re.finditer(r"SYCLFFT_B200_EXPORT[^;(]*?\b(\w+)\s*\(", text):
            syms.append(m.group(1))
    return syms


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "syclfft_b200_get_provider_v1" in syms


def test_library_exports_every_declared_symbol():
    from syclfft_b200 import _provider
    lib = _provider.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(_provider.EXPORTED_SYMBOLS) <= set(declared_symbols())


def test_provider_table_without_gpu():
    from syclfft_b200 import _provider
    api = _provider.provider()
    assert api.abi_version == _provider.ABI_VERSION
    assert api.name == b"b200"
    lib = _provider.load()
    assert lib.syclfft_b200_version().startswith(b"syclfft-b200")

"""The C-ABI library loads without a GPU and exports every symbol that
include/z2dqmc.h declares (no compute calls)."""
import os
import re

import pytest

from z2_gauge_zfy_b200 import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "z2dqmc.h")).read()
    return sorted(set(re.findall(r"\b(z2_[a-zA-Z0-9_]+)\s*\(", txt)))


def test_header_matches_binding_list():
    assert declared_symbols() == sorted(_ffi.EXPORTS)


def test_library_exports_all_symbols():
    lib = _ffi.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_no_fallback_without_library(monkeypatch, tmp_path):
    monkeypatch.setattr(_ffi, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_ffi, "_lib", None)
    with pytest.raises(ImportError):
        _ffi.load()


@pytest.mark.parametrize("bad, msg", [
    (dict(Nlx=5), "even"),
    (dict(Ltrot=25, Nwrap=10), "multiple of Nwrap"),
    (dict(absolute=7), "absolute"),
    (dict(beta=0.0), "beta"),
])
def test_create_rejects_bad_arguments(bad, msg):
    """Argument errors (the reference would print and stop) come back as
    Z2_ERR_ARG before any device work, so they are checked without a GPU."""
    from z2_gauge_zfy_b200 import Chain, Z2Batch, Z2Error
    kw = dict(RT=1.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10)
    kw.update(bad)
    with pytest.raises(Z2Error) as e:
        Z2Batch([Chain(**kw)])
    assert e.value.code == 1 and msg in str(e.value)

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
    (dict(rt_bond=[1.0] * 5), "rt_bond"),
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


def test_create_rejects_wrong_delay_list():
    """One delayed-update rank per chain, checked before any device work."""
    from z2_gauge_zfy_b200 import Chain, Z2Batch, Z2Error
    with pytest.raises(Z2Error) as e:
        Z2Batch([Chain()], delay_k_chain=[4, 4])
    assert e.value.code == 1 and "delay_k_chain" in str(e.value)


def test_null_handle_is_an_argument_error():
    """Every entry point that takes a handle returns Z2_ERR_ARG for a null one
    before touching the device (so this runs without a GPU); z2_destroy(NULL)
    is a no-op and z2_last_error(NULL) still returns text."""
    import ctypes as C
    lib = _ffi.load()
    skip = {"z2_create", "z2_tune_delay", "z2_stab_green_noalloc", "z2_last_error",
            "z2_destroy"}
    checked = 0
    for name in _ffi.EXPORTS:
        if name in skip:
            continue
        f = getattr(lib, name)
        # null for every pointer (handle and buffers), zero for every integer
        args = [0 if t in (C.c_int32, C.c_size_t) else None for t in f.argtypes]
        assert f(*args) == 1, name
        checked += 1
    assert checked == len(_ffi.EXPORTS) - len(skip)
    assert lib.z2_destroy(None) == 0
    assert lib.z2_last_error(None) == b"null handle"
    assert lib.z2_create(None, None, 1, None) == 1
    assert lib.z2_tune_delay(None, 1, None, None) == 1


def _header_arity():
    txt = open(os.path.join(ROOT, "include", "z2dqmc.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(z2_[a-zA-Z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_fortran_binding_matches_header():
    """include/z2_cuda_mod.f90's ISO_C_BINDING module binds every entry point of the
    header, each with the header's number of arguments."""
    txt = open(os.path.join(ROOT, "include", "z2_cuda_mod.f90")).read()
    txt = re.sub(r"&\s*\n\s*", " ", txt)           # join continuation lines
    fort = {}
    for m in re.finditer(r"function\s+(z2_[a-z0-9_]+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)",
                         txt, flags=re.I):
        assert m.group(1).lower() == m.group(3).lower()
        args = m.group(2).strip()
        fort[m.group(3)] = 0 if not args else args.count(",") + 1
    hdr = _header_arity()
    assert sorted(hdr) == sorted(_ffi.EXPORTS)
    assert sorted(fort) == sorted(hdr)
    for name, n in hdr.items():
        assert fort[name] == n, (name, fort[name], n)


def test_ctypes_signatures_match_header():
    """The ctypes declarations carry the header's number of arguments."""
    lib = _ffi.load()
    for name, n in _header_arity().items():
        assert len(getattr(lib, name).argtypes) == n, name


def test_fortran_module_is_well_formed():
    """No Fortran compiler is available here, so the module's structure is
    checked by reading it: free-form lines of at most 132 characters, every
    interface function closed, one interface block, module opened and closed."""
    src = open(os.path.join(ROOT, "include", "z2_cuda_mod.f90")).read()
    lines = src.splitlines()
    assert all(len(ln) <= 132 for ln in lines)
    code = [ln.split("!")[0].strip().lower() for ln in lines]
    opened = sum(1 for ln in code if re.match(r"(integer\(c_int\)|type\(c_ptr\)) function ", ln)
                 or re.match(r"function ", ln))
    closed = sum(1 for ln in code if ln == "end function")
    assert opened == closed > 0
    assert code.count("interface") == 1 and code.count("end interface") == 1
    assert sum(ln.startswith("module z2_cuda_mod") for ln in code) == 1
    assert sum(ln.startswith("end module z2_cuda_mod") for ln in code) == 1
    # continuation lines end with '&' and are followed by a line
    for i, ln in enumerate(code):
        if ln.endswith("&"):
            assert i + 1 < len(code) and code[i + 1]

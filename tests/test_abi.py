"""The C-ABI shared library loads and exports every symbol include/*.h
declares (no GPU needed: nothing here launches device work)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(sb200_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("sb200_ctx_create", "sb200_hpsi", "sb200_taylor", "sb200_rt_propagate", "sb200_calc_current"):
        assert n in names


def test_library_exports_all_declared_symbols():
    from salmon2_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    # the ctypes signature table covers the header exactly
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_library_reports_missing_device_without_crashing():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from salmon2_b200 import _lib
    h = ctypes.c_void_p()
    rc = _lib.lib().sb200_ctx_create(0, ctypes.byref(h))
    assert rc == 5  # SB200_ERR_CUDA
    assert _lib.lib().sb200_last_error()


def test_fortran_interface_binds_every_entry_point():
    """The ISO_C_BINDING module a SALMON build would use declares every entry
    point of the header under its C name (no Fortran compiler here: checked
    as text)."""
    src = open(os.path.join(ROOT, "salmon2_b200", "fortran", "salmon_b200.f90")).read()
    bound = set(re.findall(r'bind\(c,\s*name="(sb200_\w+)"\)', src))
    assert bound == set(declared_symbols())

"""CPU tests of the C-ABI library: it loads, exports every entry point the
public header declares, and rejects bad arguments before touching a device
(no compute runs here)."""
import ctypes
import subprocess

import numpy as np
import pytest

import osiris_b200 as osr
from osiris_b200.build import LIB


def test_library_exports_every_header_symbol():
    names = osr.header_symbols()
    assert "osr_flash_batch" in names and "osr_flash_batch_host" in names
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = osr.lib()
    for n in names:
        assert getattr(L, n) is not None


def test_every_entry_point_has_full_width_signature():
    """Each declared function gets argtypes from the header, so host addresses
    above 4 GiB (large numpy arrays) are never truncated to a C int."""
    L = osr.lib()
    for ret, name, params in osr.header_signatures():
        fn = getattr(L, name)
        assert fn.argtypes is not None and len(fn.argtypes) == len(params), name
        for p, t in zip(params, fn.argtypes):
            if "*" in p:
                assert t in (ctypes.c_void_p, ctypes.c_char_p), (name, p)
    assert L.osr_grid_field_size.restype is ctypes.c_long
    assert L.osr_status_string.restype is ctypes.c_char_p


def test_status_strings_and_version():
    L = osr.lib()
    assert L.osr_version() == 1
    for s in range(6):
        assert L.osr_status_string(s)


def _bad_call(fluid_nc=6, eos=1, n=10):
    tc, pc, acf, kij = (np.ones(max(fluid_nc, 1)) for _ in range(4))
    kij = np.zeros((max(fluid_nc, 1), max(fluid_nc, 1)))
    f = osr._CFluid(fluid_nc, eos, tc.ctypes.data, pc.ctypes.data, acf.ctypes.data, kij.ctypes.data)
    out = osr._CFlashOut(*([ctypes.c_void_p(8)] * 6 + [None] * 4))
    dummy = ctypes.c_void_p(8)
    return osr.lib().osr_flash_batch(ctypes.byref(f), dummy, dummy, dummy, ctypes.c_long(n), ctypes.byref(out), None)


def test_argument_validation_without_device():
    assert _bad_call(fluid_nc=0) == 2          # OSR_ERR_NC
    assert _bad_call(fluid_nc=17) == 2
    assert _bad_call(eos=7) == 1                # OSR_ERR_ARG
    assert _bad_call(n=-1) == 1
    L = osr.lib()
    assert L.osr_flash_set_shape(0, 32, 4, 8) == 1
    assert L.osr_flash_set_shape(8, 32, 0, 8) == 1
    assert L.osr_flash_set_shape(8, 0, 4, 8) == 1
    assert L.osr_flash_set_shape(8, 32, 4, -1) == 1
    a, b, c, d = osr.get_shape()
    assert 1 <= a <= 32 and 1 <= b <= 32 and 1 <= c <= 16 and 0 <= d <= 500


def test_shape_roundtrip():
    old = osr.get_shape()
    osr.set_shape(12, 30, 3, 6)
    assert osr.get_shape() == (12, 30, 3, 6)
    osr.set_shape(*old)
    with pytest.raises(osr.OsrError):
        osr.set_shape(33, 1, 1, 1)

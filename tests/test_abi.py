"""CPU tests of the C ABI boundary: the library loads, exports every symbol include/dns2d.h
declares, and its host-only entry points and error paths behave (no device work here)."""
import ctypes as C
import os
import re
import struct

import pytest

import optimizec_b200 as P

HEADER = os.path.join(P.REPO, "include", "dns2d.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dns2d_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(P.SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(P.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_supported_sizes_and_errors():
    L = P.lib()
    for n in (16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 840, 8192, 9216, 16384, 29400):
        assert L.dns2d_supported(n) == 1
    for n in (0, 7, 100, 4095):
        assert L.dns2d_supported(n) == 0
    assert L.dns2d_strerror(0) == b"ok"
    assert b"unsupported" in L.dns2d_strerror(2)
    s = C.c_void_p()
    assert L.dns2d_create(C.byref(s), 100, 1e4, 4.0, 0.1, 0) == 2  # DNS2D_ERR_SIZE
    assert not s
    assert L.dns2d_create(None, 512, 1e4, 4.0, 0.1, 0) == 1  # DNS2D_ERR_ARG
    assert L.dns2d_step(None, 1, None, None) == 1
    assert L.dns2d_k4_spectrum(12, 4.0, 0, None) == 1


def test_device_bytes_scale():
    L = P.lib()
    b512 = L.dns2d_device_bytes(512)
    b4096 = L.dns2d_device_bytes(4096)
    assert 60 * 4096 ** 2 > b4096 > 50 * 4096 ** 2
    assert b4096 / b512 == pytest.approx(64, rel=0.01)


def test_restart_header_layout():
    """restart.bin v2 header of cuda/mem_cuda.cu:1019-1054: 144 bytes, u64 counts at 112..143."""
    fmt = "<16s4I10i9f4x4Q"
    assert struct.calcsize(fmt) == 144
    assert struct.calcsize("<16s4I10i9f4x3Q") == 136

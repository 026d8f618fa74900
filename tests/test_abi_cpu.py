"""CPU checks of the C ABI: the library loads without a GPU and exports every
entry point include/starjoin.h declares; host-only calls behave."""
import ctypes as C
import os
import re

import pytest

from conftest import HAS_GPU, ROOT


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sj[bs]?_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(sj):
    lib = C.CDLL(sj.LIB_PATH)
    names = [n for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h") for n in _declared(h)]
    assert names, "no declarations found"
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(sj):
    import shared_scan
    assert set(_declared("starjoin.h")) <= set(sj.exported_symbols())
    assert set(_declared("starjoin_batch.h")) <= set(shared_scan.SYMBOLS) | set(sj.exported_symbols())
    shared_scan.load()  # every binding resolves


def test_status_strings(sj):
    lib = sj.load()
    assert lib.sj_status_string(0) == b"ok"
    assert lib.sj_status_string(sj.SJ_ERR_CAPACITY) == b"result buffer too small"


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_engine_create_without_device_fails_cleanly(sj):
    lib = sj.load()
    h = C.c_void_p()
    assert lib.sj_engine_create(0, C.byref(h)) == sj.SJ_ERR_NO_DEVICE
    assert h.value is None
    assert b"no CUDA device" in lib.sj_last_error()

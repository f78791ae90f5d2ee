"""CPU-side checks of the C ABI: the library loads and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(aoa_[a-z0-9_]+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import aoa_b200.build as build
    lib = ctypes.CDLL(build.build())
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert len(_declared()) > 10


def test_python_binding_covers_header():
    from aoa_b200 import capi
    assert set(_declared()) <= set(capi.exported_symbols())


def test_engine_create_fails_cleanly_without_gpu_or_bad_params():
    import numpy as np
    from aoa_b200 import capi
    lib = capi.load()
    p = capi.Params()
    arr = np.array([3, 5], dtype=np.uint64)
    p.log_n, p.k, p.kl, p.primes, p.generators, p.scale_bits, p.dnum = 4, 1, 1, arr.ctypes.data_as(capi.u64p), None, 0, 1
    h = ctypes.c_void_p()
    st = lib.aoa_engine_create(ctypes.byref(p), ctypes.byref(h))
    assert st != 0 and not h.value
    assert lib.aoa_last_error()


def test_reference_signature_shim_compiles_and_links(tmp_path):
    """The C++ shims (include/newckks/ckks/ckks.h, include/AOADGT/ckks.h) and a
    caller written against the reference's signatures build and link against
    libaoa_b200.so with plain g++ (running it needs a GPU:
    tests/test_gpu_shim.py)."""
    import subprocess
    import aoa_b200.build as build
    lib = os.path.dirname(build.build())
    for flags, exe in (([], "shim_check"), (["-DSHIM_DGT"], "shim_check_dgt")):
        subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror"] + flags +
                              ["-I", os.path.join(ROOT, "include"),
                               os.path.join(ROOT, "tests", "shim", "shim_check.cpp"), "-L", lib, "-laoa_b200",
                               "-Wl,-rpath," + lib, "-o", str(tmp_path / exe)])
        assert os.path.exists(tmp_path / exe)

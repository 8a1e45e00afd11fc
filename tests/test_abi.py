"""The C-ABI library: builds, loads without a GPU and exports every symbol
that include/*.h declares.  No compute calls here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, pac

HEADERS = [os.path.join(ROOT, "include", h) for h in ("fft.h", "pac.h")]


def declared_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    src = "\n".join(l for l in src.splitlines() if not l.strip().startswith("#"))
    src = re.sub(r"typedef[^;]*;", "", src, flags=re.S)
    src = re.sub(r"enum\s*\{.*?\};", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(names))


def exported(path):
    out = subprocess.check_output(["nm", "-D", "--defined-only", path], text=True)
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


def test_headers_declare_the_reference_surface():
    names = declared_functions(HEADERS[0])
    # the reference's fft.h declares 66 functions (fft.h:17-229)
    assert len(names) == 66, len(names)
    for n in ("permutation_avoiding_convolution_3d", "apply_transposed_butterflies_r8",
              "precompute_twiddles_r4", "uifft_3d", "in_place_square_array_transpose_split_2d"):
        assert n in names


def test_library_exports_every_declared_symbol():
    so = pac.build()
    have = exported(so)
    missing = []
    for h in HEADERS:
        for n in declared_functions(h):
            if n not in have:
                missing.append((os.path.basename(h), n))
    assert not missing, missing


def test_library_loads_without_gpu_and_fails_loudly():
    lib = pac.load()
    assert lib.pac_launch_count() >= 0
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    plan = C.c_void_p()
    dims = (C.c_int * 1)(64)
    st = lib.pac_plan_create(C.byref(plan), 1, dims, 1, 2, 0)
    assert st == 6  # PAC_ERROR_NO_DEVICE: no host fallback
    assert b"device" in lib.pac_last_error()


def test_invalid_arguments_rejected_before_device():
    lib = pac.load()
    plan = C.c_void_p()
    dims = (C.c_int * 1)(64)
    assert lib.pac_plan_create(C.byref(plan), 0, dims, 1, 2, 0) == 1
    assert lib.pac_plan_create(C.byref(plan), 1, dims, 1, 3, 0) == 3
    assert lib.pac_plan_create(C.byref(plan), 1, dims, 1, 2, 7) == 1
    assert lib.pac_status_string(2) == b"axis length is not a power of the radix"


def test_emulator_is_a_separate_test_build():
    """The product library carries no host replay path."""
    gpu = exported(pac.build())
    emu = exported(pac.build(emulate=True))
    gpu_only = {"pac_convolve_1d_noalloc"}  # its scratch is a static device array
    for h in HEADERS:
        for n in declared_functions(h):
            assert n in gpu and (n in emu or n in gpu_only)  # same C ABI ...
    strings = subprocess.check_output(["strings", pac.build()], text=True)
    assert "host allocation failed" not in strings  # ... but no emulator inside

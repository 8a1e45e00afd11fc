"""Shared fixtures.

* ``orc``   -- the C restatement of the reference (oracle/pac_oracle.c)
* ``ref``   -- the reference itself compiled from its sources (skips where
               oracle/_ref/libref.so was not built)
* ``emu``   -- the TEST-ONLY host replay build of the library
* ``lib``   -- the product library (GPU tests only)
* ``golden_cases`` -- the reference's outputs in tests/golden/
"""
import glob
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

pac = importlib.import_module("c-permutation-avoiding-convolution_b200")

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def orc():
    return O.Orc()


@pytest.fixture(scope="session")
def ref():
    path = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    if not os.path.exists(path):
        if O.ref_source_dir():  # PAC_REF_DIR names the reference sources
            O.build_ref()
        else:
            pytest.skip("reference library not built here")
    return O.Ref(path)


@pytest.fixture(scope="session")
def emu():
    return pac.load(emulate=True)


@pytest.fixture(scope="session")
def lib():
    return pac.load()


def load_golden(path):
    g = np.load(path)
    return {k: g[k] for k in g.files}


@pytest.fixture(scope="session", params=GOLDEN, ids=[os.path.basename(p)[2:-4] for p in GOLDEN])
def golden(request):
    return load_golden(request.param)


def rng(seed):
    return np.random.default_rng(seed)


rel_l2 = O.rel_l2
max_abs = O.max_abs

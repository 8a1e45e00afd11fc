"""pac_convolve_1d_noalloc: the entry point for callers that cannot allocate
device memory (framework memory pools, fixed budgets, code that must not
synchronise the device).  Its only scratch is a fixed static device array of
the library, shared by every call on a device.

Checked through the C ABI against the allocating entry point
(pac_filter_spectrum + pac_convolve on a plan) on two calls in a row, which
also shows that the second call does not depend on what the first left in
the shared array.  This file is collected last (test_zz_*), so a run that
stops at the first failure has run every other test before it; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import parity as P
from conftest import pac, rng

pytestmark = pytest.mark.gpu


def _noalloc(L, d, x, h, n, batch):
    xr, xi = d.put(np.ascontiguousarray(x.real)), d.put(np.ascontiguousarray(x.imag))
    hr, hi = d.put(np.ascontiguousarray(h.real)), d.put(np.ascontiguousarray(h.imag))
    yr, yi = d.zeros((batch, n), np.float64), d.zeros((batch, n), np.float64)
    st = L.pac_convolve_1d_noalloc(xr, xi, hr, hi, yr, yi, n, batch, None)
    pac.check(L, st, "pac_convolve_1d_noalloc")
    return d.get(yr, (batch, n), np.float64) + 1j * d.get(yi, (batch, n), np.float64)


@pytest.mark.parametrize("n,batch", [(4096, 3), (65536, 2), (2048, 1), (64, 5), (1, 2)])
def test_noalloc_matches_allocating_entry_point(lib, n, batch):
    g = rng(n + batch)
    x = g.standard_normal((batch, n)) + 1j * g.standard_normal((batch, n))
    h = g.standard_normal(n) + 1j * g.standard_normal(n)
    want = P.native_conv(lib, (n,), batch, 2, pac.PAC_FORM_F64, x, h)
    d = P.Dev(lib)
    try:
        first = _noalloc(lib, d, x, h, n, batch)
        # a different problem in between leaves other contents in the array
        g2 = rng(7)
        x2 = g2.standard_normal((1, 256)) + 1j * g2.standard_normal((1, 256))
        _noalloc(lib, d, x2, g2.standard_normal(256) + 0j, 256, 1)
        second = _noalloc(lib, d, x, h, n, batch)
    finally:
        d.free()
    assert P.crel(first, want) < P.TOL
    assert P.crel(second, want) < P.TOL
    assert np.array_equal(first, second)


def test_noalloc_rejects_oversize(lib):
    n = 2 * 65536
    d = P.Dev(lib)
    try:
        z = np.zeros(n)
        ptrs = [d.put(z) for _ in range(4)]
        y = d.put(np.full(n, 7.0))
        st = lib.pac_convolve_1d_noalloc(ptrs[0], ptrs[1], ptrs[2], ptrs[3], y, y, n, 1, None)
        assert st == 4  # PAC_ERROR_SIZE
        assert b"no-allocation limit" in lib.pac_last_error()
        assert np.all(d.get(y, (n,), np.float64) == 7.0)
        st = lib.pac_convolve_1d_noalloc(ptrs[0], ptrs[1], ptrs[2], ptrs[3], y, y, 96, 1, None)
        assert st == 2  # not a power of 2
        # sizes near the int range are rejected by the limit before any shift
        for big in ((1 << 30) + 1, 1 << 30, 2147483647):
            st = lib.pac_convolve_1d_noalloc(ptrs[0], ptrs[1], ptrs[2], ptrs[3], y, y, big, 1,
                                             None)
            assert st == 4
        assert np.all(d.get(y, (n,), np.float64) == 7.0)
    finally:
        d.free()

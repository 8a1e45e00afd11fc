"""Pin the oracle: the C restatement against the reference's own outputs.

The reference has no test suite or golden vectors (it only prints max
errors against FFTW in its bench drivers' verify modes), so the pins are
(1) golden vectors produced by the reference library compiled from its own
sources (tests/golden/make_golden.py), (2) the reference library run live
where it is built, (3) numpy.fft and (4) a direct O(N^2) long-double
convolution.
"""
import numpy as np
import pytest

from conftest import O, rel_l2, rng

TOL = 1e-14  # restatement vs reference: both FP64, different rounding order

OPS = ((O.OP_A, "A"), (O.OP_CONJ, "conjA"), (O.OP_AT, "At"))
KINDS = ("fft", "fft2", "ufft", "ifft", "uifft")


def test_restatement_matches_golden(orc, golden):
    g = golden
    r = int(g["r"])
    x = (g["x_re"], g["x_im"])
    h = (g["h_re"], g["h_im"])
    if "At_re" in g:
        for op, name in OPS:
            a = orc.butterflies(op, r, *x)
            assert rel_l2(*a, g[name + "_re"], g[name + "_im"]) < TOL, name
        for k, name in enumerate(KINDS):
            a = orc.transform(k, r, *x)
            assert rel_l2(*a, g[name + "_re"], g[name + "_im"]) < TOL, name
        assert np.array_equal(orc.rho(r, tuple(g["shape"])), g["rho"])
        y = orc.convolution(O.METHOD_FFT_BASED, r, *x, *h)
        assert rel_l2(y[0], y[1], g["fbc_re"], g["fbc_im"]) < TOL
        assert rel_l2(y[2], y[3], g["fbc_hre"], g["fbc_him"]) < TOL
    y = orc.convolution(O.METHOD_PAC, r, *x, *h)
    assert rel_l2(y[0], y[1], g["pac_re"], g["pac_im"]) < TOL
    assert rel_l2(y[2], y[3], g["pac_hre"], g["pac_him"]) < TOL


def test_reference_reproduces_golden(ref, golden):
    """Provenance of the fixtures: the reference library gives them bit for bit."""
    g = golden
    r = int(g["r"])
    y = ref.convolution(O.METHOD_PAC, r, g["x_re"], g["x_im"], g["h_re"], g["h_im"])
    assert np.array_equal(y[0], g["pac_re"]) and np.array_equal(y[3], g["pac_him"])
    if "At_re" in g:
        a = ref.butterflies(O.OP_AT, r, g["x_re"], g["x_im"])
        assert np.array_equal(a[0], g["At_re"]) and np.array_equal(a[1], g["At_im"])


@pytest.mark.parametrize("shape,r", [((4096,), 2), ((4096,), 4), ((4096,), 8), ((2048,), 2),
                                     ((32, 64), 2), ((64, 64), 4), ((16, 16, 16), 4),
                                     ((32, 8, 4), 2)])
def test_restatement_matches_live_reference(orc, ref, shape, r):
    g = rng(11)
    x = (g.standard_normal(shape), g.standard_normal(shape))
    h = (g.standard_normal(shape), g.standard_normal(shape))
    for op, _ in OPS:
        assert rel_l2(*orc.butterflies(op, r, *x), *ref.butterflies(op, r, *x)) < TOL
    for k in range(5):
        assert rel_l2(*orc.transform(k, r, *x), *ref.transform(k, r, *x)) < TOL
    a = orc.convolution(O.METHOD_PAC, r, *x, *h)
    b = ref.convolution(O.METHOD_PAC, r, *x, *h)
    assert rel_l2(a[0], a[1], b[0], b[1]) < TOL
    assert rel_l2(a[2], a[3], b[2], b[3]) < TOL
    assert np.array_equal(orc.rho(r, shape), ref.rho(r, shape))


@pytest.mark.parametrize("shape,r", [((512,), 8), ((1024,), 4), ((64, 16), 2), ((16, 16, 16), 4)])
def test_transposed_is_digit_reversed_dft(orc, shape, r):
    """A^T x = P_r F x (the method's factorisation, README.md:1-3)."""
    g = rng(3)
    x = (g.standard_normal(shape), g.standard_normal(shape))
    a = orc.butterflies(O.OP_AT, r, *x)
    F = np.fft.fftn(x[0] + 1j * x[1]).ravel()[orc.rho(r, shape)].reshape(shape)
    assert rel_l2(*a, F.real, F.imag) < 1e-14


@pytest.mark.parametrize("shape,r", [((256,), 2), ((256,), 4), ((512,), 8), ((16, 16), 4),
                                     ((8, 4, 8), 2)])
def test_convolution_matches_direct_sum(orc, shape, r):
    g = rng(5)
    x = (g.standard_normal(shape), g.standard_normal(shape))
    h = (g.standard_normal(shape), g.standard_normal(shape))
    y = orc.convolution(O.METHOD_PAC, r, *x, *h)
    z = orc.naive_conv(*x, *h)
    assert rel_l2(y[0], y[1], *z) < 1e-14


def test_impulse_and_unsupported_radix(orc):
    n = 64
    x = (np.zeros(n), np.zeros(n))
    x[0][0] = 1.0
    g = rng(9)
    h = (g.standard_normal(n), g.standard_normal(n))
    y = orc.convolution(O.METHOD_PAC, 4, *x, *h)
    assert rel_l2(y[0], y[1], *h) < 1e-15
    # 2D r = 8: butterflies skipped, product / n only (convolution_2d.c:41-63)
    s = (8, 8)
    x = (g.standard_normal(s), g.standard_normal(s))
    h = (g.standard_normal(s), g.standard_normal(s))
    y = orc.convolution(O.METHOD_PAC, 8, *x, *h)
    z = (x[0] + 1j * x[1]) * (h[0] + 1j * h[1]) / 64
    assert rel_l2(y[0], y[1], z.real, z.imag) < 1e-15
    assert np.array_equal(y[2], h[0])


def test_twiddle_tables_match_reference_layout(orc):
    for r, n in ((2, 64), (4, 256), (8, 512)):
        tabs = orc.twiddles(r, n)
        k = 1
        for q, tab in enumerate(tabs):
            k *= r
            ell = k // r
            m = np.repeat(np.arange(1, r), ell)
            j = np.tile(np.arange(ell), r - 1)
            want = np.exp(-2j * np.pi * m * j / k)
            assert np.max(np.abs(tab - want)) < 1e-15

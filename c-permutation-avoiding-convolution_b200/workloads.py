"""Seeded synthetic inputs of the five benchmark configurations.

No dataset is involved in the reference's benchmarks; these generators make
the inputs the configurations describe, with fixed seeds (numpy
default_rng), as complex128 arrays:

  c1  1D n = 2^12, x and h with N(0,1) real and imaginary parts
  c2  1D batch 1024 x 2^16, x N(0,1) complex; one 257-tap filter of
      N(0, 1/257) complex entries zero-padded to 2^16
  c3  2D 2048 x 2048, x with U(-1,1) real and imaginary parts; h a real
      31 x 31 Gaussian (sigma 5, normalised to sum 1), zero-padded and
      circularly centred so the centre tap sits at (0, 0)
  c4  3D 256^3 and 512 x 256 x 128, x N(0,1) complex; h a 9 x 9 x 9 complex
      stencil of N(0, 1/729) entries zero-padded
  c5  batched uneven: 4096 1D problems with log2 n uniform on 8..20 and 64 2D
      problems with log2 of each side uniform on 6..11; x, h N(0,1) complex,
      h supported on the first n/16 entries of every axis
"""
import numpy as np


def _cn(g, shape, var=1.0):
    s = np.sqrt(var)
    return s * g.standard_normal(shape) + 1j * s * g.standard_normal(shape)


def c1(n=4096):
    x = _cn(np.random.default_rng(1), n)
    h = _cn(np.random.default_rng(2), n)
    return x, h


def c2(batch=1024, n=65536, taps=257):
    x = _cn(np.random.default_rng(1), (batch, n))
    h = np.zeros(n, np.complex128)
    h[:taps] = _cn(np.random.default_rng(2), taps, 1.0 / taps)
    return x, h


def gaussian_filter_2d(n1, n2, size=31, sigma=5.0):
    r = size // 2
    i = np.arange(-r, r + 1)
    k = np.exp(-(i[:, None] ** 2 + i[None, :] ** 2) / (2 * sigma * sigma))
    k /= k.sum()
    h = np.zeros((n1, n2), np.complex128)
    rows = np.mod(i, n1)
    cols = np.mod(i, n2)
    h[np.ix_(rows, cols)] = k
    return h


def c3(n=2048):
    g = np.random.default_rng(1)
    x = g.uniform(-1, 1, (n, n)) + 1j * g.uniform(-1, 1, (n, n))
    return x, gaussian_filter_2d(n, n)


def c4(shape=(256, 256, 256), size=9):
    x = _cn(np.random.default_rng(1), shape)
    h = np.zeros(shape, np.complex128)
    h[:size, :size, :size] = _cn(np.random.default_rng(2), (size,) * 3, 1.0 / size ** 3)
    return x, h


def c5_shapes(n1d=4096, n2d=64, seed=5):
    """The problem shapes of c5 (log2 sizes drawn uniformly, rounded)."""
    g = np.random.default_rng(seed)
    one = [(1 << int(round(v)),) for v in g.uniform(8, 20, n1d)]
    two = [(1 << int(round(a)), 1 << int(round(b))) for a, b in g.uniform(6, 11, (n2d, 2))]
    return one + two


def c5_problem(shape, seed):
    g = np.random.default_rng(seed)
    x = _cn(g, shape)
    h = np.zeros(shape, np.complex128)
    sl = tuple(slice(0, max(1, s // 16)) for s in shape)
    h[sl] = _cn(g, h[sl].shape)
    return x, h

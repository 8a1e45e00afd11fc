"""Parity of the sm_100a library (libpac.so) with the oracle, on the GPU.

Every call goes through the C ABI: fft.h (host pointers, the reference's
prototypes) or pac.h (plans, device pointers).  FP64 results must match the
oracle to 1e-13 relative L2, the reference's digit-reversal order exactly
(the overwritten filter A^T h is compared position by position), and the FP32
form the FP64 oracle to 1e-6 relative L2.
"""
import importlib
import threading

import numpy as np
import pytest

import parity as P
from conftest import O, pac, rel_l2, rng

pytestmark = pytest.mark.gpu
W = importlib.import_module("c-permutation-avoiding-convolution_b200.workloads")


def test_golden(lib, golden):
    P.check_golden(lib, golden)


@pytest.mark.parametrize("shape,r", [
    ((4096,), 4), ((4096,), 2), ((4096,), 8), ((8192,), 2), ((4 ** 8,), 4), ((8 ** 5,), 8),
    ((2 ** 17,), 2), ((8192, 4), 2), ((4, 8192), 2), ((256, 256), 4), ((512, 64), 2),
    ((64, 64, 64), 4), ((128, 4, 4), 2), ((16, 32, 64), 2), ((1,), 2), ((2,), 2), ((1,), 8)])
def test_oracle_sizes(lib, orc, shape, r):
    P.check_against_oracle(lib, orc, shape, r, ops=np.prod(shape) <= 2 ** 17)


@pytest.mark.parametrize("cap", ["3", "4", "6"])
def test_multi_factor_splits(lib, orc, cap, monkeypatch):
    monkeypatch.setenv("PAC_MAX_FACTOR_LOG", cap)
    for shape, r in [((2 ** 12,), 2), ((4 ** 6,), 4), ((8 ** 4,), 8), ((128, 32), 2),
                     ((16, 64, 32), 2)]:
        if r == 4 and cap == "3":
            continue
        P.check_against_oracle(lib, orc, shape, r, seed=int(cap))


def test_c1_against_reference_and_direct_sum(lib, orc):
    """C1: n = 2^12, radix 4, N(0,1) inputs."""
    x, h = W.c1()
    xs, hs = (x.real, x.imag), (h.real, h.imag)
    y = pac.dropin_convolution(lib, O.METHOD_PAC, 4, *xs, *hs)
    z = orc.convolution(O.METHOD_PAC, 4, *xs, *hs)
    assert rel_l2(y[0], y[1], z[0], z[1]) < P.TOL
    assert rel_l2(y[2], y[3], z[2], z[3]) < P.TOL
    d = orc.naive_conv(*xs, *hs)
    assert rel_l2(y[0], y[1], *d) < P.TOL
    # the A^T x intermediate is the reference's element by element
    a = pac.dropin_butterflies(lib, O.OP_AT, 4, *xs)
    b = orc.butterflies(O.OP_AT, 4, *xs)
    assert rel_l2(*a, *b) < P.TOL
    for r in (2, 8):
        y = pac.dropin_convolution(lib, O.METHOD_PAC, r, *xs, *hs)
        assert rel_l2(y[0], y[1], *d) < P.TOL


@pytest.mark.parametrize("form", [pac.PAC_FORM_F64, pac.PAC_FORM_F32, pac.PAC_FORM_TC])
def test_c2_batched_1d(lib, orc, form):
    """C2: 1024 x 2^16 with one 257-tap filter; sampled rows against the
    oracle (reference radix 4, 2^16 = 4^8) and the whole batch through
    linearity: sum_b (x_b * h) = (sum_b x_b) * h."""
    x, h = W.c2()
    y = P.native_conv(lib, (65536,), 1024, 2, form, x, h)
    tol = {pac.PAC_FORM_F64: P.TOL, pac.PAC_FORM_F32: P.TOL_F32, pac.PAC_FORM_TC: P.TOL_TC}[form]
    for b in (0, 1, 511, 1023):
        z = orc.convolution(O.METHOD_PAC, 4, x[b].real, x[b].imag, h.real, h.imag)
        assert P.crel(y[b], z[0] + 1j * z[1]) < tol
    s = x.sum(axis=0)
    z = orc.convolution(O.METHOD_PAC, 4, s.real, s.imag, h.real, h.imag)
    assert P.crel(y.sum(axis=0), z[0] + 1j * z[1]) < tol * 4


@pytest.mark.parametrize("form", [pac.PAC_FORM_F64, pac.PAC_FORM_F32, pac.PAC_FORM_TC])
def test_c3_2d(lib, orc, form):
    """C3: 2048^2, Gaussian 31x31 filter; oracle at reference radix 2."""
    x, h = W.c3()
    y = P.native_conv(lib, (2048, 2048), 1, 2, form, x, h)[0]
    z = orc.convolution(O.METHOD_PAC, 2, x.real, x.imag, h.real, h.imag)
    tol = {pac.PAC_FORM_F64: P.TOL, pac.PAC_FORM_F32: P.TOL_F32, pac.PAC_FORM_TC: P.TOL_TC}[form]
    assert P.crel(y, z[0] + 1j * z[1]) < tol


def test_c3_dropin_matches_reference_semantics(lib, orc):
    x, h = W.c3()
    y = pac.dropin_convolution(lib, O.METHOD_PAC, 2, x.real, x.imag, h.real, h.imag)
    z = orc.convolution(O.METHOD_PAC, 2, x.real, x.imag, h.real, h.imag)
    assert rel_l2(y[0], y[1], z[0], z[1]) < P.TOL
    assert rel_l2(y[2], y[3], z[2], z[3]) < P.TOL


@pytest.mark.parametrize("shape", [(256, 256, 256), (512, 256, 128)])
def test_c4_3d_f32(lib, shape):
    """C4 in FP32 against an FP64 reference (numpy.fft), plus the impulse
    property at full size: x = delta gives y = h."""
    x, h = W.c4(shape)
    y = P.native_conv(lib, shape, 1, 2, pac.PAC_FORM_F32, x, h)[0]
    z = P.fftconv(x, h, (0, 1, 2))
    assert P.crel(y, z) < P.TOL_F32
    d = np.zeros(shape, np.complex128)
    d[0, 0, 0] = 1.0
    y = P.native_conv(lib, shape, 1, 2, pac.PAC_FORM_F32, d, h)[0]
    assert P.crel(y, h) < P.TOL_F32


@pytest.mark.parametrize("shape", [(64, 128, 32), (256, 256, 256)])
def test_c4_3d_f64_against_oracle(lib, orc, shape):
    """C4 in FP64 against the oracle, at full size too (256^3: the oracle
    takes ~16 s on one core)."""
    x, h = W.c4(shape)
    y = P.native_conv(lib, shape, 1, 2, pac.PAC_FORM_F64, x, h)[0]
    z = orc.convolution(O.METHOD_PAC, 2, x.real, x.imag, h.real, h.imag)
    assert P.crel(y, z[0] + 1j * z[1]) < P.TOL


def test_c5_full_batch(lib, orc):
    """The whole uneven C5 batch (4096 1D and 64 2D problems, 5.5e8
    elements, FP32 form) in one multi-plan call at full size:
    - x = delta in every problem gives y = h in every problem, which checks
      every problem's offsets, levels and plan-order spectrum;
    - random inputs match the oracle on sampled problems: the longest 1D,
      the largest 2D and ten drawn at random."""
    import torch

    dev = torch.device("cuda", 0)
    shapes = W.c5_shapes()
    m = pac.MultiPlan(lib, shapes, 2, pac.PAC_FORM_F32)
    try:
        off = m.offsets
        n = int(off[-1])
        g = torch.Generator(device=dev)
        g.manual_seed(5)
        f32 = dict(dtype=torch.float32, device=dev)
        hr = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
        hi = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
        Hr, Hi = torch.empty(n, **f32), torch.empty(n, **f32)
        m.filter_spectra(hr.data_ptr(), hi.data_ptr(), Hr.data_ptr(), Hi.data_ptr())
        xr, xi = torch.zeros(n, **f32), torch.zeros(n, **f32)
        xr[torch.from_numpy(off[:-1]).to(dev)] = 1.0
        yr, yi = torch.empty(n, **f32), torch.empty(n, **f32)
        m.convolve(xr.data_ptr(), xi.data_ptr(), Hr.data_ptr(), Hi.data_ptr(), yr.data_ptr(),
                   yi.data_ptr())
        torch.cuda.synchronize()
        # per-problem squared error and norm, by cumulative sums at the offsets
        ends = torch.from_numpy(off[1:] - 1).to(dev)

        def per_problem(v):
            c = torch.cumsum(v, 0)[ends]
            return torch.diff(c, prepend=torch.zeros(1, dtype=c.dtype, device=dev))

        err = per_problem((yr.double() - hr) ** 2 + (yi.double() - hi) ** 2)
        ref = per_problem(hr ** 2 + hi ** 2)
        rel = torch.sqrt(err / ref).cpu().numpy()
        assert rel.shape == (len(shapes),)
        assert np.all(rel < P.TOL_F32), (int(np.argmax(rel)), float(rel.max()))
        # random signals, sampled problems against the oracle
        xr.normal_(generator=g)
        xi.normal_(generator=g)
        m.convolve(xr.data_ptr(), xi.data_ptr(), Hr.data_ptr(), Hi.data_ptr(), yr.data_ptr(),
                   yi.data_ptr())
        torch.cuda.synchronize()
        sizes = np.diff(off)
        one = [p for p, s in enumerate(shapes) if len(s) == 1]
        two = [p for p, s in enumerate(shapes) if len(s) == 2]
        pick = {max(one, key=lambda p: sizes[p]), max(two, key=lambda p: sizes[p])}
        pick |= set(rng(17).choice(len(shapes), 10, replace=False).tolist())
        for p in sorted(pick):
            a, b = int(off[p]), int(off[p + 1])
            seg = lambda t: t[a:b].double().cpu().numpy().reshape(shapes[p])  # noqa: E731
            x = seg(xr) + 1j * seg(xi)
            h = seg(hr) + 1j * seg(hi)
            z = orc.convolution(O.METHOD_PAC, 2, x.real, x.imag, h.real, h.imag)
            y = seg(yr) + 1j * seg(yi)
            assert P.crel(y, z[0] + 1j * z[1]) < P.TOL_F32, (p, shapes[p])
    finally:
        m.close()


@pytest.mark.parametrize("dims,batch,base,form,per", [
    ((1024,), 4, 2, 0, False), ((4 ** 7,), 2, 4, 0, True), ((64, 32), 3, 2, 1, False),
    ((2 ** 14,), 2, 2, 1, True), ((16, 16, 16), 2, 4, 1, False), ((8 ** 3,), 2, 8, 0, False), ((1024,), 5, 2, 0, False),
    ((256,), 3, 4, 1, True), ((4096,), 7, 4, 0, False),
    ((2048, 64), 1, 2, 0, False), ((64, 2048), 2, 2, 0, False), ((2048, 32), 1, 2, 1, False),
    ((32, 2048), 2, 2, 1, True),
    # specialised geometries: 256-point rows and columns (FP32 16 lines, FP64 8),
    # 512-point columns and 128-point rows, base-4 4096-point rows and
    # 16-point columns
    ((256, 16, 256), 1, 2, 1, False), ((256, 8, 256), 1, 2, 0, False),
    ((512, 2, 128), 1, 2, 1, False), ((512, 2, 128), 1, 2, 0, False),
    ((2 ** 16,), 2, 4, 0, False), ((2 ** 16,), 2, 4, 1, False),
    ((2 ** 20,), 2, 2, 0, False), ((2 ** 20,), 2, 2, 1, False),
    # fused 4096-point rows (FP64 one line per CTA, FP32 two); 16-point
    # columns of 256-column tiles (2^16 = 16 x 4096, a 16 x 8192 plane)
    ((4096,), 2, 2, 0, False), ((4096,), 4, 2, 1, True), ((16, 4096), 2, 2, 1, False),
    ((2 ** 16,), 8, 2, 0, False), ((2 ** 16,), 8, 2, 1, False), ((16, 8192), 1, 2, 0, False)])
def test_native_conv(lib, dims, batch, base, form, per):
    g = rng(21)
    shape = (batch,) + dims
    x = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    hs = shape if per else dims
    h = g.standard_normal(hs) + 1j * g.standard_normal(hs)
    y = P.native_conv(lib, dims, batch, base, form, x, h, per_problem=per)
    z = P.fftconv(x, h if per else h[None], tuple(range(1, len(shape))))
    assert P.crel(y, z) < (P.TOL if form == 0 else P.TOL_F32)


@pytest.mark.parametrize("op", [pac.OP_AT, pac.OP_A, pac.OP_CONJ_A, pac.OP_FFT, pac.OP_IFFT,
                                pac.OP_UIFFT])
@pytest.mark.parametrize("dims,base", [((4096,), 4), ((2 ** 13,), 2), ((64, 128), 2),
                                       ((2 ** 16,), 4)])
def test_native_transform(lib, orc, op, dims, base):
    g = rng(4)
    x = g.standard_normal((2,) + dims) + 1j * g.standard_normal((2,) + dims)
    y = P.native_transform(lib, dims, 2, base, 0, op, x)
    for b in range(2):
        if op == pac.OP_FFT:
            z = np.fft.fftn(x[b])
        elif op == pac.OP_IFFT:
            z = np.fft.ifftn(x[b])
        else:
            oop = {pac.OP_AT: O.OP_AT, pac.OP_A: O.OP_A, pac.OP_CONJ_A: O.OP_CONJ,
                   pac.OP_UIFFT: O.OP_CONJ}[op]
            zr, zi = orc.butterflies(oop, base, x[b].real, x[b].imag)
            z = (zr + 1j * zi) / (np.prod(dims) if op == pac.OP_UIFFT else 1)
        assert P.crel(y[b], z) < P.TOL


def test_invalid_inputs_leave_data_untouched(lib):
    g = rng(1)
    x = g.standard_normal(48), g.standard_normal(48)
    h = g.standard_normal(48), g.standard_normal(48)
    y = pac.dropin_convolution(lib, 1, 2, *x, *h)
    assert lib.pac_get_last_status() == 2
    assert np.array_equal(y[0], x[0]) and np.array_equal(y[2], h[0])
    x = g.standard_normal(32), g.standard_normal(32)
    y = pac.dropin_butterflies(lib, 2, 4, *x)
    assert lib.pac_get_last_status() == 2 and np.array_equal(y[0], x[0])
    y = pac.dropin_butterflies(lib, 2, 2, *x)
    assert lib.pac_get_last_status() == 0


def test_unsupported_radix_behaviour(lib, orc):
    g = rng(2)
    s = (16, 16)
    x = g.standard_normal(s), g.standard_normal(s)
    h = g.standard_normal(s), g.standard_normal(s)
    y = pac.dropin_convolution(lib, 1, 8, *x, *h)
    z = orc.convolution(1, 8, *x, *h)
    assert rel_l2(y[0], y[1], z[0], z[1]) < 1e-15 and np.array_equal(y[2], h[0])


def test_twiddle_tables(lib, orc):
    for r, n in ((2, 1024), (4, 4096), (8, 512), (4, 2048)):
        a = pac.dropin_twiddles(lib, r, n)
        b = orc.twiddles(r, n)
        assert len(a) == len(b)
        for u, v in zip(a, b):
            assert np.max(np.abs(u - v)) < 2e-15


def test_concurrent_callers(lib, orc):
    """Two host threads on different shapes and one shape shared."""
    errs = []

    def work(shape, r, seed):
        try:
            for k in range(3):
                P.check_against_oracle(lib, orc, shape, r, seed=seed + k, ops=False)
        except AssertionError as e:  # pragma: no cover
            errs.append(e)

    ts = [threading.Thread(target=work, args=a) for a in
          (((4096,), 4, 1), ((64, 64), 2, 2), ((4096,), 4, 3))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs


@pytest.mark.parametrize("dims,base,form", [((2048,), 2, 0), ((2048, 2048), 2, 0),
                                            ((2048, 2048), 2, 1), ((4096,), 4, 1),
                                            ((8 ** 3,), 8, 0), ((16, 16, 16), 2, 1)])
def test_spectrum_orders(lib, dims, base, form):
    P.check_spectrum_orders(lib, dims, 1, base, form)


@pytest.mark.parametrize("kind", P.COLUMN_KERNELS)
@pytest.mark.parametrize("form", [0, 1])
def test_column_kernels(lib, orc, monkeypatch, form, kind):
    P.check_column_kernels(lib, orc, (2048, 32), 2, form, monkeypatch, kind)
    P.check_column_kernels(lib, orc, (2048, 256), 1, form, monkeypatch, kind)
    # more tiles than SMs: persistent CTAs walk several tiles
    P.check_column_kernels(lib, orc, (2048, 2048), 1, form, monkeypatch, kind)



@pytest.mark.parametrize("kind", ["tile", "tma1", "tma2"])
@pytest.mark.parametrize("dims", [(256, 32), (512, 32), (4, 256, 16), (256, 256, 256),
                                  (512, 256, 128)])
@pytest.mark.parametrize("form", [0, 1])
def test_column_kernels_short(lib, orc, monkeypatch, dims, kind, form):
    """256- and 512-point column passes of 64-byte rows (16 FP32 or 8 FP64
    lines; the 3D axes) through the pipelined tensor-copy kernels, at the
    C4 sizes too."""
    if np.prod(dims) > 2 ** 20:
        monkeypatch.setenv("PAC_PLANE", "0")  # every axis as column passes
        monkeypatch.setenv("PAC_COLTMA", "0" if kind == "tile" else kind[3:])
        x, h = W.c4(dims)
        y = P.native_conv(lib, dims, 1, 2, form, x, h)[0]
        tol = P.TOL if form == pac.PAC_FORM_F64 else P.TOL_F32
        assert P.crel(y, P.fftconv(x, h, (0, 1, 2))) < tol
        return
    P.check_column_kernels(lib, orc, dims, 1, form, monkeypatch, kind)


@pytest.mark.parametrize("dims,batch", [((2048, 32), 2), ((2048, 256), 1), ((2048, 2048), 1)])
def test_tc_tcgen05_columns(lib, orc, monkeypatch, dims, batch):
    """Tensor-core form with the column passes' radix-16 steps on tcgen05
    MMAs (tensor memory accumulators, operands in shared memory, one MMA of
    M = 128 butterflies per warpgroup and round) against numpy's FP64 FFT
    convolution and the oracle's butterflies, within the form's tolerance."""
    monkeypatch.setenv("PAC_COLTMA", "1")
    P.check_tc(lib, orc, dims, batch, 2, ops=dims[1] <= 256)


@pytest.mark.parametrize("dims,batch,form,per", [((256, 256, 256), 1, 1, False),
                                                  ((512, 256, 128), 1, 1, False),
                                                  ((8, 256, 256), 3, 1, True),
                                                  ((16, 256, 256), 1, 0, False),
                                                  ((16, 256, 128), 2, 0, False)])
def test_plane_schedule(lib, monkeypatch, dims, batch, form, per):
    """3D plane schedule (cluster kernel, distributed shared memory for the
    outermost axis-1 stage) at the C4 sizes and smaller FP64 shapes, against
    numpy's FP64 FFT."""
    P.check_plane(lib, dims, batch, form, monkeypatch, per_problem=per)


@pytest.mark.parametrize("kind", ["tma1", "tma2", "tma3", "pipe"])
@pytest.mark.parametrize("form", [0, 1])
def test_wait_timeout_reported(lib, monkeypatch, form, kind):
    """A wait limit of 4 SM cycles: every bounded tensor-copy wait of the
    column passes gives up before its copy lands; the kernels report
    PAC_ERROR_TIMEOUT in the plan's status word, let the copies land and
    leave; the device stays usable and the next call is correct."""
    P.check_wait_timeout(lib, form, monkeypatch, kind)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("stream", [False, True])
def test_multi_uneven_batch(lib, form, stream):
    """Uneven batch through one persistent work-queue launch per level; with
    a stream the levels are captured into a CUDA graph and replayed."""
    W5 = W.c5_shapes(48, 6, seed=9)
    shapes = W5 + [(2 ** 20,), (2048, 512), (16, 16, 16), (2,), (128, 4, 64)]
    info = P.check_multi(lib, shapes, form, stream=stream)
    assert info["graph"] == (1 if stream else 0)


@pytest.mark.parametrize("dims,bases,form", [((64, 16, 8), (8, 4, 2), 0), ((512, 64), (8, 4), 1),
                                              ((2 ** 15, 16), (8, 2), 0),
                                              ((512, 256, 128), (8, 4, 2), 1)])
def test_axis_bases(lib, dims, bases, form):
    """One digit base per axis: 512 x 256 x 128 at bases 8, 4, 2 (the
    reference runs it at radix 2 only)."""
    P.check_axis_bases(lib, dims, bases, form, batch=1 if np.prod(dims) > 2 ** 20 else 2)


# Tensor-core form (mma.sync m16n8k16, split FP16 operands): the same shapes
# as the host replay's test, against the FP64 oracle, and against the host
# replay of the same lane code (an MMA modelled from the PTX fragment
# layouts).  Device and replay round differently (MMA accumulation order,
# FMA contraction), each ~2e-7 from the exact result; a fragment placed
# wrongly would differ by O(1).
@pytest.mark.parametrize("dims,batch,base", [
    ((64, 2048), 1, 2), ((2048, 64), 1, 2), ((4096,), 3, 4), ((4096,), 2, 2),
    ((16, 16, 256), 1, 2), ((16, 16), 5, 2), ((16, 16), 3, 4), ((2048, 2048), 1, 2)])
def test_tc_form(lib, emu, orc, dims, batch, base):
    big = int(np.prod(dims)) > 2 ** 20
    P.check_tc(lib, orc, dims, batch, base, ops=not big)
    if big:
        return
    g = rng(9)
    shape = (batch,) + dims
    x = g.uniform(-1, 1, shape) + 1j * g.uniform(-1, 1, shape)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    y = P.native_conv(lib, dims, batch, base, pac.PAC_FORM_TC, x, h)
    e = P.native_conv(emu, dims, batch, base, pac.PAC_FORM_TC, x, h)
    assert P.crel(y, e) < P.TOL_TC
    y32 = P.native_conv(lib, dims, batch, base, pac.PAC_FORM_F32, x, h)
    assert not np.array_equal(y, y32)


def test_tc_form_split_axes(lib, orc, monkeypatch):
    monkeypatch.setenv("PAC_MAX_FACTOR_LOG", "8")
    P.check_tc(lib, orc, (2 ** 16,), 1, 2, ops=True)
    P.check_tc(lib, orc, (256, 1024), 1, 4, ops=False)


@pytest.mark.parametrize("stream", [False, True])
def test_tc_multi(lib, stream):
    shapes = [(256,), (2048, 16), (16, 16, 16), (4096,), (2,), (2048, 2048)]
    P.check_multi(lib, shapes, pac.PAC_FORM_TC, stream=stream)


@pytest.mark.parametrize("shape", [(256, 256, 256), (512, 256, 128)])
def test_c4_3d_tc(lib, shape):
    g = rng(12)
    x = g.uniform(-1, 1, shape) + 1j * g.uniform(-1, 1, shape)
    h = np.zeros(shape, np.complex128)
    h[:8, :8, :8] = g.standard_normal((8, 8, 8))
    y = P.native_conv(lib, shape, 1, 2, pac.PAC_FORM_TC, x, h)[0]
    z = P.fftconv(x, h, (0, 1, 2))
    assert P.crel(y, z) < P.TOL_TC


# Autotuner: every knob set of its search gives the built-in plan's
# convolution on the device (specialised kernels off, radix-8 / radix-4
# schedules, other factor splits and tile widths), and the tuner's cache
# round trip on the device's own timings.
@pytest.mark.parametrize("tune", P.TUNE_CANDIDATES)
@pytest.mark.parametrize("dims,batch,base,form", [
    ((2048, 2048), 1, 2, 1), ((65536,), 4, 2, 0), ((256, 256, 256), 1, 2, 1),
    ((64, 2048), 2, 2, 2), ((4096,), 3, 4, 0), ((65536,), 2, 2, 1),
    ((4096,), 2, 2, 1)])
def test_tuned_plans(lib, dims, batch, base, form, tune):
    P.check_tuned(lib, dims, batch, base, form, tune)


@pytest.mark.parametrize("dims,batch,base,form", [((2048, 2048), 1, 2, 1), ((65536,), 64, 2, 0)])
def test_autotune_cache(lib, tmp_path, dims, batch, base, form):
    P.check_autotune(lib, str(tmp_path / "tune.jsonl"), dims, batch, base, form)


def test_multi_autotune(lib, tmp_path):
    shapes = [(256,), (2048, 64), (4096,), (16, 16, 16), (65536,), (512, 512)]
    cache = str(tmp_path / "tune.jsonl")
    r = pac.multi_autotune(lib, shapes, 2, 1, cache=cache)
    assert r.cached == 0 and r.candidates >= 2 and r.ms <= r.default_ms
    r2 = pac.multi_autotune(lib, shapes, 2, 1, cache=cache)
    assert r2.cached == 1 and r2.tune.as_dict() == r.tune.as_dict()
    P.check_multi(lib, shapes, 1, stream=True, tune=r.tune.as_dict())



@pytest.mark.parametrize("stream", [False, True])
def test_multi_queue_fast_paths(lib, stream):
    """Fused 2048-point rows and 512/256/128-point columns on the compile-time
    bodies inside the work-queue kernel, against numpy per problem; with the
    fast paths turned off (special = -1) the same results."""
    shapes = [(2 ** 18,), (256, 2048), (512, 64), (2048,), (128, 2048), (2 ** 17,), (64, 32),
              (2 ** 20,), (2048, 2048)]
    cap11 = {"max_factor_log": 11, "max_radix_log": 0, "special": 0, "w_shift": 0}
    info = P.check_multi(lib, shapes, 1, stream=stream, tune=cap11)
    assert 0 < info["fast_items"] < sum(info["items"])
    info = P.check_multi(lib, shapes, 1, stream=stream, tune=dict(cap11, special=-1))
    assert info["fast_items"] == 0



def test_fma_peak(lib):
    """pac_fma_peak: plausible B200 figures (FP64 tens of TFLOP/s, FP32 above it)."""
    f64 = pac.fma_peak(lib, 8)
    f32 = pac.fma_peak(lib, 4)
    assert 5.0 < f64 < 200.0 and f32 > f64

"""Host replay of the device passes (TEST-ONLY libpac_emu.so) against the
oracle: the plan layer, the pass geometry, the digit-reversal index maps and
the 4-step twiddles, checked on the CPU with the same code the sm_100a
kernel runs.  The GPU versions of these checks are in test_gpu_parity.py."""
import os

import numpy as np
import pytest

import parity as P
from conftest import O, pac, rel_l2, rng


def test_golden(emu, golden):
    P.check_golden(emu, golden)


@pytest.mark.parametrize("shape,r", [((8192,), 2), ((4 ** 7,), 4), ((8 ** 5,), 8),
                                     ((8192, 4), 2), ((4, 8192), 2), ((16, 64, 16), 4),
                                     ((128, 4, 4), 2), ((1,), 2), ((2,), 2), ((1,), 8)])
def test_oracle_sizes(emu, orc, shape, r):
    P.check_against_oracle(emu, orc, shape, r, ops=np.prod(shape) <= 2 ** 15)


@pytest.mark.parametrize("cap", ["3", "4", "6"])
def test_multi_factor_splits(emu, orc, cap, monkeypatch):
    """Force 2-4 factors per axis (4-step twiddles between every pair, the
    natural-order store across factors)."""
    monkeypatch.setenv("PAC_MAX_FACTOR_LOG", cap)
    for shape, r in [((2 ** 12,), 2), ((4 ** 6,), 4), ((8 ** 4,), 8), ((128, 32), 2),
                     ((16, 64, 32), 2)]:
        if r == 4 and cap == "3":
            continue  # would need more than 4 factors
        P.check_against_oracle(emu, orc, shape, r, seed=int(cap))


@pytest.mark.parametrize("dims,batch,base,form,per", [
    ((1024,), 4, 2, 0, False), ((4 ** 7,), 2, 4, 0, True), ((64, 32), 3, 2, 1, False),
    ((2 ** 14,), 2, 2, 1, True), ((16, 16, 16), 2, 4, 1, False), ((8 ** 3,), 2, 8, 0, False), ((1024,), 5, 2, 0, False),
    ((256,), 3, 4, 1, True), ((4096,), 7, 4, 0, False),
    # geometries served by the specialised kernels (pac_special.h)
    ((2048, 64), 1, 2, 0, False), ((64, 2048), 2, 2, 0, False), ((2048, 32), 1, 2, 1, False),
    ((32, 2048), 2, 2, 1, True),
    # specialised geometries: 256-point rows and columns (FP32 16 lines, FP64 8),
    # 512-point columns and 128-point rows, base-4 4096-point rows and
    # 16-point columns
    ((256, 16, 256), 1, 2, 1, False), ((256, 8, 256), 1, 2, 0, False),
    ((512, 2, 128), 1, 2, 1, False), ((512, 2, 128), 1, 2, 0, False),
    ((2 ** 16,), 2, 4, 0, False), ((2 ** 16,), 2, 4, 1, False),
    # fused 4096-point rows (FP64 one line per CTA, FP32 two); 16-point
    # columns of 256-column tiles (2^16 = 16 x 4096, a 16 x 8192 plane)
    ((4096,), 2, 2, 0, False), ((4096,), 4, 2, 1, True), ((16, 4096), 2, 2, 1, False),
    ((2 ** 16,), 8, 2, 0, False), ((2 ** 16,), 8, 2, 1, False), ((16, 8192), 1, 2, 0, False)])
def test_native_conv(emu, dims, batch, base, form, per):
    g = rng(21)
    shape = (batch,) + dims
    x = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    hs = shape if per else dims
    h = g.standard_normal(hs) + 1j * g.standard_normal(hs)
    y = P.native_conv(emu, dims, batch, base, form, x, h, per_problem=per)
    axes = tuple(range(1, len(shape)))
    z = P.fftconv(x, h if per else h[None], axes)
    tol = P.TOL if form == 0 else P.TOL_F32
    assert P.crel(y, z) < tol


@pytest.mark.parametrize("op", [pac.OP_AT, pac.OP_A, pac.OP_CONJ_A, pac.OP_FFT, pac.OP_IFFT,
                                pac.OP_UIFFT])
@pytest.mark.parametrize("dims,base", [((4096,), 4), ((2 ** 13,), 2), ((64, 128), 2)])
def test_native_transform(emu, orc, op, dims, base):
    g = rng(4)
    x = g.standard_normal((2,) + dims) + 1j * g.standard_normal((2,) + dims)
    y = P.native_transform(emu, dims, 2, base, 0, op, x)
    for b in range(2):
        if op == pac.OP_FFT:
            z = np.fft.fftn(x[b])
        elif op == pac.OP_IFFT:
            z = np.fft.ifftn(x[b])
        else:
            oop = {pac.OP_AT: O.OP_AT, pac.OP_A: O.OP_A, pac.OP_CONJ_A: O.OP_CONJ,
                   pac.OP_UIFFT: O.OP_CONJ}[op]
            zr, zi = orc.butterflies(oop, base, x[b].real, x[b].imag)
            z = zr + 1j * zi
            if op == pac.OP_UIFFT:
                z = z / np.prod(dims)
        assert P.crel(y[b], z) < P.TOL


def test_invalid_size_leaves_data_untouched(emu):
    g = rng(1)
    x = g.standard_normal(48), g.standard_normal(48)
    h = g.standard_normal(48), g.standard_normal(48)
    y = pac.dropin_convolution(emu, 1, 2, *x, *h)
    assert emu.pac_get_last_status() == 2
    assert np.array_equal(y[0], x[0]) and np.array_equal(y[2], h[0])
    # a power of 2 that is not a power of 4
    x = g.standard_normal(32), g.standard_normal(32)
    y = pac.dropin_butterflies(emu, 2, 4, *x)
    assert emu.pac_get_last_status() == 2
    assert np.array_equal(y[0], x[0])
    # success clears nothing but reports success
    y = pac.dropin_butterflies(emu, 2, 2, *x)
    assert emu.pac_get_last_status() == 0


def test_unsupported_radix_matches_reference_behaviour(emu, orc):
    """3D r = 8 and 1D r = 3: the reference skips the butterflies."""
    g = rng(2)
    s = (8, 8, 8)
    x = g.standard_normal(s), g.standard_normal(s)
    h = g.standard_normal(s), g.standard_normal(s)
    y = pac.dropin_convolution(emu, 1, 8, *x, *h)
    z = orc.convolution(1, 8, *x, *h)
    assert rel_l2(y[0], y[1], z[0], z[1]) < 1e-15
    assert np.array_equal(y[2], h[0])
    x = g.standard_normal(9), g.standard_normal(9)
    h = g.standard_normal(9), g.standard_normal(9)
    y = pac.dropin_convolution(emu, 1, 3, *x, *h)
    z = (x[0] + 1j * x[1]) * (h[0] + 1j * h[1]) / 9
    assert P.crel(y[0] + 1j * y[1], z) < 1e-15


def test_twiddle_tables(emu, orc):
    for r, n in ((2, 1024), (4, 4096), (8, 512), (4, 2048)):
        a = pac.dropin_twiddles(emu, r, n)
        b = orc.twiddles(r, n)
        assert len(a) == len(b)
        # the reference evaluates cos/sin of a rounded angle -2*pi*m*j/k, which
        # carries up to ~|angle| * eps; the device tables use the exact
        # fraction 2*m*j/k (sincospi), so they agree to a few 1e-16
        for u, v in zip(a, b):
            assert np.max(np.abs(u - v)) < 2e-15


def test_index_reversal_tables(emu, orc):
    import ctypes as C
    for r, dims in ((2, (64,)), (4, (256,)), (8, (512,)), (2, (8, 32)), (4, (16, 64)),
                    (2, (4, 8, 16)), (4, (16, 4, 64))):
        n = int(np.prod(dims))
        f = getattr(emu, f"precompute_index_reversal_permutation_r{r}"
                    + ("" if len(dims) == 1 else f"_{len(dims)}d"))
        p = f(*dims)
        got = np.ctypeslib.as_array(p, shape=(n,)).copy()
        C.CDLL(None).free(C.cast(p, C.c_void_p))
        assert np.array_equal(got, orc.rho(r, dims))


def test_standalone_permutation(emu, orc):
    g = rng(8)
    n = 1024
    re, im = g.standard_normal(n), g.standard_normal(n)
    rho = orc.rho(4, (n,))
    a, b = re.copy(), im.copy()
    import ctypes as C
    emu.apply_permutation_split(a.ctypes.data_as(C.POINTER(C.c_double)),
                                b.ctypes.data_as(C.POINTER(C.c_double)), n,
                                rho.ctypes.data_as(C.POINTER(C.c_int)))
    assert np.array_equal(a, re[rho]) and np.array_equal(b, im[rho])
    z = np.stack([re, im], axis=1).copy()
    emu.apply_permutation(z.ctypes.data_as(C.POINTER(C.c_double)), n,
                          rho.ctypes.data_as(C.POINTER(C.c_int)))
    assert np.array_equal(z[:, 0], re[rho]) and np.array_equal(z[:, 1], im[rho])


@pytest.mark.parametrize("dims,base,form", [((2048,), 2, 0), ((64, 2048), 2, 0), ((4096,), 4, 1),
                                            ((8 ** 3,), 8, 0), ((16, 16, 16), 2, 1)])
def test_spectrum_orders(emu, dims, base, form):
    P.check_spectrum_orders(emu, dims, 1, base, form)


@pytest.mark.parametrize("kind", P.COLUMN_KERNELS)
@pytest.mark.parametrize("form", [0, 1])
def test_column_kernels(emu, orc, monkeypatch, form, kind):
    """2048-row column passes through every column kernel: the pipelined
    persistent one (its CTAs walk several tiles here: the replay backend
    reports 3 SMs), one-CTA tiles, and tiles shared by 2- and 4-CTA clusters
    (each cluster phase replayed for all ranks in turn)."""
    P.check_column_kernels(emu, orc, (2048, 32), 2, form, monkeypatch, kind)


@pytest.mark.parametrize("kind", ["tile", "tma1", "tma2"])
@pytest.mark.parametrize("dims", [(256, 32), (512, 32), (4, 256, 16)])
@pytest.mark.parametrize("form", [0, 1])
def test_column_kernels_short(emu, orc, monkeypatch, dims, kind, form):
    """256- and 512-point column passes of 64-byte rows (16 FP32 or 8 FP64
    lines; the 3D axes) through the pipelined tensor-copy kernels, with
    tensor stores and with direct stores (tma1 / tma2)."""
    P.check_column_kernels(emu, orc, dims, 1, form, monkeypatch, kind)


@pytest.mark.parametrize("dims,batch", [((2048, 32), 2), ((2048, 8), 1)])
def test_tc_tcgen05_columns(emu, orc, monkeypatch, dims, batch):
    """Tensor-core form with the column passes' radix-16 steps on tcgen05
    MMAs (PAC_COLTMA=1 picks the tensor-copy kernel's tensor-core variant):
    the replay of the A rows, the MMA (modelled from the FP16 halves) and
    the D rows against numpy and the oracle."""
    monkeypatch.setenv("PAC_COLTMA", "1")
    P.check_tc(emu, orc, dims, batch, 2, ops=True)


@pytest.mark.parametrize("dims,batch,form,per", [((2, 256, 256), 1, 1, False),
                                                  ((2, 256, 128), 2, 1, True),
                                                  ((2, 256, 256), 1, 0, False),
                                                  ((2, 256, 128), 1, 0, False)])
def test_plane_schedule(emu, monkeypatch, dims, batch, form, per):
    """3D plane schedule, replayed cluster by cluster, against numpy."""
    P.check_plane(emu, dims, batch, form, monkeypatch, per_problem=per)


@pytest.mark.parametrize("kind", ["tma1", "tma2", "tma3", "pipe"])
@pytest.mark.parametrize("form", [0, 1])
def test_wait_timeout_reported(emu, monkeypatch, form, kind):
    """The replay models a tensor copy as landing 1000 cycles after it is
    issued: a wait limit of 4 cycles gives up, and the status word, its
    read-and-clear and the recovery run through the host plan layer."""
    P.check_wait_timeout(emu, form, monkeypatch, kind)


@pytest.mark.parametrize("form", [0, 1])
def test_multi_uneven_batch(emu, form):
    """Many convolutions of uneven 1D/2D/3D shapes through the work-queue
    levels (replayed item by item)."""
    shapes = [(256,), (1024,), (2 ** 14,), (4096,), (64, 32), (16, 16, 16), (2,), (2048,),
              (32, 64), (256,), (8192, 2)]
    info = P.check_multi(emu, shapes, form)
    assert info["nprob"] == len(shapes) and info["nshapes"] == len(set(shapes))
    # the 3D shape has three factors: 5 passes, the deepest level count
    assert info["nlevels"] == 5 and info["graph"] == 0


@pytest.mark.parametrize("dims,bases,form", [((64, 16, 8), (8, 4, 2), 0), ((64, 16, 8), (8, 4, 2), 1),
                                              ((512, 64), (8, 4), 0), ((32, 8), (2, 8), 1),
                                              ((4096, 16), (4, 2), 0)])
def test_axis_bases(emu, dims, bases, form):
    """One digit base per axis (pac_plan_create_axes)."""
    P.check_axis_bases(emu, dims, bases, form)


# Tensor-core form: the lane code of the split-FP16 radix-16 stages replayed
# lane by lane around an MMA modelled from the PTX fragment layouts.
# Shapes: the specialised 2048-point row (CONV) and 8-line column kernels,
# generic radix-16 stages of base 2 and 4, 3D, and 16-point lines whose
# stages have fewer butterflies than a 16-butterfly tile.
@pytest.mark.parametrize("dims,batch,base", [
    ((64, 2048), 1, 2), ((2048, 64), 1, 2), ((4096,), 3, 4), ((4096,), 2, 2),
    ((16, 16, 256), 1, 2), ((16, 16), 5, 2), ((16, 16), 3, 4)])
def test_tc_form(emu, orc, dims, batch, base):
    errs = P.check_tc(emu, orc, dims, batch, base, ops=int(np.prod(dims)) <= 2 ** 14)
    # the radix-16 stages are on the tensor cores: the error is of the split
    # FP16 products, well above an FP64 path's and at most a few FP32 ulps,
    # and the result is not the FP32 form's
    assert errs["conv"][0] > 1e-12
    g = rng(5)
    shape = (batch,) + dims
    x = g.uniform(-1, 1, shape) + 1j * g.uniform(-1, 1, shape)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    y_tc = P.native_conv(emu, dims, batch, base, pac.PAC_FORM_TC, x, h)
    y_32 = P.native_conv(emu, dims, batch, base, pac.PAC_FORM_F32, x, h)
    assert not np.array_equal(y_tc, y_32)


def test_tc_form_split_axes(emu, orc, monkeypatch):
    """4-step twiddles on tensor-core stages: 2^16 as 256 x 256 factors
    (radix-16 stages next to the 4-step twiddle, DIF post and DIT pre)."""
    monkeypatch.setenv("PAC_MAX_FACTOR_LOG", "8")
    P.check_tc(emu, orc, (2 ** 16,), 1, 2, ops=True)
    P.check_tc(emu, orc, (256, 1024), 1, 4, ops=False)


def test_tc_multi(emu):
    shapes = [(256,), (2048, 16), (16, 16, 16), (4096,), (2,)]
    P.check_multi(emu, shapes, pac.PAC_FORM_TC)


# Autotuner knobs (pac_tune_t): every knob set of the search builds a plan
# whose convolution is the built-in plan's (factor splits, radix-8 and
# radix-4 schedules, generic kernels only, other tile widths), and the
# tuner itself over the replay backend (whose events read the host clock).
@pytest.mark.parametrize("tune", P.TUNE_CANDIDATES)
@pytest.mark.parametrize("dims,batch,base,form", [
    ((4096,), 2, 2, 0), ((64, 2048), 1, 2, 1), ((2048, 32), 1, 2, 2), ((4096,), 1, 4, 1),
    ((16, 32, 64), 2, 2, 0), ((2048, 64), 1, 2, 0), ((32, 2048), 1, 2, 0), ((4096,), 2, 2, 1)])
def test_tuned_plans(emu, dims, batch, base, form, tune):
    P.check_tuned(emu, dims, batch, base, form, tune)


def test_tune_knob_errors(emu):
    with pytest.raises(pac.PacError):
        pac.Plan(emu, (64,), 1, 2, 0, tune={"max_factor_log": 0, "max_radix_log": 5,
                                            "special": 0, "w_shift": 0})
    with pytest.raises(pac.PacError):
        pac.Plan(emu, (64,), 1, 2, 0, tune={"max_factor_log": 0, "max_radix_log": 0,
                                            "special": -2, "w_shift": 0})
    # radix-2 stages of a 2^12 factor: more stages than a pass holds
    with pytest.raises(pac.PacError):
        pac.Plan(emu, (4096,), 1, 2, 0, tune={"max_factor_log": 0, "max_radix_log": 1,
                                              "special": 0, "w_shift": 0})
    plan = pac.Plan(emu, (256,), 1, 2, 0, tune={"max_factor_log": 0, "max_radix_log": 1,
                                                "special": 0, "w_shift": 0})
    plan.close()


def test_autotune_cache(emu, tmp_path):
    P.check_autotune(emu, str(tmp_path / "tune.jsonl"), (1024,), 2, 2, 1)


def test_multi_autotune(emu, tmp_path):
    shapes = [(256,), (64, 32), (1024,), (16, 16, 16)]
    cache = str(tmp_path / "tune.jsonl")
    r = pac.multi_autotune(emu, shapes, 2, 1, cache=cache)
    assert r.cached == 0 and r.candidates >= 2 and r.tune.special == 0
    r2 = pac.multi_autotune(emu, shapes, 2, 1, cache=cache)
    assert r2.cached == 1 and r2.tune.as_dict() == r.tune.as_dict()
    for t in (r.tune.as_dict(), P.TUNE_CANDIDATES[3]):
        P.check_multi(emu, shapes, 1, tune=t)


def test_tune_knobs_take_effect(emu):
    """The factor cap changes the pass count; the radix cap changes the last
    stage radix of the innermost factor, which is the block size of the
    filter spectrum's plan order (pac_filter_spectrum output) -- while the
    convolutions agree (test_tuned_plans)."""
    def knobs(**kw):
        t = {"max_factor_log": 0, "max_radix_log": 0, "special": 0, "w_shift": 0}
        t.update(kw)
        return t
    passes = {}
    for cap in (0, 8, 6, 4):
        plan = pac.Plan(emu, (4096,), 1, 2, 0, tune=knobs(max_factor_log=cap))
        passes[cap] = plan.info().conv_passes
        plan.close()
    assert passes == {0: 1, 8: 3, 6: 3, 4: 5}
    g = rng(3)
    h = g.standard_normal(4096) + 1j * g.standard_normal(4096)
    d = P.Dev(emu)
    try:
        hr, hi = d.put(h.real.copy()), d.put(h.imag.copy())
        outs = []
        for rl in (0, 3):
            plan = pac.Plan(emu, (4096,), 1, 2, 0, tune=knobs(max_radix_log=rl))
            Hr, Hi = d.zeros(4096, np.float64), d.zeros(4096, np.float64)
            plan.filter_spectrum(hr, hi, Hr, Hi)
            outs.append(d.get(Hr, 4096, np.float64) + 1j * d.get(Hi, 4096, np.float64))
            plan.close()
    finally:
        d.free()
    # same values (the P-order spectrum), different plan orders
    assert not np.allclose(outs[0], outs[1])
    assert np.allclose(np.sort_complex(outs[0]), np.sort_complex(outs[1]), atol=1e-12)



# Work-queue fast paths (PAC_QUEUE_LIST): with factors of at most 2^11 these
# shapes put fused 2048-point rows and 512-, 256- and 128-point columns on
# the compile-time bodies inside the queue kernel.
QUEUE_FAST_SHAPES = [(2 ** 18,), (256, 2048), (512, 64), (2048,), (128, 2048), (2 ** 17,), (64, 32)]
CAP11 = {"max_factor_log": 11, "max_radix_log": 0, "special": 0, "w_shift": 0}


def test_multi_queue_fast_paths(emu):
    info = P.check_multi(emu, QUEUE_FAST_SHAPES, 1, tune=CAP11)
    assert 0 < info["fast_items"] < sum(info["items"])
    off = dict(CAP11, special=-1)
    info = P.check_multi(emu, QUEUE_FAST_SHAPES, 1, tune=off)
    assert info["fast_items"] == 0

"""Parity checks shared by the host-replay tests (test_emulated.py, CPU) and
the GPU tests (test_gpu_*.py).  Each check calls the library through its C
ABI and compares with the oracle."""
import ctypes as C

import numpy as np

from conftest import O, pac, rel_l2, rng

TOL = 1e-13  # FP64 forms vs the FP64 oracle (relative L2)
TOL_F32 = 1e-6  # FP32 form vs the FP64 oracle
TOL_TC = 1e-6  # tensor-core form (split FP16 radix-16 stages) vs the FP64 oracle

OPS = ((O.OP_A, "A"), (O.OP_CONJ, "conjA"), (O.OP_AT, "At"))
KINDS = ("fft", "fft2", "ufft", "ifft", "uifft")


def check_golden(L, g):
    """Every drop-in entry point against the reference's own outputs."""
    r = int(g["r"])
    x = (g["x_re"], g["x_im"])
    h = (g["h_re"], g["h_im"])
    errs = {}
    if "At_re" in g:
        for op, name in OPS:
            a = pac.dropin_butterflies(L, op, r, *x)
            errs[name] = rel_l2(*a, g[name + "_re"], g[name + "_im"])
        for k, name in enumerate(KINDS):
            a = pac.dropin_transform(L, k, r, *x, rho=g["rho"])
            errs[name] = rel_l2(*a, g[name + "_re"], g[name + "_im"])
        y = pac.dropin_convolution(L, O.METHOD_FFT_BASED, r, *x, *h, rho=g["rho"])
        errs["fbc"] = rel_l2(y[0], y[1], g["fbc_re"], g["fbc_im"])
        errs["fbc_h"] = rel_l2(y[2], y[3], g["fbc_hre"], g["fbc_him"])
    y = pac.dropin_convolution(L, O.METHOD_PAC, r, *x, *h)
    errs["pac"] = rel_l2(y[0], y[1], g["pac_re"], g["pac_im"])
    errs["pac_h"] = rel_l2(y[2], y[3], g["pac_hre"], g["pac_him"])
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, bad


def check_against_oracle(L, orc, shape, r, seed=0, ops=True):
    g = rng(seed)
    x = (g.standard_normal(shape), g.standard_normal(shape))
    h = (g.standard_normal(shape), g.standard_normal(shape))
    errs = {}
    if ops:
        for op, name in OPS:
            errs[name] = rel_l2(*pac.dropin_butterflies(L, op, r, *x), *orc.butterflies(op, r, *x))
        rho = orc.rho(r, shape)
        for k, name in enumerate(KINDS):
            errs[name] = rel_l2(*pac.dropin_transform(L, k, r, *x, rho=rho),
                                *orc.transform(k, r, *x))
    y = pac.dropin_convolution(L, O.METHOD_PAC, r, *x, *h)
    z = orc.convolution(O.METHOD_PAC, r, *x, *h)
    errs["pac"] = rel_l2(y[0], y[1], z[0], z[1])
    # the overwritten filter is A^T h in P_r order: the index maps must agree
    errs["pac_h"] = rel_l2(y[2], y[3], z[2], z[3])
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, bad


class Dev:
    """Device buffers through the library's own pac_malloc (host memory in
    the emulator build, device memory in the product)."""

    def __init__(self, L):
        self.L = L
        self.ptrs = []

    def put(self, a):
        a = np.ascontiguousarray(a)
        p = C.c_void_p()
        pac.check(self.L, self.L.pac_malloc(C.byref(p), max(a.nbytes, 16)), "pac_malloc")
        self.ptrs.append(p)
        pac.check(self.L, self.L.pac_memcpy_h2d(p, a.ctypes.data, a.nbytes, None), "h2d")
        return p

    def zeros(self, shape, dtype):
        return self.put(np.zeros(shape, dtype))

    def get(self, p, shape, dtype):
        out = np.empty(shape, dtype)
        pac.check(self.L, self.L.pac_memcpy_d2h(out.ctypes.data, p, out.nbytes, None), "d2h")
        pac.check(self.L, self.L.pac_stream_synchronize(None), "sync")
        return out

    def free(self):
        for p in self.ptrs:
            self.L.pac_free(p)
        self.ptrs = []


def native_conv(L, dims, batch, base, form, x, h, per_problem=False, tune=None):
    """pac_filter_spectrum + pac_convolve on host arrays; returns y (complex)."""
    dt = np.float64 if form == pac.PAC_FORM_F64 else np.float32
    d = Dev(L)
    try:
        plan = pac.Plan(L, dims, batch, base, form, tune=tune)
        nf = batch if per_problem else 1
        hshape = (nf,) + tuple(dims)
        hr = d.put(np.real(h).reshape(hshape).astype(np.float64))
        hi = d.put(np.imag(h).reshape(hshape).astype(np.float64))
        Hr, Hi = d.zeros(hshape, dt), d.zeros(hshape, dt)
        plan.filter_spectrum(hr, hi, Hr, Hi, nfilters=nf)
        shape = (batch,) + tuple(dims)
        xr = d.put(np.real(x).reshape(shape).astype(dt))
        xi = d.put(np.imag(x).reshape(shape).astype(dt))
        yr, yi = d.zeros(shape, dt), d.zeros(shape, dt)
        plan.convolve(xr, xi, Hr, Hi, yr, yi, per_problem=1 if per_problem else 0)
        y = d.get(yr, shape, dt) + 1j * d.get(yi, shape, dt)
        plan.close()
        return y
    finally:
        d.free()


def native_transform(L, dims, batch, base, form, op, x):
    dt = np.float64 if form == pac.PAC_FORM_F64 else np.float32
    d = Dev(L)
    try:
        plan = pac.Plan(L, dims, batch, base, form)
        shape = (batch,) + tuple(dims)
        xr = d.put(np.real(x).reshape(shape).astype(dt))
        xi = d.put(np.imag(x).reshape(shape).astype(dt))
        yr, yi = d.zeros(shape, dt), d.zeros(shape, dt)
        plan.transform(op, xr, xi, yr, yi)
        y = d.get(yr, shape, dt) + 1j * d.get(yi, shape, dt)
        plan.close()
        return y
    finally:
        d.free()


def fftconv(x, h, axes):
    return np.fft.ifftn(np.fft.fftn(x, axes=axes) * np.fft.fftn(h, axes=axes), axes=axes)


def crel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def check_spectrum_orders(L, dims, batch, base, form):
    """pac_transform(A^T) + pac_spectrum_to_plan_order equals
    pac_filter_spectrum, and A^T h is P_b F h (the reference's order)."""
    import ctypes as C
    dt = np.float64 if form == pac.PAC_FORM_F64 else np.float32
    g = rng(17)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    d = Dev(L)
    try:
        plan = pac.Plan(L, dims, 1, base, form)
        hr, hi = d.put(np.ascontiguousarray(h.real)), d.put(np.ascontiguousarray(h.imag))
        a_r, a_i = d.zeros(dims, dt), d.zeros(dims, dt)
        plan.filter_spectrum(hr, hi, a_r, a_i, scale=0.5)
        plan64 = pac.Plan(L, dims, 1, base, pac.PAC_FORM_F64)
        p_r, p_i = d.zeros(dims, np.float64), d.zeros(dims, np.float64)
        plan64.transform(pac.OP_AT, hr, hi, p_r, p_i)
        pv = d.get(p_r, dims, np.float64) + 1j * d.get(p_i, dims, np.float64)
        b_r, b_i = d.zeros(dims, dt), d.zeros(dims, dt)
        pac.check(L, L.pac_spectrum_to_plan_order(plan.h, p_r, p_i, 1, b_r, b_i, 0.5, None), "reorder")
        a = d.get(a_r, dims, dt) + 1j * d.get(a_i, dims, dt)
        b = d.get(b_r, dims, dt) + 1j * d.get(b_i, dims, dt)
        # the reorder is a bijection: integer labels (exact in FP32 below
        # 2^24) come out as a permutation of themselves, real and imaginary
        # parts moved together
        n = int(np.prod(dims))
        lab = np.arange(n, dtype=np.float64).reshape(dims)
        q_r, q_i = d.put(lab), d.put(-2.0 * lab)
        pac.check(L, L.pac_spectrum_to_plan_order(plan.h, q_r, q_i, 1, b_r, b_i, 1.0, None), "reorder")
        lr = d.get(b_r, dims, dt).ravel().astype(np.float64)
        li = d.get(b_i, dims, dt).ravel().astype(np.float64)
        plan.close()
        plan64.close()
    finally:
        d.free()
    tol = TOL if form == pac.PAC_FORM_F64 else TOL_F32
    assert crel(a, b) < tol
    assert np.array_equal(np.sort(lr), np.arange(n)) and np.array_equal(li, -2.0 * lr)
    # plan order is a permutation of P order (the reference's order): the
    # multiset of spectrum values is the same
    if form == pac.PAC_FORM_F64:
        assert np.allclose(np.sort_complex(a.ravel()), np.sort_complex(0.5 * pv.ravel()),
                           rtol=tol, atol=tol * np.abs(pv).max())


COLUMN_KERNELS = ("pipe", "tile", "cluster0", "cluster1", "tma1", "tma2", "tma3", "tma4", "tma5",
                  "tma6", "tma7")


def check_column_kernels(L, orc, dims, batch, form, monkeypatch, kind):
    """Column passes served by each column kernel give the oracle's results
    (the convolution, A^T, conj(A) and A): one-CTA tiles ("tile", the
    default), the pipelined persistent kernel ("pipe", PAC_PIPE=1), tiles
    shared by a CTA cluster ("clusterK", PAC_CLUSTER_VARIANT=K), or tiles
    staged by tensor copies ("tmaK", the K-th candidate, PAC_COLTMA=K)."""
    monkeypatch.delenv("PAC_CLUSTER_VARIANT", raising=False)
    monkeypatch.delenv("PAC_PIPE", raising=False)
    monkeypatch.setenv("PAC_COLTMA", "0")
    if kind == "pipe":
        monkeypatch.setenv("PAC_PIPE", "1")
    elif kind.startswith("tma"):
        monkeypatch.setenv("PAC_COLTMA", kind[len("tma"):])
    elif kind.startswith("cluster"):
        monkeypatch.setenv("PAC_CLUSTER_VARIANT", kind[len("cluster"):])
    g = rng(31)
    shape = (batch,) + tuple(dims)
    x = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    tol = TOL if form == pac.PAC_FORM_F64 else TOL_F32
    y = native_conv(L, dims, batch, 2, form, x, h)
    assert crel(y, fftconv(x, h[None], tuple(range(1, len(shape))))) < tol
    for op, oop in ((pac.OP_AT, O.OP_AT), (pac.OP_CONJ_A, O.OP_CONJ), (pac.OP_A, O.OP_A)):
        t = native_transform(L, dims, batch, 2, pac.PAC_FORM_F64, op, x)
        for b in range(batch):
            zr, zi = orc.butterflies(oop, 2, x[b].real, x[b].imag)
            assert crel(t[b], zr + 1j * zi) < TOL


def check_wait_timeout(L, form, monkeypatch, kind="tma1"):
    """Bounded waits: with a wait limit of a few SM cycles every tensor-copy
    wait of the column passes gives up; the call reports PAC_ERROR_TIMEOUT
    through pac_plan_check_status (the device stays usable), and the same
    plan with the default limit convolves correctly afterwards."""
    monkeypatch.setenv("PAC_COLTMA", "0")
    monkeypatch.delenv("PAC_PIPE", raising=False)
    if kind == "pipe":
        monkeypatch.setenv("PAC_PIPE", "1")
    else:
        monkeypatch.setenv("PAC_COLTMA", kind[len("tma"):])
    dims, batch = (2048, 64), 1
    dt = np.float64 if form == pac.PAC_FORM_F64 else np.float32
    g = rng(41)
    x = g.standard_normal((batch,) + dims) + 1j * g.standard_normal((batch,) + dims)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    d = Dev(L)
    try:
        plan = pac.Plan(L, dims, batch, 2, form)
        assert L.pac_plan_check_status(plan.h, None) == 0
        hr, hi = d.put(h.real), d.put(h.imag)
        Hr, Hi = d.zeros(dims, dt), d.zeros(dims, dt)
        plan.filter_spectrum(hr, hi, Hr, Hi)
        xr, xi = d.put(x.real.astype(dt)), d.put(x.imag.astype(dt))
        yr, yi = d.zeros((batch,) + dims, dt), d.zeros((batch,) + dims, dt)
        pac.check(L, L.pac_plan_set_wait_limit(plan.h, 4), "wait limit")
        plan.convolve(xr, xi, Hr, Hi, yr, yi)
        assert L.pac_plan_check_status(plan.h, None) == 8  # PAC_ERROR_TIMEOUT
        assert b"gave up" in L.pac_last_error()
        assert L.pac_plan_check_status(plan.h, None) == 0  # read and cleared
        pac.check(L, L.pac_plan_set_wait_limit(plan.h, 0), "wait limit")
        plan.convolve(xr, xi, Hr, Hi, yr, yi)
        assert L.pac_plan_check_status(plan.h, None) == 0
        y = d.get(yr, (batch,) + dims, dt) + 1j * d.get(yi, (batch,) + dims, dt)
        plan.close()
    finally:
        d.free()
    tol = TOL if form == pac.PAC_FORM_F64 else TOL_F32
    assert crel(y, fftconv(x, h[None], (1, 2))) < tol
    assert L.pac_plan_set_wait_limit(None, 1) == 1  # PAC_ERROR_INVALID_VALUE


def check_plane(L, dims, batch, form, monkeypatch, per_problem=False, seed=8):
    """The plane schedule of a 3D convolution (axes 1 and 2 of every plane in
    one cluster pass: 3 passes) against numpy's FP64 FFT, through the
    environment switch and through the plan knob; the knob plane = -1 keeps
    the line schedule (5 passes)."""
    monkeypatch.setenv("PAC_PLANE", "1")
    g = rng(seed)
    shape = (batch,) + tuple(dims)
    x = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    hs = shape if per_problem else dims
    h = g.standard_normal(hs) + 1j * g.standard_normal(hs)
    z = fftconv(x, h if per_problem else h[None], (1, 2, 3))
    tol = TOL if form == pac.PAC_FORM_F64 else TOL_F32
    y = native_conv(L, dims, batch, 2, form, x, h, per_problem=per_problem)
    assert crel(y, z) < tol
    plan = pac.Plan(L, dims, batch, 2, form)
    assert plan.info().conv_passes == 3
    plan.close()
    monkeypatch.delenv("PAC_PLANE")
    knob = {"max_factor_log": 0, "max_radix_log": 0, "special": 0, "w_shift": 0, "plane": 1}
    y = native_conv(L, dims, batch, 2, form, x, h, per_problem=per_problem, tune=knob)
    assert crel(y, z) < tol
    plan = pac.Plan(L, dims, batch, 2, form, tune=dict(knob, plane=-1))
    assert plan.info().conv_passes == 5
    plan.close()
    return y


def check_multi(L, shapes, form, stream=False, seed=3, tune=None):
    """pac_multi_*: every problem of an uneven batch against numpy's FP64
    FFT convolution; a second call (the CUDA-graph replay when a stream is
    given) repeats the first bit for bit."""
    dt = np.float64 if form == pac.PAC_FORM_F64 else np.float32
    tol = TOL if form == pac.PAC_FORM_F64 else TOL_TC if form == pac.PAC_FORM_TC else TOL_F32
    g = rng(seed)
    m = pac.MultiPlan(L, shapes, 2, form, tune=tune)
    off = m.offsets
    n = int(off[-1])
    xs, hs = [], []
    for s in shapes:
        x = g.standard_normal(s) + 1j * g.standard_normal(s)
        h = np.zeros(s, np.complex128)
        sl = tuple(slice(0, max(1, v // 16)) for v in s)
        h[sl] = g.standard_normal(h[sl].shape) + 1j * g.standard_normal(h[sl].shape)
        xs.append(x)
        hs.append(h)
    xp = np.concatenate([x.ravel() for x in xs])
    hp = np.concatenate([h.ravel() for h in hs])
    d = Dev(L)
    st = None
    try:
        if stream:
            st = C.c_void_p()
            pac.check(L, L.pac_stream_create(C.byref(st)), "stream")
        hr, hi = d.put(hp.real.copy()), d.put(hp.imag.copy())
        Hr, Hi = d.zeros(n, dt), d.zeros(n, dt)
        m.filter_spectra(hr, hi, Hr, Hi, stream=st)
        xr, xi = d.put(xp.real.astype(dt)), d.put(xp.imag.astype(dt))
        yr, yi = d.zeros(n, dt), d.zeros(n, dt)
        m.convolve(xr, xi, Hr, Hi, yr, yi, stream=st)
        if st is not None:
            pac.check(L, L.pac_stream_synchronize(st), "sync")
        y1 = d.get(yr, n, dt) + 1j * d.get(yi, n, dt)
        m.convolve(xr, xi, Hr, Hi, yr, yi, stream=st)
        if st is not None:
            pac.check(L, L.pac_stream_synchronize(st), "sync")
        y2 = d.get(yr, n, dt) + 1j * d.get(yi, n, dt)
        info = m.info()
    finally:
        d.free()
        if st is not None:
            L.pac_stream_destroy(st)
        m.close()
    assert np.array_equal(y1, y2)
    bad = {}
    for p, s in enumerate(shapes):
        y = y1[off[p]:off[p + 1]].reshape(s)
        z = fftconv(xs[p], hs[p], tuple(range(len(s))))
        e = crel(y, z)
        if not e < tol:
            bad[(p, s)] = e
    assert not bad, bad
    return info


def digit_reversal(base, n):
    """index -> its base-`base` digit reversal (n a power of base)"""
    k = int(round(np.log(n) / np.log(base)))
    idx = np.arange(n)
    out = np.zeros(n, dtype=np.int64)
    v = idx.copy()
    for _ in range(k):
        out = out * base + v % base
        v //= base
    return out


def check_axis_bases(L, dims, bases, form, batch=2):
    """Plans with one digit base per axis: the convolution and the natural-
    order FFT against numpy; A^T = P F, A = F P and conj(A) = n F^-1 P with
    P the per-axis digit reversal (every axis in its own base)."""
    g = rng(13)
    shape = (batch,) + tuple(dims)
    x = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    tol = TOL if form == pac.PAC_FORM_F64 else TOL_F32
    axes = tuple(range(1, len(shape)))
    y = native_conv(L, dims, batch, tuple(bases), form, x, h)
    assert crel(y, fftconv(x, h[None], axes)) < tol
    rev = np.ix_(*[digit_reversal(b, n) for b, n in zip(bases, dims)])
    n = int(np.prod(dims))
    for op in (pac.OP_AT, pac.OP_A, pac.OP_CONJ_A, pac.OP_FFT):
        t = native_transform(L, dims, batch, tuple(bases), pac.PAC_FORM_F64, op, x)
        for b in range(batch):
            if op == pac.OP_AT:
                want = np.fft.fftn(x[b])[rev]
            elif op == pac.OP_A:
                want = np.fft.fftn(x[b][rev])
            elif op == pac.OP_CONJ_A:
                want = n * np.fft.ifftn(x[b][rev])
            else:
                want = np.fft.fftn(x[b])
            assert crel(t[b], want) < TOL, (op, b)
    plan = pac.Plan(L, dims, 1, tuple(bases), form)
    info = pac.PlanInfo()
    pac.check(L, L.pac_plan_get_info(plan.h, C.byref(info)), "info")
    plan.close()
    assert list(info.digit_bases[:len(dims)]) == list(bases)


def max_rel(a, b):
    """Largest elementwise error relative to the largest reference magnitude."""
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def check_tc(L, orc, dims, batch, base, seed=5, ops=True):
    """Tensor-core form: convolution against numpy's FP64 FFT convolution and
    the transform operators against the oracle's butterflies; returns the
    relative L2 and max errors of every result."""
    g = rng(seed)
    shape = (batch,) + tuple(dims)
    x = g.uniform(-1, 1, shape) + 1j * g.uniform(-1, 1, shape)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    y = native_conv(L, dims, batch, base, pac.PAC_FORM_TC, x, h)
    z = fftconv(x, h[None], tuple(range(1, len(shape))))
    errs = {"conv": (crel(y, z), max_rel(y, z))}
    if ops:
        for op, oop in ((pac.OP_AT, O.OP_AT), (pac.OP_CONJ_A, O.OP_CONJ)):
            y = native_transform(L, dims, batch, base, pac.PAC_FORM_TC, op, x)
            for b in range(batch):
                zr, zi = orc.butterflies(oop, base, x[b].real, x[b].imag)
                z = zr + 1j * zi
                e = errs.get(op, (0.0, 0.0))
                errs[op] = (max(e[0], crel(y[b], z)), max(e[1], max_rel(y[b], z)))
        y = native_transform(L, dims, batch, base, pac.PAC_FORM_TC, pac.OP_FFT, x)
        z = np.fft.fftn(x, axes=tuple(range(1, len(shape))))
        errs[pac.OP_FFT] = (crel(y, z), max_rel(y, z))
    for k, (l2, mx) in errs.items():
        assert l2 < TOL_TC, (dims, base, k, l2, mx)
    return errs


# knob sets of the autotuner's search (pac_tune_t), each of which must give
# the same convolution as the built-in knobs
TUNE_CANDIDATES = [
    {"max_factor_log": 0, "max_radix_log": 0, "special": -1, "w_shift": 0},
    {"max_factor_log": 0, "max_radix_log": 3, "special": 0, "w_shift": 0},
    {"max_factor_log": 8, "max_radix_log": 0, "special": 0, "w_shift": 0},
    {"max_factor_log": 6, "max_radix_log": 3, "special": 0, "w_shift": 1},
    {"max_factor_log": 0, "max_radix_log": 0, "special": 0, "w_shift": -1},
    {"max_factor_log": 0, "max_radix_log": 2, "special": 0, "w_shift": 2},
    {"max_factor_log": 0, "max_radix_log": 0, "special": 1, "w_shift": 0},
    {"max_factor_log": 0, "max_radix_log": 0, "special": 2, "w_shift": 0},
    {"max_factor_log": 0, "max_radix_log": 0, "special": 3, "w_shift": 0},
    {"max_factor_log": 0, "max_radix_log": 0, "special": 4, "w_shift": 0},
]


def check_tuned(L, dims, batch, base, form, tune, seed=6):
    """A tuned plan's convolution against numpy's FP64 FFT convolution; the
    plan reports the knobs it was built with."""
    g = rng(seed)
    shape = (batch,) + tuple(dims)
    x = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    y = native_conv(L, dims, batch, base, form, x, h, tune=tune)
    z = fftconv(x, h[None], tuple(range(1, len(shape))))
    tol = {pac.PAC_FORM_F64: TOL, pac.PAC_FORM_F32: TOL_F32, pac.PAC_FORM_TC: TOL_TC}[form]
    assert crel(y, z) < tol, (dims, tune, crel(y, z))
    plan = pac.Plan(L, dims, batch, base, form, tune=tune)
    got = plan.info().tune.as_dict()
    plan.close()
    assert got == dict({"plane": 0}, **tune)  # knobs a dict leaves out are 0
    return crel(y, z)


def check_autotune(L, cache, dims, batch, base, form):
    """pac_autotune: a result, appended to the cache as one JSON line and read
    back on the second call without timing; plans made by pac_plan_create
    with PAC_TUNE_CACHE set carry the cached knobs and convolve correctly."""
    import json
    import os
    r1 = pac.autotune(L, dims, batch, base, form, cache=cache)
    assert r1.cached == 0 and r1.candidates >= 3 and r1.ms > 0 and r1.default_ms > 0
    assert r1.ms <= r1.default_ms
    lines = [json.loads(s) for s in open(cache).read().splitlines()]
    assert lines[-1]["max_radix_log"] == r1.tune.max_radix_log
    assert lines[-1]["candidates"] == r1.candidates
    r2 = pac.autotune(L, dims, batch, base, form, cache=cache)
    assert r2.cached == 1 and r2.candidates == 0
    assert r2.tune.as_dict() == r1.tune.as_dict()
    old = os.environ.get("PAC_TUNE_CACHE")
    os.environ["PAC_TUNE_CACHE"] = cache
    try:
        plan = pac.Plan(L, dims, batch, base, form)
        assert plan.info().tune.as_dict() == r1.tune.as_dict()
        plan.close()
        check_tuned(L, dims, batch, base, form, r1.tune.as_dict())
    finally:
        if old is None:
            del os.environ["PAC_TUNE_CACHE"]
        else:
            os.environ["PAC_TUNE_CACHE"] = old
    return r1

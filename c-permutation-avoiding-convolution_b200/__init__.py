"""ctypes binding of the B200 permutation-avoiding FFT convolution library.

The library itself is C/CUDA (``csrc/``, built into ``lib/libpac.so``) with
two C ABIs: the reference-compatible ``fft.h`` (host pointers, identical
prototypes) and the native ``pac.h`` (plans, device pointers, status codes).
This module only loads the shared object and declares argument types; it
does no arithmetic.  The package directory name is not a Python identifier,
so import it with ``importlib.import_module``.

``load()`` returns the product library and raises if it cannot be built or
loaded: there is no fallback.  ``load(emulate=True)`` returns the TEST-ONLY
host replay build (``lib/libpac_emu.so``) used by the CPU test suite.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib", "libpac.so")
LIB_EMU = os.path.join(HERE, "lib", "libpac_emu.so")

PAC_SUCCESS = 0
PAC_FORM_F64, PAC_FORM_F32, PAC_FORM_TC = 0, 1, 2
OP_AT, OP_A, OP_CONJ_A, OP_FFT, OP_IFFT, OP_UFFT, OP_UIFFT = range(7)

_lock = threading.Lock()
_libs: dict = {}

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


def _sources():
    out = [os.path.join(HERE, "Makefile")]
    for d in (os.path.join(HERE, "csrc"), os.path.join(ROOT, "include")):
        out += [os.path.join(d, f) for f in os.listdir(d)]
    return out


def build(emulate=False, force=False):
    """Build lib/libpac.so (and lib/libpac_emu.so with emulate=True) in-tree."""
    target = LIB_EMU if emulate else LIB
    stale = force or not os.path.exists(target) or any(
        os.path.getmtime(s) > os.path.getmtime(target) for s in _sources())
    if stale:
        subprocess.check_call(["make", "-s", "-C", HERE, "-j4", "emu" if emulate else "all"])
    return target


class PacError(RuntimeError):
    pass


def _declare(L):
    i, ll, d, sz = C.c_int, C.c_longlong, C.c_double, C.c_size_t
    L.pac_plan_create.argtypes = [C.POINTER(_vp), i, C.POINTER(i), i, i, i]
    L.pac_plan_create_axes.argtypes = [C.POINTER(_vp), i, C.POINTER(i), C.POINTER(i), i, i]
    L.pac_plan_get_info.argtypes = [_vp, C.POINTER(PlanInfo)]
    L.pac_plan_create_tuned.argtypes = [C.POINTER(_vp), i, C.POINTER(i), C.POINTER(i), i, i,
                                        C.POINTER(Tune)]
    L.pac_autotune.argtypes = [i, C.POINTER(i), C.POINTER(i), i, i, _vp, C.c_char_p,
                               C.POINTER(TuneResult)]
    L.pac_multi_create_tuned.argtypes = [C.POINTER(_vp), i, C.POINTER(i), C.POINTER(i), i, i,
                                         C.POINTER(Tune)]
    L.pac_multi_autotune.argtypes = [i, C.POINTER(i), C.POINTER(i), i, i, _vp, C.c_char_p,
                                     C.POINTER(TuneResult)]
    L.pac_plan_destroy.argtypes = [_vp]
    L.pac_plan_set_wait_limit.argtypes = [_vp, ll]
    L.pac_plan_check_status.argtypes = [_vp, _vp]
    L.pac_filter_spectrum.argtypes = [_vp, _vp, _vp, i, _vp, _vp, d, _vp]
    L.pac_convolve.argtypes = [_vp, _vp, _vp, _vp, _vp, i, _vp, _vp, d, _vp]
    L.pac_spectrum_to_plan_order.argtypes = [_vp, _vp, _vp, i, _vp, _vp, d, _vp]
    L.pac_transform.argtypes = [_vp, i, _vp, _vp, _vp, _vp, _vp]
    if hasattr(L, "pac_convolve_1d_noalloc"):  # product library only
        L.pac_convolve_1d_noalloc.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, i, i, _vp]
    L.pac_pointwise_product.argtypes = [ll, _vp, _vp, _vp, _vp, _vp, _vp, d, _vp]
    L.pac_scale.argtypes = [ll, _vp, _vp, _vp, _vp, d, _vp]
    L.pac_permute.argtypes = [ll, _vp, _vp, _vp, _vp]
    L.pac_reference_twiddles.argtypes = [i, i, _vp, _vp, _vp]
    L.pac_malloc.argtypes = [C.POINTER(_vp), sz]
    L.pac_free.argtypes = [_vp]
    for f in (L.pac_memcpy_h2d, L.pac_memcpy_d2h, L.pac_memcpy_d2d):
        f.argtypes = [_vp, _vp, sz, _vp]
    L.pac_stream_synchronize.argtypes = [_vp]
    L.pac_stream_create.argtypes = [C.POINTER(_vp)]
    L.pac_stream_destroy.argtypes = [_vp]
    L.pac_stream_wait_stream.argtypes = [_vp, _vp]
    L.pac_stream_set_l2_persisting.argtypes = [_vp, _vp, sz]
    L.pac_launch_count.restype = ll
    L.pac_fma_peak.argtypes = [i, _vp, C.POINTER(d)]
    L.pac_multi_create.argtypes = [C.POINTER(_vp), i, C.POINTER(i), C.POINTER(i), i, i]
    L.pac_multi_destroy.argtypes = [_vp]
    L.pac_multi_offsets.argtypes = [_vp, C.POINTER(ll)]
    L.pac_multi_filter_spectra.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.pac_multi_convolve.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.pac_multi_get_info.argtypes = [_vp, C.POINTER(MultiInfo)]
    L.pac_multi_set_level_timing.argtypes = [_vp, i]
    L.pac_status_string.restype = C.c_char_p
    L.pac_status_string.argtypes = [i]
    L.pac_last_error.restype = C.c_char_p
    L.pac_get_last_status.restype = i
    # fft.h: host-pointer drop-in.  Twiddle-table arguments are declared as
    # void pointers (the library never reads them).
    for r in (2, 4, 8):
        for kind in ("", "conjugate_", "transposed_"):
            getattr(L, f"apply_{kind}butterflies_r{r}").argtypes = [_dp, _dp, i, _vp, _vp]
    for r in (2, 4):
        for kind in ("", "conjugate_", "transposed_"):
            getattr(L, f"apply_{kind}butterflies_r{r}_2d").argtypes = [_dp, _dp, i, i] + [_vp] * 4
            getattr(L, f"apply_{kind}butterflies_r{r}_3d").argtypes = [_dp, _dp, i, i, i] + [_vp] * 6
    for name in ("fft", "fft2", "ifft"):
        getattr(L, name).argtypes = [_dp, _dp, i, i, _vp, _vp, _vp]
        getattr(L, name + "_2d").argtypes = [_dp, _dp, i, i, i] + [_vp] * 5
        getattr(L, name + "_3d").argtypes = [_dp, _dp, i, i, i, i] + [_vp] * 7
    for name in ("ufft", "uifft"):
        getattr(L, name).argtypes = [_dp, _dp, i, i, _vp, _vp]
        getattr(L, name + "_2d").argtypes = [_dp, _dp, i, i, i] + [_vp] * 4
        getattr(L, name + "_3d").argtypes = [_dp, _dp, i, i, i, i] + [_vp] * 6
    L.permutation_avoiding_convolution.argtypes = [_dp, _dp, i, i, _vp, _vp, _dp, _dp]
    L.permutation_avoiding_convolution_2d.argtypes = [_dp, _dp, i, i, i] + [_vp] * 4 + [_dp, _dp]
    L.permutation_avoiding_convolution_3d.argtypes = [_dp, _dp, i, i, i, i] + [_vp] * 6 + [_dp, _dp]
    L.fft_based_convolution.argtypes = [_dp, _dp, i, i, _vp, _vp, _vp, _dp, _dp]
    L.fft_based_convolution_2d.argtypes = [_dp, _dp, i, i, i] + [_vp] * 5 + [_dp, _dp]
    L.fft_based_convolution_3d.argtypes = [_dp, _dp, i, i, i, i] + [_vp] * 7 + [_dp, _dp]
    tw = C.POINTER(C.POINTER(_dp))
    for r in (2, 4, 8):
        getattr(L, f"precompute_twiddles_r{r}").argtypes = [i, tw, tw]
        getattr(L, f"precompute_index_reversal_permutation_r{r}").restype = C.POINTER(i)
        getattr(L, f"precompute_index_reversal_permutation_r{r}").argtypes = [i]
        getattr(L, f"reverse_index_r{r}").argtypes = [i, i]
    for r in (2, 4):
        getattr(L, f"precompute_index_reversal_permutation_r{r}_2d").restype = C.POINTER(i)
        getattr(L, f"precompute_index_reversal_permutation_r{r}_2d").argtypes = [i, i]
        getattr(L, f"precompute_index_reversal_permutation_r{r}_3d").restype = C.POINTER(i)
        getattr(L, f"precompute_index_reversal_permutation_r{r}_3d").argtypes = [i, i, i]
    L.free_twiddles.argtypes = [C.POINTER(_dp), C.POINTER(_dp), i]
    L.apply_permutation_split.argtypes = [_dp, _dp, i, C.POINTER(i)]
    L.apply_permutation.argtypes = [_dp, i, C.POINTER(i)]
    L.supports_radix_4.restype = C.c_bool
    L.supports_radix_8.restype = C.c_bool
    return L


def load(emulate=False):
    """Load (building first if needed) the product library, or the test-only
    emulator build with emulate=True."""
    key = "emu" if emulate else "gpu"
    with _lock:
        if key not in _libs:
            path = build(emulate=emulate)
            _libs[key] = _declare(C.CDLL(path))
        return _libs[key]


def check(L, st, what=""):
    if st != PAC_SUCCESS:
        msg = L.pac_last_error().decode(errors="replace")
        raise PacError(f"{what}: {L.pac_status_string(st).decode()} ({msg})")


def _p(a):
    return a.ctypes.data_as(_dp)


# ---------------------------------------------------------------------------
# reference-compatible calls on numpy arrays (host pointers, fft.h)
# ---------------------------------------------------------------------------
def dropin_butterflies(L, op, r, re, im):
    """apply_{,conjugate_,transposed_}butterflies_r{r}{,_2d,_3d} on copies;
    op 0 = A, 1 = conj(A), 2 = A^T (oracle numbering)."""
    re = np.ascontiguousarray(re, dtype=np.float64).copy()
    im = np.ascontiguousarray(im, dtype=np.float64).copy()
    kind = {0: "", 1: "conjugate_", 2: "transposed_"}[op]
    name = f"apply_{kind}butterflies_r{r}"
    if re.ndim > 1:
        name += f"_{re.ndim}d"
    args = [_p(re), _p(im)] + [int(v) for v in re.shape] + [None] * (2 * re.ndim)
    getattr(L, name)(*args)
    return re, im


def dropin_transform(L, kind, r, re, im, rho=None):
    """fft/fft2/ufft/ifft/uifft{,_2d,_3d}; kind 0..4 in that order."""
    re = np.ascontiguousarray(re, dtype=np.float64).copy()
    im = np.ascontiguousarray(im, dtype=np.float64).copy()
    name = ["fft", "fft2", "ufft", "ifft", "uifft"][kind]
    nd = re.ndim
    if nd > 1:
        name += f"_{nd}d"
    args = [_p(re), _p(im)] + [int(v) for v in re.shape] + [r] + [None] * (2 * nd)
    if kind in (0, 1, 3):
        rp = None
        if rho is not None:
            rho = np.ascontiguousarray(rho, dtype=np.int32)
            rp = rho.ctypes.data_as(C.POINTER(C.c_int))
        args.append(rp)
    getattr(L, name)(*args)
    return re, im


def dropin_convolution(L, method, r, re, im, h_re, h_im, rho=None):
    """permutation_avoiding_convolution* (method 1) or fft_based_convolution*
    (method 0) on copies; returns (y_re, y_im, h_re_out, h_im_out)."""
    re = np.ascontiguousarray(re, dtype=np.float64).copy()
    im = np.ascontiguousarray(im, dtype=np.float64).copy()
    hr = np.ascontiguousarray(h_re, dtype=np.float64).copy()
    hi = np.ascontiguousarray(h_im, dtype=np.float64).copy()
    nd = re.ndim
    name = ["fft_based_convolution", "permutation_avoiding_convolution"][method]
    if nd > 1:
        name += f"_{nd}d"
    args = [_p(re), _p(im)] + [int(v) for v in re.shape] + [r] + [None] * (2 * nd)
    if method == 0:
        rp = None
        if rho is not None:
            rho = np.ascontiguousarray(rho, dtype=np.int32)
            rp = rho.ctypes.data_as(C.POINTER(C.c_int))
        args.append(rp)
    args += [_p(hr), _p(hi)]
    getattr(L, name)(*args)
    return re, im, hr, hi


def dropin_twiddles(L, r, n):
    """precompute_twiddles_r{r}(n) -> list of complex arrays per level."""
    pr = C.POINTER(_dp)()
    pi = C.POINTER(_dp)()
    getattr(L, f"precompute_twiddles_r{r}")(n, C.byref(pr), C.byref(pi))
    t, v = 0, n
    if r == 2:
        while not (n >> t) & 1:
            t += 1
    else:
        sh = {4: 2, 8: 3}[r]
        while v > 1:
            v >>= sh
            t += 1
    out = []
    for q in range(t):
        cnt = (r - 1) * r ** q
        a = np.ctypeslib.as_array(pr[q], shape=(cnt,)).copy()
        b = np.ctypeslib.as_array(pi[q], shape=(cnt,)).copy()
        out.append(a + 1j * b)
    L.free_twiddles(pr, pi, t)
    return out


# ---------------------------------------------------------------------------
# native plan API (device pointers)
# ---------------------------------------------------------------------------
class Tune(C.Structure):
    """pac_tune_t: plan knobs (0 everywhere = the built-in choices)"""
    _fields_ = [("max_factor_log", C.c_int), ("max_radix_log", C.c_int), ("special", C.c_int),
                ("w_shift", C.c_int), ("plane", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneResult(C.Structure):
    """pac_tune_result_t"""
    _fields_ = [("tune", Tune), ("ms", C.c_double), ("default_ms", C.c_double),
                ("candidates", C.c_int), ("cached", C.c_int)]


def _tune(t):
    if t is None or isinstance(t, Tune):
        return t
    return Tune(**t)


class PlanInfo(C.Structure):
    """pac_plan_info_t"""
    _fields_ = [("n_elements", C.c_longlong), ("batch", C.c_longlong), ("rank", C.c_int),
                ("dims", C.c_int * 3), ("digit_base", C.c_int), ("form", C.c_int),
                ("element_bytes", C.c_int), ("conv_passes", C.c_int),
                ("transform_passes", C.c_int), ("workspace_bytes", C.c_size_t),
                ("digit_bases", C.c_int * 3), ("tune", Tune)]


def _bases(dims, digit_base):
    if isinstance(digit_base, (tuple, list)):
        return list(digit_base)
    return [digit_base] * len(dims)


def autotune(L, dims, batch=1, digit_base=2, form=PAC_FORM_F64, stream=None, cache=None):
    """pac_autotune: the fastest knobs for one problem (read from `cache`, a
    JSON-lines file, when it holds them; appended to it otherwise)."""
    r = TuneResult()
    arr = (C.c_int * len(dims))(*dims)
    bases = (C.c_int * len(dims))(*_bases(dims, digit_base))
    check(L, L.pac_autotune(len(dims), arr, bases, batch, form, stream,
                            cache.encode() if cache else None, C.byref(r)), "pac_autotune")
    return r


def fma_peak(L, elem_bytes=8, stream=None):
    """pac_fma_peak: measured FMA throughput of the device in TFLOP/s."""
    v = C.c_double()
    check(L, L.pac_fma_peak(elem_bytes, stream, C.byref(v)), "pac_fma_peak")
    return v.value


def multi_autotune(L, shapes, digit_base=2, form=PAC_FORM_F32, stream=None, cache=None):
    """pac_multi_autotune: one knob set for a whole uneven batch."""
    r = TuneResult()
    n = len(shapes)
    ranks = (C.c_int * n)(*[len(s) for s in shapes])
    dims = (C.c_int * (3 * n))(*[v for s in shapes for v in (tuple(s) + (1, 1, 1))[:3]])
    check(L, L.pac_multi_autotune(n, ranks, dims, digit_base, form, stream,
                                  cache.encode() if cache else None, C.byref(r)),
          "pac_multi_autotune")
    return r


class MultiInfo(C.Structure):
    _fields_ = [("nprob", C.c_int), ("nshapes", C.c_int), ("nlevels", C.c_int),
                ("items", C.c_longlong * 8), ("elements", C.c_longlong), ("graph", C.c_int),
                ("level_ms", C.c_double * 8), ("timed_calls", C.c_longlong),
                ("fast_items", C.c_longlong)]


class MultiPlan:
    """pac.h multi-plan: many convolutions of uneven shapes per call, over
    packed split arrays (problem p at elements offsets[p]:offsets[p+1])."""

    def __init__(self, L, shapes, digit_base=2, form=PAC_FORM_F32, tune=None):
        self.L = L
        self.h = _vp()
        n = len(shapes)
        ranks = (C.c_int * n)(*[len(s) for s in shapes])
        dims = (C.c_int * (3 * n))(*[v for s in shapes for v in (tuple(s) + (1, 1, 1))[:3]])
        t = _tune(tune)
        if t is not None:
            check(L, L.pac_multi_create_tuned(C.byref(self.h), n, ranks, dims, digit_base, form,
                                              C.byref(t)), "pac_multi_create_tuned")
        else:
            check(L, L.pac_multi_create(C.byref(self.h), n, ranks, dims, digit_base, form),
                  "pac_multi_create")
        off = (C.c_longlong * (n + 1))()
        check(L, L.pac_multi_offsets(self.h, off), "pac_multi_offsets")
        self.offsets = np.array(off[:], dtype=np.int64)
        self.shapes = [tuple(s) for s in shapes]
        self.form = form

    def filter_spectra(self, h_re, h_im, hhat_re, hhat_im, stream=None):
        check(self.L, self.L.pac_multi_filter_spectra(self.h, h_re, h_im, hhat_re, hhat_im, stream),
              "pac_multi_filter_spectra")

    def convolve(self, x_re, x_im, hhat_re, hhat_im, y_re, y_im, stream=None):
        check(self.L, self.L.pac_multi_convolve(self.h, x_re, x_im, hhat_re, hhat_im, y_re, y_im,
                                                stream), "pac_multi_convolve")

    def info(self):
        inf = MultiInfo()
        check(self.L, self.L.pac_multi_get_info(self.h, C.byref(inf)), "pac_multi_get_info")
        return {"nprob": inf.nprob, "nshapes": inf.nshapes, "nlevels": inf.nlevels,
                "items": list(inf.items[:inf.nlevels]), "elements": inf.elements,
                "graph": inf.graph, "level_ms": list(inf.level_ms[:inf.nlevels]),
                "timed_calls": inf.timed_calls, "fast_items": inf.fast_items}

    def set_level_timing(self, enable):
        check(self.L, self.L.pac_multi_set_level_timing(self.h, 1 if enable else 0),
              "pac_multi_set_level_timing")

    def close(self):
        if self.h:
            self.L.pac_multi_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """pac.h plan; device pointers are passed as integers."""

    def __init__(self, L, dims, batch=1, digit_base=2, form=PAC_FORM_F64, tune=None):
        self.L = L
        self.h = _vp()
        arr = (C.c_int * len(dims))(*dims)
        t = _tune(tune)
        if t is not None:  # explicit knobs (pac_tune_t)
            bases = (C.c_int * len(dims))(*_bases(dims, digit_base))
            check(L, L.pac_plan_create_tuned(C.byref(self.h), len(dims), arr, bases, batch, form,
                                             C.byref(t)), "pac_plan_create_tuned")
        elif isinstance(digit_base, (tuple, list)):  # one digit base per axis
            bases = (C.c_int * len(dims))(*digit_base)
            check(L, L.pac_plan_create_axes(C.byref(self.h), len(dims), arr, bases, batch, form),
                  "pac_plan_create_axes")
        else:
            check(L, L.pac_plan_create(C.byref(self.h), len(dims), arr, batch, digit_base, form),
                  "pac_plan_create")
        self.dims = tuple(dims)
        self.batch = batch
        self.form = form

    def filter_spectrum(self, h_re, h_im, hhat_re, hhat_im, nfilters=1, scale=None, stream=None):
        n = int(np.prod(self.dims))
        sc = 1.0 / n if scale is None else scale
        check(self.L, self.L.pac_filter_spectrum(self.h, h_re, h_im, nfilters, hhat_re, hhat_im,
                                                 sc, stream), "pac_filter_spectrum")

    def convolve(self, x_re, x_im, hhat_re, hhat_im, y_re, y_im, per_problem=0, scale=1.0,
                 stream=None):
        check(self.L, self.L.pac_convolve(self.h, x_re, x_im, hhat_re, hhat_im, per_problem, y_re,
                                          y_im, scale, stream), "pac_convolve")

    def transform(self, op, in_re, in_im, out_re, out_im, stream=None):
        check(self.L, self.L.pac_transform(self.h, op, in_re, in_im, out_re, out_im, stream),
              "pac_transform")

    def info(self):
        inf = PlanInfo()
        check(self.L, self.L.pac_plan_get_info(self.h, C.byref(inf)), "pac_plan_get_info")
        return inf

    def close(self):
        if self.h:
            self.L.pac_plan_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

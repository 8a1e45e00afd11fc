"""ctypes front end of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Two back ends with one Python surface:

* ``Orc``  -- the C restatement ``oracle/pac_oracle.c`` (``liborc.so``),
  available everywhere the repository is (it is rebuilt from source on
  demand with gcc).
* ``Ref``  -- the reference library compiled from the reference's own
  sources (``oracle/_ref/libref.so``, recipe in ``oracle/Makefile``),
  available where it was built.

Only ``tests/``, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
``bench.py`` import this module.  The GPU library never does.

All arrays are float64 numpy arrays, row-major, last axis contiguous; complex
data is split into separate real and imaginary arrays as in the reference.
Every wrapper works in place on copies and returns new arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()

OP_A, OP_CONJ, OP_AT = 0, 1, 2
KIND_FFT, KIND_FFT2, KIND_UFFT, KIND_IFFT, KIND_UIFFT = 0, 1, 2, 3, 4
METHOD_FFT_BASED, METHOD_PAC = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _dims(dims):
    arr = (C.c_int * len(dims))(*dims)
    return arr


def build_orc(force=False):
    """Compile liborc.so from pac_oracle.c when it is missing or stale."""
    so = os.path.join(HERE, "liborc.so")
    src = os.path.join(HERE, "pac_oracle.c")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O3", "-march=x86-64-v3", "-fno-fast-math", "-fPIC", "-shared",
             "-o", so, src, "-lm"])
    return so


def ref_source_dir():
    """The reference's source directory: the environment variable PAC_REF_DIR
    (unset: none -- the checkers that need it are skipped)."""
    d = os.environ.get("PAC_REF_DIR")
    return d if d and os.path.isdir(d) else None


def build_ref(ref_dir=None):
    """Compile the reference sources into _ref/ (only where they exist)."""
    ref_dir = ref_dir or ref_source_dir()
    if not ref_dir or not os.path.isdir(ref_dir):
        return None
    subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF_DIR={ref_dir}"])
    return os.path.join(HERE, "_ref", "libref.so")


class Orc:
    """The C restatement of the reference algorithms."""

    def __init__(self):
        with _lock:
            so = build_orc()
        L = C.CDLL(so)
        L.orc_levels.restype = C.c_int
        L.orc_levels.argtypes = [C.c_int, C.c_int]
        L.orc_butterflies_nd.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip]
        L.orc_transform_nd.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip]
        L.orc_convolution_nd.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _dp, _dp]
        L.orc_rho.argtypes = [C.c_int, C.c_int, _ip, _ip]
        L.orc_naive_circular_conv.argtypes = [_dp, _dp, _dp, _dp, C.c_int, _ip, _dp, _dp]
        L.orc_max_error.restype = C.c_double
        L.orc_max_error.argtypes = [_dp, _dp, _dp, _dp, C.c_long]
        L.orc_twiddles.argtypes = [C.c_int, C.c_int, C.POINTER(C.POINTER(_dp)),
                                   C.POINTER(C.POINTER(_dp))]
        L.orc_free_twiddles.argtypes = [C.POINTER(_dp), C.POINTER(_dp), C.c_int]
        self.lib = L

    # -- helpers ---------------------------------------------------------
    @staticmethod
    def _prep(re, im):
        re = np.ascontiguousarray(re, dtype=np.float64).copy()
        im = np.ascontiguousarray(im, dtype=np.float64).copy()
        return re, im

    def levels(self, n, r):
        return self.lib.orc_levels(n, r)

    def butterflies(self, op, r, re, im):
        """A (op 0), conj(A) (op 1) or A^T (op 2) along every axis."""
        re, im = self._prep(re, im)
        d = re.shape
        self.lib.orc_butterflies_nd(op, r, _ptr(re), _ptr(im), len(d), _dims(d))
        return re, im

    def transform(self, kind, r, re, im):
        re, im = self._prep(re, im)
        d = re.shape
        self.lib.orc_transform_nd(kind, r, _ptr(re), _ptr(im), len(d), _dims(d))
        return re, im

    def convolution(self, method, r, re, im, h_re, h_im):
        """Returns (y_re, y_im, h_re_out, h_im_out) like the reference call."""
        re, im = self._prep(re, im)
        hr, hi = self._prep(h_re, h_im)
        d = re.shape
        self.lib.orc_convolution_nd(method, r, _ptr(re), _ptr(im), len(d), _dims(d),
                                    _ptr(hr), _ptr(hi))
        return re, im, hr, hi

    def rho(self, r, dims):
        n = int(np.prod(dims))
        out = np.empty(n, dtype=np.int32)
        self.lib.orc_rho(r, len(dims), _dims(dims), out.ctypes.data_as(_ip))
        return out

    def naive_conv(self, xr, xi, hr, hi):
        xr, xi = self._prep(xr, xi)
        hr, hi = self._prep(hr, hi)
        yr = np.empty_like(xr)
        yi = np.empty_like(xi)
        d = xr.shape
        self.lib.orc_naive_circular_conv(_ptr(xr), _ptr(xi), _ptr(hr), _ptr(hi), len(d),
                                         _dims(d), _ptr(yr), _ptr(yi))
        return yr, yi

    def twiddles(self, r, n):
        """Reference-layout twiddle tables as a list of complex arrays."""
        pr = C.POINTER(_dp)()
        pi = C.POINTER(_dp)()
        self.lib.orc_twiddles(r, n, C.byref(pr), C.byref(pi))
        t = self.levels(n, r)
        out = []
        for q in range(t):
            cnt = (r - 1) * r ** q
            a = np.ctypeslib.as_array(pr[q], shape=(cnt,)).copy()
            b = np.ctypeslib.as_array(pi[q], shape=(cnt,)).copy()
            out.append(a + 1j * b)
        self.lib.orc_free_twiddles(pr, pi, t)
        return out


class Ref:
    """The reference library itself, compiled from its sources."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "_ref", "libref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        tw_t = C.POINTER(C.POINTER(_dp))
        for r in (2, 4, 8):
            getattr(self.lib, f"precompute_twiddles_r{r}").argtypes = [C.c_int, tw_t, tw_t]
            getattr(self.lib, f"precompute_index_reversal_permutation_r{r}").restype = _ip
        self.lib.free_twiddles.argtypes = [C.POINTER(_dp), C.POINTER(_dp), C.c_int]
        self.lib.free.argtypes = [C.c_void_p]

    def _tw(self, r, n):
        pr = C.POINTER(_dp)()
        pi = C.POINTER(_dp)()
        getattr(self.lib, f"precompute_twiddles_r{r}")(n, C.byref(pr), C.byref(pi))
        return pr, pi

    def _levels(self, r, n):
        t, v = 0, n
        if r == 2:
            while not (n >> t) & 1:
                t += 1
            return t
        sh = {4: 2, 8: 3}[r]
        while v > 1:
            v >>= sh
            t += 1
        return t

    def _tables(self, r, dims):
        tabs = [self._tw(r if r in (2, 4, 8) else 2, n) for n in dims]
        return tabs

    def _free(self, r, dims, tabs):
        rr = r if r in (2, 4, 8) else 2
        for n, (pr, pi) in zip(dims, tabs):
            self.lib.free_twiddles(pr, pi, self._levels(rr, n))

    def butterflies(self, op, r, re, im):
        re, im = Orc._prep(re, im)
        dims = re.shape
        name = {OP_A: "apply_butterflies", OP_CONJ: "apply_conjugate_butterflies",
                OP_AT: "apply_transposed_butterflies"}[op] + f"_r{r}"
        if len(dims) > 1:
            name += f"_{len(dims)}d"
        tabs = self._tables(r, dims)
        args = [_ptr(re), _ptr(im)] + [C.c_int(n) for n in dims]
        for pr, pi in tabs:
            args += [pr, pi]
        getattr(self.lib, name)(*args)
        self._free(r, dims, tabs)
        return re, im

    def rho(self, r, dims):
        n = int(np.prod(dims))
        if len(dims) == 1:
            p = getattr(self.lib, f"precompute_index_reversal_permutation_r{r}")(n)
        else:
            f = getattr(self.lib, f"precompute_index_reversal_permutation_r{r}_{len(dims)}d")
            f.restype = _ip
            p = f(*[C.c_int(v) for v in dims])
        out = np.ctypeslib.as_array(p, shape=(n,)).copy()
        self.lib.free(C.cast(p, C.c_void_p))
        return out

    def transform(self, kind, r, re, im):
        re, im = Orc._prep(re, im)
        dims = re.shape
        name = ["fft", "fft2", "ufft", "ifft", "uifft"][kind]
        if len(dims) > 1:
            name += f"_{len(dims)}d"
        rr = r if r in (2, 4, 8) else 2
        tabs = self._tables(r, dims)
        args = [_ptr(re), _ptr(im)] + [C.c_int(n) for n in dims] + [C.c_int(r)]
        for pr, pi in tabs:
            args += [pr, pi]
        rho = None
        if kind in (KIND_FFT, KIND_FFT2, KIND_IFFT):
            if len(dims) == 1:
                rho = getattr(self.lib, f"precompute_index_reversal_permutation_r{rr}")(dims[0])
            else:
                f = getattr(self.lib, f"precompute_index_reversal_permutation_r{rr}_{len(dims)}d")
                f.restype = _ip
                rho = f(*[C.c_int(v) for v in dims])
            args.append(rho)
        getattr(self.lib, name)(*args)
        if rho is not None:
            self.lib.free(C.cast(rho, C.c_void_p))
        self._free(r, dims, tabs)
        return re, im

    def convolution(self, method, r, re, im, h_re, h_im):
        re, im = Orc._prep(re, im)
        hr, hi = Orc._prep(h_re, h_im)
        dims = re.shape
        rr = r if r in (2, 4, 8) else 2
        name = ["fft_based_convolution", "permutation_avoiding_convolution"][method]
        if len(dims) > 1:
            name += f"_{len(dims)}d"
        tabs = self._tables(r, dims)
        args = [_ptr(re), _ptr(im)] + [C.c_int(n) for n in dims] + [C.c_int(r)]
        for pr, pi in tabs:
            args += [pr, pi]
        rho = None
        if method == METHOD_FFT_BASED:
            if len(dims) == 1:
                rho = getattr(self.lib, f"precompute_index_reversal_permutation_r{rr}")(dims[0])
            else:
                f = getattr(self.lib, f"precompute_index_reversal_permutation_r{rr}_{len(dims)}d")
                f.restype = _ip
                rho = f(*[C.c_int(v) for v in dims])
            args.append(rho)
        args += [_ptr(hr), _ptr(hi)]
        getattr(self.lib, name)(*args)
        if rho is not None:
            self.lib.free(C.cast(rho, C.c_void_p))
        self._free(r, dims, tabs)
        return re, im, hr, hi


def rel_l2(a_re, a_im, b_re, b_im):
    """||a - b||_2 / ||b||_2 over complex split arrays."""
    num = np.sqrt(np.sum((np.asarray(a_re) - b_re) ** 2 + (np.asarray(a_im) - b_im) ** 2))
    den = np.sqrt(np.sum(np.asarray(b_re) ** 2 + np.asarray(b_im) ** 2))
    return float(num / den) if den > 0 else float(num)


def max_abs(a_re, a_im, b_re, b_im):
    """max_i |a_i - b_i| by hypot, the reference's error metric (misc.c:20-30)."""
    return float(np.max(np.hypot(np.asarray(a_re) - b_re, np.asarray(a_im) - b_im)))

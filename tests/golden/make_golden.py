"""Generate the golden vectors in this directory from the reference itself.

The reference publishes no golden vectors or known-answer tests, so the
fixtures are produced by running the reference library, compiled from its
own sources by ``oracle/Makefile`` (target ``ref``), on seeded inputs.

Run from the repository root where the reference sources are present:

    python tests/golden/make_golden.py REF_DIR   (or PAC_REF_DIR=... python ...)

Each case (shape, radix) is one ``.npz`` holding the inputs and every
output of the path: the three butterfly operators (A, conj(A), A^T), the
five transforms (fft, fft2, ufft, ifft, uifft), both convolutions with the
overwritten filter, and the digit-reversal map.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# (shape, radix): 1D pure powers of 2/4/8, isotropic and anisotropic 2D/3D
# (the n1 x 4 and n1 x 4 x 4 shapes of the reference's anisotropic benches),
# and one unsupported radix (2D r = 8: the reference skips the butterflies).
CASES = [
    ((64,), 2), ((64,), 4), ((64,), 8),
    ((256,), 2), ((256,), 4),
    ((512,), 8),
    ((16, 16), 2), ((16, 16), 4), ((16, 16), 8),
    ((8, 32), 2),
    ((64, 4), 2), ((64, 4), 4),
    ((8, 8, 8), 2),
    ((4, 16, 4), 2), ((4, 16, 4), 4),
    ((16, 4, 4), 2), ((16, 4, 4), 4),
]


def case_name(shape, r):
    return "g_" + "x".join(str(s) for s in shape) + f"_r{r}.npz"


def make(ref_dir):
    if not O.build_ref(ref_dir):
        raise SystemExit(f"no reference sources at {ref_dir!r}")
    ref = O.Ref()
    for idx, (shape, r) in enumerate(CASES):
        rng = np.random.default_rng(1000 + idx)
        xr, xi = rng.standard_normal(shape), rng.standard_normal(shape)
        hr, hi = rng.standard_normal(shape), rng.standard_normal(shape)
        out = dict(shape=np.array(shape), r=np.array(r), x_re=xr, x_im=xi, h_re=hr, h_im=hi)
        supported = r in ((2, 4, 8) if len(shape) == 1 else (2, 4))
        if supported:
            for op, name in ((O.OP_A, "A"), (O.OP_CONJ, "conjA"), (O.OP_AT, "At")):
                a, b = ref.butterflies(op, r, xr, xi)
                out[name + "_re"], out[name + "_im"] = a, b
            for kind, name in enumerate(("fft", "fft2", "ufft", "ifft", "uifft")):
                a, b = ref.transform(kind, r, xr, xi)
                out[name + "_re"], out[name + "_im"] = a, b
            out["rho"] = ref.rho(r, shape).astype(np.int32)
        y = ref.convolution(O.METHOD_PAC, r, xr, xi, hr, hi)
        out["pac_re"], out["pac_im"], out["pac_hre"], out["pac_him"] = y
        if supported:
            y = ref.convolution(O.METHOD_FFT_BASED, r, xr, xi, hr, hi)
            out["fbc_re"], out["fbc_im"], out["fbc_hre"], out["fbc_him"] = y
        np.savez_compressed(os.path.join(HERE, case_name(shape, r)), **out)
        print("wrote", case_name(shape, r))


if __name__ == "__main__":
    # the reference's source directory: the first argument, else PAC_REF_DIR
    src = sys.argv[1] if len(sys.argv) > 1 else O.ref_source_dir()
    if not src:
        raise SystemExit("usage: make_golden.py REF_DIR (or set PAC_REF_DIR)")
    make(src)

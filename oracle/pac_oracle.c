/*
 * pac_oracle.c -- CPU restatement of the reference's permutation-avoiding
 * convolution path.  TEST INFRASTRUCTURE ONLY: the GPU library never links,
 * loads or calls this file.  It is the checker used by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline leg of bench.py.
 *
 * Every function restates an algorithm of venkovic/c-permutation-avoiding-
 * convolution (file:line cited per function, paths relative to that
 * project).  The restatement is written generically over the radix r: one
 * stage is "twiddle, then an r-point DFT" (A, conj(A)) or "r-point DFT, then
 * twiddle" (A^T), which is what the hand-expanded radix-2/4/8 kernels of
 * butterflies.c compute.  Arithmetic is IEEE FP64, split re/im arrays,
 * row-major multi-D arrays with the last axis contiguous -- the reference's
 * data layout.
 *
 * Pinning: tests/test_oracle.py checks this file against the reference
 * itself (oracle/_ref/libref.so, compiled from the reference sources by
 * oracle/Makefile) and against golden vectors that the reference produced
 * (tests/golden/, made by tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* --------------------------------------------------------------------- */
/* Stage count t for n and radix r.                                        */
/* r == 2: count of trailing zero bits (butterflies.c:14).                 */
/* r == 4, 8: the shift-until-1 loop (butterflies.c:101-106, :282-287).    */
/* --------------------------------------------------------------------- */
int orc_levels(int n, int r) {
  if (n <= 0) return 0;
  if (r == 2) {
    int t = 0;
    while (!((n >> t) & 1)) ++t;
    return t;
  }
  int shift = (r == 4) ? 2 : (r == 8) ? 3 : 0;
  if (!shift) return 0;
  int t = 0;
  for (int v = n; v > 1; v >>= shift) ++t;
  return t;
}

/* exp(sign * 2*pi*i * p / r) for r in {2,4,8}, exact where the value is
 * 0/+-1 and (+-1 +- i)/sqrt(2) otherwise (the r = 8 constants a, b of
 * butterflies.c:286-290). */
static void unit_root(int r, int p, int sign, double* c, double* s) {
  p %= r;
  if (p < 0) p += r;
  int e8 = p * (8 / r);          /* exponent in units of 2*pi/8 */
  double h = 1.0 / sqrt(2.0);
  static const double cr[8] = {1, 0, 0, 0, -1, 0, 0, 0};
  static const double ci[8] = {0, 0, 1, 0, 0, 0, -1, 0};
  if (e8 % 2 == 0) {
    *c = cr[e8];
    *s = ci[e8];
  } else {
    /* odd multiples of pi/4 */
    *c = (e8 == 1 || e8 == 7) ? h : -h;
    *s = (e8 == 1 || e8 == 3) ? h : -h;
  }
  *s *= (double)sign;
}

/* --------------------------------------------------------------------- */
/* Twiddle tables, reference layout (twiddle_factors.c:17-131).            */
/* Level q, k = r^(q+1), ell = k/r, holds (r-1)*ell entries; entry         */
/* (m-1)*ell + j = exp(-2*pi*i*m*j/k), m = 1..r-1.                         */
/* --------------------------------------------------------------------- */
void orc_twiddles(int r, int n, double*** tre, double*** tim) {
  int t = orc_levels(n, r);
  *tre = (double**)malloc((t > 0 ? t : 1) * sizeof(double*));
  *tim = (double**)malloc((t > 0 ? t : 1) * sizeof(double*));
  long k = 1;
  for (int q = 0; q < t; ++q) {
    k *= r;
    long ell = k / r;
    double* a = (double*)malloc((size_t)((r - 1) * ell) * sizeof(double));
    double* b = (double*)malloc((size_t)((r - 1) * ell) * sizeof(double));
    for (int m = 1; m < r; ++m)
      for (long j = 0; j < ell; ++j) {
        double ang = -2.0 * M_PI * (double)(m * j) / (double)k;
        a[(m - 1) * ell + j] = cos(ang);
        b[(m - 1) * ell + j] = sin(ang);
      }
    (*tre)[q] = a;
    (*tim)[q] = b;
  }
}

void orc_free_twiddles(double** tre, double** tim, int t) {
  for (int q = 0; q < t; ++q) {
    free(tre[q]);
    free(tim[q]);
  }
  free(tre);
  free(tim);
}

/* --------------------------------------------------------------------- */
/* 1D butterfly operators (butterflies.c).                                 */
/*   op 0  A        apply_butterflies_r{2,4,8}            :12  :99  :277   */
/*   op 1  conj(A)  apply_conjugate_butterflies_r{2,4,8}  :41  :158 :391   */
/*   op 2  A^T      apply_transposed_butterflies_r{2,4,8} :70  :217 :505   */
/* A, conj(A): stages q = 0..t-1; in each block of k = r^(q+1) elements    */
/*   z_m = w_k^{+-j m} x[i + m ell];  x[i + s ell] = sum_m z_m w_r^{-+ m s}*/
/* A^T: stages q = t-1..0;                                                 */
/*   u_m = sum_s x[i + s ell] w_r^{-m s};  x[i + m ell] = w_k^{j m} u_m    */
/* --------------------------------------------------------------------- */
#define ORC_RMAX 8

void orc_butterflies(int op, int r, double* re, double* im, int n,
                     double** tre, double** tim) {
  int t = orc_levels(n, r);
  double wr[ORC_RMAX * ORC_RMAX], wi[ORC_RMAX * ORC_RMAX];
  /* the r-point DFT matrix: forward sign for A and A^T, + for conj(A) */
  int dsign = (op == 1) ? +1 : -1;
  for (int m = 0; m < r; ++m)
    for (int s = 0; s < r; ++s) unit_root(r, m * s, dsign, &wr[m * r + s], &wi[m * r + s]);

  double zr[ORC_RMAX], zi[ORC_RMAX];
  for (int step = 0; step < t; ++step) {
    int q = (op == 2) ? (t - 1 - step) : step;
    long k = 1;
    for (int e = 0; e <= q; ++e) k *= r;
    long ell = k / r;
    long nb = n / k;
    for (long b = 0; b < nb; ++b) {
      for (long j = 0; j < ell; ++j) {
        long i = b * k + j;
        if (op != 2) {
          /* DIT: twiddle the inputs, then the r-point DFT */
          zr[0] = re[i];
          zi[0] = im[i];
          for (int m = 1; m < r; ++m) {
            double c = tre[q][(m - 1) * ell + j];
            double s = tim[q][(m - 1) * ell + j];
            if (op == 1) s = -s;
            double xr = re[i + m * ell], xi = im[i + m * ell];
            zr[m] = c * xr - s * xi;
            zi[m] = c * xi + s * xr;
          }
          for (int s = 0; s < r; ++s) {
            double ar = 0.0, ai = 0.0;
            for (int m = 0; m < r; ++m) {
              ar += zr[m] * wr[m * r + s] - zi[m] * wi[m * r + s];
              ai += zr[m] * wi[m * r + s] + zi[m] * wr[m * r + s];
            }
            re[i + s * ell] = ar;
            im[i + s * ell] = ai;
          }
        } else {
          /* DIF: the r-point DFT, then twiddle the outputs */
          for (int m = 0; m < r; ++m) {
            zr[m] = re[i + m * ell];
            zi[m] = im[i + m * ell];
          }
          for (int m = 0; m < r; ++m) {
            double ar = 0.0, ai = 0.0;
            for (int s = 0; s < r; ++s) {
              ar += zr[s] * wr[m * r + s] - zi[s] * wi[m * r + s];
              ai += zr[s] * wi[m * r + s] + zi[s] * wr[m * r + s];
            }
            if (m > 0) {
              double c = tre[q][(m - 1) * ell + j];
              double s = tim[q][(m - 1) * ell + j];
              double br = c * ar - s * ai;
              double bi = c * ai + s * ar;
              ar = br;
              ai = bi;
            }
            re[i + m * ell] = ar;
            im[i + m * ell] = ai;
          }
        }
      }
    }
  }
}

/* --------------------------------------------------------------------- */
/* Multi-D butterflies (butterflies_2d.c:12-243, butterflies_3d.c:12-382): */
/* the 1D operator along every axis, last (contiguous) axis first, other   */
/* axes gathered into a temporary line and scattered back.  Per-axis       */
/* twiddle tables are built here from (r, n_axis), as the reference        */
/* benches do with precompute_twiddles_r*(n_axis).                         */
/* --------------------------------------------------------------------- */
void orc_butterflies_nd(int op, int r, double* re, double* im, int rank, const int* dims) {
  long total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  int nmax = 1;
  for (int d = 0; d < rank; ++d) nmax = dims[d] > nmax ? dims[d] : nmax;
  double* lr = (double*)malloc(nmax * sizeof(double));
  double* li = (double*)malloc(nmax * sizeof(double));
  for (int d = rank - 1; d >= 0; --d) {
    int len = dims[d];
    long stride = 1;
    for (int e = d + 1; e < rank; ++e) stride *= dims[e];
    double **tr, **ti;
    orc_twiddles(r, len, &tr, &ti);
    long outer = total / (stride * len);
    for (long o = 0; o < outer; ++o)
      for (long s = 0; s < stride; ++s) {
        long base = o * stride * len + s;
        for (int e = 0; e < len; ++e) {
          lr[e] = re[base + e * stride];
          li[e] = im[base + e * stride];
        }
        orc_butterflies(op, r, lr, li, len, tr, ti);
        for (int e = 0; e < len; ++e) {
          re[base + e * stride] = lr[e];
          im[base + e * stride] = li[e];
        }
      }
    orc_free_twiddles(tr, ti, orc_levels(len, r));
  }
  free(lr);
  free(li);
}

/* --------------------------------------------------------------------- */
/* Index reversal (index_reversals.c:13-72, _2d.c:14-59, _3d.c:14-69):     */
/* radix-r digit reversal of each axis index independently.               */
/* --------------------------------------------------------------------- */
int orc_reverse_index(int r, int x, int t) {
  int bits = (r == 2) ? 1 : (r == 4) ? 2 : 3;
  int v = 0;
  for (int d = 0; d < t; ++d) {
    v = (v << bits) | (x & (r - 1));
    x >>= bits;
  }
  return v;
}

void orc_rho(int r, int rank, const int* dims, int* rho) {
  int t[3] = {0, 0, 0};
  for (int d = 0; d < rank; ++d) t[d] = orc_levels(dims[d], r);
  long total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  for (long idx = 0; idx < total; ++idx) {
    long rem = idx, out = 0, mul = 1;
    int digit[3];
    for (int d = rank - 1; d >= 0; --d) {
      digit[d] = (int)(rem % dims[d]);
      rem /= dims[d];
    }
    for (int d = rank - 1; d >= 0; --d) {
      out += mul * orc_reverse_index(r, digit[d], t[d]);
      mul *= dims[d];
    }
    rho[idx] = (int)out;
  }
}

/* swap-based in-place permutation (index_reversals.c:85-94).  Indices past
 * the array (a digit reversal built for a length that is not a power of r)
 * are skipped instead of written out of bounds. */
void orc_apply_permutation_split(double* re, double* im, long n, const int* rho) {
  for (long j = 0; j < n; ++j) {
    long p = rho[j];
    if (j < p && p < n) {
      double a = re[j], b = im[j];
      re[j] = re[p];
      im[j] = im[p];
      re[p] = a;
      im[p] = b;
    }
  }
}

/* --------------------------------------------------------------------- */
/* Transforms (fft.c:12-87, fft_2d.c:12-113, fft_3d.c:12-128).             */
/*   kind 0 fft   : permute, A                                             */
/*   kind 1 fft2  : A^T, permute                                           */
/*   kind 2 ufft  : A                                                      */
/*   kind 3 ifft  : permute, conj(A), divide by n                          */
/*   kind 4 uifft : conj(A), divide by n                                   */
/* An unsupported radix skips the butterflies (the if/else chains of       */
/* fft.c:16-24), the permutation and division still run.                   */
/* --------------------------------------------------------------------- */
static int radix_ok(int r, int rank) {
  if (rank == 1) return r == 2 || r == 4 || r == 8;
  return r == 2 || r == 4;
}

void orc_transform_nd(int kind, int r, double* re, double* im, int rank, const int* dims) {
  long total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  int* rho = NULL;
  if (kind == 0 || kind == 1 || kind == 3) {
    rho = (int*)malloc(total * sizeof(int));
    orc_rho(r, rank, dims, rho);
  }
  int ok = radix_ok(r, rank);
  switch (kind) {
    case 0:
      orc_apply_permutation_split(re, im, total, rho);
      if (ok) orc_butterflies_nd(0, r, re, im, rank, dims);
      break;
    case 1:
      if (ok) orc_butterflies_nd(2, r, re, im, rank, dims);
      orc_apply_permutation_split(re, im, total, rho);
      break;
    case 2:
      if (ok) orc_butterflies_nd(0, r, re, im, rank, dims);
      break;
    case 3:
    case 4:
      if (kind == 3) orc_apply_permutation_split(re, im, total, rho);
      if (ok) orc_butterflies_nd(1, r, re, im, rank, dims);
      for (long i = 0; i < total; ++i) {
        re[i] /= (double)total;
        im[i] /= (double)total;
      }
      break;
  }
  free(rho);
}

/* --------------------------------------------------------------------- */
/* Convolutions (convolution.c:12-71, _2d.c:12-69, _3d.c:12-71).           */
/* method 1 permutation-avoiding:                                          */
/*   x <- A^T x; h <- A^T h; x <- (x .* h) / n; x <- conj(A) x             */
/* method 0 FFT-based: fft(x), fft(h), x .* h, ifft(x)                     */
/* h is overwritten with A^T h (method 1) or F h (method 0), as in the     */
/* reference.  An unsupported radix skips the butterfly calls.             */
/* --------------------------------------------------------------------- */
void orc_convolution_nd(int method, int r, double* re, double* im, int rank, const int* dims,
                        double* h_re, double* h_im) {
  long total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  int ok = radix_ok(r, rank);
  if (method == 1) {
    if (ok) {
      orc_butterflies_nd(2, r, re, im, rank, dims);
      orc_butterflies_nd(2, r, h_re, h_im, rank, dims);
    }
    for (long i = 0; i < total; ++i) {
      double ar = re[i], ai = im[i], br = h_re[i], bi = h_im[i];
      re[i] = (ar * br - ai * bi) / (double)total;
      im[i] = (ar * bi + ai * br) / (double)total;
    }
    if (ok) orc_butterflies_nd(1, r, re, im, rank, dims);
  } else {
    orc_transform_nd(0, r, re, im, rank, dims);
    orc_transform_nd(0, r, h_re, h_im, rank, dims);
    for (long i = 0; i < total; ++i) {
      double ar = re[i], ai = im[i], br = h_re[i], bi = h_im[i];
      re[i] = ar * br - ai * bi;
      im[i] = ar * bi + ai * br;
    }
    orc_transform_nd(3, r, re, im, rank, dims);
  }
}

/* --------------------------------------------------------------------- */
/* Independent checks (no counterpart in the reference).                   */
/* --------------------------------------------------------------------- */
/* Direct O(N^2) circular convolution in long double over a rank-d array. */
void orc_naive_circular_conv(const double* xr, const double* xi, const double* hr,
                             const double* hi, int rank, const int* dims, double* yr,
                             double* yi) {
  long total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  int di[3], dj[3], dk[3];
  for (long a = 0; a < total; ++a) {
    long rem = a;
    for (int d = rank - 1; d >= 0; --d) {
      di[d] = (int)(rem % dims[d]);
      rem /= dims[d];
    }
    long double sr = 0.0L, si = 0.0L;
    for (long b = 0; b < total; ++b) {
      long rb = b;
      for (int d = rank - 1; d >= 0; --d) {
        dj[d] = (int)(rb % dims[d]);
        rb /= dims[d];
      }
      long c = 0;
      for (int d = 0; d < rank; ++d) {
        dk[d] = (di[d] - dj[d]) % dims[d];
        if (dk[d] < 0) dk[d] += dims[d];
        c = c * dims[d] + dk[d];
      }
      long double pr = (long double)xr[b], pi = (long double)xi[b];
      long double qr = (long double)hr[c], qi = (long double)hi[c];
      sr += pr * qr - pi * qi;
      si += pr * qi + pi * qr;
    }
    yr[a] = (double)sr;
    yi[a] = (double)si;
  }
}

/* max_i |a_i - b_i| by hypot (misc.c:20-30) */
double orc_max_error(const double* ar, const double* ai, const double* br, const double* bi,
                     long n) {
  double m = 0.0;
  for (long i = 0; i < n; ++i) {
    double e = hypot(ar[i] - br[i], ai[i] - bi[i]);
    if (e > m) m = e;
  }
  return m;
}

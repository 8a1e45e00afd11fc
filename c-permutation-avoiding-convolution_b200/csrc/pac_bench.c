/*
 * pac_bench.c -- GPU bench drivers with the command line of the reference's
 * bench*.c programs (bench1d_convolution.c:58-86 and siblings):
 *
 *   pac_bench <driver> [verify|bench] [-t power] [-r timing_runs] [--json]
 *   pac_bench sweep <1d|2d|3d> [-r timing_runs] [--json] [--list]
 *
 * drivers (the reference's executables without the "bench" prefix):
 *   1d_forward_fft 1d_backward_fft 1d_convolution
 *   2d_forward_fft 2d_backward_fft 2d_convolution 2d_convolution_anisotropic
 *   3d_forward_fft 3d_backward_fft 3d_convolution 3d_convolution_anisotropic
 *
 * Shapes follow the reference: 1D n = 2^t (default t = 24); 2D n x n with
 * n = 2^t (default 12), anisotropic 2^t x 4; 3D n^3 with n = 2^t (default 8),
 * anisotropic 2^t x 4 x 4.  Radix 2 always, 4 when every axis exponent is
 * even, 8 in 1D when t is a multiple of 3 (supports_radix_4/8, misc.c).
 * Inputs: real and imaginary parts from rand() / RAND_MAX, as
 * initialize_data_split and initialize_filter (misc.c:40-55) make them.
 *
 * bench: per radix, the mean +/- standard deviation over timing_runs of
 * every fft.h call the reference driver times (called here with host
 * buffers, so the times include the host<->device copies), followed by the
 * device-resident pac.h call on the same data (plan and filter spectrum
 * made once, untimed).  verify: the maximum error |z - z_ref| against a
 * plain FP64 CPU FFT in this file, which stands where FFTW stands in the
 * reference's drivers.  sweep: the t lists of bench1d.sh / bench2d.sh /
 * bench3d.sh, bench mode (--list prints the (driver, t) pairs instead).
 * --json: one JSON object per line instead of text.
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fft.h"
#include "pac.h"

static int g_json = 0;

static double now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + t.tv_nsec * 1e-9;
}

/* ------------------------------------------------------------------------ */
/* CPU FP64 reference FFT (radix 2, in place, split arrays)                  */
/* ------------------------------------------------------------------------ */
static void cpu_fft_line(double* re, double* im, size_t n, int sign) {
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double t = re[i]; re[i] = re[j]; re[j] = t;
      t = im[i]; im[i] = im[j]; im[j] = t;
    }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const double ang = sign * 6.283185307179586476925 / (double)len;  /* 2 pi / len */
    for (size_t k = 0; k < len / 2; ++k) {
      const double wr = cos(ang * (double)k), wi = sin(ang * (double)k);
      for (size_t s = 0; s < n; s += len) {
        size_t a = s + k, b = a + len / 2;
        double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - xr; im[b] = im[a] - xi;
        re[a] += xr; im[a] += xi;
      }
    }
  }
}

/* every axis of a row-major rank-d array; sign -1 forward, +1 inverse
 * (unnormalised) */
static void cpu_fft_nd(double* re, double* im, int d, const int* dims, int sign) {
  size_t total = 1;
  for (int a = 0; a < d; ++a) total *= (size_t)dims[a];
  size_t maxn = 0;
  for (int a = 0; a < d; ++a) if ((size_t)dims[a] > maxn) maxn = dims[a];
  double* lr = malloc(maxn * sizeof(double));
  double* li = malloc(maxn * sizeof(double));
  for (int a = 0; a < d; ++a) {
    size_t n = dims[a], stride = 1;
    for (int b = a + 1; b < d; ++b) stride *= (size_t)dims[b];
    for (size_t base = 0; base < total; ++base) {
      if ((base / stride) % n != 0) continue; /* first element of a line */
      for (size_t k = 0; k < n; ++k) { lr[k] = re[base + k * stride]; li[k] = im[base + k * stride]; }
      cpu_fft_line(lr, li, n, sign);
      for (size_t k = 0; k < n; ++k) { re[base + k * stride] = lr[k]; im[base + k * stride] = li[k]; }
    }
  }
  free(lr);
  free(li);
}

static double max_err(const double* re, const double* im, const double* zr, const double* zi,
                      size_t n) {
  double m = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double e = hypot(re[i] - zr[i], im[i] - zi[i]);
    if (e > m) m = e;
  }
  return m;
}

/* ------------------------------------------------------------------------ */
/* drivers                                                                   */
/* ------------------------------------------------------------------------ */
enum { K_FWD, K_BWD, K_CONV };

typedef struct {
  const char* name;
  int rank;
  int kind;
  int aniso;
  int t_default;
} Driver;

static const Driver DRIVERS[] = {
    {"1d_forward_fft", 1, K_FWD, 0, 24},  {"1d_backward_fft", 1, K_BWD, 0, 24},
    {"1d_convolution", 1, K_CONV, 0, 24}, {"2d_forward_fft", 2, K_FWD, 0, 12},
    {"2d_backward_fft", 2, K_BWD, 0, 12}, {"2d_convolution", 2, K_CONV, 0, 12},
    {"2d_convolution_anisotropic", 2, K_CONV, 1, 12},
    {"3d_forward_fft", 3, K_FWD, 0, 8},   {"3d_backward_fft", 3, K_BWD, 0, 8},
    {"3d_convolution", 3, K_CONV, 0, 8},  {"3d_convolution_anisotropic", 3, K_CONV, 1, 8},
};

typedef struct {
  int d;
  int dims[3];
  int logs[3];
  size_t n;
} Shape;

static Shape make_shape(const Driver* dr, int t) {
  Shape s;
  s.d = dr->rank;
  s.n = 1;
  for (int a = 0; a < s.d; ++a) {
    s.logs[a] = (dr->aniso && a > 0) ? 2 : t; /* anisotropic: 2^t x 4 (x 4) */
    s.dims[a] = 1 << s.logs[a];
    s.n *= (size_t)s.dims[a];
  }
  return s;
}

static int radix_ok(const Shape* s, int r) {
  if (r == 2) return 1;
  for (int a = 0; a < s->d; ++a) {
    if (r == 4 && s->logs[a] % 2) return 0;
    if (r == 8 && (s->d != 1 || s->logs[a] % 3)) return 0;
  }
  return 1;
}

static void fill_rand(double* v, size_t n) {
  for (size_t i = 0; i < n; ++i) v[i] = rand() / (double)RAND_MAX;
}

static void report(const Driver* dr, const Shape* s, int t, int r, const char* what,
                   const char* path, double mu, double sd) {
  if (g_json) {
    printf("{\"driver\": \"%s\", \"t\": %d, \"dims\": [", dr->name, t);
    for (int a = 0; a < s->d; ++a) printf("%s%d", a ? ", " : "", s->dims[a]);
    printf("], \"radix\": %d, \"call\": \"%s\", \"path\": \"%s\", \"mean_s\": %.9f, "
           "\"std_s\": %.9f, \"gelem_per_s\": %.6f}\n",
           r, what, path, mu, sd, mu > 0 ? (double)s->n / mu / 1e9 : 0.0);
  } else {
    char label[160];
    snprintf(label, sizeof label, "Average radix-%d %s time (%s):", r, what, path);
    printf("%-70s %.6f +/- %.6f seconds  (%.3f GElem/s)\n", label, mu, sd,
           mu > 0 ? (double)s->n / mu / 1e9 : 0.0);
  }
  fflush(stdout);
}

static void report_err(const Driver* dr, int t, int r, const char* what, double e) {
  if (g_json)
    printf("{\"driver\": \"%s\", \"t\": %d, \"radix\": %d, \"call\": \"%s\", "
           "\"max_error_vs_cpu_fft\": %.3e}\n", dr->name, t, r, what, e);
  else
    printf("Max error %s radix-%d vs CPU FFT: %.3e\n", what, r, e);
  fflush(stdout);
}

/* fft.h calls of one driver at radix r on host buffers */
static void call_fft(const Shape* s, int kind, int unordered, int r, double* re, double* im,
                     int* rho) {
  const int* n = s->dims;
  if (s->d == 1) {
    if (kind == K_FWD) { if (unordered) ufft(re, im, n[0], r, NULL, NULL); else fft(re, im, n[0], r, NULL, NULL, rho); }
    else { if (unordered) uifft(re, im, n[0], r, NULL, NULL); else ifft(re, im, n[0], r, NULL, NULL, rho); }
  } else if (s->d == 2) {
    if (kind == K_FWD) { if (unordered) ufft_2d(re, im, n[0], n[1], r, NULL, NULL, NULL, NULL); else fft_2d(re, im, n[0], n[1], r, NULL, NULL, NULL, NULL, rho); }
    else { if (unordered) uifft_2d(re, im, n[0], n[1], r, NULL, NULL, NULL, NULL); else ifft_2d(re, im, n[0], n[1], r, NULL, NULL, NULL, NULL, rho); }
  } else {
    if (kind == K_FWD) { if (unordered) ufft_3d(re, im, n[0], n[1], n[2], r, NULL, NULL, NULL, NULL, NULL, NULL); else fft_3d(re, im, n[0], n[1], n[2], r, NULL, NULL, NULL, NULL, NULL, NULL, rho); }
    else { if (unordered) uifft_3d(re, im, n[0], n[1], n[2], r, NULL, NULL, NULL, NULL, NULL, NULL); else ifft_3d(re, im, n[0], n[1], n[2], r, NULL, NULL, NULL, NULL, NULL, NULL, rho); }
  }
}

static void call_conv(const Shape* s, int pac, int r, double* re, double* im, double* hr,
                      double* hi, int* rho) {
  const int* n = s->dims;
  if (s->d == 1) {
    if (pac) permutation_avoiding_convolution(re, im, n[0], r, NULL, NULL, hr, hi);
    else fft_based_convolution(re, im, n[0], r, NULL, NULL, rho, hr, hi);
  } else if (s->d == 2) {
    if (pac) permutation_avoiding_convolution_2d(re, im, n[0], n[1], r, NULL, NULL, NULL, NULL, hr, hi);
    else fft_based_convolution_2d(re, im, n[0], n[1], r, NULL, NULL, NULL, NULL, rho, hr, hi);
  } else {
    if (pac) permutation_avoiding_convolution_3d(re, im, n[0], n[1], n[2], r, NULL, NULL, NULL, NULL, NULL, NULL, hr, hi);
    else fft_based_convolution_3d(re, im, n[0], n[1], n[2], r, NULL, NULL, NULL, NULL, NULL, NULL, rho, hr, hi);
  }
}

static int* make_rho(const Shape* s, int r) {
  const int* n = s->dims;
  if (s->d == 1) return r == 2 ? precompute_index_reversal_permutation_r2(n[0])
                     : r == 4 ? precompute_index_reversal_permutation_r4(n[0])
                              : precompute_index_reversal_permutation_r8(n[0]);
  if (s->d == 2) return r == 2 ? precompute_index_reversal_permutation_r2_2d(n[0], n[1])
                               : precompute_index_reversal_permutation_r4_2d(n[0], n[1]);
  return r == 2 ? precompute_index_reversal_permutation_r2_3d(n[0], n[1], n[2])
                : precompute_index_reversal_permutation_r4_3d(n[0], n[1], n[2]);
}

static int check_last(const char* what) {
  int st = pac_get_last_status();
  if (st) fprintf(stderr, "%s failed: %s (%s)\n", what, pac_status_string(st), pac_last_error());
  return st;
}

typedef struct {
  double sum, sq;
  int k;
} Acc;
static void acc_add(Acc* a, double v) { a->sum += v; a->sq += v * v; a->k++; }
static double acc_mu(const Acc* a) { return a->k ? a->sum / a->k : 0.0; }
static double acc_sd(const Acc* a) {
  double mu = acc_mu(a), v = a->k ? a->sq / a->k - mu * mu : 0.0;
  return v > 0 ? sqrt(v) : 0.0;
}

/* the device-resident pac.h call matching the driver, timed per call */
static int device_time(const Driver* dr, const Shape* s, int r, int runs, const double* x_re,
                       const double* x_im, const double* h_re, const double* h_im, Acc* acc) {
  pac_plan_t plan = NULL;
  void *xr = NULL, *xi = NULL, *hr = NULL, *hi = NULL, *Hr = NULL, *Hi = NULL, *yr = NULL, *yi = NULL;
  size_t B = s->n * sizeof(double);
  int st = pac_plan_create(&plan, s->d, s->dims, 1, r, PAC_FORM_F64);
  if (!st) st = pac_malloc(&xr, B);
  if (!st) st = pac_malloc(&xi, B);
  if (!st) st = pac_malloc(&yr, B);
  if (!st) st = pac_malloc(&yi, B);
  if (!st) st = pac_memcpy_h2d(xr, x_re, B, NULL);
  if (!st) st = pac_memcpy_h2d(xi, x_im, B, NULL);
  if (!st && dr->kind == K_CONV) {
    st = pac_malloc(&hr, B);
    if (!st) st = pac_malloc(&hi, B);
    if (!st) st = pac_malloc(&Hr, B);
    if (!st) st = pac_malloc(&Hi, B);
    if (!st) st = pac_memcpy_h2d(hr, h_re, B, NULL);
    if (!st) st = pac_memcpy_h2d(hi, h_im, B, NULL);
    if (!st) st = pac_filter_spectrum(plan, hr, hi, 1, Hr, Hi, 1.0 / (double)s->n, NULL);
  }
  for (int k = -1; !st && k < runs; ++k) { /* k = -1: warm-up */
    double t0 = now();
    if (dr->kind == K_CONV) st = pac_convolve(plan, xr, xi, Hr, Hi, 0, yr, yi, 1.0, NULL);
    else st = pac_transform(plan, dr->kind == K_FWD ? PAC_OP_FFT : PAC_OP_IFFT, xr, xi, yr, yi, NULL);
    if (!st) st = pac_stream_synchronize(NULL);
    if (k >= 0) acc_add(acc, now() - t0);
  }
  if (st) fprintf(stderr, "device-resident call failed: %s\n", pac_last_error());
  void* ptrs[] = {xr, xi, hr, hi, Hr, Hi, yr, yi};
  for (int i = 0; i < 8; ++i) pac_free(ptrs[i]);
  if (plan) pac_plan_destroy(plan);
  return st;
}

static int run_driver(const Driver* dr, int verify, int t, int runs) {
  Shape s = make_shape(dr, t);
  const size_t n = s.n, B = n * sizeof(double);
  double *re = malloc(B), *im = malloc(B), *x_re = malloc(B), *x_im = malloc(B);
  double *h_re = malloc(B), *h_im = malloc(B), *hr = malloc(B), *hi = malloc(B);
  double *zr = NULL, *zi = NULL;
  if (!re || !im || !x_re || !x_im || !h_re || !h_im || !hr || !hi) {
    fprintf(stderr, "host allocation of %zu bytes failed\n", 8 * B);
    return 1;
  }
  fill_rand(h_re, n); /* initialize_filter, then initialize_data_split */
  fill_rand(h_im, n);
  fill_rand(x_re, n);
  fill_rand(x_im, n);
  if (!g_json)
    printf("%s %s, t = %d (%zu elements)\n", dr->name, verify ? "verify" : "bench", t, n);
  if (verify) {
    zr = malloc(B);
    zi = malloc(B);
    memcpy(zr, x_re, B);
    memcpy(zi, x_im, B);
    if (dr->kind == K_FWD) {
      cpu_fft_nd(zr, zi, s.d, s.dims, -1);
    } else if (dr->kind == K_BWD) {
      cpu_fft_nd(zr, zi, s.d, s.dims, +1);
      for (size_t i = 0; i < n; ++i) { zr[i] /= (double)n; zi[i] /= (double)n; }
    } else {
      memcpy(hr, h_re, B);
      memcpy(hi, h_im, B);
      cpu_fft_nd(zr, zi, s.d, s.dims, -1);
      cpu_fft_nd(hr, hi, s.d, s.dims, -1);
      for (size_t i = 0; i < n; ++i) {
        double a = zr[i] * hr[i] - zi[i] * hi[i], b = zr[i] * hi[i] + zi[i] * hr[i];
        zr[i] = a / (double)n;
        zi[i] = b / (double)n;
      }
      cpu_fft_nd(zr, zi, s.d, s.dims, +1);
    }
  }
  int rc = 0;
  for (int r = 2; r <= 8 && !rc; r *= 2) {
    if (!radix_ok(&s, r)) continue;
    int* rho = make_rho(&s, r);
    if (dr->kind == K_CONV) {
      for (int pac = 0; pac < 2 && !rc; ++pac) {
        const char* what = pac ? "permutation-avoiding" : "FFT-based";
        Acc acc = {0, 0, 0};
        for (int k = verify ? 0 : -1; k < (verify ? 1 : runs); ++k) {
          memcpy(re, x_re, B); memcpy(im, x_im, B);
          memcpy(hr, h_re, B); memcpy(hi, h_im, B);
          double t0 = now();
          call_conv(&s, pac, r, re, im, hr, hi, rho);
          double dt = now() - t0;
          if ((rc = check_last(what))) break;
          if (k >= 0) acc_add(&acc, dt);
        }
        if (rc) break;
        if (verify) report_err(dr, t, r, what, max_err(re, im, zr, zi, n));
        else report(dr, &s, t, r, what, "fft.h, host buffers", acc_mu(&acc), acc_sd(&acc));
      }
    } else {
      const char* names[3] = {"FFT", "permutation", "unordered FFT"};
      for (int which = 0; which < 3 && !rc; ++which) {
        if (verify && which != 0) continue;
        Acc acc = {0, 0, 0};
        for (int k = verify ? 0 : -1; k < (verify ? 1 : runs); ++k) {
          memcpy(re, x_re, B); memcpy(im, x_im, B);
          double t0 = now();
          if (which == 1) apply_permutation_split(re, im, (int)n, rho);
          else call_fft(&s, dr->kind, which == 2, r, re, im, rho);
          double dt = now() - t0;
          if ((rc = check_last(names[which]))) break;
          if (k >= 0) acc_add(&acc, dt);
        }
        if (rc) break;
        if (verify) report_err(dr, t, r, names[which], max_err(re, im, zr, zi, n));
        else report(dr, &s, t, r, names[which], "fft.h, host buffers", acc_mu(&acc), acc_sd(&acc));
      }
    }
    free(rho);
    if (!verify && !rc) {
      Acc acc = {0, 0, 0};
      rc = device_time(dr, &s, r, runs, x_re, x_im, h_re, h_im, &acc);
      if (!rc)
        report(dr, &s, t, r, dr->kind == K_CONV ? "permutation-avoiding" : "FFT",
               "pac.h, device-resident", acc_mu(&acc), acc_sd(&acc));
    }
  }
  free(re); free(im); free(x_re); free(x_im); free(h_re); free(h_im); free(hr); free(hi);
  free(zr); free(zi);
  return rc;
}

/* the t lists of the reference's sweep scripts (bench1d.sh, bench2d.sh,
 * bench3d.sh) */
static int run_sweep(const char* which, int runs, int list_only) {
  static const int t1[] = {20, 22, 24, 26, 28}, t2[] = {10, 11, 12, 13, 14},
                   t2a[] = {20, 22, 24, 26}, t3[] = {7, 8, 9}, t3a[] = {20, 22, 24};
  struct Item { const char* name; const int* ts; int nt; } items[4];
  int ni = 0;
  if (!strcmp(which, "1d")) {
    items[ni++] = (struct Item){"1d_forward_fft", t1, 5};
    items[ni++] = (struct Item){"1d_backward_fft", t1, 5};
    items[ni++] = (struct Item){"1d_convolution", t1, 5};
  } else if (!strcmp(which, "2d")) {
    items[ni++] = (struct Item){"2d_forward_fft", t2, 5};
    items[ni++] = (struct Item){"2d_backward_fft", t2, 5};
    items[ni++] = (struct Item){"2d_convolution", t2, 5};
    items[ni++] = (struct Item){"2d_convolution_anisotropic", t2a, 4};
  } else if (!strcmp(which, "3d")) {
    items[ni++] = (struct Item){"3d_forward_fft", t3, 3};
    items[ni++] = (struct Item){"3d_backward_fft", t3, 3};
    items[ni++] = (struct Item){"3d_convolution", t3, 3};
    items[ni++] = (struct Item){"3d_convolution_anisotropic", t3a, 3};
  } else {
    fprintf(stderr, "Unknown sweep: %s (1d, 2d or 3d)\n", which);
    return 1;
  }
  for (int i = 0; i < ni; ++i)
    for (int k = 0; k < items[i].nt; ++k) {
      const Driver* dr = NULL;
      for (size_t j = 0; j < sizeof(DRIVERS) / sizeof(DRIVERS[0]); ++j)
        if (!strcmp(DRIVERS[j].name, items[i].name)) dr = &DRIVERS[j];
      if (list_only) {
        printf("{\"driver\": \"%s\", \"t\": %d}\n", dr->name, items[i].ts[k]);
        continue;
      }
      if (!g_json) printf("\n");
      int rc = run_driver(dr, 0, items[i].ts[k], runs);
      if (rc) return rc;
    }
  return 0;
}

static void usage(const char* prog) {
  fprintf(stderr,
          "Usage: %s <driver> [verify|bench] [-t power] [-r timing_runs] [--json]\n"
          "       %s sweep <1d|2d|3d> [-r timing_runs] [--json] [--list]\n"
          "drivers:", prog, prog);
  for (size_t j = 0; j < sizeof(DRIVERS) / sizeof(DRIVERS[0]); ++j)
    fprintf(stderr, " %s", DRIVERS[j].name);
  fprintf(stderr, "\n");
}

int main(int argc, char** argv) {
  if (argc < 3) {
    usage(argv[0]);
    return 1;
  }
  int runs = 10, t = -1, verify = 0, list_only = 0;
  const char* sweep = NULL;
  const Driver* dr = NULL;
  if (!strcmp(argv[1], "sweep")) {
    sweep = argv[2];
  } else {
    for (size_t j = 0; j < sizeof(DRIVERS) / sizeof(DRIVERS[0]); ++j)
      if (!strcmp(DRIVERS[j].name, argv[1])) dr = &DRIVERS[j];
    if (!dr) {
      fprintf(stderr, "Unknown driver: %s\n", argv[1]);
      usage(argv[0]);
      return 1;
    }
    if (!strcmp(argv[2], "verify")) verify = 1;
    else if (strcmp(argv[2], "bench")) {
      fprintf(stderr, "Unknown mode: %s\n", argv[2]);
      return 1;
    }
  }
  for (int i = 3; i < argc; ++i) {
    if (!strcmp(argv[i], "-t") && i + 1 < argc && !sweep) t = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-r") && i + 1 < argc) runs = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--json")) g_json = 1;
    else if (!strcmp(argv[i], "--list") && sweep) list_only = 1;
    else {
      fprintf(stderr, "Unknown or malformed option: %s\n", argv[i]);
      return 1;
    }
  }
  if (runs < 1) runs = 1;
  if (sweep) return run_sweep(sweep, runs, list_only);
  if (t < 0) t = dr->t_default;
  if (t < 1 || t > 30) {
    fprintf(stderr, "power out of range: %d\n", t);
    return 1;
  }
  return run_driver(dr, verify, t, runs);
}

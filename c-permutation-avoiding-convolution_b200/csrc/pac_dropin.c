/*
 * pac_dropin.c -- the reference's fft.h entry points on the B200 library.
 *
 * Host C over the native C ABI (pac.h).  Every function keeps the
 * reference's prototype and side effects (fft.h of the reference, lines
 * cited per function) and runs the arithmetic on the GPU:
 *
 *   host arrays --H2D--> plan kernels --D2H--> host arrays
 *
 * Plans and device staging buffers are cached per (rank, dims, radix) and
 * reused by later calls; the cache is guarded by a mutex and each entry by
 * its own lock, so concurrent callers are safe.  Calls are synchronous.
 *
 * Errors: the reference functions return void and do not validate.  Here an
 * axis length that is not a power of r, a NULL array or a CUDA failure
 * leaves the caller's data untouched, prints one line to stderr and records
 * the status for pac_get_last_status().  A device wait that gave up during
 * the call (pac_plan_check_status) is reported the same way, as
 * PAC_ERROR_TIMEOUT; the outputs of that call are then incomplete.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fft.h"
#include "pac.h"

static __thread int t_status = PAC_SUCCESS;

PAC_API int pac_get_last_status(void) {
  int s = t_status;
  t_status = PAC_SUCCESS;
  return s;
}

static int report(int st, const char* fn) {
  if (st != PAC_SUCCESS) {
    t_status = st;
    const char* msg = pac_last_error();
    fprintf(stderr, "pac: %s: %s%s%s\n", fn, pac_status_string(st), (msg && *msg) ? ": " : "",
            msg ? msg : "");
  }
  return st;
}

/* ------------------------------------------------------------------------ */
/* validation                                                               */
/* ------------------------------------------------------------------------ */
static int is_power_of(long long v, int r) {
  if (v < 1) return 0;
  while (v % r == 0) v /= r;
  return v == 1;
}

/* the radices the reference dispatches on (convolution.c:35-43,
 * convolution_2d.c:41-47, fft.c:16-24) */
static int radix_supported(int rank, int r) {
  return rank == 1 ? (r == 2 || r == 4 || r == 8) : (r == 2 || r == 4);
}

static int check_dims(int rank, const int* dims, int r, const char* fn) {
  for (int a = 0; a < rank; ++a) {
    if (!is_power_of(dims[a], r)) {
      t_status = PAC_ERROR_NOT_POWER;
      fprintf(stderr, "pac: %s: axis %d length %d is not a power of %d; data left untouched\n", fn,
              a, dims[a], r);
      return PAC_ERROR_NOT_POWER;
    }
  }
  return PAC_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* plan + staging-buffer cache                                              */
/* ------------------------------------------------------------------------ */
#define CACHE_SLOTS 16

/* An entry is pinned (pins > 0) from the moment a caller picks it under the
 * cache lock until it releases it; eviction only ever takes unpinned
 * entries, so an entry cannot be refilled with another shape between the
 * caller's lookup and its use.  When every slot is pinned (more concurrent
 * callers on distinct shapes than slots) the caller gets a private entry
 * that is freed on release. */
typedef struct {
  int used;
  int pins;        /* callers holding or waiting for this entry (cache lock) */
  int temporary;   /* private entry outside the cache, freed on release */
  int rank, dims[3], r;
  long long N;
  pac_plan_t plan; /* NULL for shapes the butterflies do not run on */
  double *x, *h;   /* device: x re|im, h re|im, each 2N doubles */
  int* rho;        /* device: N ints (permutation-only paths) */
  pac_stream_t s1, s2;
  unsigned long long last_use;
  pthread_mutex_t mu;
} entry_t;

static entry_t g_cache[CACHE_SLOTS];
static pthread_mutex_t g_cache_mu = PTHREAD_MUTEX_INITIALIZER;
static unsigned long long g_tick = 0;
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

static void cache_init(void) {
  for (int i = 0; i < CACHE_SLOTS; ++i) pthread_mutex_init(&g_cache[i].mu, NULL);
}

static void entry_release(entry_t* e) {
  if (e->plan) pac_plan_destroy(e->plan);
  pac_free(e->x);
  pac_free(e->h);
  pac_free(e->rho);
  if (e->s1) pac_stream_destroy(e->s1);
  if (e->s2) pac_stream_destroy(e->s2);
  e->plan = NULL;
  e->x = e->h = NULL;
  e->rho = NULL;
  e->s1 = e->s2 = NULL;
  e->used = 0;
}

/* plan, staging buffers and streams of an entry for (rank, dims, r) */
static int entry_fill(entry_t* e, int rank, const int* dims, int r, int want_plan) {
  e->used = 1;
  e->rank = rank;
  e->r = r;
  e->N = 1;
  for (int a = 0; a < 3; ++a) e->dims[a] = a < rank ? dims[a] : 1;
  for (int a = 0; a < rank; ++a) e->N *= dims[a];
  int st = PAC_SUCCESS;
  if (want_plan) st = pac_plan_create(&e->plan, rank, dims, 1, r, PAC_FORM_F64);
  if (st == PAC_SUCCESS) st = pac_malloc((void**)&e->x, (size_t)e->N * 16);
  if (st == PAC_SUCCESS) st = pac_malloc((void**)&e->h, (size_t)e->N * 16);
  if (st == PAC_SUCCESS) st = pac_malloc((void**)&e->rho, (size_t)e->N * sizeof(int));
  if (st == PAC_SUCCESS) st = pac_stream_create(&e->s1);
  if (st == PAC_SUCCESS) st = pac_stream_create(&e->s2);
  if (st != PAC_SUCCESS) entry_release(e);
  return st;
}

/* Returns a locked entry for (rank, dims, r); want_plan selects whether the
 * butterfly plan is built (radix supported and dims valid). */
static int acquire(int rank, const int* dims, int r, int want_plan, entry_t** out) {
  pthread_once(&g_once, cache_init);
  pthread_mutex_lock(&g_cache_mu);
  entry_t* hit = NULL;
  for (int i = 0; i < CACHE_SLOTS && !hit; ++i) {
    entry_t* e = &g_cache[i];
    if (!e->used || e->rank != rank || e->r != r || (want_plan && !e->plan)) continue;
    int same = 1;
    for (int a = 0; a < rank; ++a) same &= e->dims[a] == dims[a];
    if (same) hit = e;
  }
  if (hit) {
    hit->pins++;
    hit->last_use = ++g_tick;
    pthread_mutex_unlock(&g_cache_mu);
    pthread_mutex_lock(&hit->mu);  /* pinned: still this shape once locked */
    *out = hit;
    return PAC_SUCCESS;
  }
  /* free slot, else evict the least recently used unpinned one */
  entry_t* victim = NULL;
  for (int i = 0; i < CACHE_SLOTS && !victim; ++i)
    if (!g_cache[i].used && !g_cache[i].pins) victim = &g_cache[i];
  if (!victim) {
    for (int i = 0; i < CACHE_SLOTS; ++i) {
      entry_t* e = &g_cache[i];
      if (e->pins) continue;
      if (!victim || e->last_use < victim->last_use) victim = e;
    }
  }
  if (!victim) {
    /* every slot is in use by another caller: a private entry */
    pthread_mutex_unlock(&g_cache_mu);
    entry_t* e = (entry_t*)calloc(1, sizeof(entry_t));
    if (!e) return PAC_ERROR_ALLOC;
    pthread_mutex_init(&e->mu, NULL);
    e->temporary = 1;
    e->pins = 1;
    int st = entry_fill(e, rank, dims, r, want_plan);
    if (st != PAC_SUCCESS) {
      pthread_mutex_destroy(&e->mu);
      free(e);
      return st;
    }
    pthread_mutex_lock(&e->mu);
    *out = e;
    return PAC_SUCCESS;
  }
  /* unpinned: no caller holds its lock or waits for it */
  victim->pins++;
  pthread_mutex_lock(&victim->mu);
  if (victim->used) entry_release(victim);
  int st = entry_fill(victim, rank, dims, r, want_plan);
  if (st != PAC_SUCCESS) {
    victim->pins--;
    pthread_mutex_unlock(&victim->mu);
    pthread_mutex_unlock(&g_cache_mu);
    return st;
  }
  victim->last_use = ++g_tick;
  pthread_mutex_unlock(&g_cache_mu);
  *out = victim;
  return PAC_SUCCESS;
}

static void release(entry_t* e) {
  pthread_mutex_unlock(&e->mu);
  if (e->temporary) {
    entry_release(e);
    pthread_mutex_destroy(&e->mu);
    free(e);
    return;
  }
  pthread_mutex_lock(&g_cache_mu);
  e->pins--;
  pthread_mutex_unlock(&g_cache_mu);
}

#define TRY(x)                  \
  do {                          \
    st = (x);                   \
    if (st != PAC_SUCCESS) goto done; \
  } while (0)

/* ------------------------------------------------------------------------ */
/* operators                                                                */
/* ------------------------------------------------------------------------ */
enum {
  K_OP = 0,   /* one pac_transform op, no permutation fallback */
  K_FFT,      /* fft / fft2: natural order                       */
  K_UFFT,     /* ufft                                            */
  K_IFFT,     /* ifft                                            */
  K_UIFFT     /* uifft                                           */
};

/* x <- op(x) for the butterfly operators and the five transforms.  When
 * the radix is not supported the reference's transforms still permute by
 * rho and divide by n (fft.c:14, :57, :69-70): reproduced with rho.  */
static void run_op(const char* fn, int rank, const int* dims, int r, int kind, int op,
                   double* re, double* im, const int* rho) {
  if (!re || !im) {
    report(PAC_ERROR_INVALID_VALUE, fn);
    return;
  }
  int sup = radix_supported(rank, r);
  if (sup && check_dims(rank, dims, r, fn) != PAC_SUCCESS) return;
  entry_t* e = NULL;
  int st = acquire(rank, dims, r, sup, &e);
  if (st != PAC_SUCCESS) {
    report(st, fn);
    return;
  }
  const size_t nb = (size_t)e->N * sizeof(double);
  double* xr = e->x;
  double* xi = e->x + e->N;
  TRY(pac_memcpy_h2d(xr, re, nb, e->s1));
  TRY(pac_memcpy_h2d(xi, im, nb, e->s1));
  if (sup) {
    TRY(pac_transform(e->plan, op, xr, xi, xr, xi, e->s1));
  } else {
    int perm = (kind == K_FFT || kind == K_IFFT) && rho != NULL;
    if (perm) {
      TRY(pac_memcpy_h2d(e->rho, rho, (size_t)e->N * sizeof(int), e->s1));
      TRY(pac_permute(e->N, e->rho, xr, xi, e->s1));
    }
    if (kind == K_IFFT || kind == K_UIFFT)
      TRY(pac_scale(e->N, xr, xi, xr, xi, 1.0 / (double)e->N, e->s1));
  }
  TRY(pac_memcpy_d2h(re, xr, nb, e->s1));
  TRY(pac_memcpy_d2h(im, xi, nb, e->s1));
  TRY(pac_stream_synchronize(e->s1));
  if (e->plan) TRY(pac_plan_check_status(e->plan, e->s1));
done:
  release(e);
  report(st, fn);
}

/* permutation-avoiding convolution (convolution.c:31-71, convolution_2d.c:35,
 * convolution_3d.c:36): h <- A^T h (P_r order, unscaled, written back);
 * x <- conj(A)[(A^T x .* A^T h) / n].  Unsupported radix: x <- x .* h / n,
 * h untouched (the butterfly calls are skipped, the product loop runs). */
static void run_pac_conv(const char* fn, int rank, const int* dims, int r, double* re, double* im,
                         double* h_re, double* h_im) {
  if (!re || !im || !h_re || !h_im) {
    report(PAC_ERROR_INVALID_VALUE, fn);
    return;
  }
  int sup = radix_supported(rank, r);
  if (sup && check_dims(rank, dims, r, fn) != PAC_SUCCESS) return;
  entry_t* e = NULL;
  int st = acquire(rank, dims, r, sup, &e);
  if (st != PAC_SUCCESS) {
    report(st, fn);
    return;
  }
  const long long N = e->N;
  const size_t nb = (size_t)N * sizeof(double);
  double *xr = e->x, *xi = e->x + N, *hr = e->h, *hi = e->h + N;
  if (!sup) {
    TRY(pac_memcpy_h2d(xr, re, nb, e->s1));
    TRY(pac_memcpy_h2d(xi, im, nb, e->s1));
    TRY(pac_memcpy_h2d(hr, h_re, nb, e->s1));
    TRY(pac_memcpy_h2d(hi, h_im, nb, e->s1));
    TRY(pac_pointwise_product(N, xr, xi, hr, hi, xr, xi, 1.0 / (double)N, e->s1));
    TRY(pac_memcpy_d2h(re, xr, nb, e->s1));
    TRY(pac_memcpy_d2h(im, xi, nb, e->s1));
    TRY(pac_stream_synchronize(e->s1));
    goto done;
  }
  /* stream 1: filter in, A^T h, filter out; stream 2: signal in, convolve
   * once the filter spectrum is ready, signal out.  The filter's D2H and the
   * signal's H2D run in opposite directions and overlap. */
  TRY(pac_memcpy_h2d(hr, h_re, nb, e->s1));
  TRY(pac_memcpy_h2d(hi, h_im, nb, e->s1));
  /* A^T h in the reference's order goes back to the caller; the same
   * buffer is then reordered in place into the plan's spectrum order */
  TRY(pac_transform(e->plan, PAC_OP_AT, hr, hi, hr, hi, e->s1));
  TRY(pac_memcpy_h2d(xr, re, nb, e->s2));
  TRY(pac_memcpy_h2d(xi, im, nb, e->s2));
  TRY(pac_memcpy_d2h(h_re, hr, nb, e->s1));
  TRY(pac_memcpy_d2h(h_im, hi, nb, e->s1));
  TRY(pac_spectrum_to_plan_order(e->plan, hr, hi, 1, hr, hi, 1.0, e->s1));
  TRY(pac_stream_wait_stream(e->s2, e->s1));
  TRY(pac_convolve(e->plan, xr, xi, hr, hi, 0, xr, xi, 1.0 / (double)N, e->s2));
  TRY(pac_memcpy_d2h(re, xr, nb, e->s2));
  TRY(pac_memcpy_d2h(im, xi, nb, e->s2));
  TRY(pac_stream_synchronize(e->s1));
  TRY(pac_stream_synchronize(e->s2));
  if (e->plan) TRY(pac_plan_check_status(e->plan, e->s1));
done:
  release(e);
  report(st, fn);
}

/* FFT-based convolution (convolution.c:12-29, _2d.c:12, _3d.c:12):
 * h <- F h (natural order, written back); x <- F^-1 (F x .* F h).
 * Unsupported radix: the reference's fft() permutes by rho and skips the
 * butterflies, ifft() permutes and divides: reproduced with rho. */
static void run_fft_conv(const char* fn, int rank, const int* dims, int r, double* re, double* im,
                         const int* rho, double* h_re, double* h_im) {
  if (!re || !im || !h_re || !h_im) {
    report(PAC_ERROR_INVALID_VALUE, fn);
    return;
  }
  int sup = radix_supported(rank, r);
  if (sup && check_dims(rank, dims, r, fn) != PAC_SUCCESS) return;
  entry_t* e = NULL;
  int st = acquire(rank, dims, r, sup, &e);
  if (st != PAC_SUCCESS) {
    report(st, fn);
    return;
  }
  const long long N = e->N;
  const size_t nb = (size_t)N * sizeof(double);
  double *xr = e->x, *xi = e->x + N, *hr = e->h, *hi = e->h + N;
  TRY(pac_memcpy_h2d(xr, re, nb, e->s1));
  TRY(pac_memcpy_h2d(xi, im, nb, e->s1));
  TRY(pac_memcpy_h2d(hr, h_re, nb, e->s1));
  TRY(pac_memcpy_h2d(hi, h_im, nb, e->s1));
  if (sup) {
    TRY(pac_transform(e->plan, PAC_OP_FFT, hr, hi, hr, hi, e->s1));
    TRY(pac_transform(e->plan, PAC_OP_FFT, xr, xi, xr, xi, e->s1));
    TRY(pac_pointwise_product(N, xr, xi, hr, hi, xr, xi, 1.0, e->s1));
    TRY(pac_transform(e->plan, PAC_OP_IFFT, xr, xi, xr, xi, e->s1));
  } else {
    if (rho) {
      TRY(pac_memcpy_h2d(e->rho, rho, (size_t)N * sizeof(int), e->s1));
      TRY(pac_permute(N, e->rho, xr, xi, e->s1));
      TRY(pac_permute(N, e->rho, hr, hi, e->s1));
    }
    TRY(pac_pointwise_product(N, xr, xi, hr, hi, xr, xi, 1.0 / (double)N, e->s1));
    if (rho) TRY(pac_permute(N, e->rho, xr, xi, e->s1));
  }
  TRY(pac_memcpy_d2h(h_re, hr, nb, e->s1));
  TRY(pac_memcpy_d2h(h_im, hi, nb, e->s1));
  TRY(pac_memcpy_d2h(re, xr, nb, e->s1));
  TRY(pac_memcpy_d2h(im, xi, nb, e->s1));
  TRY(pac_stream_synchronize(e->s1));
  if (e->plan) TRY(pac_plan_check_status(e->plan, e->s1));
done:
  release(e);
  report(st, fn);
}

/* ------------------------------------------------------------------------ */
/* twiddle_factors.c (reference fft.h:17-21): tables generated on the GPU  */
/* in FP64, returned in the reference's jagged layout.                     */
/* ------------------------------------------------------------------------ */
static int ref_levels(int n, int r) {
  int t = 0;
  if (n < 1) return 0;
  if (r == 2) {
    while (!((n >> t) & 1)) ++t;
    return t;
  }
  int sh = r == 4 ? 2 : 3;
  for (int v = n; v > 1; v >>= sh) ++t;
  return t;
}

static void make_twiddles(const char* fn, int r, int n, double*** tre, double*** tim) {
  int t = ref_levels(n, r);
  *tre = (double**)malloc((t > 0 ? t : 1) * sizeof(double*));
  *tim = (double**)malloc((t > 0 ? t : 1) * sizeof(double*));
  long long total = 1;
  for (int q = 0; q < t; ++q) total *= r;
  total -= 1;
  double* hbuf = (double*)calloc((size_t)(total > 0 ? total : 1) * 2, sizeof(double));
  int st = PAC_SUCCESS;
  if (total > 0) {
    double* d = NULL;
    st = pac_malloc((void**)&d, (size_t)total * 2 * sizeof(double));
    if (st == PAC_SUCCESS) st = pac_reference_twiddles(r, n, d, d + total, NULL);
    if (st == PAC_SUCCESS) st = pac_memcpy_d2h(hbuf, d, (size_t)total * 2 * sizeof(double), NULL);
    if (st == PAC_SUCCESS) st = pac_stream_synchronize(NULL);
    pac_free(d);
  }
  long long off = 0, ell = 1;
  for (int q = 0; q < t; ++q) {
    long long cnt = (r - 1) * ell;
    (*tre)[q] = (double*)malloc((size_t)cnt * sizeof(double));
    (*tim)[q] = (double*)malloc((size_t)cnt * sizeof(double));
    memcpy((*tre)[q], hbuf + off, (size_t)cnt * sizeof(double));
    memcpy((*tim)[q], hbuf + total + off, (size_t)cnt * sizeof(double));
    off += cnt;
    ell *= r;
  }
  free(hbuf);
  report(st, fn);
}

void precompute_twiddles_r2(int n, double*** twiddle_re, double*** twiddle_im) {
  make_twiddles("precompute_twiddles_r2", 2, n, twiddle_re, twiddle_im);
}
void precompute_twiddles_r4(int n, double*** twiddle_re, double*** twiddle_im) {
  make_twiddles("precompute_twiddles_r4", 4, n, twiddle_re, twiddle_im);
}
void precompute_twiddles_r8(int n, double*** twiddle_re, double*** twiddle_im) {
  make_twiddles("precompute_twiddles_r8", 8, n, twiddle_re, twiddle_im);
}
void free_twiddles(double** twiddle_re, double** twiddle_im, int t) {
  if (twiddle_re)
    for (int q = 0; q < t; ++q) free(twiddle_re[q]);
  if (twiddle_im)
    for (int q = 0; q < t; ++q) free(twiddle_im[q]);
  free(twiddle_re);
  free(twiddle_im);
}

/* ------------------------------------------------------------------------ */
/* butterflies.c, butterflies_2d.c, butterflies_3d.c (reference fft.h:23-99) */
/* ------------------------------------------------------------------------ */
#define ONE_D(name, r, op)                                                              \
  void name(double* restrict re, double* restrict im, int n, const double** twiddle_re, \
            const double** twiddle_im) {                                                \
    (void)twiddle_re;                                                                   \
    (void)twiddle_im;                                                                   \
    int dims[1] = {n};                                                                  \
    run_op(#name, 1, dims, r, K_OP, op, re, im, NULL);                                  \
  }
ONE_D(apply_butterflies_r2, 2, PAC_OP_A)
ONE_D(apply_conjugate_butterflies_r2, 2, PAC_OP_CONJ_A)
ONE_D(apply_transposed_butterflies_r2, 2, PAC_OP_AT)
ONE_D(apply_butterflies_r4, 4, PAC_OP_A)
ONE_D(apply_conjugate_butterflies_r4, 4, PAC_OP_CONJ_A)
ONE_D(apply_transposed_butterflies_r4, 4, PAC_OP_AT)
ONE_D(apply_butterflies_r8, 8, PAC_OP_A)
ONE_D(apply_conjugate_butterflies_r8, 8, PAC_OP_CONJ_A)
ONE_D(apply_transposed_butterflies_r8, 8, PAC_OP_AT)

#define TWO_D(name, r, op)                                                              \
  void name(double* restrict re, double* restrict im, int n1, int n2,                   \
            const double** twiddle_re1, const double** twiddle_im1,                     \
            const double** twiddle_re2, const double** twiddle_im2) {                   \
    (void)twiddle_re1;                                                                  \
    (void)twiddle_im1;                                                                  \
    (void)twiddle_re2;                                                                  \
    (void)twiddle_im2;                                                                  \
    int dims[2] = {n1, n2};                                                             \
    run_op(#name, 2, dims, r, K_OP, op, re, im, NULL);                                  \
  }
TWO_D(apply_butterflies_r2_2d, 2, PAC_OP_A)
TWO_D(apply_conjugate_butterflies_r2_2d, 2, PAC_OP_CONJ_A)
TWO_D(apply_transposed_butterflies_r2_2d, 2, PAC_OP_AT)
TWO_D(apply_butterflies_r4_2d, 4, PAC_OP_A)
TWO_D(apply_conjugate_butterflies_r4_2d, 4, PAC_OP_CONJ_A)
TWO_D(apply_transposed_butterflies_r4_2d, 4, PAC_OP_AT)

#define THREE_D(name, r, op)                                                            \
  void name(double* restrict re, double* restrict im, int n1, int n2, int n3,           \
            const double** twiddle_re1, const double** twiddle_im1,                     \
            const double** twiddle_re2, const double** twiddle_im2,                     \
            const double** twiddle_re3, const double** twiddle_im3) {                   \
    (void)twiddle_re1;                                                                  \
    (void)twiddle_im1;                                                                  \
    (void)twiddle_re2;                                                                  \
    (void)twiddle_im2;                                                                  \
    (void)twiddle_re3;                                                                  \
    (void)twiddle_im3;                                                                  \
    int dims[3] = {n1, n2, n3};                                                         \
    run_op(#name, 3, dims, r, K_OP, op, re, im, NULL);                                  \
  }
THREE_D(apply_butterflies_r2_3d, 2, PAC_OP_A)
THREE_D(apply_conjugate_butterflies_r2_3d, 2, PAC_OP_CONJ_A)
THREE_D(apply_transposed_butterflies_r2_3d, 2, PAC_OP_AT)
THREE_D(apply_butterflies_r4_3d, 4, PAC_OP_A)
THREE_D(apply_conjugate_butterflies_r4_3d, 4, PAC_OP_CONJ_A)
THREE_D(apply_transposed_butterflies_r4_3d, 4, PAC_OP_AT)

/* ------------------------------------------------------------------------ */
/* fft.c, fft_2d.c, fft_3d.c (reference fft.h:120-185)                      */
/* ------------------------------------------------------------------------ */
void fft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
         double** twiddle_im, const int* rho) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_op("fft", 1, dims, r, K_FFT, PAC_OP_FFT, re, im, rho);
}
void fft2(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
          double** twiddle_im, const int* rho) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_op("fft2", 1, dims, r, K_FFT, PAC_OP_FFT, re, im, rho);
}
void ufft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
          double** twiddle_im) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_op("ufft", 1, dims, r, K_UFFT, PAC_OP_UFFT, re, im, NULL);
}
void ifft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
          double** twiddle_im, const int* rho) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_op("ifft", 1, dims, r, K_IFFT, PAC_OP_IFFT, re, im, rho);
}
void uifft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
           double** twiddle_im) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_op("uifft", 1, dims, r, K_UIFFT, PAC_OP_UIFFT, re, im, NULL);
}

#define FFT2D(name, kind, op, RHO_PARAM, RHO)                                              \
  void name(double* restrict re, double* restrict im, int n1, int n2, int r,               \
            double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,              \
            double** twiddle_im2 RHO_PARAM) {                                              \
    (void)twiddle_re1;                                                                     \
    (void)twiddle_im1;                                                                     \
    (void)twiddle_re2;                                                                     \
    (void)twiddle_im2;                                                                     \
    int dims[2] = {n1, n2};                                                                \
    run_op(#name, 2, dims, r, kind, op, re, im, RHO);                                      \
  }
#define FFT3D(name, kind, op, RHO_PARAM, RHO)                                              \
  void name(double* restrict re, double* restrict im, int n1, int n2, int n3, int r,       \
            double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,              \
            double** twiddle_im2, double** twiddle_re3, double** twiddle_im3 RHO_PARAM) {  \
    (void)twiddle_re1;                                                                     \
    (void)twiddle_im1;                                                                     \
    (void)twiddle_re2;                                                                     \
    (void)twiddle_im2;                                                                     \
    (void)twiddle_re3;                                                                     \
    (void)twiddle_im3;                                                                     \
    int dims[3] = {n1, n2, n3};                                                            \
    run_op(#name, 3, dims, r, kind, op, re, im, RHO);                                      \
  }
#define WITH_RHO , const int* rho
#define NO_RHO
FFT2D(fft_2d, K_FFT, PAC_OP_FFT, WITH_RHO, rho)
FFT2D(fft2_2d, K_FFT, PAC_OP_FFT, WITH_RHO, rho)
FFT2D(ufft_2d, K_UFFT, PAC_OP_UFFT, NO_RHO, NULL)
FFT2D(ifft_2d, K_IFFT, PAC_OP_IFFT, WITH_RHO, rho)
FFT2D(uifft_2d, K_UIFFT, PAC_OP_UIFFT, NO_RHO, NULL)
FFT3D(fft_3d, K_FFT, PAC_OP_FFT, WITH_RHO, rho)
FFT3D(fft2_3d, K_FFT, PAC_OP_FFT, WITH_RHO, rho)
FFT3D(ufft_3d, K_UFFT, PAC_OP_UFFT, NO_RHO, NULL)
FFT3D(ifft_3d, K_IFFT, PAC_OP_IFFT, WITH_RHO, rho)
FFT3D(uifft_3d, K_UIFFT, PAC_OP_UIFFT, NO_RHO, NULL)

/* ------------------------------------------------------------------------ */
/* convolution.c, _2d.c, _3d.c (reference fft.h:187-221)                    */
/* ------------------------------------------------------------------------ */
void fft_based_convolution(double* restrict re, double* restrict im, int n, int r,
                           double** twiddle_re, double** twiddle_im, const int* rho,
                           double* restrict g_re, double* restrict g_im) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_fft_conv("fft_based_convolution", 1, dims, r, re, im, rho, g_re, g_im);
}
void permutation_avoiding_convolution(double* restrict re, double* restrict im, int n, int r,
                                      double** twiddle_re, double** twiddle_im,
                                      double* restrict Pg_re, double* restrict Pg_im) {
  (void)twiddle_re;
  (void)twiddle_im;
  int dims[1] = {n};
  run_pac_conv("permutation_avoiding_convolution", 1, dims, r, re, im, Pg_re, Pg_im);
}
void fft_based_convolution_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
                              double** twiddle_re1, double** twiddle_im1,
                              double** twiddle_re2, double** twiddle_im2, const int* rho,
                              double* restrict g_re, double* restrict g_im) {
  (void)twiddle_re1;
  (void)twiddle_im1;
  (void)twiddle_re2;
  (void)twiddle_im2;
  int dims[2] = {n1, n2};
  run_fft_conv("fft_based_convolution_2d", 2, dims, r, re, im, rho, g_re, g_im);
}
void permutation_avoiding_convolution_2d(double* restrict re, double* restrict im, int n1,
                                         int n2, int r, double** twiddle_re1,
                                         double** twiddle_im1, double** twiddle_re2,
                                         double** twiddle_im2, double* restrict Pg_re,
                                         double* restrict Pg_im) {
  (void)twiddle_re1;
  (void)twiddle_im1;
  (void)twiddle_re2;
  (void)twiddle_im2;
  int dims[2] = {n1, n2};
  run_pac_conv("permutation_avoiding_convolution_2d", 2, dims, r, re, im, Pg_re, Pg_im);
}
void fft_based_convolution_3d(double* restrict re, double* restrict im, int n1, int n2, int n3,
                              int r, double** twiddle_re1, double** twiddle_im1,
                              double** twiddle_re2, double** twiddle_im2,
                              double** twiddle_re3, double** twiddle_im3, const int* rho,
                              double* restrict g_re, double* restrict g_im) {
  (void)twiddle_re1;
  (void)twiddle_im1;
  (void)twiddle_re2;
  (void)twiddle_im2;
  (void)twiddle_re3;
  (void)twiddle_im3;
  int dims[3] = {n1, n2, n3};
  run_fft_conv("fft_based_convolution_3d", 3, dims, r, re, im, rho, g_re, g_im);
}
void permutation_avoiding_convolution_3d(double* restrict re, double* restrict im, int n1,
                                         int n2, int n3, int r, double** twiddle_re1,
                                         double** twiddle_im1, double** twiddle_re2,
                                         double** twiddle_im2, double** twiddle_re3,
                                         double** twiddle_im3, double* restrict Pg_re,
                                         double* restrict Pg_im) {
  (void)twiddle_re1;
  (void)twiddle_im1;
  (void)twiddle_re2;
  (void)twiddle_im2;
  (void)twiddle_re3;
  (void)twiddle_im3;
  int dims[3] = {n1, n2, n3};
  run_pac_conv("permutation_avoiding_convolution_3d", 3, dims, r, re, im, Pg_re, Pg_im);
}

/* ------------------------------------------------------------------------ */
/* index_reversals*.c (reference fft.h:101-118): host-side table builders  */
/* ------------------------------------------------------------------------ */
static int digit_reverse(int x, int t, int bits) {
  int v = 0;
  for (int i = 0; i < t; ++i) {
    v = (v << bits) | (x & ((1 << bits) - 1));
    x >>= bits;
  }
  return v;
}
int reverse_index_r2(int x, int t) { return digit_reverse(x, t, 1); }
int reverse_index_r4(int x, int t) { return digit_reverse(x, t, 2); }
int reverse_index_r8(int x, int t) { return digit_reverse(x, t, 3); }

static int* rho_nd(int rank, const int* dims, int r) {
  int bits = r == 2 ? 1 : r == 4 ? 2 : 3;
  long long n = 1;
  int t[3] = {0, 0, 0};
  for (int a = 0; a < rank; ++a) {
    n *= dims[a];
    t[a] = ref_levels(dims[a], r);
  }
  int* rho = (int*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
  if (!rho) return NULL;
  for (long long idx = 0; idx < n; ++idx) {
    long long rem = idx, out = 0, mul = 1;
    for (int a = rank - 1; a >= 0; --a) {
      int i = (int)(rem % dims[a]);
      rem /= dims[a];
      out += mul * digit_reverse(i, t[a], bits);
      mul *= dims[a];
    }
    rho[idx] = (int)out;
  }
  return rho;
}
int* precompute_index_reversal_permutation_r2(int n) { return rho_nd(1, &n, 2); }
int* precompute_index_reversal_permutation_r4(int n) { return rho_nd(1, &n, 4); }
int* precompute_index_reversal_permutation_r8(int n) { return rho_nd(1, &n, 8); }
int* precompute_index_reversal_permutation_r2_2d(int n1, int n2) {
  int d[2] = {n1, n2};
  return rho_nd(2, d, 2);
}
int* precompute_index_reversal_permutation_r4_2d(int n1, int n2) {
  int d[2] = {n1, n2};
  return rho_nd(2, d, 4);
}
int* precompute_index_reversal_permutation_r2_3d(int n1, int n2, int n3) {
  int d[3] = {n1, n2, n3};
  return rho_nd(3, d, 2);
}
int* precompute_index_reversal_permutation_r4_3d(int n1, int n2, int n3) {
  int d[3] = {n1, n2, n3};
  return rho_nd(3, d, 4);
}

/* standalone permutations (index_reversals.c:74-94) on the GPU */
static void run_permute(const char* fn, double* re, double* im, int n, const int* rho) {
  if (!re || !rho || n < 0) {
    report(PAC_ERROR_INVALID_VALUE, fn);
    return;
  }
  if (n == 0) return;
  int st;
  void *d = NULL, *dr = NULL;
  size_t nb = (size_t)n * sizeof(double) * (im ? 1 : 2);
  st = pac_malloc(&d, nb * (im ? 2 : 1));
  if (st == PAC_SUCCESS) st = pac_malloc(&dr, (size_t)n * sizeof(int));
  double* dre = (double*)d;
  double* dim = im ? dre + n : NULL;
  if (st == PAC_SUCCESS) st = pac_memcpy_h2d(dre, re, nb, NULL);
  if (st == PAC_SUCCESS && im) st = pac_memcpy_h2d(dim, im, nb, NULL);
  if (st == PAC_SUCCESS) st = pac_memcpy_h2d(dr, rho, (size_t)n * sizeof(int), NULL);
  if (st == PAC_SUCCESS) st = pac_permute(n, (const int*)dr, dre, dim, NULL);
  if (st == PAC_SUCCESS) st = pac_memcpy_d2h(re, dre, nb, NULL);
  if (st == PAC_SUCCESS && im) st = pac_memcpy_d2h(im, dim, nb, NULL);
  if (st == PAC_SUCCESS) st = pac_stream_synchronize(NULL);
  pac_free(d);
  pac_free(dr);
  report(st, fn);
}
void apply_permutation(PAC_FFT_H_COMPLEX* x, int n, const int* rho) {
  run_permute("apply_permutation", (double*)x, NULL, n, rho);
}
void apply_permutation_split(double* restrict re, double* restrict im, int n, const int* rho) {
  if (!im) {
    report(PAC_ERROR_INVALID_VALUE, "apply_permutation_split");
    return;
  }
  run_permute("apply_permutation_split", re, im, n, rho);
}

/* ------------------------------------------------------------------------ */
/* misc.c (reference fft.h:223-229): host utilities of the reference's     */
/* drivers (timing, error metric, rand() inputs); not on the device path.  */
/* ------------------------------------------------------------------------ */
double time_diff(struct timespec start, struct timespec end) {
  return (double)(end.tv_sec - start.tv_sec) + (double)(end.tv_nsec - start.tv_nsec) * 1e-9;
}

double get_max_error(double* re, double* im, double* fftw_flat, int n) {
  double m = 0.0;
  for (int i = 0; i < n; ++i) {
    double e = hypot(re[i] - fftw_flat[2 * i], im[i] - fftw_flat[2 * i + 1]);
    if (e > m) m = e;
  }
  return m;
}

void initialize_data(PAC_FFT_H_COMPLEX* x, double* fftw_in_flat, int n) {
  double* z = (double*)x;
  for (int i = 0; i < n; ++i) {
    double a = rand() / (double)RAND_MAX;
    double b = rand() / (double)RAND_MAX;
    z[2 * i] = a;
    z[2 * i + 1] = b;
    fftw_in_flat[2 * i] = a;
    fftw_in_flat[2 * i + 1] = b;
  }
}

void initialize_data_split(double* re, double* im, double* fftw_in_flat, int n) {
  for (int i = 0; i < n; ++i) {
    re[i] = rand() / (double)RAND_MAX;
    im[i] = rand() / (double)RAND_MAX;
    fftw_in_flat[2 * i] = re[i];
    fftw_in_flat[2 * i + 1] = im[i];
  }
}

void initialize_filter(double* g_re, double* g_im, int n) {
  for (int i = 0; i < n; ++i) {
    g_re[i] = rand() / (double)RAND_MAX;
    g_im[i] = rand() / (double)RAND_MAX;
  }
}

bool supports_radix_4(int t2) { return t2 % 2 == 0; }
bool supports_radix_8(int t2) { return t2 % 3 == 0; }

void in_place_square_array_transpose_split_2d(double* re, double* im, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) {
      size_t a = (size_t)i * n + j, b = (size_t)j * n + i;
      double t = re[a];
      re[a] = re[b];
      re[b] = t;
      t = im[a];
      im[a] = im[b];
      im[b] = t;
    }
}

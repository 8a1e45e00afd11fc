/*
 * fft.h -- drop-in C ABI of venkovic/c-permutation-avoiding-convolution,
 * served by the B200 library (libpac.so).
 *
 * Every prototype below is the reference's own (reference fft.h:17-229,
 * line cited per group), with the same argument meaning, so code written
 * against the reference (its bench*.c drivers included) compiles and links
 * unchanged.  Behaviour follows the reference:
 *
 *  - arrays are host pointers, split complex (re[], im[]), row-major;
 *  - every call is synchronous and returns after the result is back in the
 *    caller's arrays;
 *  - permutation_avoiding_convolution* overwrite re/im with the circular
 *    convolution and h_re/h_im with A^T h (convolution.c:45-53);
 *  - an unsupported radix skips the butterflies exactly as the reference's
 *    if/else chains do (e.g. r = 8 in 2D leaves x .* h / n);
 *  - twiddle tables passed in are accepted and not read: the device
 *    generates its own in FP64;
 *  - rho arguments are accepted and not read: natural order is produced by
 *    the device passes, never by a separate permutation pass.
 *
 * Differences (the reference has no error reporting): an axis length that
 * is not a power of r, a NULL array or a CUDA failure leaves the data
 * untouched, prints one line to stderr and records a status that
 * pac_get_last_status() (pac.h) returns.
 */
#ifndef FFT_H
#define FFT_H

#include <stdbool.h>
#include <stdlib.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#define restrict __restrict__
typedef struct {
  double re, im;
} pac_fft_h_complex_;
#define PAC_FFT_H_COMPLEX pac_fft_h_complex_
#else
#include <complex.h>
#define PAC_FFT_H_COMPLEX double complex
#endif

/* twiddle_factors.c (reference fft.h:17-21) */
void precompute_twiddles_r2(int n, double*** twiddle_re, double*** twiddle_im);
void precompute_twiddles_r4(int n, double*** twiddle_re, double*** twiddle_im);
void precompute_twiddles_r8(int n, double*** twiddle_re, double*** twiddle_im);
void free_twiddles(double** twiddle_re, double** twiddle_im, int t);

/* butterflies.c (reference fft.h:23-41) */
void apply_butterflies_r2(double* restrict re, double* restrict im, int n,
                          const double** twiddle_re, const double** twiddle_im);
void apply_conjugate_butterflies_r2(double* restrict re, double* restrict im, int n,
                                    const double** twiddle_re, const double** twiddle_im);
void apply_transposed_butterflies_r2(double* restrict re, double* restrict im, int n,
                                     const double** twiddle_re, const double** twiddle_im);
void apply_butterflies_r4(double* restrict re, double* restrict im, int n,
                          const double** twiddle_re, const double** twiddle_im);
void apply_conjugate_butterflies_r4(double* restrict re, double* restrict im, int n,
                                    const double** twiddle_re, const double** twiddle_im);
void apply_transposed_butterflies_r4(double* restrict re, double* restrict im, int n,
                                     const double** twiddle_re, const double** twiddle_im);
void apply_butterflies_r8(double* restrict re, double* restrict im, int n,
                          const double** twiddle_re, const double** twiddle_im);
void apply_conjugate_butterflies_r8(double* restrict re, double* restrict im, int n,
                                    const double** twiddle_re, const double** twiddle_im);
void apply_transposed_butterflies_r8(double* restrict re, double* restrict im, int n,
                                     const double** twiddle_re, const double** twiddle_im);

/* butterflies_2d.c (reference fft.h:43-71) */
void apply_butterflies_r2_2d(double* restrict re, double* restrict im, int n1, int n2,
                             const double** twiddle_re1, const double** twiddle_im1,
                             const double** twiddle_re2, const double** twiddle_im2);
void apply_conjugate_butterflies_r2_2d(double* restrict re, double* restrict im, int n1, int n2,
                                       const double** twiddle_re1, const double** twiddle_im1,
                                       const double** twiddle_re2, const double** twiddle_im2);
void apply_transposed_butterflies_r2_2d(double* restrict re, double* restrict im, int n1, int n2,
                                        const double** twiddle_re1, const double** twiddle_im1,
                                        const double** twiddle_re2, const double** twiddle_im2);
void apply_butterflies_r4_2d(double* restrict re, double* restrict im, int n1, int n2,
                             const double** twiddle_re1, const double** twiddle_im1,
                             const double** twiddle_re2, const double** twiddle_im2);
void apply_conjugate_butterflies_r4_2d(double* restrict re, double* restrict im, int n1, int n2,
                                       const double** twiddle_re1, const double** twiddle_im1,
                                       const double** twiddle_re2, const double** twiddle_im2);
void apply_transposed_butterflies_r4_2d(double* restrict re, double* restrict im, int n1, int n2,
                                        const double** twiddle_re1, const double** twiddle_im1,
                                        const double** twiddle_re2, const double** twiddle_im2);

/* butterflies_3d.c (reference fft.h:73-99) */
void apply_butterflies_r2_3d(double* restrict re, double* restrict im, int n1, int n2, int n3,
                             const double** twiddle_re1, const double** twiddle_im1,
                             const double** twiddle_re2, const double** twiddle_im2,
                             const double** twiddle_re3, const double** twiddle_im3);
void apply_conjugate_butterflies_r2_3d(double* restrict re, double* restrict im, int n1, int n2,
                                       int n3, const double** twiddle_re1,
                                       const double** twiddle_im1, const double** twiddle_re2,
                                       const double** twiddle_im2, const double** twiddle_re3,
                                       const double** twiddle_im3);
void apply_transposed_butterflies_r2_3d(double* restrict re, double* restrict im, int n1, int n2,
                                        int n3, const double** twiddle_re1,
                                        const double** twiddle_im1, const double** twiddle_re2,
                                        const double** twiddle_im2, const double** twiddle_re3,
                                        const double** twiddle_im3);
void apply_butterflies_r4_3d(double* restrict re, double* restrict im, int n1, int n2, int n3,
                             const double** twiddle_re1, const double** twiddle_im1,
                             const double** twiddle_re2, const double** twiddle_im2,
                             const double** twiddle_re3, const double** twiddle_im3);
void apply_conjugate_butterflies_r4_3d(double* restrict re, double* restrict im, int n1, int n2,
                                       int n3, const double** twiddle_re1,
                                       const double** twiddle_im1, const double** twiddle_re2,
                                       const double** twiddle_im2, const double** twiddle_re3,
                                       const double** twiddle_im3);
void apply_transposed_butterflies_r4_3d(double* restrict re, double* restrict im, int n1, int n2,
                                        int n3, const double** twiddle_re1,
                                        const double** twiddle_im1, const double** twiddle_re2,
                                        const double** twiddle_im2, const double** twiddle_re3,
                                        const double** twiddle_im3);

/* index_reversals.c, _2d.c, _3d.c (reference fft.h:101-118).  Host-side
 * table builders and the standalone permutation; the transforms never use
 * them. */
int reverse_index_r2(int x, int t);
int* precompute_index_reversal_permutation_r2(int n);
int reverse_index_r4(int x, int t);
int* precompute_index_reversal_permutation_r4(int n);
int reverse_index_r8(int x, int t);
int* precompute_index_reversal_permutation_r8(int n);
void apply_permutation(PAC_FFT_H_COMPLEX* x, int n, const int* rho);
void apply_permutation_split(double* restrict re, double* restrict im, int n, const int* rho);
int* precompute_index_reversal_permutation_r2_2d(int n1, int n2);
int* precompute_index_reversal_permutation_r4_2d(int n1, int n2);
int* precompute_index_reversal_permutation_r2_3d(int n1, int n2, int n3);
int* precompute_index_reversal_permutation_r4_3d(int n1, int n2, int n3);

/* fft.c (reference fft.h:120-131) */
void fft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
         double** twiddle_im, const int* rho);
void fft2(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
          double** twiddle_im, const int* rho);
void ufft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
          double** twiddle_im);
void ifft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
          double** twiddle_im, const int* rho);
void uifft(double* restrict re, double* restrict im, int n, int r, double** twiddle_re,
           double** twiddle_im);

/* fft_2d.c (reference fft.h:133-157) */
void fft_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
            double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
            double** twiddle_im2, const int* rho);
void fft2_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
             double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
             double** twiddle_im2, const int* rho);
void ufft_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
             double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
             double** twiddle_im2);
void ifft_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
             double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
             double** twiddle_im2, const int* rho);
void uifft_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
              double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
              double** twiddle_im2);

/* fft_3d.c (reference fft.h:159-185) */
void fft_3d(double* restrict re, double* restrict im, int n1, int n2, int n3, int r,
            double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
            double** twiddle_im2, double** twiddle_re3, double** twiddle_im3, const int* rho);
void fft2_3d(double* restrict re, double* restrict im, int n1, int n2, int n3, int r,
             double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
             double** twiddle_im2, double** twiddle_re3, double** twiddle_im3, const int* rho);
void ufft_3d(double* restrict re, double* restrict im, int n1, int n2, int n3, int r,
             double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
             double** twiddle_im2, double** twiddle_re3, double** twiddle_im3);
void ifft_3d(double* restrict re, double* restrict im, int n1, int n2, int n3, int r,
             double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
             double** twiddle_im2, double** twiddle_re3, double** twiddle_im3, const int* rho);
void uifft_3d(double* restrict re, double* restrict im, int n1, int n2, int n3, int r,
              double** twiddle_re1, double** twiddle_im1, double** twiddle_re2,
              double** twiddle_im2, double** twiddle_re3, double** twiddle_im3);

/* convolution.c (reference fft.h:187-193) */
void fft_based_convolution(double* restrict re, double* restrict im, int n, int r,
                           double** twiddle_re, double** twiddle_im, const int* rho,
                           double* restrict g_re, double* restrict g_im);
void permutation_avoiding_convolution(double* restrict re, double* restrict im, int n, int r,
                                      double** twiddle_re, double** twiddle_im,
                                      double* restrict Pg_re, double* restrict Pg_im);

/* convolution_2d.c (reference fft.h:195-206) */
void fft_based_convolution_2d(double* restrict re, double* restrict im, int n1, int n2, int r,
                              double** twiddle_re1, double** twiddle_im1,
                              double** twiddle_re2, double** twiddle_im2, const int* rho,
                              double* restrict g_re, double* restrict g_im);
void permutation_avoiding_convolution_2d(double* restrict re, double* restrict im, int n1,
                                         int n2, int r, double** twiddle_re1,
                                         double** twiddle_im1, double** twiddle_re2,
                                         double** twiddle_im2, double* restrict Pg_re,
                                         double* restrict Pg_im);

/* convolution_3d.c (reference fft.h:208-221) */
void fft_based_convolution_3d(double* restrict re, double* restrict im, int n1, int n2, int n3,
                              int r, double** twiddle_re1, double** twiddle_im1,
                              double** twiddle_re2, double** twiddle_im2,
                              double** twiddle_re3, double** twiddle_im3, const int* rho,
                              double* restrict g_re, double* restrict g_im);
void permutation_avoiding_convolution_3d(double* restrict re, double* restrict im, int n1,
                                         int n2, int n3, int r, double** twiddle_re1,
                                         double** twiddle_im1, double** twiddle_re2,
                                         double** twiddle_im2, double** twiddle_re3,
                                         double** twiddle_im3, double* restrict Pg_re,
                                         double* restrict Pg_im);

/* misc.c (reference fft.h:223-229): host utilities of the reference drivers */
double time_diff(struct timespec start, struct timespec end);
double get_max_error(double* re, double* im, double* fftw_flat, int n);
void initialize_data(PAC_FFT_H_COMPLEX* x, double* fftw_in_flat, int n);
void initialize_data_split(double* re, double* im, double* fftw_in_flat, int n);
void initialize_filter(double* g_re, double* g_im, int n);
bool supports_radix_4(int t2);
bool supports_radix_8(int t2);
void in_place_square_array_transpose_split_2d(double* re, double* im, int n);

#ifdef __cplusplus
#undef restrict
}
#endif

#endif /* FFT_H */

/*
 * pac.h -- native C ABI of the B200 permutation-avoiding FFT convolution.
 *
 * Plain C: opaque plan handles, device pointers, sizes and int status codes.
 * The reference (venkovic/c-permutation-avoiding-convolution) has no plan
 * object and no device API; every entry point below states which reference
 * function(s) it stands in for.  The reference-compatible host-pointer
 * entry points (identical prototypes) are declared in fft.h and are built
 * on top of this header.
 *
 * Data layout (the reference's): split complex arrays -- one array of real
 * parts, one of imaginary parts -- row-major with the last axis contiguous
 * (butterflies_3d.c:24-26).  A plan covers `batch` independent problems
 * stored back to back.
 *
 * Spectrum order: the forward stages leave the spectrum of every axis in
 * base-b digit-reversed order P_b (b = the plan's digit base), exactly as
 * the reference's transposed butterflies do (A^T x = P_b F x).  With b equal
 * to the reference radix r the order is bit-identical to the reference's.
 *
 * Forms: PAC_FORM_F64 computes and stores complex FP64.  PAC_FORM_F32 stores
 * and computes FP32, with twiddles and the filter spectrum computed in FP64
 * on the device and rounded once.  PAC_FORM_TC is PAC_FORM_F32 with every
 * radix-16 stage run on the tensor cores: dense 16 x 16 complex DFT products
 * on split hi + lo FP16 operands (three products, FP32 accumulation, a
 * power-of-two scale per butterfly); the other stages, the twiddles and the
 * filter product stay FP32 on the CUDA cores.
 *
 * Threading: plans are immutable after creation; calls on one plan from
 * several host threads are safe when they use distinct buffers (the plan's
 * workspace is locked internally).  All device work is asynchronous on the
 * given stream unless stated otherwise.
 */
#ifndef PAC_H
#define PAC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PAC_API __attribute__((visibility("default")))
#else
#define PAC_API
#endif

typedef struct pac_plan_s* pac_plan_t;
typedef void* pac_stream_t; /* a cudaStream_t; NULL is the legacy default stream */

/* status codes */
enum {
  PAC_SUCCESS = 0,
  PAC_ERROR_INVALID_VALUE = 1,     /* NULL pointer, bad rank/batch/op      */
  PAC_ERROR_NOT_POWER = 2,         /* an axis length is not a power of b   */
  PAC_ERROR_UNSUPPORTED_RADIX = 3, /* digit base / radix not supported     */
  PAC_ERROR_SIZE = 4,              /* problem larger than the int index range */
  PAC_ERROR_CUDA = 5,              /* a CUDA runtime call failed           */
  PAC_ERROR_NO_DEVICE = 6,         /* no usable sm_100 device              */
  PAC_ERROR_ALLOC = 7,             /* device or host allocation failed     */
  PAC_ERROR_TIMEOUT = 8,           /* a bounded device wait gave up        */
  PAC_ERROR_INTERNAL = 9
};

/* storage / compute forms */
enum { PAC_FORM_F64 = 0, PAC_FORM_F32 = 1, PAC_FORM_TC = 2 };

/* transform operators (per axis, all axes of the plan) */
enum {
  PAC_OP_AT = 0,      /* x <- A^T x = P_b F x      apply_transposed_butterflies_r* */
  PAC_OP_A = 1,       /* x <- A x   = F P_b x      apply_butterflies_r*            */
  PAC_OP_CONJ_A = 2,  /* x <- conj(A) x            apply_conjugate_butterflies_r*  */
  PAC_OP_FFT = 3,     /* natural -> natural F x    fft, fft2                       */
  PAC_OP_IFFT = 4,    /* natural -> natural F^-1 x ifft                            */
  PAC_OP_UFFT = 5,    /* = PAC_OP_A                ufft                            */
  PAC_OP_UIFFT = 6    /* conj(A) x / N             uifft                           */
};

/* Plan knobs the autotuner chooses (0 everywhere = the built-in choices,
 * which the environment variables PAC_MAX_FACTOR_LOG and
 * PAC_SPECIAL_VARIANT may still adjust):
 *   max_factor_log  longest axis factor one CTA transforms, log2 (lower
 *                   values split an axis into more, shorter factors)
 *   max_radix_log   largest stage radix, log2: 4 (radix 16) or 3 (radix 8)
 *   special         -1: every pass on the generic kernel; 0: the specialised
 *                   kernel of the pass's geometry where one exists; k > 0:
 *                   its k-th candidate
 *   w_shift         lines per CTA of generic passes times 2^w_shift
 *   plane           3D convolutions: 1 runs axes 1 and 2 of every plane in
 *                   one pass on a thread-block cluster (3 passes over HBM in
 *                   all) where a plane kernel exists for the shape, -1 the
 *                   line schedule (5 passes), 0 the built-in choice (the
 *                   line schedule, unless PAC_PLANE=1)
 * No counterpart in the reference, which has one fixed schedule per radix. */
typedef struct {
  int max_factor_log;
  int max_radix_log;
  int special;
  int w_shift;
  int plane;
} pac_tune_t;

typedef struct {
  long long n_elements;   /* elements of one problem (product of dims)    */
  long long batch;
  int rank;
  int dims[3];
  int digit_base;
  int form;
  int element_bytes;      /* bytes of one real component (8 or 4)        */
  int conv_passes;        /* kernel launches of one pac_convolve          */
  int transform_passes;   /* kernel launches of one forward transform     */
  size_t workspace_bytes; /* device workspace held by the plan            */
  int digit_bases[3];     /* per axis (digit_base is axis 0's)            */
  pac_tune_t tune;        /* the knobs the plan was built with            */
} pac_plan_info_t;

/* Plan for `batch` problems of shape dims[0..rank-1] (rank 1..3).  Every
 * axis length must be a power of digit_base (2, 4 or 8); digit_base 0 picks
 * 2.  Allocates the twiddle tables on the current device.
 * Stands in for precompute_twiddles_r{2,4,8} (twiddle_factors.c:17,39,76):
 * the tables are generated on the device in FP64. */
PAC_API int pac_plan_create(pac_plan_t* plan, int rank, const int* dims, int batch,
                            int digit_base, int form);
/* As pac_plan_create with one digit base per axis (digit_bases[a] in
 * {2, 4, 8}, 0 picks 2): axis a's spectrum is in base-digit_bases[a] digit-
 * reversed order, A^T = (P_b0 F) x (P_b1 F) x ...  No counterpart in the
 * reference, which uses one radix for every axis (convolution_2d.c:41-47,
 * convolution_3d.c:44-49) and so runs 512 x 256 x 128 at radix 2 only; here
 * it runs at bases 8, 4 and 2. */
PAC_API int pac_plan_create_axes(pac_plan_t* plan, int rank, const int* dims,
                                 const int* digit_bases, int batch, int form);
/* As pac_plan_create_axes with explicit knobs (tune NULL: the built-in
 * choices).  pac_plan_create and pac_plan_create_axes use the knobs cached
 * for the problem in the file named by the environment variable
 * PAC_TUNE_CACHE, when it names one and holds an entry for this device and
 * problem (pac_autotune writes them). */
PAC_API int pac_plan_create_tuned(pac_plan_t* plan, int rank, const int* dims,
                                  const int* digit_bases, int batch, int form,
                                  const pac_tune_t* tune);

/* Autotuner: times candidate knob sets for one problem on the current
 * device (convolutions of device buffers it allocates and frees itself,
 * issued on `stream`, which it synchronises) -- a coordinate descent over
 * the kernel choice, the largest stage radix, the factor length and the
 * tile width, each step kept only if it is at least 2% faster -- and
 * returns the fastest.  With cache_path non-NULL it first looks the
 * problem up there and, when it tuned, appends the result as one JSON line
 * ({"key": ..., "max_factor_log": ..., ..., "ms": ..., "default_ms": ...}).
 * While it times, the output buffer (the passes' intermediate) is kept
 * persisting in L2 when it fits in three quarters of L2, so a knob set is
 * timed under the cache policy of a caller that does the same.
 * No counterpart in the reference. */
typedef struct {
  pac_tune_t tune;     /* the fastest knobs                               */
  double ms;           /* its time per convolution                        */
  double default_ms;   /* the built-in knobs' time                        */
  int candidates;      /* knob sets timed (0 when read from the cache)    */
  int cached;          /* 1: read from cache_path, nothing was timed      */
} pac_tune_result_t;
PAC_API int pac_autotune(int rank, const int* dims, const int* digit_bases, int batch, int form,
                         pac_stream_t stream, const char* cache_path, pac_tune_result_t* result);
/* free_twiddles (twiddle_factors.c:133) */
PAC_API int pac_plan_destroy(pac_plan_t plan);
PAC_API int pac_plan_get_info(pac_plan_t plan, pac_plan_info_t* info);

/* Filter spectrum: hhat = scale * A^T h, computed in FP64 and rounded once
 * to the plan's storage type, stored in the plan's spectrum order: the P_b
 * (digit-reversed) order of A^T h in which, on the innermost axis, every
 * block of R consecutive positions (R the radix of the plan's last stage)
 * is transposed to stride L/R, so that the fused pass of pac_convolve reads
 * it coalesced.  h_re/h_im are FP64 device arrays of nfilters problems (1,
 * or the plan's batch); hhat has the plan's element type.  In place
 * (h == hhat) is allowed for PAC_FORM_F64.  The reference recomputes A^T h
 * inside every call (convolution.c:45-53); the plan API computes it once.
 * A^T h in the reference's own order is pac_transform(PAC_OP_AT). */
PAC_API int pac_filter_spectrum(pac_plan_t plan, const double* h_re, const double* h_im,
                                int nfilters, void* hhat_re, void* hhat_im, double scale,
                                pac_stream_t stream);

/* A P_b-order FP64 spectrum (e.g. from pac_transform(PAC_OP_AT), or the
 * reference's A^T h) to the plan's spectrum order, scaled and rounded once.
 * In place allowed for PAC_FORM_F64.  Set-up work: the convolution itself
 * never reorders. */
PAC_API int pac_spectrum_to_plan_order(pac_plan_t plan, const double* p_re, const double* p_im,
                                       int nfilters, void* hhat_re, void* hhat_im, double scale,
                                       pac_stream_t stream);

/* Circular convolution of every problem of the batch:
 *   y = conj(A)[ scale * (A^T x) .* hhat ]
 * hhat in the plan's spectrum order (pac_filter_spectrum,
 * pac_spectrum_to_plan_order); hhat_per_problem = 0 applies one filter
 * spectrum to every problem, 1 reads one spectrum per problem.  x may alias
 * y.  permutation_avoiding_convolution{,_2d,_3d} (convolution.c:31,
 * convolution_2d.c:35, convolution_3d.c:36) with the filter transform
 * hoisted into the plan. */
PAC_API int pac_convolve(pac_plan_t plan, const void* x_re, const void* x_im,
                         const void* hhat_re, const void* hhat_im, int hhat_per_problem,
                         void* y_re, void* y_im, double scale, pac_stream_t stream);

/* Bounded device waits.  Kernels that wait on an mbarrier for their tensor
 * copies (the tensor-copy column passes, the opt-in pipelined column kernel)
 * give up after a limit of SM clock cycles instead of spinning forever: a
 * CTA whose wait gives up writes PAC_ERROR_TIMEOUT into the plan's device
 * status word, issues nothing more, lets the copies it has in flight land
 * and leaves -- the output of that call is then incomplete, and the device
 * stays usable.  pac_plan_check_status synchronises `stream`, reads and
 * clears the status word and returns PAC_ERROR_TIMEOUT if a wait of any
 * call of this plan gave up since the last check (PAC_SUCCESS otherwise);
 * the fft.h functions check it after every call.  pac_plan_set_wait_limit
 * sets the limit, in SM cycles, for the plan's later calls (<= 0: the
 * default 2^31, about a second); a tiny limit makes the waits run out.
 * No counterpart in the reference (whose calls never wait on a device). */
PAC_API int pac_plan_set_wait_limit(pac_plan_t plan, long long cycles);
PAC_API int pac_plan_check_status(pac_plan_t plan, pac_stream_t stream);

/* One operator over all axes of every problem, in -> out (may alias).
 * See PAC_OP_*.  For PAC_OP_FFT / PAC_OP_IFFT an axis split over several
 * passes needs the plan workspace (allocated on first use). */
PAC_API int pac_transform(pac_plan_t plan, int op, const void* in_re, const void* in_im,
                          void* out_re, void* out_im, pac_stream_t stream);

/* No counterpart in the reference.  Circular convolution of each of `batch`
 * complex FP64 signals of length n (a power of 2, at most
 * PAC_NOALLOC_MAX_N) with one filter h, for callers that cannot allocate
 * device memory (inside another framework's memory pool, under a fixed
 * memory budget, or where an allocation could synchronise the device).
 * x, h and y are device arrays the caller owns (x may alias y; x is
 * batch * n elements, h is n).  The call allocates nothing: its twiddle
 * tables and filter spectrum live in a fixed static device array of this
 * library, held by every GPU that loads it until the process exits.  The
 * first call on a device looks up that array's address once.  Calls whose
 * device work overlaps (other streams or host threads) race on the shared
 * array; queue them on one stream.  n above the limit returns
 * PAC_ERROR_SIZE and leaves y untouched. */
#define PAC_NOALLOC_MAX_N 65536
PAC_API int pac_convolve_1d_noalloc(const double* x_re, const double* x_im, const double* h_re,
                                    const double* h_im, double* y_re, double* y_im, int n,
                                    int batch, pac_stream_t stream);

/* ---- Many convolutions of uneven shapes in one call ----------------------
 * No counterpart in the reference, which convolves one signal per call
 * (bench1d_convolution.c loops over sizes).  A multi-plan covers nprob
 * problems of any mix of ranks and power-of-b shapes (every problem at
 * least 2 elements); problem p's data occupies elements
 * [offsets[p], offsets[p+1]) of packed split arrays (pac_multi_offsets),
 * in the problem's own row-major layout.  Problems of one shape share their
 * plan and twiddles.
 *
 * pac_multi_convolve runs every problem's convolution passes level by level
 * (level k = the k-th pass of every problem that has one): a level is one
 * persistent launch whose CTAs take work items (pass, tile) from a device
 * work queue, largest tiles first, so small and large problems share the
 * GPU -- or two such launches side by side when the level mixes tiles of
 * more and less than 72 KB of shared memory.  With a non-NULL stream the
 * launches are captured once into a CUDA graph per set of buffer addresses
 * and replayed afterwards (the first call for new addresses captures; later
 * calls launch the graph).  Calls on one multi-plan are serialised by a
 * lock on the host, but its work-queue counters are one device block per
 * multi-plan: calls whose device work overlaps (different streams, or graph
 * replays on different streams) take items from the same counters and
 * corrupt each other's results.  Queue the calls of one multi-plan on one
 * stream, or use one multi-plan per stream. */
typedef struct pac_multi_s* pac_multi_t;

/* ranks[p] in 1..3; dims holds 3 entries per problem (the first ranks[p]
 * are used). */
PAC_API int pac_multi_create(pac_multi_t* multi, int nprob, const int* ranks, const int* dims,
                             int digit_base, int form);
PAC_API int pac_multi_destroy(pac_multi_t multi);
/* offsets[0..nprob]: element offset of every problem; offsets[nprob] is the
 * total element count of one packed array */
PAC_API int pac_multi_offsets(pac_multi_t multi, long long* offsets);
/* filter spectra of every problem (packed FP64 h -> packed hhat of the
 * form's type, each scaled by 1/N of its problem and in its plan's order) */
PAC_API int pac_multi_filter_spectra(pac_multi_t multi, const double* h_re, const double* h_im,
                                     void* hhat_re, void* hhat_im, pac_stream_t stream);
/* y = x (*) h for every problem; x may alias y */
PAC_API int pac_multi_convolve(pac_multi_t multi, const void* x_re, const void* x_im,
                               const void* hhat_re, const void* hhat_im, void* y_re, void* y_im,
                               pac_stream_t stream);

typedef struct {
  int nprob;
  int nshapes;            /* distinct shapes (plans) */
  int nlevels;            /* levels of passes per pac_multi_convolve */
  long long items[8];     /* work items (CTAs) of each level */
  long long elements;     /* total elements of one packed array */
  int graph;              /* 1 once a CUDA graph replays the levels */
  double level_ms[8];     /* per-level mean time of the timed calls */
  long long timed_calls;  /* calls behind level_ms */
  long long fast_items;   /* work items on compile-time bodies (work-queue fast paths) */
} pac_multi_info_t;
PAC_API int pac_multi_get_info(pac_multi_t multi, pac_multi_info_t* info);
/* As pac_multi_create with one set of knobs for every shape's plan. */
PAC_API int pac_multi_create_tuned(pac_multi_t* multi, int nprob, const int* ranks,
                                   const int* dims, int digit_base, int form,
                                   const pac_tune_t* tune);
/* pac_autotune for a whole uneven batch: the knob set under which one
 * pac_multi_convolve of all the problems is fastest (the work-queue kernel
 * is generic, so `special` is not searched); cached under a key that lists
 * every problem's shape. */
PAC_API int pac_multi_autotune(int nprob, const int* ranks, const int* dims, int digit_base,
                               int form, pac_stream_t stream, const char* cache_path,
                               pac_tune_result_t* result);
/* Level timing: while enabled, pac_multi_convolve issues the levels
 * directly (no graph), records a CUDA event around every level on the
 * caller's stream and waits for them (calls become synchronous);
 * pac_multi_get_info reports the per-level means.  Enabling resets them. */
PAC_API int pac_multi_set_level_timing(pac_multi_t multi, int enable);

/* y = scale * x .* h elementwise over n complex FP64 values (the product
 * loop of convolution.c:55-62 on its own; the reference's convolution
 * reduces to it when the radix is not supported). */
PAC_API int pac_pointwise_product(long long n, const double* x_re, const double* x_im,
                                  const double* h_re, const double* h_im, double* y_re,
                                  double* y_im, double scale, pac_stream_t stream);

/* y = scale * x elementwise over n complex FP64 values (the division by n
 * of ifft / uifft, fft.c:69-70, on its own). x may alias y. */
PAC_API int pac_scale(long long n, const double* x_re, const double* x_im, double* y_re,
                      double* y_im, double scale, pac_stream_t stream);

/* Swap x[j] <-> x[rho[j]] for j < rho[j], rho an involution
 * (apply_permutation_split, index_reversals.c:85; apply_permutation,
 * index_reversals.c:74).  rho is a device int array of n entries.  With
 * im == NULL, re is an interleaved complex array of n (re, im) pairs. */
PAC_API int pac_permute(long long n, const int* rho, double* re, double* im,
                        pac_stream_t stream);

/* Stage twiddles in the reference layout (twiddle_factors.c:17-131):
 * level q (k = r^(q+1), ell = k/r) has (r-1)*ell entries, entry
 * (m-1)*ell + j = exp(-2 pi i m j / k).  Writes all levels back to back
 * into the device arrays re/im ((n-1) entries in total). */
PAC_API int pac_reference_twiddles(int r, int n, double* re, double* im, pac_stream_t stream);

/* Device memory and streams (thin wrappers so that C callers need no CUDA
 * headers). */
PAC_API int pac_malloc(void** ptr, size_t bytes);
PAC_API int pac_free(void* ptr);
PAC_API int pac_memcpy_h2d(void* dst, const void* src, size_t bytes, pac_stream_t stream);
PAC_API int pac_memcpy_d2h(void* dst, const void* src, size_t bytes, pac_stream_t stream);
PAC_API int pac_memcpy_d2d(void* dst, const void* src, size_t bytes, pac_stream_t stream);
PAC_API int pac_stream_create(pac_stream_t* stream);
PAC_API int pac_stream_destroy(pac_stream_t stream);
PAC_API int pac_stream_synchronize(pac_stream_t stream);
/* Work queued on `waiter` after this call starts when the work queued so far
 * on `waitee` has finished (an event recorded on waitee). */
PAC_API int pac_stream_wait_stream(pac_stream_t waiter, pac_stream_t waitee);

/* Keep [base, base + bytes) resident in L2 for work queued on `stream`
 * (CUDA access-policy window, persisting hits, streaming misses; the
 * persisting set-aside is a limit of this process's context only).
 * Meant for the convolution output, which the passes of pac_convolve use as
 * their intermediate, when it fits in L2: on 2048^2 FP64 a 64 MiB window
 * gains 7%, while a window of several times the L2 (268 MB) made the same
 * passes 36% slower than none.  bytes == 0 removes the window. */
PAC_API int pac_stream_set_l2_persisting(pac_stream_t stream, const void* base, size_t bytes);

/* Per-pass timing: while enabled, pac_convolve and pac_transform record a
 * CUDA event before the first and after every pass on the caller's stream
 * and wait for them at the end of the call (so calls become synchronous).
 * pac_plan_get_pass_timing returns, per pass slot of the last operator, the
 * summed milliseconds and the number of timed calls, then resets them. */
PAC_API int pac_plan_set_pass_timing(pac_plan_t plan, int enable);
PAC_API int pac_plan_get_pass_timing(pac_plan_t plan, int max_passes, double* ms,
                                     long long* calls, int* npasses);

/* Number of this library's kernel launches since load (for accounting). */
PAC_API long long pac_launch_count(void);
/* The current device's measured arithmetic peak, the denominator of the
 * flop-rate fraction bench.py reports beside the HBM roofline: a kernel of
 * independent fused multiply-add chains (8 per thread, 8 CTAs of 256
 * threads per SM), best of three timed launches on `stream`;
 * *tflops = 2 x FMAs per second / 1e12.  elem_bytes 8: FP64, 4: FP32.
 * No counterpart in the reference. */
PAC_API int pac_fma_peak(int elem_bytes, pac_stream_t stream, double* tflops);

PAC_API const char* pac_status_string(int status);
/* Message of the last failed call on this host thread ("" if none). */
PAC_API const char* pac_last_error(void);
/* Status of the last failed fft.h drop-in call on this thread, then clears it
 * (the fft.h entry points return void, as in the reference). */
PAC_API int pac_get_last_status(void);

#ifdef __cplusplus
}
#endif

#endif /* PAC_H */

// pac_backend.h -- what the plan layer needs from a device.
//
// The product library implements this interface on CUDA (pac_cuda.cu).
// The test-only emulator (pac_emu.cpp, built as libpac_emu.so and loaded
// only by tests/) implements it on host memory by replaying the same
// pass_body phases on the CPU, so that the plan layer and the kernels' index
// arithmetic can be checked without a GPU.
#pragma once
#include <stddef.h>

#include "pac_engine.cuh"

namespace pac {

enum { CPY_H2D = 0, CPY_D2H = 1, CPY_D2D = 2 };

int be_init();  // PAC_SUCCESS when a usable device is present
int be_num_sms();  // streaming multiprocessors of the current device (>= 1)
int be_device_name(char* buf, int n);  // the current device's name (tuning cache key)
int be_malloc(void** p, size_t bytes);
int be_free(void* p);
int be_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream);
int be_memset(void* dst, int value, size_t bytes, void* stream);
int be_stream_create(void** s);
int be_stream_destroy(void* s);
int be_stream_sync(void* s);
int be_stream_wait(void* waiter, void* waitee);
int be_l2_persist(void* stream, const void* base, size_t bytes);
long long be_l2_bytes();  // L2 cache size of the current device (0: none / unknown)
// timing events: record on a stream, elapsed milliseconds between two
int be_event_create(void** ev);
int be_event_destroy(void* ev);
int be_event_record(void* ev, void* stream);
int be_event_elapsed(void* a, void* b, float* ms);  // waits for b

// one pass over `grid` CTAs (elem_bytes 8: double, 4: float; b2 = log2 base)
int be_launch_pass(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                   size_t smem, void* stream);
// stage table (K = 2^logK, R = 2^logR): entry j*(R-1) + s-1 = w_K^{j s}, forward sign
int be_fill_stage_tw(void* dst, int elem_bytes, int logK, int logR, void* stream);
// the tensor-core form's DFT operand table: TC_CONST_SETS x 32 TcConst
int be_fill_tc_const(void* dst, void* stream);
// dst[k] = w_N^{k * stride} for k < count, N = 2^logN, forward sign
int be_fill_pow_tw(void* dst, int elem_bytes, long long count, long long stride, int logN,
                   void* stream);
// reference-layout tables of t levels for radix r (r^t - 1 entries)
int be_fill_ref_tw(int r, int t, double* re, double* im, void* stream);
int be_round_to_f32(const double* src, float* dst, long long n, void* stream);
// P-order FP64 spectrum lines (length 2^logL) -> plan order (every block of
// 2^logR positions transposed to stride L/R), scaled, stored as elem_bytes;
// in == out allowed for elem_bytes 8
int be_plan_order(const double* in_re, const double* in_im, void* out_re, void* out_im,
                  int elem_bytes, int logL, int logR, long long nlines, double scale,
                  void* stream);
// y = scale * x .* h[i & hmask] (complex, split); elem_bytes 8 or 4
int be_pointwise(long long n, int elem_bytes, const void* xr, const void* xi, const void* hr,
                 const void* hi, long long hmask, void* yr, void* yi, double scale,
                 void* stream);
int be_scale_copy(long long n, int elem_bytes, const void* xr, const void* xi, void* yr,
                  void* yi, double scale, void* stream);
int be_permute(long long n, const int* rho, double* re, double* im, void* stream);
long long be_launch_count();
// FMA throughput of the device (pac_fma_peak)
int be_fma_peak(int elem_bytes, void* stream, double* tflops);

// Persistent launch over a device work queue (pac_multi.cpp): the CTAs take
// work items from *counter (zeroed beforehand) until `total` are done; item
// i belongs to descriptor k = item_desc[i] and is CTA i - starts[k] of that
// pass.  descs (ndesc), starts (ndesc + 1) and item_desc (total) live in
// device memory; smem is the largest shared-memory size of the passes.
// tc = 1: the tensor-core form's kernel (PassDesc.tc set in every descriptor).
int be_queue_prepare(int elem_bytes, int b2, int tc, size_t smem);  // outside graph capture
int be_launch_queue(const PassDesc* descs, const long long* starts, const int* item_desc,
                    int ndesc, long long total, unsigned long long* counter, int elem_bytes,
                    int b2, int tc, size_t smem, void* stream);
// CUDA graphs: capture what a thread issues on `stream` between begin and
// end, then replay it.  be_graph_supported() is 0 where nothing can be
// captured (the host replay), and callers then issue the work directly.
int be_graph_supported();
int be_graph_begin(void* stream);
int be_graph_end(void* stream, void** exec);
int be_graph_launch(void* exec, void* stream);
int be_graph_destroy(void* exec);

}  // namespace pac

// kernels.h -- host-side view of the device engine (shared with plan.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>


#define CFFT_DT_C128 0
#define CFFT_DT_C64 1
#define CFFT_EMAX 16
#define CFFT_THREADS 256

#include "engine_types.h"

// generic kernel for a mode, or nullptr
const void* cfft_kernel_for(int mode, int dtype);
// statically shaped FOUR kernel matching (N1, N2, C, radix multiplicities), or
// nullptr; *single (if given) = 1 when it keeps one buffer for both layouts
const void* cfft_static_four(int dtype, int N1, int N2, int C, const unsigned char* ca,
                             const unsigned char* cc, int* single = nullptr);
// n = 4096 register kernel (KParams of a one-transform-per-CTA ROWS stage
// plus t4 = the two-level table of w_4096) and its shared memory
const void* cfft_r4096_kernel(int dtype);
size_t cfft_r4096_smem(size_t elem_bytes);
// power-of-two lengths n = N1 x 4096 (N1 = 2 .. 1024, pow2.cuh): pass A
// (KParams: batch = rows = transforms x N1, PA = log2 N1, t4 = table of
// w_4096, t4n = table of w_n, staged in shared memory after the kernel's own
// when pre = 1; shared memory cfft_r4096_smem + the staged table) and pass B
// (batch = column tiles = transforms x N1, twN1 = w_N1^e for e < N1; shared
// memory cfft_p2col_smem), built for mb = 3 or 2 CTAs per SM (ComplexF64;
// ComplexF32 is always 3)
const void* cfft_p2col_kernel(int dtype, int N1, int mb);
// single-pass power-of-two n = C x 4096 (C in {2, 4, 8, 16}) on clusters of C
// register 4096-point CTAs, mb = 2 or 3 CTAs per SM; shared memory
// cfft_r4096_smem
const void* cfft_p2cl_kernel(int dtype, int C, int mb);
// ComplexF64, the stride-C subsequences by tensor copies (two CTAs per SM),
// and its launcher (cluster of C CTAs)
const void* cfft_p2cl_tma_kernel(int C);
cudaError_t cfft_launch_p2cl_tma(const void* fn, const KParams& p, unsigned grid, size_t smem, int cluster,
                                 cudaStream_t st);
// both power-of-two passes in one persistent dataflow launch (N1 = 8 ..
// 1024): kernel, shared memory (staged_entries = w_n table entries staged,
// or 0) and launcher; ctr (ticket, abort flag, 2 nb counters) must be zero,
// ring holds depth intermediates of N1 x 4096 elements
const void* cfft_p2flow_kernel(int dtype, int N1);
size_t cfft_p2flow_smem(size_t elem_bytes, int N1, int staged_entries);
cudaError_t cfft_launch_p2flow(const void* fn, const KParams& pa, const KParams& pb, int* ctr, void* ring, int nb,
                               int lag, int depth, unsigned grid, size_t smem, cudaStream_t st);
// pass A with tensor copies (ComplexF64), and its launcher (encodes the
// tensor map of p.in for this launch)
const void* cfft_p2row_tma_kernel(int mb);
cudaError_t cfft_launch_p2row_tma(const void* fn, const KParams& p, unsigned grid, size_t smem, cudaStream_t st);
// ComplexF32 pass A with tensor copies of subsequence pairs (two CTAs per
// SM; batch = rows, even), its shared memory and launcher
const void* cfft_p2row_tma2_kernel();
size_t cfft_p2row_tma2_smem();
cudaError_t cfft_launch_p2row_tma2(const void* fn, const KParams& p, unsigned grid, size_t smem, cudaStream_t st);
// Rader for primes on a cluster of C in {3, 4, 5, 7, 8} register 4096-point
// CTAs (convc.cuh; M = 4096 C), built for mb = 3 or 2 CTAs per SM
// (ComplexF64; ComplexF32 is always 3), and its shared memory
const void* cfft_convc_kernel(int dtype, int C, int mb);
size_t cfft_convc_smem(size_t elem_bytes);
// mixed-radix lengths with a cluster kernel of C register L-point CTAs
// (mixc.cuh): 1 and the kernel, C, L and threads per CTA, else 0; variant 0
// stages both twiddle tables (two CTAs per SM), variant 1 reads the w_n
// table through L2 (three CTAs per SM), variants 2 and 3 are another split
// of n at three and two CTAs per SM, variants 4 and 5 the two splits with
// the input by tensor copies (ComplexF64 only)
int cfft_mixc_lookup(long long n, int dtype, int variant, const void** fn, int* C, int* L, int* threads);
// variants 4 and 5 (ComplexF64, the strided input by tensor copies) launch
// through this (a cluster of `cluster` CTAs of `threads`; KParams C, N2 = L)
cudaError_t cfft_launch_mixc_tma(const void* fn, const KParams& p, unsigned grid, int threads, size_t smem,
                                 int cluster, cudaStream_t st);
// launch a one-thread kernel whose bounded wait (at most `polls` polls) runs
// out on an mbarrier no one completes, and wait for it
cudaError_t cfft_wait_probe(int polls);
// the device fault word (bit 0: a tensor-copy wait timed out), optionally cleared
cudaError_t cfft_device_fault_word(unsigned* out, int clear);
const void* cfft_p2row_kernel(int dtype, int mb);
size_t cfft_p2col_smem(size_t elem_bytes, int N1);
cudaError_t cfft_prepare_fn(const void* fn, size_t smem, int cluster);
cudaError_t cfft_launch_fn(const void* fn, const KParams& p, unsigned grid, int threads, size_t smem,
                           int cluster, cudaStream_t stream);
cudaError_t cfft_max_active_clusters_fn(const void* fn, int threads, size_t smem, int cluster, int* out);
// batched (descriptor-driven) kernels
const void* cfft_batch_kernel_for(int mode, int dtype);
cudaError_t cfft_launch_batch(const void* fn, const BatchLaunch& L, unsigned grid, size_t smem,
                              int cluster, cudaStream_t stream);
// the batched form's persistent queue kernel (QueueLaunch, queue.cu), built
// for mb = 2 or 3 CTAs per SM, its launcher (ctl must be zero) and its
// translation unit's copy of the device fault word
const void* cfft_queue_kernel(int dtype, int mb);
cudaError_t cfft_launch_queue(const void* fn, const QueueLaunch& L, unsigned grid, size_t smem, cudaStream_t st);
cudaError_t cfft_queue_fault_word(unsigned* out, int clear);
// convolution tables on the device (tables.cu)
cudaError_t cfft_gen_chirp(double2* ch, long long n, cudaStream_t st);
cudaError_t cfft_gen_bluestein_b(double2* b, const double2* ch, long long n, long long M, cudaStream_t st);
cudaError_t cfft_gen_rader_b(double2* b, const int* iperm, long long n, long long M, int exact,
                             double2 winv, cudaStream_t st);
cudaError_t cfft_scale(double2* v, long long M, double s, cudaStream_t st);
cudaError_t cfft_spec_rowmajor(double2* dst, const double2* src, long long N1, long long N2, cudaStream_t st);
// real-input transforms (real.cu)
cudaError_t cfft_r2c_post(void* out, long long N, long long n, long long batch, long long dist, int dtype,
                          cudaStream_t st);
cudaError_t cfft_c2r_pre(const void* in, void* z, long long N, long long n, long long batch, long long in_dist,
                         double scale, int dtype, cudaStream_t st);
cudaError_t cfft_r2c_widen(const void* x, void* s, long long n, long long batch, int dtype, cudaStream_t st);
cudaError_t cfft_r2c_keep(const void* s, void* out, long long n, long long batch, int dtype, cudaStream_t st);
cudaError_t cfft_c2r_expand(const void* in, void* s, long long n, long long batch, double scale, int dtype,
                            cudaStream_t st);
cudaError_t cfft_c2r_real(const void* s, void* x, long long n, long long batch, int dtype, cudaStream_t st);
// ComplexF16 <-> ComplexF32 element conversion (real.cu)
cudaError_t cfft_half_to_float(const void* in, void* out, long long count, cudaStream_t st);
cudaError_t cfft_float_to_half(const void* in, void* out, long long count, cudaStream_t st);
// strided layouts <-> contiguous working buffer (real.cu)
cudaError_t cfft_gather(const void* in, void* w, long long n, long long batch, long long stride, long long dist,
                        int dtype, cudaStream_t st);
cudaError_t cfft_scatter(const void* w, void* out, long long n, long long batch, long long stride, long long dist,
                         int dtype, cudaStream_t st);
// set the thread-local text returned by cfft_last_error() (fixed buffer)
void cfft_set_last_error(const char* msg);

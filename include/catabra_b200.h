/*
 * catabra_b200.h -- C ABI of the B200-native 1D complex FFT.
 *
 * Drop-in boundary for CatabraFFT.jl's public FFT path.  Every entry point is
 * plain C (pointers, sizes, status codes); no exception or abort crosses it.
 * Each declaration names the reference interface it replaces (paths relative
 * to the CatabraFFT.jl project).
 *
 * Data layout: interleaved complex, contiguous, `batch` transforms of length
 * n back to back ([batch][n]); CFFT_C128 = ComplexF64 (16 B per element),
 * CFFT_C64 = ComplexF32 (8 B per element).
 *
 * Threading: plans are immutable after creation; one plan may be executed
 * concurrently on different streams as long as each concurrent call uses
 * its own output buffer (plans whose strategy needs device scratch -- see
 * cfft_plan_workspace_bytes -- serialise on that scratch: give each stream
 * its own plan).  Inputs are never modified (the reference's p * x can
 * overwrite x, src/CatabraFFT.jl:186-196).
 */
#ifndef CATABRA_B200_H
#define CATABRA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* element types: the reference's Complex{T}, T in {Float64, Float32} and
 * Float16 (ComplexF16, which the reference's self-test uses,
 * test/runtests.jl:39): ComplexF16 data is transformed with FP32 arithmetic
 * and rounded once on output; plans, execution, cfft_fft and the host entry
 * accept it (the batched, serving and real-input forms do not). */
enum { CFFT_C128 = 0, CFFT_C64 = 1, CFFT_C32 = 2 };

/* directions: fft (CatabraFFT.jl:65-72), ifft with 1/n (:88-101),
 * bfft without scaling (:103-115) */
enum { CFFT_FORWARD = 0, CFFT_INVERSE = 1, CFFT_BACKWARD = 2 };

/* planner flags, same values as the reference's FLAG (src/spells.jl:4-8):
 * NO_FLAG = heuristic plan, MEASURE = time candidate plans on the device,
 * ENCHANT = wider timed search (factorisations x cluster sizes x radix
 * orders).  Bit 4 (CFFT_EXACT_TWIDDLES) replaces the reference's Rader
 * twiddle recurrence (src/prime.jl:36-37) by exactly rounded twiddles.
 * Bit 5 (CFFT_BATCH_GROUPED, cfft_batch_create only) selects the grouped
 * schedule of the batched form instead of its single queue launch. */
enum { CFFT_NO_FLAG = 0, CFFT_MEASURE = 1, CFFT_ENCHANT = 2, CFFT_EXACT_TWIDDLES = 16, CFFT_BATCH_GROUPED = 32 };

/* status codes */
enum {
    CFFT_OK = 0,
    CFFT_ERR_INVALID = 1,     /* bad argument (n < 1, batch < 1, null pointer, ...) */
    CFFT_ERR_CUDA = 2,        /* a CUDA call failed; cfft_last_error() has the text  */
    CFFT_ERR_NOMEM = 3,       /* device or host allocation failed                    */
    CFFT_ERR_UNSUPPORTED = 4  /* size or configuration outside what the build covers */
};

typedef struct cfft_plan_s* cfft_plan;

/* Replaces plan_fft(x, flag) -> Spell (src/CatabraFFT.jl:149-167) and the
 * strategy choice of generate_and_cache_fft! (src/kernel.jl:72-92).
 * Builds twiddle tables, Rader/Bluestein spectra and scratch on the current
 * device.  batch >= 1 transforms of length n per execution. */
int cfft_plan_create(cfft_plan* plan, int64_t n, int64_t batch, int dtype, int flags);

/* Replaces mul!(y, p, x) / p * x (src/CatabraFFT.jl:186-196) and
 * fft_kernel! (src/kernel.jl:95-100): device pointers, enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  in == out is allowed. */
int cfft_execute(cfft_plan plan, const void* d_in, void* d_out, int direction, void* stream);

/* Replaces fft(x) / ifft(x) / bfft(x) (src/CatabraFFT.jl:65-115) for callers
 * holding host memory (the Julia ccall path): copies in, transforms, copies
 * out and synchronises.  Host buffers may be pinned (copied by DMA directly)
 * or pageable (staged through the plan's pinned buffers by host threads,
 * overlapped with the device work). */
int cfft_execute_host(cfft_plan plan, const void* h_in, void* h_out, int direction);

/* Strided layouts -- the reference's `region` argument, which it ignores
 * (src/CatabraFFT.jl:169): element i of transform b is read at
 * d_in[b * idist + i * istride] and written at d_out[b * odist + i * ostride]
 * (elements, not bytes).  Transforming the second axis of a column-major
 * n1 x n2 Julia matrix is n = n2, batch = n1, stride = n1, dist = 1.  The
 * data is gathered into a contiguous working buffer, transformed and
 * scattered back; cfft_execute only (device buffers). */
int cfft_plan_create_many(cfft_plan* plan, int64_t n, int64_t batch, int dtype, int flags, int64_t istride,
                          int64_t idist, int64_t ostride, int64_t odist);

/* Releases a plan and its device tables. */
int cfft_plan_destroy(cfft_plan plan);

/* One-call form with an internal plan cache keyed by (n, batch, dtype,
 * flags), mirroring fft_kernel!'s cached lookup (src/kernel.jl:72-100). */
int cfft_fft(int64_t n, int64_t batch, int dtype, int flags, const void* d_in, void* d_out,
             int direction, void* stream);

/* Replaces empty_cache() (src/CatabraFFT.jl:39-43): frees cached plans. */
int cfft_empty_cache(void);

/* Thread-local text of the last error on this thread ("" if none). */
const char* cfft_last_error(void);

/* Plan introspection: strategy string, e.g.
 * "four(C=12,N1=180,N2=168)[8,9,5,4|8,7,3]"; no device work. */
int cfft_plan_describe(cfft_plan plan, char* buf, int len);

/* Planner decision for (n, dtype) without touching the GPU (host logic only,
 * usable on machines without a device). */
int cfft_describe_strategy(int64_t n, int dtype, char* buf, int len);

/* Bytes of device scratch a plan holds beyond its tables (0 for the
 * one-HBM-round-trip strategies). */
int64_t cfft_plan_workspace_bytes(cfft_plan plan);

/* Number of kernel launches one cfft_execute of this plan issues. */
int cfft_plan_launches(cfft_plan plan);

/* Batched form: `count` transforms of mixed lengths packed back to back in
 * the order given (transform i starts at element sum(lengths[:i])).  The
 * reference transforms one vector per call (fft_kernel!, src/kernel.jl:95-100,
 * with one cached function per length); this plans every distinct length
 * once and runs the whole batch as one CUDA graph holding one kernel
 * launch: its CTAs claim work items by atomic ticket (whole single-CTA
 * transforms, and the tiles of two-pass transforms, whose stages wait for
 * one another through counters with bounded waits) from a queue built
 * here, largest transforms first.  A wait that runs out stops the launch and sets bit 1
 * of cfft_device_faults.  With CFFT_BATCH_GROUPED the graph instead holds
 * grouped descriptor-driven launches (single-kernel transforms by kernel
 * variant, cluster size and shared-memory class; two-pass transforms pass by
 * pass on a shared scratch).  flags: CFFT_EXACT_TWIDDLES, CFFT_BATCH_GROUPED. */
typedef struct cfft_batch_s* cfft_batch;
int cfft_batch_create(cfft_batch* batch, int64_t count, const int64_t* lengths, int dtype, int flags);

/* Runs the batch (device pointers, in == out allowed) on `stream` as one
 * graph launch; the graph is captured on the first call for a given
 * (d_in, d_out, direction) and replayed after that. */
int cfft_batch_execute(cfft_batch batch, const void* d_in, void* d_out, int direction, void* stream);

/* Releases the batch, its plans, descriptors, scratch and graph. */
int cfft_batch_destroy(cfft_batch batch);

/* Total elements of the packed batch; kernel launches in its graph. */
int64_t cfft_batch_elements(cfft_batch batch);
int cfft_batch_launches(cfft_batch batch);

/* Real-input transforms: plan_rfft / plan_brfft (src/CatabraFFT.jl:199-209,
 * stubs in the reference) with AbstractFFTs semantics.  A plan covers
 * `batch` transforms of n reals (CFFT_C128: double, CFFT_C64: float) and
 * their n/2 + 1 complex spectra, both packed back to back.
 *   cfft_rfft_execute          n reals -> n/2 + 1 complex (rfft)
 *   cfft_rfft_execute_inverse  n/2 + 1 complex -> n reals, CFFT_INVERSE =
 *                              irfft (scaled 1/n), CFFT_BACKWARD = brfft; the
 *                              imaginary parts of X[0] (and X[n/2], n even)
 *                              are ignored.  The complex input is not modified.
 * Buffers must be aligned to the complex element size (16 / 8 bytes). */
typedef struct cfft_rplan_s* cfft_rplan;
int cfft_rfft_plan_create(cfft_rplan* plan, int64_t n, int64_t batch, int dtype, int flags);
int cfft_rfft_execute(cfft_rplan plan, const void* d_real, void* d_complex, void* stream);
int cfft_rfft_execute_inverse(cfft_rplan plan, const void* d_complex, void* d_real, int direction, void* stream);
/* Host-buffer form (the ccall path): direction CFFT_FORWARD takes n reals
 * per transform and returns n/2 + 1 complex; CFFT_INVERSE / CFFT_BACKWARD the
 * reverse.  Copies in, transforms, copies out, synchronises. */
int cfft_rfft_execute_host(cfft_rplan plan, const void* h_in, void* h_out, int direction);
int cfft_rfft_plan_destroy(cfft_rplan plan);

/* Wisdom: the shapes MEASURE / ENCHANT chose, saved across processes --
 * the reference meant its Spell to be serialisable (src/spells.jl:180-375,
 * never finished).  A plan created with MEASURE or ENCHANT whose key
 * (n, batch, dtype, flags) has wisdom builds that shape without timing, as
 * long as it is still one of the planner's candidates.  Export writes every
 * entry of this process; import merges a file's entries (a bad file changes
 * nothing and returns CFFT_ERR_INVALID); forget drops them all. */
int cfft_wisdom_export(const char* path);
int cfft_wisdom_import(const char* path);
int cfft_wisdom_forget(void);
int64_t cfft_wisdom_entries(void);

/* Serving form: requests of any length arrive one at a time, from any host
 * thread, with device buffers; the reference runs each call to completion on
 * the calling thread (fft/ifft/bfft, src/CatabraFFT.jl:65-115).
 *   CFFT_SERVE_BATCHED  a worker thread batches whatever is queued whenever a
 *                       launch slot is idle (continuous batching), admitting
 *                       requests in arrival order while the bytes in flight
 *                       (input + output + two-pass scratch) stay under
 *                       max_inflight_bytes (0: 64 GiB);
 *   CFFT_SERVE_DIRECT   every request launches on arrival through its own
 *                       cached plan (the per-request path, for comparison).
 * A request's result is the same whichever requests share its batch.
 * max_requests bounds the tickets of the server's lifetime (0: 2^18).
 * Buffers must stay valid until the request completes. */
typedef struct cfft_server_s* cfft_server;
enum { CFFT_SERVE_BATCHED = 0, CFFT_SERVE_DIRECT = 1 };
int cfft_serve_create(cfft_server* server, int dtype, int64_t max_inflight_bytes, int64_t max_requests,
                      int mode);

/* Builds the plans of these lengths ahead of traffic (plan_fft for each). */
int cfft_serve_prepare(cfft_server server, int64_t count, const int64_t* lengths);

/* Queues one transform of length n (direction as cfft_execute); returns its
 * ticket.  Lengths without a plan are planned on first use. */
int cfft_serve_submit(cfft_server server, int64_t n, const void* d_in, void* d_out, int direction,
                      int64_t* ticket);

/* *done = 1 once the request has finished (its status is then returned and
 * latency_us, if not null, receives completion - submission in microseconds). */
int cfft_serve_query(cfft_server server, int64_t ticket, int* done, double* latency_us);

/* Blocks until the request finishes; status and latency as cfft_serve_query. */
int cfft_serve_wait(cfft_server server, int64_t ticket, double* latency_us);

/* Blocks until every submitted request has finished. */
int cfft_serve_drain(cfft_server server);

/* Requests submitted, batches formed, kernel launches issued so far. */
int cfft_serve_stats(cfft_server server, int64_t* requests, int64_t* batches, int64_t* launches);

/* Finishes queued requests, stops the worker and releases everything. */
int cfft_serve_destroy(cfft_server server);

/* No counterpart in the reference.  The two-pass FFT for callers that cannot
 * allocate device memory (a pool that forbids cudaMalloc, a framework that
 * owns every allocation): the scratch and twiddle tables live in one fixed
 * __device__ array (32 MiB + 256 KiB per GPU, held until exit), so nothing is
 * allocated.  n must be
 * 7-smooth, split as N1*N2 with N1, N2 <= 4096, and hold at most 2^21
 * ComplexF64 / 2^22 ComplexF32 elements; otherwise CFFT_ERR_UNSUPPORTED.
 * The first call on a device does a one-time set-up (make it before any
 * stream capture).  All calls share the array: calls that overlap on the
 * GPU race -- serialise them. */
int cfft_fft_twopass_noalloc(int64_t n, int64_t batch, int dtype, const void* d_in, void* d_out,
                             int direction, void* stream);

/* No counterpart in the reference.  The device fault word of the current
 * device: bit 0 is set when a kernel's bounded wait on its tensor copies (an
 * mbarrier) gave up, in which case that launch left its results incomplete.
 * Returns the word (0 = no fault; cleared when `clear` is nonzero), or -1 if
 * it could not be read (cfft_last_error() has the reason). */
int cfft_device_faults(int clear);

/* Test hook, no counterpart in the reference.  Runs a one-thread kernel whose
 * bounded wait (at most `polls` polls, 1 .. 2^20) on an mbarrier that nothing
 * completes gives up, and waits for it: the same timeout path a kernel takes
 * when its tensor copies never land, exercised without any fault.  Afterwards
 * cfft_device_faults reports bit 0 and the context stays usable. */
int cfft_debug_wait_timeout(int polls);

/* Test hook, no counterpart in the reference (whose failures are Julia
 * exceptions from @assert / error, src/kernel.jl:113,187, src/prime.jl:6,27,43).
 * From the nth device or pinned host allocation the library makes after this
 * call (nth >= 1), every allocation fails as out of memory until the hook is
 * called again; nth = 0 turns the injection off.  Returns the number of the
 * library's device and pinned host allocations that are live at the call, so
 * a test can show that a failed create released what it had allocated. */
int64_t cfft_debug_alloc_hook(int64_t nth);

/* ABI version (major*100 + minor). */
int cfft_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CATABRA_B200_H */

// real.cu -- real-input transforms (rfft / irfft / brfft) on top of the
// complex engine.
//
// Even n = 2N: the n reals of a transform are read as N complex values
// z[m] = x[2m] + i x[2m+1] (no copy), Z = FFT_N(z), and
//     X[k] = Fe[k] + w^k Fo[k],   Fe[k] = (Z[k] + conj Z[N-k]) / 2,
//                                 Fo[k] = (Z[k] - conj Z[N-k]) / 2i,
// for k = 0..N (Z[N] = Z[0]), w = exp(-2 pi i / n).  The inverse forms
//     Z'[k] = s ((X[k] + conj X[N-k]) + i w^-k (X[k] - conj X[N-k])),
// k < N, into the real output buffer and runs the unscaled backward FFT_N
// there in place: x[2m] = Re z[m], x[2m+1] = Im z[m] (s = 1/n for irfft, 1
// for brfft; the imaginary parts of X[0] and X[N] are ignored, as a
// Hermitian spectrum has none).
// Odd n: the reals are widened to complex in a scratch buffer, transformed
// by the complex path, and the first n/2 + 1 outputs kept; the inverse
// rebuilds the full Hermitian spectrum there.  Twiddles are evaluated in
// FP64 (sincospi) and rounded once to the data type.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "engine.cuh"
#include "kernels.h"

// w^k with w = exp(sign * 2 pi i / n), in FP64
__device__ __forceinline__ double2 wpow(long long k, long long n, int sign) {
    double s, c;
    sincospi(2.0 * (double)k / (double)n, &s, &c);
    return make_double2(c, sign * s);
}

template <typename V>
__global__ void k_r2c_post(V* out, long long N, long long n, long long batch, long long dist) {
    const long long half = N / 2 + 1;             // pairs (k, N - k), k = 0..N/2
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < half * batch;
         i += (long long)gridDim.x * blockDim.x) {
        const long long t = i / half, k = i - t * half;
        V* X = out + t * dist;
        if (k == 0) {
            const V z0 = X[0];
            X[0] = mk<V>(z0.x + z0.y, 0);
            X[N] = mk<V>(z0.x - z0.y, 0);
            continue;
        }
        const long long j = N - k;
        const double2 A = tod(X[k]), B = conjv(tod(X[j]));
        const double2 fe = make_double2(0.5 * (A.x + B.x), 0.5 * (A.y + B.y));
        // (A - B) / 2i = (Im(A - B) / 2, -Re(A - B) / 2)
        const double2 fo = make_double2(0.5 * (A.y - B.y), -0.5 * (A.x - B.x));
        const double2 wk = wpow(k, n, -1), wj = wpow(j, n, -1);
        const double2 a = cmul(wk, fo), b = cmul(wj, conjv(fo));
        X[k] = fromd<V>(make_double2(fe.x + a.x, fe.y + a.y));
        if (j != k) X[j] = fromd<V>(make_double2(fe.x + b.x, -fe.y + b.y));
    }
}

template <typename V>
__global__ void k_c2r_pre(const V* in, V* z, long long N, long long n, long long batch, long long in_dist,
                          double scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N * batch;
         i += (long long)gridDim.x * blockDim.x) {
        const long long t = i / N, k = i - t * N;
        const V* X = in + t * in_dist;
        double2 A = tod(X[k]), B = conjv(tod(X[N - k]));
        if (k == 0) {
            A.y = 0;
            B.y = 0;
        }
        const double2 fe = make_double2(A.x + B.x, A.y + B.y);
        const double2 fo = cmul(make_double2(A.x - B.x, A.y - B.y), wpow(k, n, +1));
        // fe + i fo
        z[t * N + k] = fromd<V>(make_double2(scale * (fe.x - fo.y), scale * (fe.y + fo.x)));
    }
}

// odd n: widen reals to complex; keep the first n/2 + 1 outputs
template <typename V, typename R>
__global__ void k_r2c_widen(const R* x, V* s, long long n, long long batch) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * batch;
         i += (long long)gridDim.x * blockDim.x)
        s[i] = mk<V>(x[i], 0);
}
template <typename V>
__global__ void k_r2c_keep(const V* s, V* out, long long n, long long batch) {
    const long long h = n / 2 + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < h * batch;
         i += (long long)gridDim.x * blockDim.x) {
        const long long t = i / h, k = i - t * h;
        out[i] = s[t * n + k];
    }
}
// odd n inverse: full Hermitian spectrum from the n/2 + 1 given values
template <typename V>
__global__ void k_c2r_expand(const V* in, V* s, long long n, long long batch, double scale) {
    const long long h = n / 2 + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * batch;
         i += (long long)gridDim.x * blockDim.x) {
        const long long t = i / n, k = i - t * n;
        V v = (k < h) ? in[t * h + k] : conjv(in[t * h + (n - k)]);
        if (k == 0) v.y = 0;
        s[i] = mk<V>(scale * v.x, scale * v.y);
    }
}
template <typename V, typename R>
__global__ void k_c2r_real(const V* s, R* x, long long n, long long batch) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * batch;
         i += (long long)gridDim.x * blockDim.x)
        x[i] = s[i].x;
}

static unsigned grid_for(long long work) {
    long long g = (work + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > 8192 ? 8192 : g));
}

cudaError_t cfft_r2c_post(void* out, long long N, long long n, long long batch, long long dist, int dtype,
                          cudaStream_t st) {
    const long long work = (N / 2 + 1) * batch;
    if (dtype == CFFT_DT_C128) k_r2c_post<double2><<<grid_for(work), 256, 0, st>>>((double2*)out, N, n, batch, dist);
    else k_r2c_post<float2><<<grid_for(work), 256, 0, st>>>((float2*)out, N, n, batch, dist);
    return cudaGetLastError();
}
cudaError_t cfft_c2r_pre(const void* in, void* z, long long N, long long n, long long batch, long long in_dist,
                         double scale, int dtype, cudaStream_t st) {
    const long long work = N * batch;
    if (dtype == CFFT_DT_C128)
        k_c2r_pre<double2><<<grid_for(work), 256, 0, st>>>((const double2*)in, (double2*)z, N, n, batch, in_dist, scale);
    else
        k_c2r_pre<float2><<<grid_for(work), 256, 0, st>>>((const float2*)in, (float2*)z, N, n, batch, in_dist, scale);
    return cudaGetLastError();
}
cudaError_t cfft_r2c_widen(const void* x, void* s, long long n, long long batch, int dtype, cudaStream_t st) {
    if (dtype == CFFT_DT_C128) k_r2c_widen<double2, double><<<grid_for(n * batch), 256, 0, st>>>((const double*)x, (double2*)s, n, batch);
    else k_r2c_widen<float2, float><<<grid_for(n * batch), 256, 0, st>>>((const float*)x, (float2*)s, n, batch);
    return cudaGetLastError();
}
cudaError_t cfft_r2c_keep(const void* s, void* out, long long n, long long batch, int dtype, cudaStream_t st) {
    const long long work = (n / 2 + 1) * batch;
    if (dtype == CFFT_DT_C128) k_r2c_keep<double2><<<grid_for(work), 256, 0, st>>>((const double2*)s, (double2*)out, n, batch);
    else k_r2c_keep<float2><<<grid_for(work), 256, 0, st>>>((const float2*)s, (float2*)out, n, batch);
    return cudaGetLastError();
}
cudaError_t cfft_c2r_expand(const void* in, void* s, long long n, long long batch, double scale, int dtype,
                            cudaStream_t st) {
    if (dtype == CFFT_DT_C128) k_c2r_expand<double2><<<grid_for(n * batch), 256, 0, st>>>((const double2*)in, (double2*)s, n, batch, scale);
    else k_c2r_expand<float2><<<grid_for(n * batch), 256, 0, st>>>((const float2*)in, (float2*)s, n, batch, scale);
    return cudaGetLastError();
}
cudaError_t cfft_c2r_real(const void* s, void* x, long long n, long long batch, int dtype, cudaStream_t st) {
    if (dtype == CFFT_DT_C128) k_c2r_real<double2, double><<<grid_for(n * batch), 256, 0, st>>>((const double2*)s, (double*)x, n, batch);
    else k_c2r_real<float2, float><<<grid_for(n * batch), 256, 0, st>>>((const float2*)s, (float*)x, n, batch);
    return cudaGetLastError();
}

// ComplexF16 input/output around the ComplexF32 path (FP32 arithmetic)
__global__ void k_h2f(const __half2* in, float2* out, long long count) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = __half22float2(in[i]);
}
__global__ void k_f2h(const float2* in, __half2* out, long long count) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = __float22half2_rn(in[i]);
}
cudaError_t cfft_half_to_float(const void* in, void* out, long long count, cudaStream_t st) {
    k_h2f<<<grid_for(count), 256, 0, st>>>((const __half2*)in, (float2*)out, count);
    return cudaGetLastError();
}
cudaError_t cfft_float_to_half(const void* in, void* out, long long count, cudaStream_t st) {
    k_f2h<<<grid_for(count), 256, 0, st>>>((const float2*)in, (__half2*)out, count);
    return cudaGetLastError();
}

// strided layouts: element i of transform b at base[b * dist + i * stride]
// gathered into / scattered out of a contiguous [batch][n] working buffer
template <typename V>
__global__ void k_gather(const V* in, V* w, long long n, long long batch, long long stride, long long dist) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * batch;
         i += (long long)gridDim.x * blockDim.x) {
        const long long b = i / n, k = i - b * n;
        w[i] = in[b * dist + k * stride];
    }
}
template <typename V>
__global__ void k_scatter(const V* w, V* out, long long n, long long batch, long long stride, long long dist) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * batch;
         i += (long long)gridDim.x * blockDim.x) {
        const long long b = i / n, k = i - b * n;
        out[b * dist + k * stride] = w[i];
    }
}
cudaError_t cfft_gather(const void* in, void* w, long long n, long long batch, long long stride, long long dist,
                        int dtype, cudaStream_t st) {
    if (dtype == CFFT_DT_C128) k_gather<double2><<<grid_for(n * batch), 256, 0, st>>>((const double2*)in, (double2*)w, n, batch, stride, dist);
    else k_gather<float2><<<grid_for(n * batch), 256, 0, st>>>((const float2*)in, (float2*)w, n, batch, stride, dist);
    return cudaGetLastError();
}
cudaError_t cfft_scatter(const void* w, void* out, long long n, long long batch, long long stride, long long dist,
                         int dtype, cudaStream_t st) {
    if (dtype == CFFT_DT_C128) k_scatter<double2><<<grid_for(n * batch), 256, 0, st>>>((const double2*)w, (double2*)out, n, batch, stride, dist);
    else k_scatter<float2><<<grid_for(n * batch), 256, 0, st>>>((const float2*)w, (float2*)out, n, batch, stride, dist);
    return cudaGetLastError();
}

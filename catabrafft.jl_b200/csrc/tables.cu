// tables.cu -- convolution tables (Rader / Bluestein) built on the device.
//
// Building the kernel vector b' and its spectrum on the host costs O(M)
// long-double trigonometry and two PCIe round trips per length; a mixed
// batch has thousands of distinct lengths, so the vector is generated here
// and transformed with this library's own FP64 path.
//
//   Bluestein:  chirp[j] = exp(-i pi (j^2 mod 2n) / n),   b'[m] = conj(chirp[|m|])
//   Rader:      W[m] = w^(-g^-m), b'[m] = W[m] (m < L), b'[M-L+m] = W[m] (1 <= m < L)
//               with w^(-k) either exactly rounded (sincospi of the reduced
//               fraction) or the reference's recurrence: Julia's
//               power_by_squaring of inv(cispi(2/n)), evaluated here with
//               unfused multiplies and adds so it rounds like the host copy.
#include <cuda_runtime.h>

#include "kernels.h"

__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
    const double re1 = __dmul_rn(a.x, b.x), re2 = __dmul_rn(a.y, b.y);
    const double im1 = __dmul_rn(a.x, b.y), im2 = __dmul_rn(a.y, b.x);
    return make_double2(__dsub_rn(re1, re2), __dadd_rn(im1, im2));
}
// power_by_squaring as in Julia Base (the reference's w^k, prime.jl:37)
__device__ double2 pow_sq_dev(double2 x, long long p) {
    if (p == 1) return x;
    if (p == 0) return make_double2(1, 0);
    if (p == 2) return cmul_rn(x, x);
    int t = __ffsll(p);              // trailing zeros + 1
    p >>= t;
    while ((t -= 1) > 0) x = cmul_rn(x, x);
    double2 y = x;
    while (p > 0) {
        t = __ffsll(p);
        p >>= t;
        while ((t -= 1) >= 0) x = cmul_rn(x, x);
        y = cmul_rn(y, x);
    }
    return y;
}
__device__ __forceinline__ double2 expi_frac(long long num, long long den, int sign) {
    // exp(sign * i * pi * num / den), num reduced to [0, 2 den)
    num %= 2 * den;
    if (num < 0) num += 2 * den;
    double s, c;
    sincospi((double)num / (double)den, &s, &c);
    return make_double2(c, sign * s);
}

__global__ void k_chirp(double2* ch, long long n) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const long long e = (long long)(((unsigned long long)j * (unsigned long long)j) %
                                        (unsigned long long)(2 * n));
        ch[j] = expi_frac(e, n, -1);
    }
}
__global__ void k_bluestein_b(double2* b, const double2* ch, long long n, long long M) {
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
         m += (long long)gridDim.x * blockDim.x) {
        double2 v = make_double2(0, 0);
        if (m < n) v = make_double2(ch[m].x, -ch[m].y);
        else if (M - m < n) v = make_double2(ch[M - m].x, -ch[M - m].y);
        b[m] = v;
    }
}
__global__ void k_rader_b(double2* b, const int* iperm, long long n, long long M, int exact,
                          double2 winv) {
    const long long L = n - 1;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
         m += (long long)gridDim.x * blockDim.x) {
        long long k = -1;
        if (m < L) k = m;
        else if (m >= M - L + 1) k = m - (M - L);
        double2 v = make_double2(0, 0);
        if (k >= 0) {
            const long long e = iperm[k];
            v = exact ? expi_frac(2 * e, n, -1) : pow_sq_dev(winv, e);
        }
        b[m] = v;
    }
}
__global__ void k_scale(double2* v, long long M, double s) {
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
         m += (long long)gridDim.x * blockDim.x) {
        v[m].x *= s;
        v[m].y *= s;
    }
}

static unsigned grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (unsigned)(g < 4096 ? (g < 1 ? 1 : g) : 4096);
}
cudaError_t cfft_gen_chirp(double2* ch, long long n, cudaStream_t st) {
    k_chirp<<<grid_for(n), 256, 0, st>>>(ch, n);
    return cudaGetLastError();
}
cudaError_t cfft_gen_bluestein_b(double2* b, const double2* ch, long long n, long long M, cudaStream_t st) {
    k_bluestein_b<<<grid_for(M), 256, 0, st>>>(b, ch, n, M);
    return cudaGetLastError();
}
cudaError_t cfft_gen_rader_b(double2* b, const int* iperm, long long n, long long M, int exact,
                             double2 winv, cudaStream_t st) {
    k_rader_b<<<grid_for(M), 256, 0, st>>>(b, iperm, n, M, exact, winv);
    return cudaGetLastError();
}
cudaError_t cfft_scale(double2* v, long long M, double s, cudaStream_t st) {
    k_scale<<<grid_for(M), 256, 0, st>>>(v, M, s);
    return cudaGetLastError();
}

// spectrum in the cluster kernels' row-major (k1, k2) order: dst[k1 N2 + k2]
// = src[k1 + N1 k2], so each CTA reads its rows contiguously
__global__ void k_spec_rowmajor(double2* dst, const double2* src, long long N1, long long N2) {
    const long long M = N1 * N2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        const long long k1 = i / N2, k2 = i - k1 * N2;
        dst[i] = src[k1 + N1 * k2];
    }
}
cudaError_t cfft_spec_rowmajor(double2* dst, const double2* src, long long N1, long long N2, cudaStream_t st) {
    k_spec_rowmajor<<<grid_for(N1 * N2), 256, 0, st>>>(dst, src, N1, N2);
    return cudaGetLastError();
}

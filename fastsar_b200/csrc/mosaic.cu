// A patch mosaic's per-patch phase history (fastsar/patches.py:315-500): the history re-referenced to the patch
// centre and gated in range to the patch, on the device. Three steps around the caller's transforms (cuFFT):
//
//   mosaic_pad     a pulse's samples placed on the padded frequency axis (zeros outside), optionally times the
//                  re-referencing phase exp(-4 pi i f shift / c) (the direct form, and the shared range profiles'
//                  input without a phase)
//   mosaic_gather  the gate's N range bins of each pulse's profile, the whole-bin part of its shift taken as an
//                  index offset: u[p, n] = Q[p, (j_n - m_p) mod K2], j_n = n for n < N / 2, n - N otherwise
//   mosaic_gate    the gated spectrum's kept samples times the fractional-bin ramp exp(-2 pi i d_p k / N), a
//                  per-pulse constant, a scale and the guard taper
//
// Each is one pass over its rows (HBM-bound, 8 bytes in and 8 out per sample); phases in float64.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {
namespace {

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void mosaic_pad_kernel(const float2 *__restrict__ S, long ldS, int rows, int K, int K2, int npl,
                                  const double *__restrict__ shift, double f0, double df, float2 *__restrict__ out)
{
    const long n = (long)rows * K2;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int p = (int)(e / K2), k = (int)(e - (long)p * K2);
        float2 v = make_float2(0.f, 0.f);
        if (k >= npl && k < npl + K) {
            v = S[(size_t)p * ldS + (k - npl)];
            if (shift) {
                // exp(-4 pi i f_k shift / c) = exp(2 pi i (-2 f_k shift / c)), f_k = f0 + k df
                const double cyc = -2.0 * fma((double)k, df, f0) * shift[p] / C_LIGHT;
                v = cmulf(v, cis_cycles_d(cyc));
            }
        }
        out[e] = v;
    }
}

__global__ void mosaic_gather_kernel(const float2 *__restrict__ Q, long ldQ, int rows, int K2, int N,
                                     const int *__restrict__ m, float2 *__restrict__ u)
{
    const long n = (long)rows * N;
    const int half = N / 2;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int p = (int)(e / N), q = (int)(e - (long)p * N);
        const int j = (q + half) % N - half;                  // the gate's bins about the centre: 0, 1, .., -1
        long col = (long)j - (m ? m[p] : 0);
        col %= K2;
        if (col < 0) col += K2;
        u[e] = Q[(size_t)p * ldQ + col];
    }
}

__global__ void mosaic_gate_kernel(const float2 *__restrict__ U, long ldU, int rows, int k0, int nk, int N,
                                   const double *__restrict__ d, const double2 *__restrict__ cph, double scale,
                                   const float *__restrict__ taper, float2 *__restrict__ out)
{
    const long n = (long)rows * nk;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int p = (int)(e / nk), k = (int)(e - (long)p * nk);
        float2 v = U[(size_t)p * ldU + k0 + k];
        double cr = scale * taper[k], ci = 0.0;
        if (cph) {
            const double2 c = cph[p];
            ci = cr * c.y;
            cr = cr * c.x;
        }
        float2 f = make_float2((float)cr, (float)ci);
        if (d) f = cmulf(f, cis_cycles_d(-d[p] * (double)(k0 + k) / (double)N));
        out[e] = cmulf(v, f);
    }
}

int grid_of(long n)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long want = (n + 255) / 256, cap = (long)nsm * 16;
    return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

cudaError_t launch_mosaic_pad(const float2 *S, long ldS, int rows, int K, int K2, int npl, const double *shift,
                              double f0, double df, float2 *out, cudaStream_t s)
{
    if ((long)rows * K2 == 0) return cudaSuccess;
    mosaic_pad_kernel<<<grid_of((long)rows * K2), 256, 0, s>>>(S, ldS, rows, K, K2, npl, shift, f0, df, out);
    return cudaGetLastError();
}

cudaError_t launch_mosaic_gather(const float2 *Q, long ldQ, int rows, int K2, int N, const int *m, float2 *u,
                                 cudaStream_t s)
{
    if ((long)rows * N == 0) return cudaSuccess;
    mosaic_gather_kernel<<<grid_of((long)rows * N), 256, 0, s>>>(Q, ldQ, rows, K2, N, m, u);
    return cudaGetLastError();
}

cudaError_t launch_mosaic_gate(const float2 *U, long ldU, int rows, int k0, int nk, int N, const double *d,
                               const double2 *cph, double scale, const float *taper, float2 *out, cudaStream_t s)
{
    if ((long)rows * nk == 0) return cudaSuccess;
    mosaic_gate_kernel<<<grid_of((long)rows * nk), 256, 0, s>>>(U, ldU, rows, k0, nk, N, d, cph, scale, taper, out);
    return cudaGetLastError();
}

}  // namespace ffbp

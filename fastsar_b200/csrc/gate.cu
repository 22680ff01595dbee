// The range gate on the device (the reference's range_gate, fastsar/ffbp_cuda.py:767-864, and ImageFormer._gate,
// fastsar/api.py:525-564). Per block of pulses: gate_pad places the windowed samples at npl .. npl + K - 1 of a zeroed
// row of Kp (recording the first pulse with a non-finite sample); the caller takes the inverse FFT of each row
// (cuFFT); gate_fold gathers the N bins about bin 0 (0 .. N - h - 1 and Kp - h .. Kp - 1, h = N / 2) into a row of N;
// the caller takes the forward FFT; gate_taper keeps samples k0 .. k1 - 1 times the taper (which carries the scale
// Kp / N) as the gated history. Each kernel is a thread per output sample: plain coalesced copies, HBM-bound.
#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

__global__ void gate_pad_kernel(const float2 *__restrict__ S, int n, int K, const float *__restrict__ wp,
                                const float *__restrict__ wk, int npl, int Kp, float2 *__restrict__ z, int *bad,
                                int p_off)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * Kp) return;
    const int p = (int)(idx / Kp), j = (int)(idx - (long)p * Kp), k = j - npl;
    float2 v = make_float2(0.f, 0.f);
    if (k >= 0 && k < K) {
        v = S[(long)p * K + k];
        if (bad && !(isfinite(v.x) && isfinite(v.y))) atomicMin(bad, p_off + p);
        if (wp) {
            const float w = wp[p_off + p] * wk[k];
            v.x *= w;
            v.y *= w;
        }
    }
    z[idx] = v;
}

__global__ void gate_fold_kernel(const float2 *__restrict__ q, int n, int Kp, int N, float2 *__restrict__ u)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * N) return;
    const int p = (int)(idx / N), i = (int)(idx - (long)p * N), h = N / 2;
    u[idx] = q[(long)p * Kp + (i < N - h ? i : Kp - N + i)];
}

__global__ void gate_taper_kernel(const float2 *__restrict__ u, int n, int N, int k0, int k1,
                                  const float *__restrict__ taper, float2 *__restrict__ out)
{
    const int W = k1 - k0;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * W) return;
    const int p = (int)(idx / W), k = (int)(idx - (long)p * W);
    const float2 v = u[(long)p * N + k0 + k];
    const float t = taper[k];
    out[idx] = make_float2(v.x * t, v.y * t);
}

unsigned blocks_for(long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t launch_gate_pad(const float2 *S, int n, int K, const float *wp, const float *wk, int npl, int Kp,
                            float2 *z, int *bad, int p_off, cudaStream_t s)
{
    const long total = (long)n * Kp;
    if (total <= 0) return cudaSuccess;
    gate_pad_kernel<<<blocks_for(total), 256, 0, s>>>(S, n, K, wp, wk, npl, Kp, z, bad, p_off);
    return cudaGetLastError();
}

cudaError_t launch_gate_fold(const float2 *q, int n, int Kp, int N, float2 *u, cudaStream_t s)
{
    const long total = (long)n * N;
    if (total <= 0) return cudaSuccess;
    gate_fold_kernel<<<blocks_for(total), 256, 0, s>>>(q, n, Kp, N, u);
    return cudaGetLastError();
}

cudaError_t launch_gate_taper(const float2 *u, int n, int N, int k0, int k1, const float *taper, float2 *out,
                              cudaStream_t s)
{
    const long total = (long)n * (k1 - k0);
    if (total <= 0) return cudaSuccess;
    gate_taper_kernel<<<blocks_for(total), 256, 0, s>>>(u, n, N, k0, k1, taper, out);
    return cudaGetLastError();
}

}  // namespace ffbp

// Stack products on images formed on one grid: the registration's detected images, the cross-spectrum of a
// correlation, the sub-pixel translation's ramp and crop, the running incoherent average with its tile statistics,
// and the pair products multilook, interferogram and coherence (fastsar/stack.py:485-1124, fastsar/products.py:28-67).
//
// Every kernel here moves a few bytes per pixel and does a few operations on them: they are bound by HBM, so each
// reads its inputs once in coalesced rows (a block's halo from L1/L2) and writes its output once. The float32
// arithmetic the reference's results depend on bit for bit (the box means' sums in their order, the average's
// products and sums) is written with the round-to-nearest intrinsics, which the library's fast-math build neither
// contracts nor approximates.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace ffbp {
namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// the intensity of pixel k: kind 0 the float as is, 1 |z|^2 of a complex64 (re re + im im, each product rounded),
// 2 x^2 of a float
__device__ __forceinline__ float pixel_value(const void *in, int kind, size_t k)
{
    if (kind == 1) {
        const float2 z = static_cast<const float2 *>(in)[k];
        return __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y));
    }
    const float x = static_cast<const float *>(in)[k];
    return kind == 2 ? __fmul_rn(x, x) : x;
}

// ------------------------------------------------------------------------------------------------ box means
// Output tile BR x BC per block; the input tile with its halo ((BR + w - 1) x (BC + w - 1), edge pixels repeated)
// in shared memory, then the w rows' means per column, then the w columns' means of those: the sums in index order
// and one division each, as the reference's float32 _box (fastsar/stack.py:493-528) forms them.
constexpr int BOX_BR = 32, BOX_BC = 64;

__global__ void __launch_bounds__(256) box_kernel(const void *__restrict__ in, int kind, int n1, int n2, int w,
                                                  int to_db, float *__restrict__ out)
{
    extern __shared__ float sbox[];
    const int W = BOX_BC + w - 1, H = BOX_BR + w - 1;
    float *sin = sbox, *sv = sbox + H * W;
    const int r0 = blockIdx.y * BOX_BR, c0 = blockIdx.x * BOX_BC, before = (w - 1) / 2;
    for (int idx = threadIdx.x; idx < H * W; idx += blockDim.x) {
        const int rr = idx / W, cc = idx - rr * W;
        const int r = clampi(r0 - before + rr, 0, n1 - 1), c = clampi(c0 - before + cc, 0, n2 - 1);
        sin[idx] = pixel_value(in, kind, (size_t)r * n2 + c);
    }
    __syncthreads();
    const float fw = (float)w;
    for (int idx = threadIdx.x; idx < BOX_BR * W; idx += blockDim.x) {
        const int rr = idx / W, cc = idx - rr * W;
        float acc = sin[rr * W + cc];
        for (int k = 1; k < w; ++k) acc = __fadd_rn(acc, sin[(rr + k) * W + cc]);
        sv[idx] = __fdiv_rn(acc, fw);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < BOX_BR * BOX_BC; idx += blockDim.x) {
        const int rr = idx / BOX_BC, cc = idx - rr * BOX_BC;
        const int r = r0 + rr, c = c0 + cc;
        if (r >= n1 || c >= n2) continue;
        float acc = sv[rr * W + cc];
        for (int k = 1; k < w; ++k) acc = __fadd_rn(acc, sv[rr * W + cc + k]);
        float m = __fdiv_rn(acc, fw);
        if (to_db) m = 10.f * log10f(fmaxf(m, 1e-30f));
        out[(size_t)r * n2 + c] = m;
    }
}

// ------------------------------------------------------------------------------------------------ coherence
// Sample coherence over w1 x w2 windows, the edge pixels repeated, the window of pixel i spanning i - w / 2 to
// i - w / 2 + w - 1 along each axis (scipy.ndimage.uniform_filter's placement, fastsar/products.py:35-39). A block
// of 128 threads owns 128 - (w2 - 1) output columns and a run of rows: each thread keeps the float64 running sums
// of (Re a b*, Im a b*, |a|^2, |b|^2) over the w1 rows of its column (one row in and one out per output row, fetched
// an output row ahead of their use); the row's 128 column sums go through shared memory as float32 (16 bytes a
// column: the shared-memory traffic of the w2-wide sums, which bounds the kernel, halved) to the horizontal sums,
// and the coherence is formed from those in float64. Rounding the column sums to float32 moves a coherence by about
// 1e-7.
constexpr int COH_NT = 128;

__global__ void __launch_bounds__(COH_NT) coherence_kernel(const float2 *__restrict__ a, const float2 *__restrict__ b,
                                                           int n1, int n2, int w1, int w2, int rows,
                                                           float *__restrict__ out)
{
    __shared__ float4 sv[COH_NT];
    const int t = threadIdx.x, oc = COH_NT - (w2 - 1);
    const int c0 = blockIdx.x * oc, lo1 = w1 / 2, lo2 = w2 / 2;
    const int c = clampi(c0 - lo2 + t, 0, n2 - 1);
    const int rbeg = blockIdx.y * rows, rend = min(rbeg + rows, n1);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    auto fetch = [&](int r, float2 &za, float2 &zb) {
        const size_t k = (size_t)clampi(r, 0, n1 - 1) * n2 + c;
        za = a[k];
        zb = b[k];
    };
    auto apply = [&](float2 za, float2 zb, double sign) {
        const double ar = za.x, ai = za.y, br = zb.x, bi = zb.y;
        s0 += sign * (ar * br + ai * bi);
        s1 += sign * (ai * br - ar * bi);
        s2 += sign * (ar * ar + ai * ai);
        s3 += sign * (br * br + bi * bi);
    };
    for (int k = 0; k < w1; ++k) {
        float2 za, zb;
        fetch(rbeg - lo1 + k, za, zb);
        apply(za, zb, 1.0);
    }
    // the rows that enter and leave the window at the next slide, fetched an output row ahead of their use
    float2 ia, ib, xa, xb;
    fetch(rbeg + 1 - lo1 + w1 - 1, ia, ib);
    fetch(rbeg - lo1, xa, xb);
    for (int r = rbeg; r < rend; ++r) {
        sv[t] = make_float4((float)s0, (float)s1, (float)s2, (float)s3);
        __syncthreads();
        if (t < oc && c0 + t < n2) {
            float h0 = 0.f, h1 = 0.f, h2 = 0.f, h3 = 0.f;
            for (int k = 0; k < w2; ++k) {
                const float4 v = sv[t + k];
                h0 += v.x; h1 += v.y; h2 += v.z; h3 += v.w;
            }
            // |sum a b*|^2 / (sum |a|^2 sum |b|^2): the windows' 1 / (w1 w2) cancels; the ratio in float64 (the
            // product of two intensity sums can pass float32's range), its square root to float32
            const double num = (double)h0 * h0 + (double)h1 * h1, den = (double)fmaxf(h2, 0.f) * fmaxf(h3, 0.f);
            out[(size_t)r * n2 + c0 + t] = sqrtf((float)(num / fmax(den, 1e-300)));
        }
        __syncthreads();
        if (r + 1 < rend) {
            apply(ia, ib, 1.0);
            apply(xa, xb, -1.0);
            if (r + 2 < rend) {
                fetch(r + 2 - lo1 + w1 - 1, ia, ib);
                fetch(r + 1 - lo1, xa, xb);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------ multilook
// out[i, j] = the mean over the la x lr box (i la.., j lr..) of |img|^2 (float32 output of float64 sums), or of
// a b* (complex64 output) when b is given.
__global__ void multilook_kernel(const float2 *__restrict__ a, const float2 *__restrict__ b, int n2, int m1, int m2,
                                 int la, int lr, void *__restrict__ out)
{
    const long n = (long)m1 * m2;
    const double inv = 1.0 / ((double)la * lr);
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int i = (int)(k / m2), j = (int)(k - (long)i * m2);
        double sr = 0.0, si = 0.0;
        for (int u = 0; u < la; ++u) {
            const size_t row = (size_t)(i * la + u) * n2 + (size_t)j * lr;
            for (int v = 0; v < lr; ++v) {
                const float2 za = a[row + v];
                if (b) {
                    const float2 zb = b[row + v];
                    sr += (double)za.x * zb.x + (double)za.y * zb.y;
                    si += (double)za.y * zb.x - (double)za.x * zb.y;
                } else {
                    sr += (double)za.x * za.x + (double)za.y * za.y;
                }
            }
        }
        if (b) static_cast<float2 *>(out)[k] = make_float2((float)(sr * inv), (float)(si * inv));
        else static_cast<float *>(out)[k] = (float)(sr * inv);
    }
}

// ------------------------------------------------------------------------------------------------ the average
// sum = (first ? 0 : sum) + p w and wsum = (first ? 0 : wsum) + (p > 0 ? weight : 0), p the pixel's intensity,
// each product and sum rounded once as the reference's float32 arrays are (fastsar/stack.py:1060-1083).
__global__ void mean_add_kernel(const void *__restrict__ img, int kind, long n, float w, float weight, int first,
                                float *__restrict__ sum, float *__restrict__ wsum)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const float p = pixel_value(img, kind, (size_t)k);
        const float s = __fmul_rn(p, w), v = p > 0.f ? weight : 0.f;
        sum[k] = first ? s : __fadd_rn(sum[k], s);
        wsum[k] = first ? v : __fadd_rn(wsum[k], v);
    }
}

__global__ void mean_image_kernel(const float *__restrict__ sum, const float *__restrict__ wsum, long n,
                                  float *__restrict__ out)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const float ws = wsum[k];
        out[k] = ws > 0.f ? __fdiv_rn(sum[k], fmaxf(ws, 1e-30f)) : 0.f;
    }
}

// One warp per T x T tile, eight neighbouring tiles of a tile row per block (coalesced rows): the mean and the
// (population) variance of x gain over the tile, from float64 sums.
constexpr int TS_WARPS = 8;

__global__ void __launch_bounds__(TS_WARPS * 32) tile_stats_kernel(const float *__restrict__ x, int n2, int t2, int T,
                                                                   float gain, float *__restrict__ mean,
                                                                   float *__restrict__ var)
{
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int ti = blockIdx.y, tj = blockIdx.x * TS_WARPS + warp;
    if (tj >= t2) return;
    const float *base = x + (size_t)ti * T * n2 + (size_t)tj * T;
    double s = 0.0, q = 0.0;
#pragma unroll 8
    for (int u = 0; u < T; ++u) {
        for (int v = lane; v < T; v += 32) {
            const double val = __fmul_rn(base[(size_t)u * n2 + v], gain);
            s += val;
            q += val * val;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        q += __shfl_xor_sync(0xffffffffu, q, o);
    }
    if (lane == 0) {
        const double nn = (double)T * T, m = s / nn;
        mean[(size_t)ti * t2 + tj] = (float)m;
        var[(size_t)ti * t2 + tj] = (float)fmax(q / nn - m * m, 0.0);
    }
}

// ------------------------------------------------------------------------------------------------ correlation
// X = conj(A) B hp over a real transform's half plane [m1, m2h], hp = 1 - e1[i] e2[j] (the separable Gaussian's
// complement; no high pass when e1 is null), and the two spectra's energies under the same weights, each column
// counted twice but the zero frequency and (nyquist) the last: energy[0] += |A|^2 wk hp, energy[1] += |B|^2 wk hp.
// blockIdx.y: the image of a batch (A, B, X advance by m1 m2h per image, energy by 2).
__global__ void __launch_bounds__(256) cross_spectrum_kernel(const float2 *__restrict__ A, const float2 *__restrict__ B,
                                                             int m1, int m2h, int nyquist, const float *__restrict__ e1,
                                                             const float *__restrict__ e2, float2 *__restrict__ X,
                                                             double *__restrict__ energy)
{
    __shared__ double red[2][8];
    const long n = (long)m1 * m2h;
    const size_t img = (size_t)blockIdx.y * n;
    A += img;
    B += img;
    X += img;
    energy += 2 * blockIdx.y;
    double ea = 0.0, eb = 0.0;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int i = (int)(k / m2h), j = (int)(k - (long)i * m2h);
        const float hp = e1 ? 1.f - e1[i] * e2[j] : 1.f;
        const float2 za = A[k], zb = B[k];
        const float xr = za.x * zb.x + za.y * zb.y, xi = za.x * zb.y - za.y * zb.x;
        X[k] = make_float2(xr * hp, xi * hp);
        const double wk = (j == 0 || (nyquist && j == m2h - 1) ? 1.0 : 2.0) * hp;
        ea += ((double)za.x * za.x + (double)za.y * za.y) * wk;
        eb += ((double)zb.x * zb.x + (double)zb.y * zb.y) * wk;
    }
    for (int o = 16; o > 0; o >>= 1) {
        ea += __shfl_xor_sync(0xffffffffu, ea, o);
        eb += __shfl_xor_sync(0xffffffffu, eb, o);
    }
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) { red[0][warp] = ea; red[1][warp] = eb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int k = 0; k < (int)(blockDim.x / 32); ++k) { sa += red[0][k]; sb += red[1][k]; }
        atomicAdd(&energy[0], sa);
        atomicAdd(&energy[1], sb);
    }
}

// out[b, i, j] = ((x[b, i, j] - mean[b]) w1[i]) w2[j], each step rounded to float32 as the reference's separate
// array operations round them (fastsar/stack.py:567-568): the correlation's mean removal and Hann windows, one pass
// over a batch of images [nb, n1, n2] (blockIdx.y: the image).
__global__ void window_kernel(const float *__restrict__ x, int n1, int n2, const float *__restrict__ mean,
                              const float *__restrict__ w1, const float *__restrict__ w2, float *__restrict__ out)
{
    const long n = (long)n1 * n2;
    const size_t img = (size_t)blockIdx.y * n;
    const float m = mean[blockIdx.y];
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int i = (int)(k / n2), j = (int)(k - (long)i * n2);
        out[img + k] = __fmul_rn(__fmul_rn(__fsub_rn(x[img + k], m), w1[i]), w2[j]);
    }
}

// F[i, j] *= r1[i] r2[j] (complex64): a separable phase ramp on a spectrum [m1, m2]
__global__ void ramp_multiply_kernel(float2 *__restrict__ F, int m1, int m2, const float2 *__restrict__ r1,
                                     const float2 *__restrict__ r2)
{
    const long n = (long)m1 * m2;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int i = (int)(k / m2), j = (int)(k - (long)i * m2);
        const float2 a = r1[i], b = r2[j], f = F[k];
        const float2 r = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
        F[k] = make_float2(f.x * r.x - f.y * r.y, f.x * r.y + f.y * r.x);
    }
}

// out[i, j] = moved[i + w0, j + w1] where that source pixel lies in the image and is not 0 there, else 0; moved
// is the sub-pixel-shifted image (complex, leading dimension ld) or, when null, the source itself. A real source
// gives a real, non-negative output (the shifted image's real part, clipped at 0).
__global__ void shift_crop_kernel(const float2 *__restrict__ shifted, int ld, const void *__restrict__ src,
                                  int src_complex, int n1, int n2, int w0, int w1, void *__restrict__ out)
{
    const long n = (long)n1 * n2;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int i = (int)(k / n2), j = (int)(k - (long)i * n2);
        const int si = i + w0, sj = j + w1;
        const bool in = si >= 0 && si < n1 && sj >= 0 && sj < n2;
        const size_t s = in ? (size_t)si * n2 + sj : 0;
        if (src_complex) {
            const float2 z = in ? static_cast<const float2 *>(src)[s] : make_float2(0.f, 0.f);
            float2 v = make_float2(0.f, 0.f);
            if (in && (z.x != 0.f || z.y != 0.f)) v = shifted ? shifted[(size_t)si * ld + sj] : z;
            static_cast<float2 *>(out)[k] = v;
        } else {
            const float x = in ? static_cast<const float *>(src)[s] : 0.f;
            float v = 0.f;
            if (in && x != 0.f) v = shifted ? fmaxf(shifted[(size_t)si * ld + sj].x, 0.f) : x;
            static_cast<float *>(out)[k] = v;
        }
    }
}

int grid_for(long n, int threads)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long want = (n + threads - 1) / threads, cap = (long)nsm * 16;
    return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

cudaError_t launch_box_mean(const void *in, int kind, int n1, int n2, int w, int to_db, float *out, cudaStream_t s)
{
    const dim3 grid((n2 + BOX_BC - 1) / BOX_BC, (n1 + BOX_BR - 1) / BOX_BR);
    const size_t smem = (size_t)((BOX_BR + w - 1) * (BOX_BC + w - 1) + BOX_BR * (BOX_BC + w - 1)) * sizeof(float);
    box_kernel<<<grid, 256, smem, s>>>(in, kind, n1, n2, w, to_db, out);
    return cudaGetLastError();
}

cudaError_t launch_coherence(const float2 *a, const float2 *b, int n1, int n2, int w1, int w2, float *out,
                             cudaStream_t s)
{
    const int oc = COH_NT - (w2 - 1), rows = 64;
    const dim3 grid((n2 + oc - 1) / oc, (n1 + rows - 1) / rows);
    coherence_kernel<<<grid, COH_NT, 0, s>>>(a, b, n1, n2, w1, w2, rows, out);
    return cudaGetLastError();
}

cudaError_t launch_multilook(const float2 *a, const float2 *b, int n1, int n2, int la, int lr, void *out,
                             cudaStream_t s)
{
    const int m1 = n1 / la, m2 = n2 / lr;
    if ((long)m1 * m2 == 0) return cudaSuccess;
    multilook_kernel<<<grid_for((long)m1 * m2, 256), 256, 0, s>>>(a, b, n2, m1, m2, la, lr, out);
    return cudaGetLastError();
}

cudaError_t launch_mean_add(const void *img, int kind, long n, float w, float weight, int first, float *sum,
                            float *wsum, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    mean_add_kernel<<<grid_for(n, 256), 256, 0, s>>>(img, kind, n, w, weight, first, sum, wsum);
    return cudaGetLastError();
}

cudaError_t launch_mean_image(const float *sum, const float *wsum, long n, float *out, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    mean_image_kernel<<<grid_for(n, 256), 256, 0, s>>>(sum, wsum, n, out);
    return cudaGetLastError();
}

cudaError_t launch_tile_stats(const float *x, int n1, int n2, int T, float gain, float *mean, float *var,
                              cudaStream_t s)
{
    const int t1 = n1 / T, t2 = n2 / T;
    if (t1 * t2 == 0) return cudaSuccess;
    if (t1 > 65535) return cudaErrorInvalidValue;
    tile_stats_kernel<<<dim3((t2 + TS_WARPS - 1) / TS_WARPS, t1), TS_WARPS * 32, 0, s>>>(x, n2, t2, T, gain, mean, var);
    return cudaGetLastError();
}

cudaError_t launch_cross_spectrum(const float2 *A, const float2 *B, int batch, int m1, int m2h, int nyquist,
                                  const float *e1, const float *e2, float2 *X, double *energy, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(energy, 0, 2 * sizeof(double) * (size_t)batch, s);
    if (e != cudaSuccess) return e;
    const int gx = (grid_for((long)m1 * m2h, 256) + batch - 1) / batch;
    cross_spectrum_kernel<<<dim3(gx < 1 ? 1 : gx, batch), 256, 0, s>>>(A, B, m1, m2h, nyquist, e1, e2, X, energy);
    return cudaGetLastError();
}

cudaError_t launch_window(const float *x, int batch, int n1, int n2, const float *mean, const float *w1, const float *w2,
                          float *out, cudaStream_t s)
{
    const int gx = (grid_for((long)n1 * n2, 256) + batch - 1) / batch;
    window_kernel<<<dim3(gx < 1 ? 1 : gx, batch), 256, 0, s>>>(x, n1, n2, mean, w1, w2, out);
    return cudaGetLastError();
}

cudaError_t launch_ramp_multiply(float2 *F, int m1, int m2, const float2 *r1, const float2 *r2, cudaStream_t s)
{
    ramp_multiply_kernel<<<grid_for((long)m1 * m2, 256), 256, 0, s>>>(F, m1, m2, r1, r2);
    return cudaGetLastError();
}

cudaError_t launch_shift_crop(const float2 *shifted, int ld, const void *src, int src_complex, int n1, int n2, int w0,
                              int w1, void *out, cudaStream_t s)
{
    shift_crop_kernel<<<grid_for((long)n1 * n2, 256), 256, 0, s>>>(shifted, ld, src, src_complex, n1, n2, w0, w1, out);
    return cudaGetLastError();
}

}  // namespace ffbp

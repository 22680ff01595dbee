// The learned-tap network on the GPU (no counterpart in the reference): an MLP 5 -> 64 -> 64 -> 64 -> 16 with GELU
// after the hidden layers. A query is one phase of one axis of a merge stage's decimation filter (features: the
// phase, the axis's pass fraction, 1 / D, the stage and the axis, scaled by the caller); its outputs are corrections
// to the 8 taps of that phase, 8 for the range axis and 8 for the angle axis (a query uses the ones of its axis).
// Forward pass, the decimation loss over point-target pairs, backward pass and Adam are hand-written kernels.
// Weights and hidden activations are bfloat16 values (rounded to nearest even and kept in float32 registers and
// buffers), every sum is float32. The network is small and its batches are a few thousand queries: CUDA-core
// kernels, not tensor cores.
//
// Parameters: one float32 array, per layer W [out, in] then b [out] (layers (5, 64), (64, 64), (64, 64), (64, 16)):
// 9,744 values. Work buffer (ffbp_mlp_work_bytes): the bfloat16-rounded weights, per layer the pre-activations Z
// and activations H of the queries, the gradient of the outputs and two back-propagation buffers.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int NL = 4;
constexpr int h_in[NL] = {5, 64, 64, 64};
constexpr int h_out[NL] = {64, 64, 64, 16};

__host__ __device__ constexpr int param_count()
{
    return 64 * 5 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 16 * 64 + 16;
}

int param_off(int l)                                          // offset of layer l's W (its b follows it)
{
    int o = 0;
    for (int i = 0; i < l; ++i) o += h_out[i] * h_in[i] + h_out[i];
    return o;
}

__device__ __forceinline__ float round_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * expf(-0.5f * z * z) * 0.39894228040143268f;
}

__global__ void round_kernel(const float *__restrict__ s, float *__restrict__ d, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = round_bf16(s[i]);
}

// Z = X W^T + b, H = bfloat16(gelu(Z)) (act) or Z; thread per (sample, output); W in shared memory
__global__ void dense_fwd(const float *__restrict__ X, int B, int in, const float *__restrict__ W,
                          const float *__restrict__ b, int out, int act, float *__restrict__ Z, float *__restrict__ H)
{
    extern __shared__ float sW[];                              // [out][in + 1]
    for (int i = threadIdx.x; i < out * (in + 1); i += blockDim.x) {
        const int o = i / (in + 1), k = i - o * (in + 1);
        sW[i] = k < in ? W[o * in + k] : b[o];
    }
    __syncthreads();
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)B * out) return;
    const int s = (int)(idx / out), o = (int)(idx - (long)s * out);
    const float *x = X + (long)s * in, *w = sW + o * (in + 1);
    float z = w[in];
    for (int k = 0; k < in; ++k) z = fmaf(w[k], __ldg(&x[k]), z);
    Z[idx] = z;
    H[idx] = act ? round_bf16(gelu(z)) : z;
}

// dW[o][k] += sum_s dZ[s][o] X[s][k], db[o] += sum_s dZ[s][o]: thread per (o, k) (k == in: the bias), over a slice
// of the batch (blockIdx.y), accumulated with atomics
__global__ void dense_bwd_w(const float *__restrict__ X, const float *__restrict__ dZ, int B, int in, int out,
                            int slice, float *__restrict__ dW, float *__restrict__ db)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= out * (in + 1)) return;
    const int o = idx / (in + 1), k = idx - o * (in + 1);
    const int s0 = blockIdx.y * slice, s1 = min(B, s0 + slice);
    float acc = 0.f;
    for (int s = s0; s < s1; ++s) acc = fmaf(__ldg(&dZ[(long)s * out + o]), k < in ? __ldg(&X[(long)s * in + k]) : 1.f, acc);
    if (k < in) atomicAdd(&dW[o * in + k], acc);
    else atomicAdd(&db[o], acc);
}

// dZp[s][k] = (sum_o dZ[s][o] W[o][k]) gelu'(Zp[s][k]): thread per (sample, input)
__global__ void dense_bwd_x(const float *__restrict__ dZ, const float *__restrict__ W, int B, int in, int out,
                            const float *__restrict__ Zp, float *__restrict__ dZp)
{
    extern __shared__ float sW[];                              // [out][in]
    for (int i = threadIdx.x; i < out * in; i += blockDim.x) sW[i] = W[i];
    __syncthreads();
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)B * in) return;
    const int s = (int)(idx / in), k = (int)(idx - (long)s * in);
    float acc = 0.f;
    for (int o = 0; o < out; ++o) acc = fmaf(__ldg(&dZ[(long)s * out + o]), sW[o * in + k], acc);
    dZp[idx] = acc * gelu_grad(Zp[idx]);
}

// The decimation loss of the learned taps. Instance i (inst[i] = first query q0, decimation D, axis a) owns the D
// queries q0 .. q0 + D - 1; query q holds the 8 taps of phase q at offsets t = phi_q - 4 + n (n = 0..7) in output
// samples, phi_q = (q + 1/2) / D for even D and q / D for odd D, each tap = prior + scale * (output 8 a + n of the
// network). A sample is a point target's parent samples e^{2 pi i f t} (f in cycles per output sample, float64) and
// its exact child value y; the decimated value is v = (1 / D) sum_{q, n} tap x; instance i's pairs weigh wt[i] (1
// without wt). Block (x, i) takes samples 256 x .. of instance i: the loss sum wt |v - y|^2 (atomic) and
// d (mean wt |v - y|^2) / d output, reduced per tap over the
// block in shared memory before one atomic per tap. An instance outside the query table (or D outside 1..32, or an
// axis other than 0 or 1) adds NaN to the loss and is skipped.
constexpr int LOSS_THREADS = 256;
constexpr int MAX_D = 32;

__device__ __forceinline__ float2 cis_frac(double c)       // e^{2 pi i c}, the argument reduced in float64
{
    float sn, cs;
    sincospif(2.f * (float)(c - rint(c)), &sn, &cs);
    return make_float2(cs, sn);
}

__global__ void __launch_bounds__(LOSS_THREADS) fir_loss(const float *__restrict__ out, const float *__restrict__ prior,
                                                         float scale, const int *__restrict__ inst,
                                                         const float *__restrict__ wt, int nq, int S,
                                                         const double *__restrict__ f, const float2 *__restrict__ y,
                                                         float gscale, float *__restrict__ dout, float *__restrict__ loss)
{
    __shared__ float s_k[8 * MAX_D], s_g[8 * MAX_D];
    const int i = blockIdx.y, q0 = inst[3 * i], D = inst[3 * i + 1], ax = inst[3 * i + 2], L = 8 * D;
    if (q0 < 0 || D < 1 || D > MAX_D || q0 > nq - D || (ax != 0 && ax != 1)) {   // a bad instance: the loss is NaN
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(loss, __int_as_float(0x7fc00000));
        return;
    }
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
        const int q = j >> 3, n = j & 7;
        s_k[j] = prior[(long)(q0 + q) * 8 + n] + scale * out[(long)(q0 + q) * 16 + 8 * ax + n];
        s_g[j] = 0.f;
    }
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = s < S;
    const double fs = live ? f[(long)i * S + s] : 0.0;
    const float2 step = cis_frac(fs);
    const double half = (D & 1) ? 0.0 : 0.5;
    float vx = 0.f, vy = 0.f;
    for (int q = 0; q < D; ++q) {
        float2 x = cis_frac(fs * ((q + half) / D - 4.0));
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const float k = s_k[8 * q + n];
            vx = fmaf(k, x.x, vx);
            vy = fmaf(k, x.y, vy);
            x = make_float2(x.x * step.x - x.y * step.y, x.x * step.y + x.y * step.x);
        }
    }
    const float invD = 1.f / (float)D, wi = wt ? wt[i] : 1.f;
    float ex = 0.f, ey = 0.f;
    if (live) {
        const float2 yy = y[(long)i * S + s];
        ex = vx * invD - yy.x;
        ey = vy * invD - yy.y;
    }
    float l = wi * (ex * ex + ey * ey);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
    const int lane = threadIdx.x & 31;
    for (int q = 0; q < D; ++q) {
        float2 x = cis_frac(fs * ((q + half) / D - 4.0));
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            float c = ex * x.x + ey * x.y;                     // Re(conj(e) x)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0) atomicAdd(&s_g[8 * q + n], c);
            x = make_float2(x.x * step.x - x.y * step.y, x.x * step.y + x.y * step.x);
        }
    }
    __syncthreads();
    const float g = gscale * scale * invD * wi;
    for (int j = threadIdx.x; j < L; j += blockDim.x)
        atomicAdd(&dout[(long)(q0 + (j >> 3)) * 16 + 8 * ax + (j & 7)], g * s_g[j]);
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct Work {
    float *Wr, *grad, *dA, *dB, *dtaps;
    float *Z[NL], *H[NL];
};

Work carve(float *w, int B)
{
    Work k;
    k.Wr = w;
    w += param_count();
    k.grad = w;
    w += param_count();
    for (int l = 0; l < NL; ++l) {
        k.Z[l] = w;
        w += (size_t)B * h_out[l];
        k.H[l] = w;
        w += (size_t)B * h_out[l];
    }
    k.dtaps = w;
    w += (size_t)B * 16;
    k.dA = w;
    w += (size_t)B * 64;
    k.dB = w;
    return k;
}

cudaError_t forward(const float *params, const float *x, int B, Work &k, cudaStream_t s)
{
    const int P = param_count();
    round_kernel<<<(P + 255) / 256, 256, 0, s>>>(params, k.Wr, P);
    const float *in = x;
    for (int l = 0; l < NL; ++l) {
        const float *W = k.Wr + param_off(l), *b = W + h_out[l] * h_in[l];
        const long n = (long)B * h_out[l];
        dense_fwd<<<(unsigned)((n + 127) / 128), 128, (size_t)h_out[l] * (h_in[l] + 1) * sizeof(float), s>>>(
            in, B, h_in[l], W, b, h_out[l], l < NL - 1, k.Z[l], k.H[l]);
        in = k.H[l];
    }
    return cudaGetLastError();
}

cudaError_t backward(const float *x, int B, Work &k, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(k.grad, 0, param_count() * sizeof(float), s);
    if (e != cudaSuccess) return e;
    const float *dZ = k.dtaps;
    for (int l = NL - 1; l >= 0; --l) {
        const float *X = l == 0 ? x : k.H[l - 1];
        float *dW = k.grad + param_off(l), *db = dW + h_out[l] * h_in[l];
        const int nw = h_out[l] * (h_in[l] + 1), slice = 512;
        dense_bwd_w<<<dim3((nw + 127) / 128, (B + slice - 1) / slice), 128, 0, s>>>(X, dZ, B, h_in[l], h_out[l], slice, dW, db);
        if (l > 0) {
            float *dZp = (dZ == k.dA) ? k.dB : k.dA;
            const long n = (long)B * h_in[l];
            dense_bwd_x<<<(unsigned)((n + 127) / 128), 128, (size_t)h_out[l] * h_in[l] * sizeof(float), s>>>(
                dZ, k.Wr + param_off(l), B, h_in[l], h_out[l], k.Z[l - 1], dZp);
            dZ = dZp;
        }
    }
    return cudaGetLastError();
}

}  // namespace

int mlp_param_count() { return param_count(); }

size_t mlp_work_bytes(int B)
{
    size_t n = 2 * (size_t)param_count();
    for (int l = 0; l < NL; ++l) n += 2 * (size_t)B * h_out[l];
    n += (size_t)B * (16 + 64 + 64);
    return n * sizeof(float);
}

cudaError_t mlp_taps(const float *params, const float *x, int B, float *taps, float *work, cudaStream_t s)
{
    Work k = carve(work, B);
    cudaError_t e = forward(params, x, B, k, s);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(taps, k.H[NL - 1], (size_t)B * 16 * sizeof(float), cudaMemcpyDeviceToDevice, s);
}

cudaError_t mlp_grad(const float *params, const float *x, int nq, const float *prior, float scale, const int *inst,
                     const float *wt, int ninst, const double *f, const float2 *y, int S, float *grad, float *loss,
                     float *work, cudaStream_t s)
{
    Work k = carve(work, nq);
    cudaError_t e = forward(params, x, nq, k, s);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(loss, 0, sizeof(float), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(k.dtaps, 0, (size_t)nq * 16 * sizeof(float), s)) != cudaSuccess) return e;
    fir_loss<<<dim3((S + LOSS_THREADS - 1) / LOSS_THREADS, ninst), LOSS_THREADS, 0, s>>>(
        k.H[NL - 1], prior, scale, inst, wt, nq, S, f, y, 2.f / ((float)ninst * (float)S), k.dtaps, loss);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = backward(x, nq, k, s)) != cudaSuccess) return e;
    if (grad) return cudaMemcpyAsync(grad, k.grad, param_count() * sizeof(float), cudaMemcpyDeviceToDevice, s);
    return cudaGetLastError();
}

cudaError_t mlp_train_step(float *params, float *adam, const float *x, int nq, const float *prior, float scale,
                           const int *inst, const float *wt, int ninst, const double *f, const float2 *y, int S,
                           float lr, int t, float *loss, float *work, cudaStream_t s)
{
    cudaError_t e = mlp_grad(params, x, nq, prior, scale, inst, wt, ninst, f, y, S, nullptr, loss, work, s);
    if (e != cudaSuccess) return e;
    Work k = carve(work, nq);
    const int P = param_count();
    const float b1 = 0.9f, b2 = 0.999f;
    adam_kernel<<<(P + 255) / 256, 256, 0, s>>>(params, k.grad, adam, adam + P, P, lr, b1, b2, 1e-8f,
                                                 1.f - powf(b1, (float)t), 1.f - powf(b2, (float)t));
    return cudaGetLastError();
}

int mlp_max_decimation() { return MAX_D; }

}  // namespace ffbp

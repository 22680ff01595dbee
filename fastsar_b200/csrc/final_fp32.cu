// The final stage on the CUDA cores in float32: the plain path (fastsar/ffbp_cpu.cpp:302-469 final_tiles,
// fastsar/ffbp_cuda.py:258-380 final_tile).
//
// Each final T x T tile is the separable sum
//   out[i, j] = sum_{p, q} A_p[i, q] B_p[j, q],   A_p[i, q] = d[p, q] wx exp(-2 pi i ux_p dlx_i (a0 + a1 q)),
//                                                  B_p[j, q] = wy exp(-2 pi i uy_p dly_j (a0 + a1 q)),
// then times the per-pixel quadratic phase exp(2 pi i qc_ij). One block of 64 threads forms one tile: per final
// subaperture p, threads build the two ramp tables in shared memory (one row each, by a complex recurrence over q
// seeded in float64), then every thread accumulates a RI x RI block of pixels (4 x 4 for T = 32) from them: per q,
// 2 RI float2 loads feed 4 RI^2 fused multiply-adds. The quadratic correction, the crop of the padded grid and
// the placement of the tile in the image are applied as the pixels are stored.
#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int FT = 64;     // threads per block
constexpr int QC = 48;     // frequency samples per table fill

struct FinalArgs {
    const float2 *__restrict__ d;
    int B, Pf, Qf;
    const double *__restrict__ ux;
    const double *__restrict__ uy;
    double spx, spy, a0, a1, fc2;
    const double *__restrict__ ucx;
    const double *__restrict__ ucy;
    const double *__restrict__ rc;
    const float *__restrict__ w;
    float2 *tiles;
    float2 *img;
    const int2 *__restrict__ first;
    int nx, ny, ox, oy;
    float scale;
};

__device__ __forceinline__ float2 cis_accurate(double cyc)
{
    const float f = (float)(cyc - rint(cyc));
    float s, c;
    sincospif(2.f * f, &s, &c);
    return make_float2(c, s);
}

template <int T>
__global__ void __launch_bounds__(FT) final_fp32_kernel(const FinalArgs a)
{
    constexpr int R = T / 8;                              // pixels per thread along each axis
    __shared__ __align__(16) float2 sA[QC][T];
    __shared__ __align__(16) float2 sB[QC][T];
    const int b = blockIdx.x;
    const int t = threadIdx.x;
    const int ti = t >> 3, tj = t & 7;
    const bool buildA = t < T, buildB = t >= T && t < 2 * T;
    const int row = buildA ? t : t - T;
    const double c = 0.5 * (T - 1);

    float2 acc[R][R];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) acc[i][j] = make_float2(0.f, 0.f);

    const float2 *__restrict__ db = a.d + (size_t)b * a.Pf * a.Qf;
    for (int p = 0; p < a.Pf; ++p) {
        float2 wv = make_float2(0.f, 0.f), st = make_float2(0.f, 0.f);
        float wt = 1.f;
        if (buildA || buildB) {
            const size_t bp = (size_t)b * a.Pf + p;
            const double u = buildA ? a.ux[bp] : a.uy[bp];
            const double dl = ((double)row - c) * (buildA ? a.spx : a.spy);
            wv = cis_accurate(-(u * dl) * a.a0);
            st = cis_accurate(-(u * dl) * a.a1);
            if (a.w) {
                const size_t nbp = (size_t)a.B * a.Pf;
                wt = buildA ? a.w[bp] + a.w[nbp + bp] * (float)dl : 1.f + a.w[2 * nbp + bp] * (float)dl;
            }
        }
        const float2 *__restrict__ dp = db + (size_t)p * a.Qf;
        for (int q0 = 0; q0 < a.Qf; q0 += QC) {
            const int qn = min(QC, a.Qf - q0);
            if (buildA) {
                for (int qq = 0; qq < qn; ++qq) {
                    const float2 v = cmul(__ldg(&dp[q0 + qq]), wv);
                    sA[qq][row] = make_float2(v.x * wt, v.y * wt);
                    wv = cmul(wv, st);
                }
            } else if (buildB) {
                for (int qq = 0; qq < qn; ++qq) {
                    sB[qq][row] = make_float2(wv.x * wt, wv.y * wt);
                    wv = cmul(wv, st);
                }
            }
            __syncthreads();
            for (int qq = 0; qq < qn; ++qq) {
                float2 av[R], bv[R];
#pragma unroll
                for (int i = 0; i < R; ++i) av[i] = sA[qq][R * ti + i];
#pragma unroll
                for (int j = 0; j < R; ++j) bv[j] = sB[qq][R * tj + j];
#pragma unroll
                for (int i = 0; i < R; ++i)
#pragma unroll
                    for (int j = 0; j < R; ++j) {
                        acc[i][j].x = fmaf(av[i].x, bv[j].x, acc[i][j].x);
                        acc[i][j].x = fmaf(-av[i].y, bv[j].y, acc[i][j].x);
                        acc[i][j].y = fmaf(av[i].x, bv[j].y, acc[i][j].y);
                        acc[i][j].y = fmaf(av[i].y, bv[j].x, acc[i][j].y);
                    }
            }
            __syncthreads();
        }
    }

    // quadratic phase, crop and store
    const double cx = a.ucx[b], cy = a.ucy[b], f = a.fc2 / (2.0 * a.rc[b]);
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int ii = R * ti + i;
        const double dx = ((double)ii - c) * a.spx;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int jj = R * tj + j;
            const double dy = ((double)jj - c) * a.spy;
            const double los = cx * dx + cy * dy;
            const float2 e = cis_cycles_d((dx * dx + dy * dy - los * los) * f);
            float2 v = cmul(acc[i][j], e);
            v.x *= a.scale;
            v.y *= a.scale;
            if (a.img) {
                const int2 f0 = a.first[b];
                const int x = f0.x + ii - a.ox, y = f0.y + jj - a.oy;
                if (x >= 0 && x < a.nx && y >= 0 && y < a.ny) a.img[(size_t)x * a.ny + y] = v;
            } else {
                a.tiles[((size_t)b * T + ii) * T + jj] = v;
            }
        }
    }
}

}  // namespace

cudaError_t launch_final_fp32(const FinalLaunch &F, cudaStream_t s, const char **why)
{
    *why = nullptr;
    FinalArgs a;
    a.d = F.d; a.B = F.B; a.Pf = F.Pf; a.Qf = F.Qf; a.ux = F.ux; a.uy = F.uy; a.spx = F.spx; a.spy = F.spy;
    a.a0 = F.a0; a.a1 = F.a1; a.fc2 = F.fc2; a.ucx = F.ucx; a.ucy = F.ucy; a.rc = F.rc; a.w = F.w;
    a.tiles = F.tiles; a.img = F.img; a.first = F.first; a.nx = F.nx; a.ny = F.ny; a.ox = F.ox; a.oy = F.oy;
    a.scale = F.scale;
    if (F.B <= 0) return cudaSuccess;
    if (F.T == 32) final_fp32_kernel<32><<<F.B, FT, 0, s>>>(a);
    else if (F.T == 16) final_fp32_kernel<16><<<F.B, FT, 0, s>>>(a);
    else { *why = "final tile size must be 16 or 32"; return cudaErrorInvalidValue; }
    return cudaGetLastError();
}

}  // namespace ffbp

// Exact backprojection onto a regular grid (the reference's ExactFormer, fastsar/exact.py:404-801, and its CUDA
// kernels bp_tiles, pad_window and crop, fastsar/exact.py:58-206), as B200 kernels behind the C ABI.
//
// Per chunk of pulses the caller windows and zero-pads the history (exact_pad: the window wp[p] wk[k] applied, the
// centre sample moved to bin 0, i.e. the fftshift folded in), takes the inverse FFT of length nfft (cuFFT), and
// calls exact_tiles: the reachable bins of each profile are cropped into a window of W bins (circularly, scaled by
// nfft) and backprojected onto the grid's tiles. A block owns one tile of TX x TY pixels; per group of TB pulses its
// threads compute the tile centre's terms in float64 (unit vector u, 1 / 2r, 1 / 2r^2, the fractional bin and the
// reduced phase) into shared memory; per pixel, with d its offset from the centre, du = d.u and D2 = |d|^2 - du^2,
// the range difference to third order is du + D2 / (2r) - du D2 / (2r^2), read from the profile by cubic Lagrange
// (four samples) or linear interpolation, and turned by exp(2 pi i (kcyc del + phase)). Consecutive blocks run
// along the grid axis closer to constant range (along1), so that resident blocks read the same bins from L2.
// The interpolation index is clamped into the window (the window covers the grid with a tile of margin on each
// side, so only pixels past the grid, which are not stored, can reach the clamp).
#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

__global__ void exact_pad_kernel(const float2 *__restrict__ s, int n, int K, const float *__restrict__ wp,
                                 const float *__restrict__ wk, int nfft, float2 *__restrict__ pad, int *bad, int p_off)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * K) return;
    const int p = (int)(idx / K), k = (int)(idx - (long)p * K), h = K / 2;
    const float g = (wp ? wp[p_off + p] : 1.f) * (wk ? wk[k] : 1.f);
    const float2 v = s[idx];
    if (bad && !(isfinite(v.x) && isfinite(v.y))) atomicMin(bad, p_off + p);
    pad[(long)p * nfft + (k >= h ? k - h : nfft - h + k)] = make_float2(v.x * g, v.y * g);
}

__global__ void exact_crop_kernel(const float2 *__restrict__ prof, const long long *__restrict__ blo, int n, int nfft,
                                  int W, float scale, float2 *__restrict__ win)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * W) return;
    const int p = (int)(idx / W), m = (int)(idx - (long)p * W);
    long long src = blo[p] + m - nfft / 2;
    src = ((src % nfft) + nfft) % nfft;
    const float2 v = prof[(long)p * nfft + src];
    win[idx] = make_float2(v.x * scale, v.y * scale);
}

struct TileArgs {
    const float2 *__restrict__ win;     // [n, W]
    const int *__restrict__ lo;         // [n] first bin of each window, relative to the profile's centre
    const double *__restrict__ ant;     // [n, 3]
    const double *__restrict__ ref;     // [n]
    const double *__restrict__ cen;     // [ntx nty, 3]
    float2 *out;                        // [nx, ny], accumulated
    int n, W, ntx, nty, nx, ny, along1;
    float spx, spy, e1x, e1y, e1z, e2x, e2y, e2z;
    double inv_dr, kcyc;
};

template <int TX, int TY, int TB, bool CUBIC>
__global__ void __launch_bounds__(TB) exact_tiles_kernel(const TileArgs a)
{
    constexpr int PX = TX * TY / TB;                          // pixels per thread
    __shared__ float s_ux[TB], s_uy[TB], s_uz[TB], s_hir[TB], s_hi2[TB], s_tf[TB], s_ph[TB];
    __shared__ int s_ti[TB];
    const int j = threadIdx.x;
    int bx, by;
    if (a.along1) {                                           // consecutive blocks along e1
        bx = blockIdx.x % a.ntx;
        by = blockIdx.x / a.ntx;
    } else {
        bx = blockIdx.x / a.nty;
        by = blockIdx.x % a.nty;
    }
    const int b = bx * a.nty + by;
    const double cx = a.cen[3 * b], cy = a.cen[3 * b + 1], cz = a.cen[3 * b + 2];
    float dx[PX], dy[PX], dz[PX], dd[PX], are[PX], aim[PX];
    int ix[PX], iy[PX];
#pragma unroll
    for (int m = 0; m < PX; ++m) {
        const int q = m * TB + j, li = q / TY, lj = q - li * TY;
        ix[m] = bx * TX + li;
        iy[m] = by * TY + lj;
        const float u = (li - 0.5f * (TX - 1)) * a.spx, v = (lj - 0.5f * (TY - 1)) * a.spy;
        dx[m] = u * a.e1x + v * a.e2x;
        dy[m] = u * a.e1y + v * a.e2y;
        dz[m] = u * a.e1z + v * a.e2z;
        dd[m] = dx[m] * dx[m] + dy[m] * dy[m] + dz[m] * dz[m];
        are[m] = 0.f;
        aim[m] = 0.f;
    }
    const float fdr = (float)a.inv_dr, fk = (float)a.kcyc;
    const int tmax = CUBIC ? a.W - 3 : a.W - 2, tmin = CUBIC ? 1 : 0;
    for (int p0 = 0; p0 < a.n; p0 += TB) {
        const int p = p0 + j;
        if (p < a.n) {
            const double *A = a.ant + 3 * p;
            const double wx = cx - A[0], wy = cy - A[1], wz = cz - A[2];
            const double r = sqrt(wx * wx + wy * wy + wz * wz), ir = 1.0 / r, dR = r - a.ref[p];
            const double t = dR * a.inv_dr - a.lo[p], tf = floor(t), ph = a.kcyc * dR;
            s_ux[j] = (float)(wx * ir);
            s_uy[j] = (float)(wy * ir);
            s_uz[j] = (float)(wz * ir);
            s_hir[j] = (float)(0.5 * ir);
            s_hi2[j] = (float)(0.5 * ir * ir);
            s_ti[j] = (int)tf;
            s_tf[j] = (float)(t - tf);
            s_ph[j] = (float)(ph - rint(ph));
        }
        __syncthreads();
        const int np = min(TB, a.n - p0);
        for (int k = 0; k < np; ++k) {
            const float ux = s_ux[k], uy = s_uy[k], uz = s_uz[k], hir = s_hir[k], hi2 = s_hi2[k], tfk = s_tf[k],
                        phk = s_ph[k];
            const int tik = s_ti[k];
            const float2 *row = a.win + (long)(p0 + k) * a.W;
#pragma unroll
            for (int m = 0; m < PX; ++m) {
                const float du = dx[m] * ux + dy[m] * uy + dz[m] * uz;
                const float del = du + (dd[m] - du * du) * (hir - du * hi2);
                const float t = tfk + del * fdr, fl = floorf(t), w = t - fl;
                const int i = min(max(tik + (int)fl, tmin), tmax);
                float vre, vim;
                if (CUBIC) {
                    const float2 a0 = __ldg(&row[i - 1]), a1 = __ldg(&row[i]), a2 = __ldg(&row[i + 1]), a3 = __ldg(&row[i + 2]);
                    const float wm1 = w - 1.f, wm2 = w - 2.f, wp1 = w + 1.f;
                    const float c0 = -w * wm1 * wm2 * (1.f / 6.f), c1 = wp1 * wm1 * wm2 * 0.5f;
                    const float c2 = -wp1 * w * wm2 * 0.5f, c3 = wp1 * w * wm1 * (1.f / 6.f);
                    vre = c0 * a0.x + c1 * a1.x + c2 * a2.x + c3 * a3.x;
                    vim = c0 * a0.y + c1 * a1.y + c2 * a2.y + c3 * a3.y;
                } else {
                    const float2 r0 = __ldg(&row[i]), r1 = __ldg(&row[i + 1]);
                    vre = fmaf(w, r1.x - r0.x, r0.x);
                    vim = fmaf(w, r1.y - r0.y, r0.y);
                }
                const float2 e = cis_cycles(fmaf(fk, del, phk));
                are[m] = fmaf(vre, e.x, fmaf(-vim, e.y, are[m]));
                aim[m] = fmaf(vre, e.y, fmaf(vim, e.x, aim[m]));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < PX; ++m)
        if (ix[m] < a.nx && iy[m] < a.ny) {
            const long o = (long)ix[m] * a.ny + iy[m];
            const float2 v = a.out[o];
            a.out[o] = make_float2(v.x + are[m], v.y + aim[m]);
        }
}

}  // namespace

cudaError_t launch_exact_pad(const float2 *s, int n, int K, const float *wp, const float *wk, int nfft, float2 *pad,
                             int *bad, int p_off, cudaStream_t st)
{
    const long total = (long)n * K;
    if (total <= 0) return cudaSuccess;
    exact_pad_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(s, n, K, wp, wk, nfft, pad, bad, p_off);
    return cudaGetLastError();
}

cudaError_t launch_exact_tiles(const float2 *prof, int n, int nfft, int W, const long long *blo, const int *lo,
                               const double *ant, const double *ref, const double *cen, int ntx, int nty, int tx,
                               int ty, int nx, int ny, double spx, double spy, const double *e1, const double *e2,
                               double inv_dr, double kcyc, int cubic, int along1, float2 *win, float2 *out,
                               cudaStream_t st, const char **why)
{
    *why = nullptr;
    if (n <= 0) return cudaSuccess;
    if (W < 4) { *why = "window of fewer than 4 bins"; return cudaErrorInvalidValue; }
    const long total = (long)n * W;
    exact_crop_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(prof, blo, n, nfft, W, (float)nfft, win);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    TileArgs a;
    a.win = win; a.lo = lo; a.ant = ant; a.ref = ref; a.cen = cen; a.out = out;
    a.n = n; a.W = W; a.ntx = ntx; a.nty = nty; a.nx = nx; a.ny = ny; a.along1 = along1;
    a.spx = (float)spx; a.spy = (float)spy;
    a.e1x = (float)e1[0]; a.e1y = (float)e1[1]; a.e1z = (float)e1[2];
    a.e2x = (float)e2[0]; a.e2y = (float)e2[1]; a.e2z = (float)e2[2];
    a.inv_dr = inv_dr; a.kcyc = kcyc;
    const unsigned nb = (unsigned)(ntx * nty);
#define FFBP_EXACT(TXV, TYV, TBV)                                                                     \
    (cubic ? (exact_tiles_kernel<TXV, TYV, TBV, true><<<nb, TBV, 0, st>>>(a), cudaGetLastError())     \
           : (exact_tiles_kernel<TXV, TYV, TBV, false><<<nb, TBV, 0, st>>>(a), cudaGetLastError()))
    if (tx == 32 && ty == 32) return FFBP_EXACT(32, 32, 128);
    if (tx == 16 && ty == 16) return FFBP_EXACT(16, 16, 128);
    if (tx == 8 && ty == 16) return FFBP_EXACT(8, 16, 128);
    if (tx == 8 && ty == 8) return FFBP_EXACT(8, 8, 64);
#undef FFBP_EXACT
    *why = "tile sizes are 32 x 32, 16 x 16, 8 x 16 or 8 x 8";
    return cudaErrorInvalidValue;
}

}  // namespace ffbp

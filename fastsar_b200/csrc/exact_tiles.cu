// Exact backprojection onto a regular grid: the device side of ExactFormer (the reference's exact former,
// fastsar/exact.py:404-801, whose mathematics this keeps: per tile a float64 centre, per pixel a third-order
// expansion of the range about it, cubic Lagrange or linear reads of the range profiles at 8x oversampling).
//
// Per chunk of pulses the caller pads and windows the history (exact_pad: the window wp[p] wk[k], the centre
// sample moved to bin 0, so that bin 0 of a profile is zero delay) and takes the inverse FFT of length nfft (cuFFT).
// exact_backproject then reads those full profiles directly; there is no cropped copy of them:
//
//  * A block owns one tile of TX x TY pixels (a thread PX of them, their offsets d from the tile centre in
//    registers). It sweeps the chunk's pulses in groups of G, double-buffered in shared memory.
//  * For a group, warp 0 computes in float64, one pulse per lane, the centre's line of sight u, 1 / 2r, 1 / 2r^2, the
//    centre's profile bin b + f (f in [0, 1)) and its reduced phase. Only the bins the tile can reach matter: a band
//    of BW bins from the even bin s = b - HB rounded down (HB: the tile's largest range offset in bins, with the
//    interpolation's margin). One thread copies each pulse's band into shared memory with one or two bulk copies
//    (cp.async.bulk, the copy engine; two where the band wraps past the profile's end, the profile being circular),
//    completing on the group's mbarrier; the next group's bands are in flight while this group is summed.
//  * Per pixel and pulse: du = d.u, D2 = |d|^2 - du^2, del = du + D2 (1/2r - du / 2r^2); the band is read at
//    (b - s) + f + del inv_dr by cubic Lagrange (4 samples) or linearly, rotated by exp(2 pi i (kcyc del + phase)) and
//    accumulated in float32. The profiles' 1 / nfft (cuFFT's inverse is unnormalised here, torch's normalised) is
//    undone once per pixel at the end, where the tile adds its sums into the image.
//  * Consecutive blocks run along the grid axis closer to constant range (along1), so that resident blocks read the
//    same profile bins from L2.
// Every wait on a group's mbarrier is bounded; a wait that runs out skips the group's sums and sets *err.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr uint64_t EXACT_WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t exact_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__global__ void exact_pad_kernel(const float2 *__restrict__ s, int n, int K, const float *__restrict__ wp,
                                 const float *__restrict__ wk, int nfft, float2 *__restrict__ pad, int *bad, int p_off)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * K) return;
    const int p = (int)(idx / K), k = (int)(idx - (long)p * K), h = K / 2;
    const float g = (wp ? wp[p_off + p] : 1.f) * (wk ? wk[k] : 1.f);
    const float2 v = s[idx];
    if (bad && !(isfinite(v.x) && isfinite(v.y))) atomicMin(bad, p_off + p);
    // sample k at bin k - K / 2 modulo nfft: zero delay at bin 0 of the inverse transform
    pad[(long)p * nfft + (k >= h ? k - h : nfft - h + k)] = make_float2(v.x * g, v.y * g);
}

struct ExactArgs {
    const float2 *__restrict__ prof;   // [n, nfft] inverse-FFT profiles, zero delay at bin 0
    const double *__restrict__ ant;    // [n, 3]
    const double *__restrict__ ref;    // [n]
    const double *__restrict__ cen;    // [ntx nty, 3] tile centres, tile (bx, by) at bx nty + by
    float2 *out;                       // [nx, ny], added to
    int *err;                          // raised when a bounded wait ran out (or null)
    int n, nfft, ntx, nty, nx, ny, along1, G, HB, BW;
    float spx, spy, e1x, e1y, e1z, e2x, e2y, e2z, scale;
    double inv_dr, kcyc;
};

// Per pulse of a group, what the pixels need (float32 after the float64 geometry).
struct PulseTerms {
    float ux, uy, uz, hir, hi2, off, ph;   // line of sight, 1/2r, 1/2r^2, (b - s) + f, reduced phase (cycles)
    int pad;
};

__device__ __forceinline__ bool exact_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t addr = exact_smem_u32(bar);
    uint32_t done = 0;
    uint64_t t0 = 0;
    for (uint32_t it = 0;; ++it) {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 200;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
        uint64_t now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if (it == 0) t0 = now;
        else if (now - t0 > EXACT_WAIT_NS) return false;
    }
}

template <int TX, int TY, int NT, bool CUBIC>
__global__ void __launch_bounds__(NT) exact_tiles_kernel(const ExactArgs a)
{
    constexpr int PX = TX * TY / NT;                          // pixels per thread
    extern __shared__ __align__(128) unsigned char smem[];
    float2 *band = reinterpret_cast<float2 *>(smem);                                 // [2][G][BW]
    PulseTerms *terms = reinterpret_cast<PulseTerms *>(band + 2 * (size_t)a.G * a.BW); // [2][G]
    uint64_t *bar = reinterpret_cast<uint64_t *>(terms + 2 * a.G);                     // [2]
    __shared__ volatile int s_fail;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int bx, by;
    if (a.along1) {
        bx = blockIdx.x % a.ntx;
        by = blockIdx.x / a.ntx;
    } else {
        bx = blockIdx.x / a.nty;
        by = blockIdx.x % a.nty;
    }
    const int tile = bx * a.nty + by;
    const double cx = a.cen[3 * tile], cy = a.cen[3 * tile + 1], cz = a.cen[3 * tile + 2];

    // this thread's pixels: pixel q = m NT + t of the tile, row q / TY along e1, column q % TY along e2
    float dx[PX], dy[PX], dz[PX], dd[PX];
    float2 acc[PX];
#pragma unroll
    for (int m = 0; m < PX; ++m) {
        const int q = m * NT + t, li = q / TY, lj = q % TY;
        const float o1 = ((float)li - 0.5f * (TX - 1)) * a.spx, o2 = ((float)lj - 0.5f * (TY - 1)) * a.spy;
        dx[m] = fmaf(o1, a.e1x, o2 * a.e2x);
        dy[m] = fmaf(o1, a.e1y, o2 * a.e2y);
        dz[m] = fmaf(o1, a.e1z, o2 * a.e2z);
        dd[m] = o1 * o1 + o2 * o2;                            // e1, e2 orthonormal
        acc[m] = make_float2(0.f, 0.f);
    }
    if (t == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(exact_smem_u32(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(exact_smem_u32(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int ngroups = (a.n + a.G - 1) / a.G;
    // warp 0: the float64 terms of group g's pulses (lane k: pulse k), then lane 0 issues their bands' bulk copies
    auto stage = [&](int g) {
        const int buf = g & 1, p0 = g * a.G, np = min(a.G, a.n - p0);
        int sm = 0;                                           // lane's band start, a bin of the profile (even)
        if (lane < np) {
            const double *A = a.ant + 3 * (size_t)(p0 + lane);
            const double wx = cx - A[0], wy = cy - A[1], wz = cz - A[2];
            const double r = sqrt(wx * wx + wy * wy + wz * wz), ir = 1.0 / r;
            const double dR = r - a.ref[p0 + lane];
            const double tc = dR * a.inv_dr, bf = floor(tc);
            const long long bb = (long long)bf;
            long long s0 = bb - a.HB;
            s0 -= (s0 & 1);                                   // down to an even bin
            const double ph = a.kcyc * dR;
            PulseTerms q;
            q.ux = (float)(wx * ir);
            q.uy = (float)(wy * ir);
            q.uz = (float)(wz * ir);
            q.hir = (float)(0.5 * ir);
            q.hi2 = (float)(0.5 * ir * ir);
            q.off = (float)((double)(bb - s0) + (tc - bf));
            q.ph = (float)(ph - rint(ph));
            q.pad = 0;
            terms[buf * a.G + lane] = q;
            long long w = s0 % a.nfft;
            sm = (int)(w < 0 ? w + a.nfft : w);
        }
        __syncwarp();
        const uint32_t b = exact_smem_u32(&bar[buf]);
        if (lane == 0) {
            // the band buffer was last read by the group two back (every thread is past it): order those reads
            // before the copy engine's writes
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         :: "r"(b), "r"((uint32_t)np * (uint32_t)a.BW * 8u) : "memory");
        }
        for (int k = 0; k < np; ++k) {
            const int s = __shfl_sync(0xffffffffu, sm, k);
            if (lane == 0) {
                const float2 *row = a.prof + (size_t)(p0 + k) * a.nfft;
                const uint32_t dst = exact_smem_u32(band + ((size_t)buf * a.G + k) * a.BW);
                const int l1 = min(a.BW, a.nfft - s);         // up to the profile's end, then from its start
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             :: "r"(dst), "l"(row + s), "r"((uint32_t)l1 * 8u), "r"(b) : "memory");
                if (l1 < a.BW)
                    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                                 :: "r"(dst + (uint32_t)l1 * 8u), "l"(row), "r"((uint32_t)(a.BW - l1) * 8u), "r"(b)
                                 : "memory");
            }
        }
    };

    const float fdr = (float)a.inv_dr, fk = (float)a.kcyc;
    const int imin = CUBIC ? 1 : 0, imax = CUBIC ? a.BW - 3 : a.BW - 2;
    if (warp == 0) stage(0);
    for (int g = 0; g < ngroups; ++g) {
        const int buf = g & 1, np = min(a.G, a.n - g * a.G);
        // the next group's terms and bands go to the other buffers, last used by group g - 1 (done: the barrier
        // at the end of the previous iteration)
        if (warp == 0 && g + 1 < ngroups && !s_fail) stage(g + 1);
        const bool ok = exact_wait(&bar[buf], (uint32_t)((g >> 1) & 1));
        if (!ok) {
            s_fail = 1;
            if (a.err) atomicAdd(a.err, 1);
        }
        if (ok && !s_fail) {
            const PulseTerms *T = terms + buf * a.G;
            const float2 *B = band + (size_t)buf * a.G * a.BW;
            for (int k = 0; k < np; ++k) {
                const PulseTerms q = T[k];
                const float2 *row = B + (size_t)k * a.BW;
#pragma unroll
                for (int m = 0; m < PX; ++m) {
                    const float du = fmaf(dx[m], q.ux, fmaf(dy[m], q.uy, dz[m] * q.uz));
                    const float del = fmaf(fmaf(-du, du, dd[m]), fmaf(-du, q.hi2, q.hir), du);
                    const float x = fmaf(del, fdr, q.off), fl = floorf(x), w = x - fl;
                    const int i = min(max((int)fl, imin), imax);
                    float2 v;
                    if (CUBIC) {
                        // Lagrange weights of the samples at -1, 0, 1, 2 for the offset w in [0, 1)
                        const float2 s0 = row[i - 1], s1 = row[i], s2 = row[i + 1], s3 = row[i + 2];
                        const float wa = w + 1.f, wb = w - 1.f, wc = w - 2.f;
                        const float l0 = -(1.f / 6.f) * w * wb * wc, l1 = 0.5f * wa * wb * wc;
                        const float l2 = -0.5f * wa * w * wc, l3 = (1.f / 6.f) * wa * w * wb;
                        v.x = fmaf(l0, s0.x, fmaf(l1, s1.x, fmaf(l2, s2.x, l3 * s3.x)));
                        v.y = fmaf(l0, s0.y, fmaf(l1, s1.y, fmaf(l2, s2.y, l3 * s3.y)));
                    } else {
                        const float2 s0 = row[i], s1 = row[i + 1];
                        v.x = fmaf(w, s1.x - s0.x, s0.x);
                        v.y = fmaf(w, s1.y - s0.y, s0.y);
                    }
                    const float2 e = cis_cycles(fmaf(fk, del, q.ph));
                    acc[m].x = fmaf(v.x, e.x, fmaf(-v.y, e.y, acc[m].x));
                    acc[m].y = fmaf(v.x, e.y, fmaf(v.y, e.x, acc[m].y));
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < PX; ++m) {
        const int q = m * NT + t, ix = bx * TX + q / TY, iy = by * TY + q % TY;
        if (ix < a.nx && iy < a.ny) {
            float2 *o = a.out + (size_t)ix * a.ny + iy;
            const float2 v = *o;
            *o = make_float2(fmaf(acc[m].x, a.scale, v.x), fmaf(acc[m].y, a.scale, v.y));
        }
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

cudaError_t launch_exact_tiles(const float2 *prof, int n, int nfft, const double *ant, const double *ref,
                               const double *cen, int ntx, int nty, int tx, int ty, int nx, int ny, double spx,
                               double spy, const double *e1, const double *e2, double inv_dr, double kcyc, int cubic,
                               int along1, float2 *out, int *err, cudaStream_t st, const char **why)
{
    *why = nullptr;
    if (n <= 0) return cudaSuccess;
    if (((uintptr_t)prof & 15) != 0) { *why = "profiles must be 16-byte aligned"; return cudaErrorInvalidValue; }
    if (nfft < 8 || (nfft & 1)) { *why = "nfft must be even and at least 8"; return cudaErrorInvalidValue; }
    ExactArgs a;
    a.prof = prof; a.ant = ant; a.ref = ref; a.cen = cen; a.out = out; a.err = err;
    a.n = n; a.nfft = nfft; a.ntx = ntx; a.nty = nty; a.nx = nx; a.ny = ny; a.along1 = along1;
    a.spx = (float)spx; a.spy = (float)spy;
    a.e1x = (float)e1[0]; a.e1y = (float)e1[1]; a.e1z = (float)e1[2];
    a.e2x = (float)e2[0]; a.e2y = (float)e2[1]; a.e2z = (float)e2[2];
    a.inv_dr = inv_dr; a.kcyc = kcyc; a.scale = (float)nfft;
    // the band: a pixel's range offset from its tile centre is at most 1.16 h (h the tile's half-diagonal; the
    // set-up keeps the tiles at least 4 h from every antenna position), plus the interpolation's samples
    const double h = 0.5 * sqrt(((tx - 1) * spx) * ((tx - 1) * spx) + ((ty - 1) * spy) * ((ty - 1) * spy));
    a.HB = (int)ceil(1.2 * h * inv_dr) + 3;
    a.BW = 2 * a.HB + 6;
    if (a.BW > nfft) { *why = "a tile spans more range bins than a profile holds"; return cudaErrorInvalidValue; }
    // pulses per group: both groups' bands within about 48 KB, so that several blocks share a multiprocessor
    const size_t per = (size_t)a.BW * sizeof(float2) + sizeof(PulseTerms);
    a.G = (int)std::max<size_t>(1, std::min<size_t>(32, (48u * 1024u) / (2 * per)));
    const size_t smem = 2 * (size_t)a.G * per + 2 * sizeof(uint64_t);
    if (smem > 200u * 1024u) { *why = "a tile's range band does not fit shared memory"; return cudaErrorInvalidValue; }
    const unsigned nb = (unsigned)(ntx * nty);
    auto run = [&](auto kern, int nt) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<nb, nt, smem, st>>>(a);
        return cudaGetLastError();
    };
    if (tx == 32 && ty == 32) return cubic ? run(exact_tiles_kernel<32, 32, 256, true>, 256) : run(exact_tiles_kernel<32, 32, 256, false>, 256);
    if (tx == 16 && ty == 16) return cubic ? run(exact_tiles_kernel<16, 16, 256, true>, 256) : run(exact_tiles_kernel<16, 16, 256, false>, 256);
    if (tx == 8 && ty == 16) return cubic ? run(exact_tiles_kernel<8, 16, 128, true>, 128) : run(exact_tiles_kernel<8, 16, 128, false>, 128);
    if (tx == 8 && ty == 8) return cubic ? run(exact_tiles_kernel<8, 8, 64, true>, 64) : run(exact_tiles_kernel<8, 8, 64, false>, 64);
    *why = "tile sizes are 32 x 32, 16 x 16, 8 x 16 or 8 x 8";
    return cudaErrorInvalidValue;
}

}  // namespace ffbp

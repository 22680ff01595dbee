// The final stage on the tcgen05 tensor cores (sm_100a): the chosen form of fastsar/ffbp_cpu.cpp:302-469's
// final_tiles (the reference's CUDA counterpart is the wmma kernel final_tile_tc2, fastsar/ffbp_cuda.py:1371-1524).
//
// Each T = 32 tile is the complex sum out[i, j] = sum_n A[i, n] B[j, n] over n = (p, q) (final subaperture p,
// frequency sample q) with A = d wx exp(-2 pi i ux dlx (a0 + a1 q)) and B = wy exp(-2 pi i uy dly (a0 + a1 q)).
// As one real product, D = [Ar; Ai] [Br; Bi]^T (64 x 64, K = Pf Qfp with Qf padded to a multiple of 16 by zeros):
// re = D[i][j] - D[i+32][j+32], im = D[i][j+32] + D[i+32][j].
//
// Block roles (persistent over tiles; one block per SM):
//   warps 5..12  producers: per final subaperture they build A' and B' (64 rows x Qfp) in shared memory, a row's
//                ramp by a complex recurrence along q seeded in float64, converted to the MMA operand type, into a
//                ring of S stages (K-major, no swizzle: core matrices of 8 rows x 16 bytes);
//   warp 4       one thread issues tcgen05.mma (M = 64, N = 64, K = 16) from each stage into a TMEM accumulator
//                and commits to the stage's "empty" barrier; after a tile's last stage it commits to the
//                accumulator's "full" barrier. The warp allocates two 64-column accumulators (128 TMEM columns);
//   warps 0..3   epilogue: reads the accumulator (rows 16w..16w+15 sit in TMEM lanes 32w..32w+15), releases it,
//                combines re/im through shared memory, applies the quadratic phase and writes the tile into the
//                image (cropped).
// Operand types: FFBP_FINAL_TC_F16 one float16 product; FFBP_FINAL_TC_BF16X3 three bfloat16 products
// (hi hi + hi lo + lo hi, with x = hi + lo), float32 accumulation in both.
//
// Every wait on a barrier is bounded: a wait that runs out sets *err (when given) and the block winds down without
// touching the barrier again; the MMA thread drains its MMAs (bounded) before the accumulator columns are freed.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int TT = 32;                     // tile side
constexpr int NTHREADS = 13 * 32;          // 4 epilogue warps, 1 MMA warp, 8 producer warps
constexpr int PRODUCER0 = 5 * 32;
constexpr int NPROD = 8 * 32;
constexpr long WAIT_LIMIT = 1L << 24;      // polls of a barrier before it counts as stuck

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint32_t mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done;
}

// Bounded wait for the phase of parity `parity` of *bar; false (and the block's abort flag and *err set) when it
// does not complete, or when another thread of the block has aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort, int *err)
{
    for (long it = 0; it < WAIT_LIMIT; ++it) {
        if (mbar_test(bar, parity)) return true;
        if (*abort) return false;
    }
    *abort = 1;
    if (err) atomicExch(err, 1);
    return false;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    // sm_100 shared-memory matrix descriptor: start address, leading (K) and stride (M/N) byte offsets in 16-byte
    // units, version 1 at bit 46, no swizzle
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_f16kind(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

struct TcArgs {
    const float2 *__restrict__ d;
    int B, Pf, Qf, Qfp, S, parts;
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
    int *err;
};

__device__ __forceinline__ float2 cis_acc(double cyc)
{
    const float f = (float)(cyc - rint(cyc));
    float s, c;
    sincospif(2.f * f, &s, &c);
    return make_float2(c, s);
}

// 8 values -> 16 bytes of operand: float16, or bfloat16 high parts (lo = nullptr) and low parts
template <bool BF>
__device__ __forceinline__ void pack8(const float *v, uint4 &hi, uint4 &lo)
{
    uint32_t h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (BF) {
            const __nv_bfloat162 x = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
            const float r0 = v[2 * e] - __low2float(x), r1 = v[2 * e + 1] - __high2float(x);
            const __nv_bfloat162 y = __floats2bfloat162_rn(r0, r1);
            h[e] = *reinterpret_cast<const uint32_t *>(&x);
            l[e] = *reinterpret_cast<const uint32_t *>(&y);
        } else {
            const __half2 x = __floats2half2_rn(v[2 * e], v[2 * e + 1]);
            h[e] = *reinterpret_cast<const uint32_t *>(&x);
            l[e] = 0;
        }
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

template <bool BF, bool WEIGHTED, int MAXIT>
__global__ void __launch_bounds__(NTHREADS, 1) final_tc_kernel(const TcArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    // layout: [S stages][parts][A', B'] operand buffers (64 x Qfp elements of 2 bytes each), then sD, then barriers
    const int ng = a.Qfp / 8;                                   // core matrices along K per operand
    const uint32_t opbytes = 64u * a.Qfp * 2u;                  // one operand buffer
    const uint32_t stagebytes = opbytes * 2u * a.parts;
    float *sD = reinterpret_cast<float *>(smem + (size_t)a.S * stagebytes);           // [64][65]
    uint64_t *bars = reinterpret_cast<uint64_t *>(sD + 64 * 65);
    uint64_t *full = bars, *empty = bars + a.S, *accf = bars + 2 * a.S, *acce = accf + 2;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;

    const int t = threadIdx.x, warp = t / 32, lane = t % 32;
    if (t == 0) {
        s_abort = 0;
        for (int s = 0; s < a.S; ++s) {
            mbar_init(&full[s], 8);
            mbar_init(&empty[s], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&accf[k], 1);
            mbar_init(&acce[k], 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" :: "r"(smem_u32(&s_tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t smem0 = smem_u32(smem);

    if (t >= PRODUCER0) {
        // ------------------------------------------------------------------ producers
        // Work items: (row pair, group of 8 frequency samples). Pixel rows r and 31 - r have offsets dl and -dl,
        // so their ramps are complex conjugates: one recurrence serves both rows of a pair. An A item writes
        // Ar, Ai of rows r and 31 - r (d times the ramp and d times its conjugate); a B item writes Br, Bi of row r
        // and, for row 31 - r, the same real part and the negated imaginary part (a sign flip of the packed words).
        // Each thread's next stage's data (its d samples and the geometry) are loaded a stage ahead.
        const int pt = t - PRODUCER0;
        const int nitems = 32 * ng;                             // 16 A pairs and 16 B pairs per group
        const float sp32x = (float)a.spx, sp32y = (float)a.spy;
        // the items of this thread
        int it_kind[MAXIT], it_pair[MAXIT], it_g[MAXIT], nmine = 0;
        uint32_t it_off[MAXIT][4];                              // byte offsets of rows r, r+32, 31-r, 63-r at group g
        for (int item = pt; item < nitems && nmine < MAXIT; item += NPROD) {
            const bool A = item < 16 * ng;
            const int rel = A ? item : item - 16 * ng;
            it_kind[nmine] = A ? 1 : 0;
            const int r = rel & 15, g = rel >> 4;
            it_pair[nmine] = r;
            it_g[nmine] = g;
            const int rows[4] = {r, r + 32, 31 - r, 63 - r};
#pragma unroll
            for (int q = 0; q < 4; ++q)
                it_off[nmine][q] = (uint32_t)(((rows[q] >> 3) * ng + g) * 128 + (rows[q] & 7) * 16) + (A ? 0u : opbytes);
            ++nmine;
        }
        // the next tile's samples and geometry into L2 while this tile is formed (128-byte lines, spread over the
        // producer threads)
        auto prefetch_tile = [&](int tile) {
            if (tile >= a.B) return;
            const char *dbeg = reinterpret_cast<const char *>(a.d + (size_t)tile * a.Pf * a.Qf);
            const size_t dbytes = (size_t)a.Pf * a.Qf * sizeof(float2);
            for (size_t o = (size_t)pt * 128; o < dbytes; o += (size_t)NPROD * 128)
                asm volatile("prefetch.global.L2 [%0];" :: "l"(dbeg + o));
            if (pt < 8) {
                const double *src = (pt < 4 ? a.ux : a.uy) + (size_t)tile * a.Pf;
                const size_t ub = (size_t)a.Pf * sizeof(double);
                for (size_t o = (size_t)(pt & 3) * 128; o < ub; o += 4 * 128)
                    asm volatile("prefetch.global.L2 [%0];" :: "l"(reinterpret_cast<const char *>(src) + o));
            }
        };
        // prefetched data of the next stage: per item 8 d samples (A) and the direction cosine (A: ux, B: uy)
        float2 dnext[MAXIT][8];
        double unext[MAXIT];
        float wnext[MAXIT][3];
        auto fetch = [&](int tile, int p) {
            const size_t bp = (size_t)tile * a.Pf + p;
            const float2 *dp = a.d + bp * a.Qf;
#pragma unroll
            for (int k = 0; k < MAXIT; ++k) {
                if (k >= nmine) break;
                unext[k] = it_kind[k] ? __ldg(&a.ux[bp]) : __ldg(&a.uy[bp]);
                if (it_kind[k]) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int q = 8 * it_g[k] + e;
                        dnext[k][e] = q < a.Qf ? __ldg(&dp[q]) : make_float2(0.f, 0.f);
                    }
                }
                if (WEIGHTED) {
                    const size_t nbp = (size_t)a.B * a.Pf;
                    wnext[k][0] = __ldg(&a.w[bp]);
                    wnext[k][1] = __ldg(&a.w[nbp + bp]);
                    wnext[k][2] = __ldg(&a.w[2 * nbp + bp]);
                }
            }
        };
        long it = 0;
        int tile = blockIdx.x, p = 0;
        if (tile < a.B) fetch(tile, 0);
        prefetch_tile(tile + gridDim.x);
        for (; tile < a.B && !s_abort; ++it) {
            float2 dcur[MAXIT][8];
            double ucur[MAXIT];
            float wcur[MAXIT][3];
#pragma unroll
            for (int k = 0; k < MAXIT; ++k) {
                ucur[k] = unext[k];
#pragma unroll
                for (int e = 0; e < 8; ++e) dcur[k][e] = dnext[k][e];
                wcur[k][0] = wnext[k][0]; wcur[k][1] = wnext[k][1]; wcur[k][2] = wnext[k][2];
            }
            int ntile = tile, np_ = p + 1;
            if (np_ == a.Pf) { np_ = 0; ntile += gridDim.x; prefetch_tile(ntile + gridDim.x); }
            if (ntile < a.B) fetch(ntile, np_);
            const int stg = (int)(it % a.S);
            if (!mbar_wait(&empty[stg], (uint32_t)(((it / a.S) & 1) ^ 1), &s_abort, a.err)) break;
            unsigned char *sbase = smem + (size_t)stg * stagebytes;
#pragma unroll
            for (int k = 0; k < MAXIT; ++k) {
                if (k >= nmine) break;
                const bool isA = it_kind[k];
                const int r = it_pair[k], g = it_g[k];
                const float dlf = ((float)r - 0.5f * (TT - 1)) * (isA ? sp32x : sp32y);       // r < 16: dl < 0
                const double dl = ((double)r - 0.5 * (TT - 1)) * (isA ? a.spx : a.spy);
                float2 wv = cis_cycles_d(-(ucur[k] * dl) * (a.a0 + a.a1 * (8.0 * g)));
                const float2 st = cis_cycles_d(-(ucur[k] * dl) * a.a1);
                float w1 = 1.f, w2 = 1.f;                       // the weights of rows r and 31 - r
                if (WEIGHTED) {
                    if (isA) { w1 = wcur[k][0] + wcur[k][1] * dlf; w2 = wcur[k][0] - wcur[k][1] * dlf; }
                    else { w1 = 1.f + wcur[k][2] * dlf; w2 = 1.f - wcur[k][2] * dlf; }
                }
                float r1[8], i1[8], r2[8], i2[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    if (isA) {
                        const float2 dd = dcur[k][e];
                        const float p1 = dd.x * wv.x, p2 = dd.y * wv.y, p3 = dd.x * wv.y, p4 = dd.y * wv.x;
                        r1[e] = (p1 - p2) * w1; i1[e] = (p3 + p4) * w1;       // d x
                        r2[e] = (p1 + p2) * w2; i2[e] = (p4 - p3) * w2;       // d conj(x)
                    } else {
                        r1[e] = wv.x * w1; i1[e] = wv.y * w1;
                        // row 31 - r: the conjugate ramp; without weights it is written from row r's packed words
                        r2[e] = WEIGHTED ? wv.x * w2 : 0.f;
                        i2[e] = WEIGHTED ? -wv.y * w2 : 0.f;
                    }
                    wv = cmul(wv, st);
                }
                uint4 h, l;
                pack8<BF>(r1, h, l);
                *reinterpret_cast<uint4 *>(sbase + it_off[k][0]) = h;
                if (BF) *reinterpret_cast<uint4 *>(sbase + 2 * opbytes + it_off[k][0]) = l;
                const bool mirror = !isA && !WEIGHTED;          // B row 31 - r from row r's words
                if (mirror) {                                   // row 31 - r: the same real part
                    *reinterpret_cast<uint4 *>(sbase + it_off[k][2]) = h;
                    if (BF) *reinterpret_cast<uint4 *>(sbase + 2 * opbytes + it_off[k][2]) = l;
                }
                pack8<BF>(i1, h, l);
                *reinterpret_cast<uint4 *>(sbase + it_off[k][1]) = h;
                if (BF) *reinterpret_cast<uint4 *>(sbase + 2 * opbytes + it_off[k][1]) = l;
                if (mirror) {                                   // row 31 - r: the imaginary part negated
                    const uint32_t sg = 0x80008000u;
                    h.x ^= sg; h.y ^= sg; h.z ^= sg; h.w ^= sg;
                    *reinterpret_cast<uint4 *>(sbase + it_off[k][3]) = h;
                    if (BF) {
                        l.x ^= sg; l.y ^= sg; l.z ^= sg; l.w ^= sg;
                        *reinterpret_cast<uint4 *>(sbase + 2 * opbytes + it_off[k][3]) = l;
                    }
                } else {
                    pack8<BF>(r2, h, l);
                    *reinterpret_cast<uint4 *>(sbase + it_off[k][2]) = h;
                    if (BF) *reinterpret_cast<uint4 *>(sbase + 2 * opbytes + it_off[k][2]) = l;
                    pack8<BF>(i2, h, l);
                    *reinterpret_cast<uint4 *>(sbase + it_off[k][3]) = h;
                    if (BF) *reinterpret_cast<uint4 *>(sbase + 2 * opbytes + it_off[k][3]) = l;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&full[stg]);
            p = np_;
            tile = ntile;
        }
    } else if (warp == 4) {
        // ------------------------------------------------------------------ MMA issue
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | ((BF ? 1u : 0u) << 7) | ((BF ? 1u : 0u) << 10) | ((64u >> 3) << 17) |
                                   ((64u >> 4) << 24);
            const uint32_t lbo = 128, sbo = (uint32_t)ng * 128;
            long it = 0;
            int lt = 0;
            for (int tile = blockIdx.x; tile < a.B && !s_abort; tile += gridDim.x, ++lt) {
                const int ab = lt & 1;
                if (!mbar_wait(&acce[ab], (uint32_t)(((lt >> 1) & 1) ^ 1), &s_abort, a.err)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t dt = tmem + (uint32_t)(ab * 64);
                bool ok = true;
                for (int p = 0; p < a.Pf; ++p, ++it) {
                    const int stg = (int)(it % a.S);
                    if (!mbar_wait(&full[stg], (uint32_t)((it / a.S) & 1), &s_abort, a.err)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sb = smem0 + (uint32_t)stg * stagebytes;
                    for (int ks = 0; ks < a.Qfp / 16; ++ks) {
                        const uint32_t koff = (uint32_t)ks * 256;
                        const uint64_t ah = smem_desc(sb + koff, lbo, sbo);
                        const uint64_t bh = smem_desc(sb + opbytes + koff, lbo, sbo);
                        const uint32_t accum = (p > 0 || ks > 0) ? 1u : 0u;
                        mma_f16kind(dt, ah, bh, idesc, accum);
                        if (BF) {
                            const uint64_t al = smem_desc(sb + 2 * opbytes + koff, lbo, sbo);
                            const uint64_t bl = smem_desc(sb + 3 * opbytes + koff, lbo, sbo);
                            mma_f16kind(dt, ah, bl, idesc, 1u);
                            mma_f16kind(dt, al, bh, idesc, 1u);
                        }
                    }
                    mma_commit(&empty[stg]);
                }
                if (!ok) break;
                mma_commit(&accf[ab]);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------------ epilogue (warps 0..3)
        int lt = 0;
        for (int tile = blockIdx.x; tile < a.B && !s_abort; tile += gridDim.x, ++lt) {
            const int ab = lt & 1;
            if (!mbar_wait(&accf[ab], (uint32_t)((lt >> 1) & 1), &s_abort, a.err)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(ab * 64);
            float v[16];
            const int m = 16 * warp + lane;                      // the accumulator row of this lane (lanes < 16)
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                tmem_ld16(base + (uint32_t)c0, v);
                if (lane < 16) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) sD[m * 65 + c0 + j] = v[j];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[ab]);
            asm volatile("bar.sync 1, 128;" ::: "memory");
            // pixels: thread -> row i, eight consecutive columns
            const int i = t >> 2, jb = (t & 3) * 8;
            const double cx = a.ucx[tile], cy = a.ucy[tile];
            const float f = (float)(a.fc2 / (2.0 * a.rc[tile]));
            const float dx = ((float)i - 0.5f * (TT - 1)) * (float)a.spx;
            const int2 f0 = a.img ? a.first[tile] : make_int2(0, 0);
            const int x = f0.x + i - a.ox;
            float2 outv[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const int j = jb + jj;
                const float re = sD[i * 65 + j] - sD[(i + 32) * 65 + j + 32];
                const float im = sD[i * 65 + j + 32] + sD[(i + 32) * 65 + j];
                const float dy = ((float)j - 0.5f * (TT - 1)) * (float)a.spy;
                const float los = (float)cx * dx + (float)cy * dy;
                const float qc = (dx * dx + dy * dy - los * los) * f;
                const float2 e = cis_cycles(qc);
                const float2 o = cmul(make_float2(re, im), e);
                outv[jj] = make_float2(o.x * a.scale, o.y * a.scale);
            }
            if (a.img) {
                if (x >= 0 && x < a.nx) {
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const int y = f0.y + jb + jj - a.oy;
                        if (y >= 0 && y < a.ny) a.img[(size_t)x * a.ny + y] = outv[jj];
                    }
                }
            } else {
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) a.tiles[((size_t)tile * TT + i) * TT + jb + jj] = outv[jj];
            }
            asm volatile("bar.sync 1, 128;" ::: "memory");
        }
    }

    // teardown: every role is done (or aborted); drain outstanding MMAs before freeing the accumulators
    __syncthreads();
    if (warp == 4) {
        if (lane == 0) {
            // a final commit on a fresh barrier arrives once every earlier MMA of this thread has completed
            uint64_t *drain = &acce[0];
            mbar_init(drain, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            mma_commit(drain);
            for (long it = 0; it < WAIT_LIMIT && !mbar_test(drain, 0); ++it) {
            }
        }
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" :: "r"(tmem));
    }
}

}  // namespace

cudaError_t launch_final_tc(const FinalLaunch &F, int mode, cudaStream_t s, const char **why)
{
    *why = nullptr;
    if (F.T != 32) { *why = "the tensor-core final stage is built for T = 32"; return cudaErrorNotSupported; }
    if (F.B <= 0) return cudaSuccess;
    TcArgs a;
    a.d = F.d; a.B = F.B; a.Pf = F.Pf; a.Qf = F.Qf; a.Qfp = (F.Qf + 15) & ~15;
    a.parts = (mode == 2) ? 2 : 1;
    a.ux = F.ux; a.uy = F.uy; a.spx = F.spx; a.spy = F.spy; a.a0 = F.a0; a.a1 = F.a1; a.fc2 = F.fc2;
    a.ucx = F.ucx; a.ucy = F.ucy; a.rc = F.rc; a.w = F.w; a.tiles = F.tiles; a.img = F.img; a.first = F.first;
    a.nx = F.nx; a.ny = F.ny; a.ox = F.ox; a.oy = F.oy; a.scale = F.scale; a.err = F.err;
    int dev = 0, nsm = 148, maxsmem = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t stage = (size_t)64 * a.Qfp * 2 * 2 * a.parts;
    const size_t fixed = (size_t)64 * 65 * 4 + 16 * 8 + 64;
    int S = 4;
    while (S > 2 && (size_t)S * stage + fixed > (size_t)maxsmem - 2048) --S;
    if ((size_t)S * stage + fixed > (size_t)maxsmem - 2048) {
        *why = "a final subaperture's operands do not fit shared memory (Qf too large for the tensor-core stage)";
        return cudaErrorNotSupported;
    }
    if (a.Qfp / 8 > 32) { *why = "more than 256 frequency samples per final tile"; return cudaErrorNotSupported; }
    a.S = S;
    const size_t smem = (size_t)S * stage + fixed;
    const int grid = F.B < nsm ? F.B : nsm;
    cudaError_t e;
    auto run = [&](auto kern) -> cudaError_t {
        cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r != cudaSuccess) return r;
        kern<<<grid, NTHREADS, smem, s>>>(a);
        return cudaGetLastError();
    };
    // items (row pair, group of 8 samples) per producer thread: 32 ng items over 256 threads
    const int maxit = (32 * (a.Qfp / 8) + NPROD - 1) / NPROD;
    if (maxit <= 1) {
        if (a.parts == 2) e = a.w ? run(final_tc_kernel<true, true, 1>) : run(final_tc_kernel<true, false, 1>);
        else e = a.w ? run(final_tc_kernel<false, true, 1>) : run(final_tc_kernel<false, false, 1>);
    } else if (maxit <= 2) {
        if (a.parts == 2) e = a.w ? run(final_tc_kernel<true, true, 2>) : run(final_tc_kernel<true, false, 2>);
        else e = a.w ? run(final_tc_kernel<false, true, 2>) : run(final_tc_kernel<false, false, 2>);
    } else {
        if (a.parts == 2) e = a.w ? run(final_tc_kernel<true, true, 4>) : run(final_tc_kernel<true, false, 4>);
        else e = a.w ? run(final_tc_kernel<false, true, 4>) : run(final_tc_kernel<false, false, 4>);
    }
    return e;
}

}  // namespace ffbp

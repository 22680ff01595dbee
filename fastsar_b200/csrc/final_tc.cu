// The final stage on the tcgen05 tensor cores (sm_100a): the chosen form of fastsar/ffbp_cpu.cpp:302-469's
// final_tiles (the reference's CUDA counterpart is the wmma kernel final_tile_tc2, fastsar/ffbp_cuda.py:1371-1524).
//
// Each T = 32 tile is the complex sum out[i, j] = sum_n A[i, n] B[j, n] over n = (p, q) (final subaperture p,
// frequency sample q) with A = d wx exp(-2 pi i ux dlx (a0 + a1 q)) and B = wy exp(-2 pi i uy dly (a0 + a1 q)).
// As one real product, D = [Ar; Ai] [Br; Bi]^T (64 x 64, K = Pf Qfp with Qf padded to a multiple of 16 by zeros):
// re = D[i][j] - D[i+32][j+32], im = D[i][j+32] + D[i+32][j].
//
// One MMA is M = 128, N = 128, K = 16, and a "unit" is what one accumulator holds:
//   FFBP_FINAL_TC_BF16X3  one tile, operands split x = hi + lo in bfloat16: A' = [A_hi; A_lo], B' = [B_hi; B_lo], so
//                         one product gives hi hi, hi lo, lo hi and lo lo of the tile, summed in the epilogue;
//   FFBP_FINAL_TC_F16     two T = 32 tiles in float16, A' = [A_1; A_2], B' = [B_1; B_2]: the two diagonal 64 x 64
//                         blocks of the product are the tiles; or four T = 16 tiles, whose 32 x 32 diagonal blocks
//                         are, each epilogue warp reading one of them from its own lane quarter. The samples are
//                         scaled by a power of two (from the largest sample component, which the last level kernel
//                         records) into float16's range, and the pixels by its inverse.
// The per-instruction issue cost of tcgen05.mma is the same for a 64 x 64 and a 128 x 128 product, so the larger
// shape does two or four times the work per instruction; two issuing warps double the rate again.
//
// Block roles (persistent over units; one block per SM):
//   warp 6       loader: stages each final subaperture's samples and geometry by cp.async into a ring of LS
//                slots, LS - 1 subapertures ahead (its copies' completion arrives on the slot's barrier);
//   warps 7..18  producers: per final subaperture they build A' and B' (128 rows x Qfp each) in shared memory from
//                the staged slot, a row's ramp by a complex recurrence along q seeded in float64, converted to the
//                operand type, into a ring of S stages (K-major, no swizzle: core matrices of 8 rows x 16 bytes);
//   warps 4, 5   one thread each issues tcgen05.mma: warp 4 + k takes the final subapertures p = k mod 2 of every
//                unit into its own accumulator (two 128-column accumulators per issuer, 512 TMEM columns), from its
//                own stages k, k + 2, ... of the ring (a stage with one consumer, so that no parity wait can run two
//                phases ahead of its barrier), commits each stage to the stage's "empty" barrier and the unit to the
//                accumulator's "full" barrier;
//   warps 0..3   epilogue: sum the issuers' accumulators (and, for bfloat16, the four split products), combine
//                re/im through shared memory, apply the quadratic phase and write the tile into the image (cropped).
//
// Every wait on a barrier is bounded: a wait that runs out sets *err (when given) and the block winds down without
// touching the barrier again; each issuing thread drains its MMAs (bounded) before the accumulator columns are freed.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int NEPI = 4;                    // epilogue warps 0..3 (TMEM lane quarters 0..3)
constexpr int NISS = 2;                    // MMA issuing warps 4, 5
constexpr int NLD = 1;                     // loader warp 6
constexpr int NPW = 12;                    // producer warps 7..18
constexpr int PW0 = NEPI + NISS + NLD;
constexpr int NTHREADS = (NEPI + NISS + NLD + NPW) * 32;
constexpr int LS = 8;                      // the loader's ring of staged final subapertures
constexpr int TMEM_COLS = 512;             // NISS issuers x 2 accumulators x 128 columns
constexpr uint64_t WAIT_NS = 2000000000ull;   // a barrier that has not completed after 2 s counts as stuck
constexpr uint32_t PRODUCER_HINT_NS = 1000;   // suspend-time hints of the waits: producers on a free stage or
                                              // a staged subaperture, the loader on a free ring slot,
constexpr uint32_t ISSUER_HINT_NS = 2000;     // the issuers on a filled stage,
constexpr uint32_t EPILOGUE_HINT_NS = 4000;   // the epilogue on a finished accumulator

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

__device__ __forceinline__ uint32_t mbar_test_sleep(uint64_t *bar, uint32_t parity, uint32_t hint_ns)
{
    // the thread may be suspended until the phase completes or about hint_ns have passed
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns) : "memory");
    return done;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase of parity `parity` of *bar: false (and the block's abort flag and *err set) when it
// has not completed after limit_ns of wall time, or when another thread of the block has aborted. HINT_NS is the
// suspend-time hint of each poll (0: poll without one).
template <uint32_t HINT_NS>
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort, int *err,
                                          uint64_t limit_ns = WAIT_NS)
{
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it) {
        if (HINT_NS ? mbar_test_sleep(bar, parity, HINT_NS) : mbar_test(bar, parity)) return true;
        if ((it & 255u) == 0) {
            if (*abort) return false;
            if (global_ns() - t0 > limit_ns) break;
        }
    }
    *abort = 1;
    if (err) atomicAdd(err, 1);
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

// 16 consecutive accumulator columns of this thread's TMEM lane, without waiting
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t *r)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(addr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// bytes = 4, 8 or 16 (dst and src aligned to it); the copy of an invalid element reads nothing and zero-fills the
// destination
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src, int bytes, bool valid)
{
    if (bytes == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" :: "r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" :: "r"(dst), "l"(src), "r"(valid ? 8 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"(dst), "l"(src), "r"(valid ? 4 : 0) : "memory");
}

struct TcArgs {
    const float2 *__restrict__ d;
    int B, Pf, Qf, Qfp, S, nunits, nis;
    const double *__restrict__ ux;
    const double *__restrict__ uy;
    const float4 *__restrict__ seeds;      // float16 form: the ramp seeds per tile and subaperture (or null)
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
    const int *amax;
    int interleave;                        // the order of the producer warps' items (final_tc_kernel)
    unsigned test_wait_ns;                 // tests only: the issuers' wait on a barrier nothing completes (0: none)
};

// The power of two s that brings samples whose components are at most *amax (a float's bits; null: unknown) to
// below 2^13 in magnitude, so that d s times a ramp and a weight stays inside float16's range (65504).
__device__ __forceinline__ float operand_scale(const int *amax)
{
    if (!amax) return 1.f;
    const float m = __int_as_float(*amax);
    if (!(m > 0.f) || !isfinite(m)) return 1.f;
    int ex;
    frexpf(m, &ex);                                             // m < 2^ex
    ex = ex < -100 ? -100 : (ex > 100 ? 100 : ex);
    return ldexpf(1.f, 13 - ex);
}

// 8 values -> 16 bytes of operand: float16, or bfloat16 high parts (and the low parts in lo)
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

__device__ __forceinline__ uint4 flip_sign(uint4 v)
{
    const uint32_t sg = 0x80008000u;
    return make_uint4(v.x ^ sg, v.y ^ sg, v.z ^ sg, v.w ^ sg);
}

// The tile of slot ts (float16: 128 / (2 TT) tiles per unit, split bfloat16: one) of this block's local unit ul
// (>= B when none).
template <bool BF, int TT>
__device__ __forceinline__ int unit_tile(int ul, int ts)
{
    const int u = (int)blockIdx.x + ul * (int)gridDim.x;
    return BF ? u : (64 / TT) * u + ts;
}

// The pixels of one T = 32 tile from P0 = D'[0:32, :] and P1 = D'[32:64, :] (rows of 64 + 1 floats in shared
// memory): thread t of the 128 epilogue threads takes row i = t / 4 and eight consecutive columns.
__device__ __forceinline__ void tile_pixels(const TcArgs &a, int tile, const float *P0, const float *P1, int t,
                                            float scale)
{
    constexpr int TT = 32;
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
        const float re = P0[i * 65 + j] - P1[i * 65 + j + 32];
        const float im = P0[i * 65 + j + 32] + P1[i * 65 + j];
        const float dy = ((float)j - 0.5f * (TT - 1)) * (float)a.spy;
        const float los = (float)cx * dx + (float)cy * dy;
        const float qc = (dx * dx + dy * dy - los * los) * f;
        const float2 e = cis_cycles(qc);
        const float2 o = cmul(make_float2(re, im), e);
        outv[jj] = make_float2(o.x * scale, o.y * scale);
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
}

// The pixels of one T = 16 tile: lane l < 16 of the warp holds accumulator row l (Ar row i = l) at the tile's 32
// columns (Br then Bi: v0 = D[i][j], v1 = D[i][j + 16]), lane l + 16 row Ai (v0 = D[i + 16][j], v1 = D[i + 16][j + 16]);
// re = D[i][j] - D[i + 16][j + 16], im = D[i][j + 16] + D[i + 16][j]. Lanes 0..15 write row i's 16 pixels.
__device__ __forceinline__ void tile16_pixels(const TcArgs &a, int tile, const float *v0, const float *v1, int lane,
                                              float scale)
{
    constexpr int TT = 16;
    float re[16], im[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const float d11 = __shfl_down_sync(0xffffffffu, v1[j], 16), d10 = __shfl_down_sync(0xffffffffu, v0[j], 16);
        re[j] = v0[j] - d11;
        im[j] = v1[j] + d10;
    }
    if (lane >= 16 || tile >= a.B) return;
    const int i = lane;
    const double cx = a.ucx[tile], cy = a.ucy[tile];
    const float f = (float)(a.fc2 / (2.0 * a.rc[tile]));
    const float dx = ((float)i - 0.5f * (TT - 1)) * (float)a.spx;
    const int2 f0 = a.img ? a.first[tile] : make_int2(0, 0);
    const int x = f0.x + i - a.ox;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const float dy = ((float)j - 0.5f * (TT - 1)) * (float)a.spy;
        const float los = (float)cx * dx + (float)cy * dy;
        const float qc = (dx * dx + dy * dy - los * los) * f;
        const float2 o = cmul(make_float2(re[j], im[j]), cis_cycles(qc));
        const float2 ov = make_float2(o.x * scale, o.y * scale);
        if (a.img) {
            const int y = f0.y + j - a.oy;
            if (x >= 0 && x < a.nx && y >= 0 && y < a.ny) a.img[(size_t)x * a.ny + y] = ov;
        } else {
            a.tiles[((size_t)tile * TT + i) * TT + j] = ov;
        }
    }
}

template <bool BF, bool WEIGHTED, int MAXWI, int TT>
__global__ void __launch_bounds__(NTHREADS, 1) final_tc_kernel(const TcArgs a)
{
    constexpr int NTS = BF ? 1 : 64 / TT;                       // tiles per unit
    extern __shared__ __align__(1024) unsigned char smem[];
    const int ng = a.Qfp / 8;                                   // core matrices along K per operand
    const uint32_t H = 64u * a.Qfp * 2u;                        // 64 operand rows
    const uint32_t HS = 2u * TT * a.Qfp * 2u;                   // one tile's operand rows (float16), 2 TT rows
    const uint32_t stagebytes = 4u * H;                         // A' (128 rows), B' (128 rows)
    float *sP = reinterpret_cast<float *>(smem + (size_t)a.S * stagebytes);             // [2][32][65]
    // the loader's ring: per slot and tile slot, the subaperture's Qfp samples (zero past Qf), ux, uy and the
    // three weights (tsb bytes)
    unsigned char *ring = reinterpret_cast<unsigned char *>(sP + 2 * 32 * 65);
    const uint32_t tsb = 8u * a.Qfp + 32u, slotbytes = (uint32_t)NTS * tsb;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + (size_t)LS * slotbytes);
    uint64_t *full = bars, *empty = bars + a.S, *accf = bars + 2 * a.S, *acce = accf + 2, *drain = acce + 2;
    uint64_t *lfull = drain + 2, *lempty = lfull + LS;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ uint64_t s_never;                                // a barrier nothing arrives on (the tests' stuck wait)

    const int t = threadIdx.x, warp = t / 32, lane = t % 32;
    const int nis = a.nis;
    // this block's units: blockIdx.x + ul gridDim.x
    const int nul = a.nunits > (int)blockIdx.x ? (a.nunits - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    if (t == 0) {
        s_abort = 0;
        for (int s = 0; s < a.S; ++s) {
            mbar_init(&full[s], NPW);
            mbar_init(&empty[s], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&accf[k], (uint32_t)nis);
            mbar_init(&acce[k], NEPI);
            mbar_init(&drain[k], 1);
        }
        for (int k = 0; k < LS; ++k) {
            mbar_init(&lfull[k], 32);                      // the loader's 32 threads, once their copies have landed
            mbar_init(&lempty[k], NPW);
        }
        mbar_init(&s_never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == NEPI) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&s_tmem)), "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t smem0 = smem_u32(smem);

    if (warp == NEPI + NISS) {
        // ------------------------------------------------------------------ loader
        // Stages every final subaperture of this block's units LS - 1 ahead of the producers: per tile slot the
        // Qfp samples (8 bytes each, zero past Qf and for a tile past the last), ux, uy and the weights, by cp.async
        // into ring slot it % LS; the copies' completion arrives on lfull (each thread's, .noinc), the producers'
        // reads of the slot on lempty. The next unit's samples and geometry are prefetched into L2 a unit ahead.
        const int nts = NTS;
        const int ntot = nul * a.Pf;
        const size_t nbp = (size_t)a.B * a.Pf;
        const bool fs = !BF && a.seeds;                         // stage the float32 seeds in place of ux, uy
        auto prefetch_unit = [&](int ul) {
            if (ul >= nul) return;
            for (int ts = 0; ts < nts; ++ts) {
                const int tile = unit_tile<BF, TT>(ul, ts);
                if (tile >= a.B) break;
                const char *dbeg = reinterpret_cast<const char *>(a.d + (size_t)tile * a.Pf * a.Qf);
                const int dbytes = a.Pf * a.Qf * (int)sizeof(float2);
                for (int o = lane * 128; o < dbytes; o += 32 * 128)
                    asm volatile("prefetch.global.L2 [%0];" :: "l"(dbeg + o));
                const char *src = fs ? reinterpret_cast<const char *>(a.seeds + (size_t)tile * a.Pf)
                                     : reinterpret_cast<const char *>((lane < 16 ? a.ux : a.uy) + (size_t)tile * a.Pf);
                const int ub = a.Pf * (fs ? 16 : 8);
                for (int o = (lane & 15) * 128; o < ub; o += 16 * 128)
                    asm volatile("prefetch.global.L2 [%0];" :: "l"(src + o));
            }
        };
        int ul = 0, p = 0;
        for (int it = 0; it < ntot; ++it) {
            const int ls = it % LS;
            if (it >= LS && !mbar_wait<PRODUCER_HINT_NS>(&lempty[ls], (uint32_t)((it / LS - 1) & 1), &s_abort, a.err))
                break;
            if (p == 0) prefetch_unit(ul + 1);
            const uint32_t sl = smem_u32(ring) + (uint32_t)ls * slotbytes;
            for (int ts = 0; ts < nts; ++ts) {
                const int tile = unit_tile<BF, TT>(ul, ts);
                const bool tv = tile < a.B;
                const size_t bp = tv ? (size_t)tile * a.Pf + p : 0;
                const float2 *src = a.d + bp * a.Qf;
                const uint32_t dst = sl + (uint32_t)ts * tsb;
                for (int q = lane; q < a.Qfp; q += 32) {
                    const bool v = tv && q < a.Qf;
                    cp_async(dst + 8u * q, v ? (const void *)(src + q) : (const void *)a.d, 8, v);
                }
                const uint32_t gd = dst + 8u * a.Qfp;
                if (fs) {
                    if (lane == 0) cp_async(gd, (const void *)(a.seeds + bp), 16, tv);
                } else if (lane < 2) cp_async(gd + 8u * lane, (const void *)((lane ? a.uy : a.ux) + bp), 8, tv);
                else if (WEIGHTED && lane < 5)
                    cp_async(gd + 16u + 4u * (lane - 2), (const void *)(a.w + (size_t)(lane - 2) * nbp + bp), 4, tv);
            }
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" :: "r"(smem_u32(&lfull[ls])) : "memory");
            if (++p == a.Pf) { p = 0; ++ul; }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp >= PW0) {
        // ------------------------------------------------------------------ producers
        // Warp items: (tile slot ts, operand A or B, pair of 8-sample groups gp). Lane l of the warp takes pixel
        // row pair r = l % 16 (rows r and 31 - r, whose offsets are dl and -dl, so that their ramps are complex
        // conjugates and one recurrence serves both) and group g = 2 gp + l / 16. An A item writes Ar, Ai of rows
        // r and 31 - r (d times the ramp and d times its conjugate); a B item writes Br, Bi of row r and, without
        // weights, row 31 - r from row r's words (the same real part, the imaginary part's sign flipped).
        const int pw = warp - PW0;
        constexpr int GPI = 64 / TT;                            // 8-sample groups per item: a lane per row pair
        const int hg = (ng + GPI - 1) / GPI;
        const int nts = NTS;
        const int nwi = nts * 2 * hg;
        const int ntot = nul * a.Pf;
        const int r = lane % (TT / 2), sub = lane / (TT / 2);
        // byte offsets (without the group) of rows r, r + TT, TT - 1 - r, 2 TT - 1 - r within a tile's 2 TT rows
        uint32_t roff[4];
        {
            const int rows[4] = {r, r + TT, TT - 1 - r, 2 * TT - 1 - r};
#pragma unroll
            for (int k = 0; k < 4; ++k) roff[k] = (uint32_t)(((rows[k] >> 3) * ng) * 128 + (rows[k] & 7) * 16);
        }
        // this warp's items (the same in every stage): tile slot, operand (0 = A), pair of groups; -1 = none
        int it_ts[MAXWI], it_op[MAXWI], it_gp[MAXWI];
#pragma unroll
        for (int k = 0; k < MAXWI; ++k) {
            if (a.interleave) {
                // A items first, then B items, dealt out to the warps forwards and backwards in turn, so that
                // with an even count per warp each warp builds as many A items (the heavier) as B items
                const int j = (k & 1) ? k * NPW + (NPW - 1 - pw) : k * NPW + pw;
                const int half = nwi / 2;
                it_ts[k] = j < nwi ? (j % half) / hg : -1;
                it_op[k] = j >= half ? 1 : 0;
                it_gp[k] = (j % half) % hg;
            } else {
                const int wi = pw + k * NPW;
                it_ts[k] = wi < nwi ? wi / (2 * hg) : -1;
                it_op[k] = (wi / hg) & 1;
                it_gp[k] = wi % hg;
            }
        }
        const float sp32x = (float)a.spx, sp32y = (float)a.spy;
        // the float16 operands carry d scaled by a power of two that keeps them inside the format's range
        const float dscale = BF ? 1.f : operand_scale(a.amax);
        // issuer k's stages are k + nis s for s < S / nis, filled and consumed in that issuer's order (one
        // consumer per stage: no wait can run two phases ahead); (ps_k, pp_k) is issuer k's next slot and parity
        const int rs = a.S / nis;
        int ps0 = 0, ps1 = 0;
        uint32_t pp0 = 0, pp1 = 0;
        int p = 0;
        for (int it = 0; it < ntot; ++it) {
            const int ls = it % LS;
            const int kq = nis == 2 ? (p & 1) : 0;
            const int stg = kq + nis * (kq ? ps1 : ps0);
            if (!mbar_wait<PRODUCER_HINT_NS>(&lfull[ls], (uint32_t)((it / LS) & 1), &s_abort, a.err)) break;
            if (!mbar_wait<PRODUCER_HINT_NS>(&empty[stg], (kq ? pp1 : pp0) ^ 1u, &s_abort, a.err)) break;
            const unsigned char *slotb = ring + (size_t)ls * slotbytes;
            unsigned char *sbase = smem + (size_t)stg * stagebytes;
#pragma unroll
            for (int k = 0; k < MAXWI; ++k) {
                if (it_ts[k] < 0) break;
                const int ts = it_ts[k], op = it_op[k];
                const int g = GPI * it_gp[k] + sub;
                if (g >= ng) continue;
                const unsigned char *tsp = slotb + (uint32_t)ts * tsb;
                const float *gw = reinterpret_cast<const float *>(tsp + 8 * a.Qfp + 16);   // the weights
                const bool isA = op == 0;
                const float dlf = ((float)r - 0.5f * (TT - 1)) * (isA ? sp32x : sp32y);      // r < TT / 2: dl < 0
                // the ramp of row offset dl = m sp / 2 (m = 2 r - (TT - 1)) at sample q: -u dl (a0 + a1 q) cycles,
                // seeded at q = 8 g with step -u dl a1
                float2 wv, st;
                if (!BF && a.seeds) {
                    // float32 from the plan's seeds (Y = frac(u sp a0 / 2), V = u sp a1 / 2): m Y carries the
                    // phase modulo 1 exactly as m u sp a0 / 2 does, to float32's rounding of Y and V
                    const float4 sd = *reinterpret_cast<const float4 *>(tsp + 8 * a.Qfp);
                    const float Y = isA ? sd.x : sd.z, V = isA ? sd.y : sd.w;
                    const float m = (float)(2 * r - (TT - 1)), mv = m * V;
                    wv = cis_cycles(-fmaf(m, Y, mv * (8.f * (float)g)));
                    st = cis_cycles(-mv);
                } else {
                    const double u = *reinterpret_cast<const double *>(tsp + 8 * a.Qfp + (isA ? 0 : 8));
                    const double dl = ((double)r - 0.5 * (TT - 1)) * (isA ? a.spx : a.spy);
                    const double ud = -(u * dl);
                    wv = cis_cycles_d(ud * fma(a.a1, 8.0 * g, a.a0));
                    st = cis_cycles_d(ud * a.a1);
                }
                if (isA) { wv.x *= dscale; wv.y *= dscale; }
                float w1 = 1.f, w2 = 1.f;                       // the weights of rows r and 31 - r
                if (WEIGHTED) {
                    if (isA) { w1 = gw[0] + gw[1] * dlf; w2 = gw[0] - gw[1] * dlf; }
                    else { w1 = 1.f + gw[2] * dlf; w2 = 1.f - gw[2] * dlf; }
                }
                // operand base: A' or B'; half: bfloat16 hi (lo one half further), float16 the tile slot's; group g
                unsigned char *ob = sbase + (isA ? 0u : 2u * H) + (BF ? 0u : (uint32_t)ts * HS) + (uint32_t)g * 128u;
                float r1[8], i1[8], r2[8], i2[8];
                if (isA) {
                    const float4 *dq = reinterpret_cast<const float4 *>(tsp + 64 * g);
#pragma unroll
                    for (int e2 = 0; e2 < 4; ++e2) {
                        const float4 dd = dq[e2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int e = 2 * e2 + h;
                            const float dr = h ? dd.z : dd.x, di = h ? dd.w : dd.y;
                            const float p1 = dr * wv.x, p2 = di * wv.y, p3 = dr * wv.y, p4 = di * wv.x;
                            r1[e] = (p1 - p2) * w1; i1[e] = (p3 + p4) * w1;       // d x
                            r2[e] = (p1 + p2) * w2; i2[e] = (p4 - p3) * w2;       // d conj(x)
                            wv = cmul(wv, st);
                        }
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        r1[e] = wv.x * w1; i1[e] = wv.y * w1;
                        r2[e] = WEIGHTED ? wv.x * w2 : 0.f;
                        i2[e] = WEIGHTED ? -wv.y * w2 : 0.f;
                        wv = cmul(wv, st);
                    }
                }
                uint4 h, l;
                const bool mirror = !isA && !WEIGHTED;
                pack8<BF>(r1, h, l);
                *reinterpret_cast<uint4 *>(ob + roff[0]) = h;
                if (BF) *reinterpret_cast<uint4 *>(ob + H + roff[0]) = l;
                if (mirror) {
                    *reinterpret_cast<uint4 *>(ob + roff[2]) = h;
                    if (BF) *reinterpret_cast<uint4 *>(ob + H + roff[2]) = l;
                }
                pack8<BF>(i1, h, l);
                *reinterpret_cast<uint4 *>(ob + roff[1]) = h;
                if (BF) *reinterpret_cast<uint4 *>(ob + H + roff[1]) = l;
                if (mirror) {
                    *reinterpret_cast<uint4 *>(ob + roff[3]) = flip_sign(h);
                    if (BF) *reinterpret_cast<uint4 *>(ob + H + roff[3]) = flip_sign(l);
                } else {
                    pack8<BF>(r2, h, l);
                    *reinterpret_cast<uint4 *>(ob + roff[2]) = h;
                    if (BF) *reinterpret_cast<uint4 *>(ob + H + roff[2]) = l;
                    pack8<BF>(i2, h, l);
                    *reinterpret_cast<uint4 *>(ob + roff[3]) = h;
                    if (BF) *reinterpret_cast<uint4 *>(ob + H + roff[3]) = l;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&full[stg]);
                mbar_arrive(&lempty[ls]);
            }
            if (kq) {
                if (++ps1 == rs) { ps1 = 0; pp1 ^= 1u; }
            } else if (++ps0 == rs) {
                ps0 = 0;
                pp0 ^= 1u;
            }
            if (++p == a.Pf) p = 0;
        }
    } else if (warp >= NEPI) {
        // ------------------------------------------------------------------ MMA issue
        const int k = warp - NEPI;
        if (lane == 0 && k < nis) {
            const uint32_t idesc = (1u << 4) | ((BF ? 1u : 0u) << 7) | ((BF ? 1u : 0u) << 10) | ((128u >> 3) << 17) |
                                   ((128u >> 4) << 24);
            const uint32_t lbo = 128, sbo = (uint32_t)ng * 128;
            const int nks = a.Qfp / 16;
            // descriptors of stage 0's A' and B'; stage s adds s stagebytes, K step ks adds 256 bytes (16 units)
            const uint64_t da0 = smem_desc(smem0, lbo, sbo), db0 = smem_desc(smem0 + 2u * H, lbo, sbo);
            const uint64_t dstage = (uint64_t)(stagebytes >> 4);
            const int rs = a.S / nis;
            int slot = 0;                                       // this issuer's stages: k + nis slot
            uint32_t par = 0;
            // tests of the failure report: a wait that runs out before any MMA, as a stuck pipeline's would
            const bool stuck = a.test_wait_ns &&
                               !mbar_wait<ISSUER_HINT_NS>(&s_never, 0, &s_abort, a.err, a.test_wait_ns);
            for (int ul = stuck ? nul : 0; ul < nul; ++ul) {
                const int ab = ul & 1;
                if (!mbar_wait<ISSUER_HINT_NS>(&acce[ab], (uint32_t)(((ul >> 1) & 1) ^ 1), &s_abort, a.err)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t dt = tmem + (uint32_t)((k * 2 + ab) * 128);
                bool ok = true;
                uint32_t accum = 0;
                for (int p = k; p < a.Pf; p += nis) {
                    const int stg = k + nis * slot;
                    if (!mbar_wait<ISSUER_HINT_NS>(&full[stg], par, &s_abort, a.err)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint64_t da = da0 + dstage * (uint64_t)stg, db = db0 + dstage * (uint64_t)stg;
                    for (int ks = 0; ks < nks; ++ks) {
                        mma_f16kind(dt, da + 16u * ks, db + 16u * ks, idesc, accum);
                        accum = 1u;
                    }
                    mma_commit(&empty[stg]);
                    if (++slot == rs) { slot = 0; par ^= 1u; }
                }
                if (!ok) break;
                mma_commit(&accf[ab]);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------------ epilogue (warps 0..3)
        float *P0 = sP, *P1 = sP + 32 * 65;
        const float oscale = a.scale / (BF ? 1.f : operand_scale(a.amax));
        // after a failed wait a warp keeps stepping through the units (and the epilogue's named barriers, which all
        // four warps must reach) without waiting, reading or writing
        bool live = true;
        for (int ul = 0; ul < nul; ++ul) {
            const int ab = ul & 1;
            if (live) live = mbar_wait<EPILOGUE_HINT_NS>(&accf[ab], (uint32_t)((ul >> 1) & 1), &s_abort, a.err);
            live = __all_sync(0xffffffffu, live);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t lanes = (uint32_t)(32 * warp) << 16;
            float *mine = (warp & 1) ? P1 : P0;                 // accumulator rows 32..63 (mod 64) are the Ai rows
            // the sum over the issuers' accumulators of columns [c0, c0 + 16), plus [c0 + c1, c0 + c1 + 16) if c1
            auto gather = [&](int c0, int c1, float *v) {
                uint32_t q0[16], q1[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = 0.f;
                for (int k = 0; k < nis; ++k) {
                    const uint32_t base = tmem + lanes + (uint32_t)((k * 2 + ab) * 128);
                    tmem_ld16(base + (uint32_t)c0, q0);
                    if (c1) tmem_ld16(base + (uint32_t)(c0 + c1), q1);
                    tmem_wait_ld();
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] += __uint_as_float(q0[j]) + (c1 ? __uint_as_float(q1[j]) : 0.f);
                }
            };
            if (BF) {
                // warps 0, 1: hi rows (hi hi + hi lo); then warps 2, 3 add the lo rows (lo hi + lo lo)
                float v[16];
                if (live && warp < 2) {
#pragma unroll
                    for (int c0 = 0; c0 < 64; c0 += 16) {
                        gather(c0, 64, v);
#pragma unroll
                        for (int j = 0; j < 16; ++j) mine[lane * 65 + c0 + j] = v[j];
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acce[ab]);
                }
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (live && warp >= 2) {
#pragma unroll
                    for (int c0 = 0; c0 < 64; c0 += 16) {
                        gather(c0, 64, v);
#pragma unroll
                        for (int j = 0; j < 16; ++j) mine[lane * 65 + c0 + j] += v[j];
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acce[ab]);
                }
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (live) tile_pixels(a, unit_tile<BF, TT>(ul, 0), P0, P1, t, oscale);
                asm volatile("bar.sync 1, 128;" ::: "memory");
            } else if (TT == 16) {
                // tile slot ts = warp: accumulator rows [32 ts, 32 ts + 32) (this warp's lane quarter) at columns
                // [32 ts, 32 ts + 32)
                if (live) {
                    float v0[16], v1[16];
                    gather(32 * warp, 0, v0);
                    gather(32 * warp + 16, 0, v1);
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acce[ab]);
                    tile16_pixels(a, unit_tile<BF, TT>(ul, warp), v0, v1, lane, oscale);
                }
            } else {
                // tile slot ts: accumulator rows and columns [64 ts, 64 ts + 64), read by warps 2 ts and 2 ts + 1
                for (int ts = 0; ts < 2; ++ts) {
                    if (live && (warp >> 1) == ts) {
                        float v[16];
#pragma unroll
                        for (int c0 = 0; c0 < 64; c0 += 16) {
                            gather(64 * ts + c0, 0, v);
#pragma unroll
                            for (int j = 0; j < 16; ++j) mine[lane * 65 + c0 + j] = v[j];
                        }
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&acce[ab]);
                    }
                    asm volatile("bar.sync 1, 128;" ::: "memory");
                    const int tile = unit_tile<BF, TT>(ul, ts);
                    if (live && tile < a.B) tile_pixels(a, tile, P0, P1, t, oscale);
                    asm volatile("bar.sync 1, 128;" ::: "memory");
                }
            }
        }
    }

    // teardown: every role is done (or aborted); each issuer drains its MMAs before the accumulators are freed
    __syncthreads();
    if (warp >= NEPI && warp < NEPI + NISS && lane == 0) {
        // a commit on a fresh barrier arrives once every earlier MMA of this thread has completed
        uint64_t *dr = &drain[warp - NEPI];
        mma_commit(dr);
        const uint64_t t0 = global_ns();
        bool drained = false;
        while (!(drained = mbar_test(dr, 0)) && global_ns() - t0 < WAIT_NS) {
        }
        if (!drained && a.err) atomicAdd(a.err, 1);              // an MMA still running: reported
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == NEPI) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS));
}

__global__ void final_seeds_kernel(const double *__restrict__ ux, const double *__restrict__ uy, long n, double spx,
                                   double spy, double a0, double a1, float4 *__restrict__ out)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double yx = 0.5 * ux[i] * spx * a0, yy = 0.5 * uy[i] * spy * a0;
        out[i] = make_float4((float)(yx - floor(yx)), (float)(0.5 * ux[i] * spx * a1), (float)(yy - floor(yy)),
                             (float)(0.5 * uy[i] * spy * a1));
    }
}

}  // namespace

cudaError_t launch_final_seeds(const double *ux, const double *uy, long n, double spx, double spy, double a0,
                               double a1, float4 *out, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const long nb = (n + 255) / 256;
    final_seeds_kernel<<<(int)(nb < 4096 ? nb : 4096), 256, 0, s>>>(ux, uy, n, spx, spy, a0, a1, out);
    return cudaGetLastError();
}

cudaError_t launch_final_tc(const FinalLaunch &F, int mode, cudaStream_t s, const char **why)
{
    *why = nullptr;
    const bool bf = mode == 2;
    if (F.T != 32 && (F.T != 16 || bf)) {
        *why = "the tensor-core final stage takes T = 32 (split bfloat16 or float16) or T = 16 (float16)";
        return cudaErrorNotSupported;
    }
    if (F.B <= 0) return cudaSuccess;
    if ((long long)F.B * F.Pf >= (1LL << 31)) { *why = "more than 2^31 final tile subapertures"; return cudaErrorNotSupported; }
    const int nts = bf ? 1 : 64 / F.T;                          // tiles per unit
    TcArgs a;
    a.d = F.d; a.B = F.B; a.Pf = F.Pf; a.Qf = F.Qf; a.Qfp = (F.Qf + 15) & ~15;
    a.nunits = (F.B + nts - 1) / nts;
    a.nis = F.Pf >= NISS ? NISS : 1;
    a.ux = F.ux; a.uy = F.uy; a.seeds = F.seeds; a.spx = F.spx; a.spy = F.spy; a.a0 = F.a0; a.a1 = F.a1; a.fc2 = F.fc2;
    a.ucx = F.ucx; a.ucy = F.ucy; a.rc = F.rc; a.w = F.w; a.tiles = F.tiles; a.img = F.img; a.first = F.first;
    a.nx = F.nx; a.ny = F.ny; a.ox = F.ox; a.oy = F.oy; a.scale = F.scale; a.err = F.err; a.amax = F.amax;
    a.test_wait_ns = F.test_wait_ns;
    int dev = 0, nsm = 148, maxsmem = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // warp items per stage: (tile slots) x (A, B) x (pairs of 8-sample groups) over the NPW producer warps; when
    // every warp gets the same even number of items they are interleaved (as many A items, the heavier, as B
    // items on each warp: 3 % faster at 47 x 91 in float16; 1 % slower at 38 x 71, whose count is uneven)
    const int ng = a.Qfp / 8, gpi = 64 / F.T, hg = (ng + gpi - 1) / gpi;
    const int nwi = nts * 2 * hg;
    a.interleave = nwi % (2 * NPW) == 0 ? 1 : 0;
    const int maxwi = (nwi + NPW - 1) / NPW;
    if (maxwi > 4) { *why = "more than 256 frequency samples per final tile"; return cudaErrorNotSupported; }
    const int mw = maxwi <= 1 ? 1 : (maxwi <= 2 ? 2 : 4);
    const size_t stage = (size_t)4 * 64 * a.Qfp * 2;
    const size_t slotbytes = (size_t)nts * (8 * a.Qfp + 32);
    const size_t fixed = (size_t)2 * 32 * 65 * 4 + (size_t)LS * slotbytes + (size_t)(2 * 4 + 6 + 2 * LS) * 8;
    const size_t avail = (size_t)maxsmem - 1024;                // static shared memory and slack
    // stages: a multiple of the issuers (each owns S / nis of them)
    int S = 4;
    while (S > 2 && ((size_t)S * stage + fixed > avail || S % a.nis)) --S;
    if ((size_t)S * stage + fixed > avail) {
        *why = "a final subaperture's operands do not fit shared memory (Qf too large for the tensor-core stage)";
        return cudaErrorNotSupported;
    }
    a.S = S;
    const size_t smem = (size_t)S * stage + fixed;
    const int grid = a.nunits < nsm ? a.nunits : nsm;
    auto run = [&](auto kern) -> cudaError_t {
        cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r != cudaSuccess) return r;
        kern<<<grid, NTHREADS, smem, s>>>(a);
        return cudaGetLastError();
    };
#define FFBP_TC_RUN(MW)                                                                                       \
    (bf ? (a.w ? run(final_tc_kernel<true, true, MW, 32>) : run(final_tc_kernel<true, false, MW, 32>))        \
        : F.T == 16 ? (a.w ? run(final_tc_kernel<false, true, MW, 16>) : run(final_tc_kernel<false, false, MW, 16>)) \
                    : (a.w ? run(final_tc_kernel<false, true, MW, 32>) : run(final_tc_kernel<false, false, MW, 32>)))
    cudaError_t e;
    if (mw == 1) e = FFBP_TC_RUN(1);
    else if (mw == 2) e = FFBP_TC_RUN(2);
    else e = FFBP_TC_RUN(4);
#undef FFBP_TC_RUN
    return e;
}

}  // namespace ffbp

// A level on the tcgen05 tensor cores (sm_100a): the chosen form of one merge stage of the FFBP (the reference's
// rot_fir_k + fir_p: fastsar/ffbp_cpu.cpp:146-293, fastsar/ffbp_cuda.py:48-256), in two passes.
//
// The rotation of child c at input pulse p and sample k, exp(2 pi i (c0 + sl (k - kc))), followed by the frequency
// FIR y[j] = sum_r hk[r] x[Dk j + r - plk] rot(Dk j + r - plk), factors as
//     y_c[p, j] = R_c,p[j] sum_r m_c,p[r] x[p, Dk j + r - plk],
//     m_c,p[r] = hk[r] exp(2 pi i sl r)                         (the child's modulated taps),
//     R_c,p[j] = exp(2 pi i (c0 + sl (Dk j - plk - kc)))        (a ramp along the output columns).
// Per pulse the sum is a dense product: the modulated taps of every child (children x taps) times the Hankel
// windows of the parent's row (taps x output columns), shared by all children. The pulse FIR that follows acts on
// the frequency-decimated columns.
//
// Pass 1 (level_tc_gemm): per parent and pulse the product on the tensor cores, three bfloat16 products (x = hi + lo:
// hi hi + hi lo + lo hi) accumulated in float32; then the ramp, a power-of-two scale into float16's range, and the
// intermediate y [Np, C, P, Kop] as float16 pairs. Real form: A' (128 rows, two per child: Mr, Mi; K = the taps
// padded to Lkp), B' = [Xr_j; Xi_j] (2 Nt rows: the real and imaginary Hankel rows of the tile's Nt columns),
// D = A' B'^T: re = MrXr - MiXi, im = MrXi + MiXr.
// Block roles: warps 8..23 produce, per pulse, the modulated taps (once per pulse, for all column tiles) and per
// (pulse, tile) the bfloat16 hi/lo planes of the parent row's window and from them the Hankel rows; warp 24 issues the
// MMAs (M = 128, N = 2 Nt, K = 16) into one of two TMEM accumulators; warps 0..7 read the accumulator (warp w reads
// lane quarter w % 4, i.e. children 16 (w % 4) .. + 15, and half of the columns), combine re/im, apply the ramp and
// store. Two read-outs, chosen by the tap count: with up to 32 taps (light producers, the consumers bound the stage)
// A' holds in each group of 16 rows the Mr rows of 8 children and then their Mi rows, and 16-row accumulator loads
// give each thread both rows of a child (no exchange between threads); with more taps A' = [Mr_0; Mi_0; Mr_1; ...]
// and the two lanes of a child exchange halves (measured faster there: 11.7 against 12.4 ms at the 12,288 x 8,832
// spotlight's third level, 8.2 against 7.1 ms the other way at its first). The producers' phases bound a stage at
// more taps, so they get two warps of every three (with 16 consumer and 8 producer warps a stage took 8-10 % longer
// at the second and third levels).
//
// Pass 2: the pulse FIR of the intermediate, written as complex64 with the largest component recorded: on the tensor
// cores as a banded product per row (level_fir_tc.cu), or on the CUDA cores in float32 (level_fir: a thread per two
// columns with the ceil(Lp / Dp) outputs it feeds in registers); a launch option, by default the tensor cores for
// output pulse axes of 512 or more.
//
// Every wait on a barrier is bounded in time; a wait that runs out sets *err and the block winds down.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int NCW = 8;                        // consumer warps 0..7 (a multiple of 4: the TMEM lane quarters)
constexpr int NPW = 16;                       // producer warps 8..23:
constexpr int NAW = 4;                        //   warps 8..11 build the modulated taps (A'),
constexpr int NBW = NPW - NAW;                //   warps 12..23 B': 12..15 the planes, 16..23 the Hankel rows
constexpr int NLW = 4, NHW = NBW - NLW;
constexpr int NAT = NAW * 32, NLT = NLW * 32, NHT = NHW * 32;
constexpr int MMAW = NCW + NPW;               // warp 24
constexpr int NTHR = (NCW + NPW + 1) * 32;
constexpr uint64_t WAIT_NS = 2000000000ull;
constexpr int XS = 4;                         // the producers' ring of parent-row windows, XS - 1 stages ahead

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint32_t mbar_test(uint64_t *bar, uint32_t parity, uint32_t hint_ns)
{
    uint32_t done;
    if (hint_ns)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done) : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns) : "memory");
    else
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase of parity `parity`: false (the block's abort flag set and *err raised) after limit_ns,
// or when another thread of the block has aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t hint_ns, volatile int *abort, int *err,
                                          uint64_t limit_ns = WAIT_NS)
{
    if (mbar_test(bar, parity, 0)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_test(bar, parity, hint_ns)) return true;
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

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
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

__device__ __forceinline__ void tmem_ld8(uint32_t addr, float *v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 8 consecutive bfloat16 samples from a plane copy: four 4-byte loads (PC = 2) or two 8-byte loads (PC = 4)
template <int PC>
__device__ __forceinline__ uint4 ld_run(const uint32_t *s)
{
    if constexpr (PC == 4) {
        const uint2 a = *reinterpret_cast<const uint2 *>(s), b = *reinterpret_cast<const uint2 *>(s + 2);
        return make_uint4(a.x, a.y, b.x, b.y);
    } else {
        return make_uint4(s[0], s[1], s[2], s[3]);
    }
}

// 8 bytes global -> shared by cp.async (zero-filled when !valid)
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;"
                 :: "r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src), "r"(valid ? 8 : 0) : "memory");
}

// x = hi + lo with hi = bfloat16(x) and lo = bfloat16(x - hi), two values per 32-bit word (first value low)
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const __nv_bfloat162 l = __floats2bfloat162_rn(a - __low2float(h), b - __high2float(h));
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

// byte offset of element (row, k) of a K-major operand without swizzle: core matrices of 8 rows x 8 elements
__device__ __forceinline__ uint32_t core_off(int row, int kchunk, int nkc)
{
    return (uint32_t)(((row >> 3) * nkc + kchunk) * 128 + (row & 7) * 16);
}

// 16 accumulator lanes x 8 columns from (lane, column) addr: thread l gets lane l / 4 at columns 2 (l % 4) and
// 2 (l % 4) + 1 (v[0], v[1]) and lane l / 4 + 8 at the same columns (v[2], v[3]); without waiting
__device__ __forceinline__ void tmem_ld16x256(uint32_t addr, float *v)
{
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr));
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}

struct GemmArgs {
    const float2 *__restrict__ x;     // [Np, P, K]
    const float2 *__restrict__ ph;    // [Np, C, P] (c0, sl)
    const float *__restrict__ tk;     // [Lk]
    const float *__restrict__ wp;     // [P] or null
    const float *__restrict__ wk;     // [K] or null
    int *bad;                         // first non-finite pulse (level 0) or null
    const int *amax_in;               // largest |component| of x (float bits)
    __half2 *y;                       // [Np, C, P, Kop]
    int *err;
    int Np, C, P, K, Ko, Kop, Dk, Lk, plk, Lkp, Nt, ntile, W, pseg, nseg, SB;
    int rp;                           // 2: A' rows 64..127 repeat rows 0..63 (more than 32 taps, at most 32 children)
    float kc;
    unsigned test_wait_ns;            // tests only: the MMA issuer's wait on a barrier nothing completes (0: none)
};

// The plane length in elements of a window of W samples held in PC shifted copies: a multiple of 2 PC, with slack.
__host__ __device__ constexpr int plane_len(int W, int PC) { return PC == 4 ? (W + 11) & ~3 : (W + 9) & ~1; }

// The power of two that brings values up to 4 amax (the taps' absolute sum is below 4 for the decimators of any
// plan) below 2^13: the float16 intermediate then stays in range and keeps 11 significant bits.
__device__ __forceinline__ float y_scale(const int *amax)
{
    const float m = amax ? __int_as_float(*amax) : 0.f;
    if (!(m > 0.f) || !isfinite(m)) return 1.f;
    int ex;
    frexpf(4.f * m, &ex);
    ex = ex < -100 ? -100 : (ex > 100 ? 100 : ex);
    return ldexpf(1.f, 13 - ex);
}

template <int NKC, int PC, int CW>
__global__ void __launch_bounds__(NTHR, 1) level_tc_gemm(const GemmArgs a)
{
    // CW consumer warps (8; 4 where the consumers idle and the Hankel copies bound the stage; 12 where the
    // accumulator read-out does), the other warps' roles after them: 4 A', 4 planes, 16 - CW Hankel rows, the MMA
    // issuer last (warp 24)
    constexpr int NCW_ = CW, NHW_ = NBW + NCW - CW - NLW, NHT_ = NHW_ * 32;
    static_assert(NCW_ + NAW + NLW + NHW_ == MMAW, "warp roles");
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int nkc = NKC;                                 // core matrices along K (Lkp = 8 NKC)
    const uint32_t apart = 128u * a.Lkp * 2u;                // one part (hi or lo) of A'
    const uint32_t bpart = 2u * a.Nt * a.Lkp * 2u;           // one part of B'
    unsigned char *sA = smem;                                // [2 pulses][hi, lo]
    unsigned char *sB = sA + 2 * 2 * apart;                  // [SB stages][hi, lo]
    const int Wp = plane_len(a.W, PC);                       // plane length in elements
    // planes: [xr hi, xr lo, xi hi, xi lo][copy c < PC][Wp / 2] words; copy c's word w holds samples 2w + c and
    // 2w + c + 1. With PC = 2 any 8 consecutive samples o .. o + 7 are the 4 aligned words (o - c) / 2 .. + 3 of copy
    // c = o mod 2; with PC = 4 they are the two 8-byte-aligned word pairs there of copy c = o mod 4 (copies 2 and 3
    // are copies 0 and 1 a word on): half the shared loads, twice the plane stores and space
    uint32_t *pl = reinterpret_cast<uint32_t *>(sB + (size_t)a.SB * 2 * bpart);   // two stages' planes
    float *s_tk = reinterpret_cast<float *>(pl + 2 * 4 * PC * (Wp / 2));           // [Lkp]
    float2 *s_x = reinterpret_cast<float2 *>(s_tk + a.Lkp);                        // [XS][Wp] staged windows
    uint64_t *bars = reinterpret_cast<uint64_t *>(s_x + (size_t)XS * Wp);
    uint64_t *afull = bars, *aempty = bars + 2, *bfull = bars + 4, *bempty = bfull + a.SB, *dfull = bempty + a.SB,
             *dempty = dfull + 2, *pfull = dempty + 2, *pempty = pfull + 2, *drain = pempty + 2;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ float s_scale;
    __shared__ uint64_t s_never;                             // a barrier nothing arrives on (the tests' stuck wait)
    __shared__ float2 s_ph[2][64];                           // the children's (c0, sl) of a pulse and the next

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int n = blockIdx.x / a.nseg, seg = blockIdx.x % a.nseg;
    const int p0 = seg * a.pseg, p1 = min(a.P, p0 + a.pseg);
    const int npl = p1 - p0;                                  // pulses of this block
    const int nst = npl * a.ntile;                            // stages (pulse, tile)
    const int ncol = 2 * a.Nt;                                // accumulator columns per stage

    if (t == 0) {
        s_abort = 0;
        s_scale = y_scale(a.amax_in);
        for (int i = 0; i < 2; ++i) {
            mbar_init(&afull[i], NAW);
            mbar_init(&aempty[i], 1);
            mbar_init(&dfull[i], 1);
            mbar_init(&dempty[i], NCW_);
        }
        for (int i = 0; i < a.SB; ++i) {
            mbar_init(&bfull[i], NHW_);
            mbar_init(&bempty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&pfull[i], NLT);
            mbar_init(&pempty[i], NHT_);
        }
        mbar_init(&s_never, 1);
        mbar_init(drain, 1);                             // the issuer's commit at the end
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = t; i < a.Lkp; i += NTHR) s_tk[i] = i < a.Lk ? (a.tk ? a.tk[i] : 1.f) : 0.f;   // Dk = 1: one tap 1
    // A' rows of no child stay zero: clear both pulses' buffers once
    for (int i = t; i < (int)(4 * apart / 16); i += NTHR) reinterpret_cast<uint4 *>(sA)[i] = make_uint4(0, 0, 0, 0);
    if (warp == MMAW) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" :: "r"(smem_u32(&s_tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const float scale = s_scale;

    if (warp >= NCW_ && warp < NCW_ + NAW) {
        // ------------------------------------------------------------------ A' producers
        // the modulated taps of each pulse into A' buffer pulse & 1, a pulse ahead of the B' producers (the
        // buffer is free once the MMAs of the pulse two back have completed); no named barrier
        const int at = t - NCW_ * 32;
        const float2 *__restrict__ phn = a.ph + (size_t)n * a.C * a.P;
        // the children's phases of each pulse are copied into s_ph a pulse ahead (cp.async, thread c: child c), so
        // that no item waits on a global load; after a failed wait a thread keeps stepping through the pulses (and
        // the named barrier, which all A' threads must reach) without waiting or working
        if (at < a.C && npl > 0) cp_async8(&s_ph[0][at], &phn[(size_t)at * a.P + p0], true);
        asm volatile("cp.async.commit_group;" ::: "memory");
        bool ok = true;
        for (int pl_i = 0; pl_i < npl; ++pl_i) {
            const int ab = pl_i & 1, p = p0 + pl_i;
            asm volatile("cp.async.wait_all;" ::: "memory");
            // every thread's phases of pulse p are in, and its reads of the other buffer (pulse p - 1) are done
            asm volatile("bar.sync 2, %0;" :: "n"(NAT) : "memory");
            if (at < a.C && pl_i + 1 < npl) cp_async8(&s_ph[(pl_i + 1) & 1][at], &phn[(size_t)at * a.P + p + 1], true);
            asm volatile("cp.async.commit_group;" ::: "memory");
            if (ok) ok = mbar_wait(&aempty[ab], (uint32_t)(((pl_i >> 1) & 1) ^ 1), 1000, &s_abort, a.err);
            if (!ok) continue;
            unsigned char *Ab = sA + ab * 2 * apart;
            const float2 *sph = s_ph[pl_i & 1];
            for (int item = at; item < a.C * nkc; item += NAT) {
                const int u = item / a.C, c = item - u * a.C;   // consecutive threads: consecutive children
                const float sl = sph[c].y;
                // exp(2 pi i sl r) for r = 8u .. 8u + 7: two independent recurrences (even and odd r)
                const float2 st = cis_cycles(sl), st2 = cmul(st, st);
                float2 ze = cis_cycles(sl * (float)(8 * u)), zo = cmul(ze, st);
                float mr[8], mi[8];
#pragma unroll
                for (int e = 0; e < 8; e += 2) {
                    const float h0 = s_tk[8 * u + e], h1 = s_tk[8 * u + e + 1];
                    mr[e] = h0 * ze.x;
                    mi[e] = h0 * ze.y;
                    mr[e + 1] = h1 * zo.x;
                    mi[e + 1] = h1 * zo.y;
                    ze = cmul(ze, st2);
                    zo = cmul(zo, st2);
                }
                uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    split2(mr[2 * e], mr[2 * e + 1], rh[e], rl[e]);
                    split2(mi[2 * e], mi[2 * e + 1], ih[e], il[e]);
                }
                // the rows of child c's Mr and Mi: with up to 32 taps, in each group of 16 rows the Mr rows of 8
                // children and then their Mi rows (the consumers' 16-row read-out); else rows 2 c and 2 c + 1
                const int row = NKC <= 4 ? 16 * (c >> 3) + (c & 7) : 2 * c, row2 = NKC <= 4 ? row + 8 : row + 1;
                const uint32_t o0 = core_off(row, u, nkc), o1 = core_off(row2, u, nkc);
                *reinterpret_cast<uint4 *>(Ab + o0) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
                *reinterpret_cast<uint4 *>(Ab + apart + o0) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
                *reinterpret_cast<uint4 *>(Ab + o1) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
                *reinterpret_cast<uint4 *>(Ab + apart + o1) = make_uint4(il[0], il[1], il[2], il[3]);
                if (NKC > 4 && a.rp == 2) {
                    // at most 32 children: rows 64 .. 127 repeat rows 0 .. 63, so that all four lane quarters of the
                    // accumulator hold children and the consumers split the columns four ways
                    const uint32_t d0 = core_off(row + 64, u, nkc), d1 = core_off(row2 + 64, u, nkc);
                    *reinterpret_cast<uint4 *>(Ab + d0) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
                    *reinterpret_cast<uint4 *>(Ab + apart + d0) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
                    *reinterpret_cast<uint4 *>(Ab + d1) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
                    *reinterpret_cast<uint4 *>(Ab + apart + d1) = make_uint4(il[0], il[1], il[2], il[3]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&afull[ab]);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp >= NCW_ + NAW && warp < NCW_ + NAW + NLW) {
        // ------------------------------------------------------------------ B' producers: planes
        const int pt = t - (NCW_ + NAW) * 32;
        const float2 *__restrict__ xn = a.x + (size_t)n * a.P * a.K;
        const int npair = (a.W + 1) / 2;                      // window samples in pairs (2i, 2i + 1)
        // the window of stage (pulse p, tile tt): samples k = kb + i, kb = Dk Nt tt - plk, i < W, copied XS - 1
        // stages ahead into ring slot (stage % XS) (zero outside [0, K)); one cp.async group per stage
        auto stage_x = [&](int st) {
            if (st < nst) {
                const int q = st / a.ntile, tt = st - q * a.ntile, p = p0 + q;
                const int kb = a.Dk * a.Nt * tt - a.plk;
                float2 *dst = s_x + (size_t)(st % XS) * Wp;
                for (int i = pt; i < a.W; i += NLT) {
                    const int k = kb + i;
                    const bool v = k >= 0 && k < a.K;
                    const float2 *src = v ? xn + (size_t)p * a.K + k : xn;
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;"
                                 :: "r"(smem_u32(dst + i)), "l"(src), "r"(v ? 8 : 0) : "memory");
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
#pragma unroll
        for (int d = 0; d < XS - 1; ++d) stage_x(d);
        // after a failed wait a warp keeps stepping through the stages (and the named barrier, which every planes
        // warp must reach) without waiting or working
        bool ok = true;
        for (int s = 0; s < nst; ++s) {
            const int pl_i = s / a.ntile, tt = s - pl_i * a.ntile, p = p0 + pl_i;
            asm volatile("cp.async.wait_group %0;" :: "n"(XS - 2) : "memory");   // this thread's copies of stage s
            // every planes thread's copies of stage s are in, and its reads of stage s - 1's window done: that
            // ring slot takes the window XS - 1 stages ahead
            asm volatile("bar.sync 1, %0;" :: "n"(NLT) : "memory");
            stage_x(s + XS - 1);
            if (ok) ok = mbar_wait(&pempty[s & 1], (uint32_t)(((s >> 1) & 1) ^ 1), 1000, &s_abort, a.err);
            // the window's planes: xr hi, xr lo, xi hi, xi lo as bfloat16 pairs (copy 0's word i = samples 2i,
            // 2i + 1), into plane buffer s & 1
            if (ok) {
                uint32_t *plb = pl + (s & 1) * 4 * PC * (Wp / 2);
                const float2 *xs = s_x + (size_t)(s % XS) * Wp;
                const int kb = a.Dk * a.Nt * tt - a.plk;
                const float wpp = a.wp ? a.wp[p] : 1.f;
                for (int i = pt; i < npair; i += NLT) {
                    float2 v[3];                              // samples 2i, 2i + 1, 2i + 2 (windowed)
#pragma unroll
                    for (int h = 0; h < 3; ++h) {
                        const int e = 2 * i + h, k = kb + e;
                        v[h] = e < a.W ? xs[e] : make_float2(0.f, 0.f);
                        if (a.wp && k >= 0 && k < a.K && e < a.W) {
                            const float w = wpp * a.wk[k];
                            v[h].x *= w;
                            v[h].y *= w;
                        }
                        if (h < 2 && a.bad && !(isfinite(v[h].x) && isfinite(v[h].y))) atomicMin(a.bad, p);
                    }
                    uint32_t rh, rl, ih, il, orh, orl, oih, oil;
                    split2(v[0].x, v[1].x, rh, rl);
                    split2(v[0].y, v[1].y, ih, il);
                    split2(v[1].x, v[2].x, orh, orl);
                    split2(v[1].y, v[2].y, oih, oil);
                    // copies 0, 1 at word i; copies 2, 3 (the same words) at word i - 1
                    const int hw = Wp / 2;
                    const uint32_t w4[4][2] = {{rh, orh}, {rl, orl}, {ih, oih}, {il, oil}};
#pragma unroll
                    for (int pq = 0; pq < 4; ++pq) {
                        uint32_t *q = plb + PC * pq * hw + i;
                        q[0] = w4[pq][0];
                        q[hw] = w4[pq][1];
                        if (PC == 4 && i > 0) {
                            q[2 * hw - 1] = w4[pq][0];
                            q[3 * hw - 1] = w4[pq][1];
                        }
                    }
                }
                mbar_arrive(&pfull[s & 1]);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp >= NCW_ + NAW + NLW && warp < MMAW) {
        // ------------------------------------------------------------------ B' producers: Hankel rows
        int sb = 0;
        uint32_t sbpar = 0;
        for (int s = 0; s < nst; ++s) {
            if (!mbar_wait(&pfull[s & 1], (uint32_t)((s >> 1) & 1), 1000, &s_abort, a.err)) break;
            if (!mbar_wait(&bempty[sb], sbpar ^ 1u, 1000, &s_abort, a.err)) break;
            // Hankel rows: row j < Nt: xr window from Dk j; row Nt + j: xi; 8 elements (16 bytes) per chunk.
            // A warp takes 8 rows (lane % 8) x 4 K chunks (lane / 8) at a time: the 8 rows' 16-byte stores fill one
            // 128-byte core matrix (no bank conflicts)
            unsigned char *Bb = sB + sb * 2 * bpart;
            const uint32_t *plb = pl + (s & 1) * 4 * PC * (Wp / 2);
            {
                // lane (r8 = lane % 8, uq = lane / 8) keeps its row within a block of 8 and its K chunk within a
                // group of 4; warp pw takes the row blocks pw, pw + NHW_, ... of each (part, re/im, chunk group).
                // Along a warp's row blocks the window offset, the plane copy and the store move by constants.
                constexpr int UB = (NKC + 3) / 4;
                const int r8 = lane & 7, uq = lane >> 3, pw = warp - NCW_ - NAW - NLW;
                const int nrb = a.Nt / 8;
                const int nmine = nrb > pw ? (nrb - 1 - pw) / NHW_ + 1 : 0;
                const int ostep = 8 * NHW_ * a.Dk, wstep = ostep >> 1;               // ostep: a multiple of 8
                const uint32_t bstep = (uint32_t)(NHW_ * nkc * 128);
#pragma unroll
                for (int ub = 0; ub < UB; ++ub) {
                    const int u = ub * 4 + uq;
                    if (u >= NKC) continue;
                    const int o0 = a.Dk * (8 * pw + r8) + 8 * u;                    // first element, first block
                    const int cp = o0 & (PC - 1);                                   // the same in every block
#pragma unroll
                    for (int pi = 0; pi < 4; ++pi) {                              // (part, re/im)
                        const int part = pi & 1, im = pi >> 1;
                        const uint32_t *src = plb + (PC * (2 * im + part) + cp) * (Wp / 2) + ((o0 - cp) >> 1);
                        unsigned char *dst = Bb + part * bpart + core_off(im * a.Nt + 8 * pw + r8, u, nkc);
                        int m = 0;
                        for (; m + 2 <= nmine; m += 2) {
                            const uint32_t *s0 = src + m * wstep, *s1 = s0 + wstep;
                            const uint4 v0 = ld_run<PC>(s0), v1 = ld_run<PC>(s1);
                            *reinterpret_cast<uint4 *>(dst + m * bstep) = v0;
                            *reinterpret_cast<uint4 *>(dst + (m + 1) * bstep) = v1;
                        }
                        if (m < nmine) {
                            const uint32_t *s0 = src + m * wstep;
                            *reinterpret_cast<uint4 *>(dst + m * bstep) = ld_run<PC>(s0);
                        }
                    }
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            mbar_arrive(&pempty[s & 1]);                      // this thread's reads of the planes are done
            if (lane == 0) mbar_arrive(&bfull[sb]);
            if (++sb == a.SB) { sb = 0; sbpar ^= 1u; }
        }
    } else if (warp == MMAW) {
        // ------------------------------------------------------------------ MMA issue
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(ncol >> 3) << 17) | ((128u >> 4) << 24);
            const uint32_t sbo = (uint32_t)nkc * 128;
            const uint32_t sA0 = smem_u32(sA), sB0 = smem_u32(sB);
            int sb = 0;
            uint32_t sbpar = 0;
            // tests of the failure report: a wait that runs out before any MMA, as a stuck pipeline's would
            const bool stuck = a.test_wait_ns && !mbar_wait(&s_never, 0, 0, &s_abort, a.err, a.test_wait_ns);
            for (int s = stuck ? nst : 0; s < nst; ++s) {
                const int pl_i = s / a.ntile, tt = s - pl_i * a.ntile;
                const int ab = pl_i & 1, db = s & 1;
                if (tt == 0 && !mbar_wait(&afull[ab], (uint32_t)((pl_i >> 1) & 1), 0, &s_abort, a.err)) break;
                if (!mbar_wait(&bfull[sb], sbpar, 0, &s_abort, a.err)) break;
                if (!mbar_wait(&dempty[db], (uint32_t)(((s >> 1) & 1) ^ 1), 0, &s_abort, a.err)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t dt = tmem + (uint32_t)(db * 256);
                const uint32_t ah = sA0 + (uint32_t)ab * 2 * apart, al = ah + apart;
                const uint32_t bh = sB0 + (uint32_t)sb * 2 * bpart, bl = bh + bpart;
                for (int ks = 0; ks < a.Lkp / 16; ++ks) {
                    const uint32_t ko = 256u * ks;
                    mma_bf16(dt, smem_desc(ah + ko, 128, sbo), smem_desc(bh + ko, 128, sbo), idesc, ks > 0 ? 1u : 0u);
                    mma_bf16(dt, smem_desc(ah + ko, 128, sbo), smem_desc(bl + ko, 128, sbo), idesc, 1u);
                    mma_bf16(dt, smem_desc(al + ko, 128, sbo), smem_desc(bh + ko, 128, sbo), idesc, 1u);
                }
                mma_commit(&bempty[sb]);
                mma_commit(&dfull[db]);
                if (tt == a.ntile - 1) mma_commit(&aempty[ab]);
                if (++sb == a.SB) { sb = 0; sbpar ^= 1u; }
            }
        }
        __syncwarp();
    } else {
        if constexpr (NKC <= 4) {
            // ------------------------------------------------------------------ consumers (warps 0..7), up to 32 taps
            // Warp w reads TMEM lane quarter q = w % 4 (A' rows 32 q .. 32 q + 31: children 16 q .. 16 q + 15) and
            // column half g = w / 4 of the tile. A 16x256b load of row group h (rows 32 q + 16 h ..) gives thread l the
            // Mr and Mi rows of child cc + 8 h (cc = 16 q + l / 4) at columns jl, jl + 1 (jl = 2 (l % 4)) of an 8-column
            // chunk: each thread forms re/im of its two children at two columns with no exchange between threads.
            const int q = warp & 3, g = warp >> 2;
            const int cc = 16 * q + (lane >> 2), jl = 2 * (lane & 3);
            const int cw = a.Nt / (NCW_ / 4);                      // columns of this warp per tile
            // child cc + 8 h's phases and intermediate rows (child 0's for a child past the last, whose results are
            // not stored)
            auto phc = [&](int h) {
                const int c = cc + 8 * h;
                return a.ph + ((size_t)n * a.C + (c < a.C ? c : 0)) * a.P;
            };
            float2 q0[2], qn[2];                                  // the children's (c0, sl): this pulse, the next
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                q0[h] = make_float2(0.f, 0.f);
                qn[h] = (cc + 8 * h < a.C && npl > 0) ? __ldg(phc(h) + p0) : make_float2(0.f, 0.f);
            }
            for (int s = 0; s < nst; ++s) {
                const int pl_i = s / a.ntile, tt = s - pl_i * a.ntile, p = p0 + pl_i;
                const int db = s & 1;
                if (tt == 0) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        q0[h] = qn[h];
                        if (cc + 8 * h < a.C && pl_i + 1 < npl) qn[h] = __ldg(phc(h) + p + 1);
                    }
                }
                // warp-uniform: the accumulator loads below are warp-collective
                if (!__all_sync(0xffffffffu, mbar_wait(&dfull[db], (uint32_t)((s >> 1) & 1), 200, &s_abort, a.err))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(db * 256);
                // per child: the ramp at this thread's first column of the first chunk, its step of one column and of
                // 8 columns
                float2 wv[2], st1[2], st8[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    st1[h] = cis_cycles(q0[h].y * (float)a.Dk);
                    st8[h] = cis_cycles(q0[h].y * (float)(8 * a.Dk));
                    float2 w0 = cis_cycles(fmaf(q0[h].y, (float)(a.Dk * (tt * a.Nt + g * cw + jl) - a.plk) - a.kc, q0[h].x));
                    w0.x *= scale;
                    w0.y *= scale;
                    wv[h] = w0;
                }
                // units (chunk of 8 columns, row group h) in order, the next unit's accumulator loads in flight while
                // one is processed; a unit's registers: (Mr, Mr, Mi, Mi) x (column jl, jl + 1) of the Xr and the Xi
                // columns
                float ua[8], ub[8];
                auto load = [&](int k8, int h, float *v) {
                    const uint32_t bh = base + ((uint32_t)(16 * h) << 16) + (uint32_t)(g * cw + k8);
                    tmem_ld16x256(bh, v);
                    tmem_ld16x256(bh + (uint32_t)a.Nt, v + 4);
                };
                auto unit = [&](int k8, int h, const float *v) {
                    // re = Mr Xr - Mi Xi, im = Mr Xi + Mi Xr at the two columns; times the ramp; the ramp 8 columns on
                    const float2 w0 = wv[h], w1 = cmul(w0, st1[h]);
                    const float2 o0 = cmul(w0, make_float2(v[0] - v[6], v[4] + v[2]));
                    const float2 o1 = cmul(w1, make_float2(v[1] - v[7], v[5] + v[3]));
                    const int c = cc + 8 * h, j = tt * a.Nt + g * cw + k8 + jl;
                    if (c < a.C && j < a.Ko) {
                        const __half2 h0 = __floats2half2_rn(o0.x, o0.y), h1 = __floats2half2_rn(o1.x, o1.y);
                        *reinterpret_cast<uint2 *>(a.y + (((size_t)n * a.C + c) * a.P + p) * a.Kop + j) =
                            make_uint2(*reinterpret_cast<const uint32_t *>(&h0), *reinterpret_cast<const uint32_t *>(&h1));
                    }
                    wv[h] = cmul(w0, st8[h]);
                };
                load(0, 0, ua);
                tmem_wait_ld();
                for (int k8 = 0; k8 < cw; k8 += 8) {
                    load(k8, 1, ub);
                    unit(k8, 0, ua);
                    tmem_wait_ld();
                    if (k8 + 8 == cw) {
                        // the accumulator's last unit is in registers: release it to the MMA issuer
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&dempty[db]);
                    } else {
                        load(k8 + 8, 0, ua);
                    }
                    unit(k8, 1, ub);
                    tmem_wait_ld();
                }
            }
        } else {
            // ------------------------------------------------------------------ consumers (warps 0..7), more taps
            // with at most 32 children lane quarters 2, 3 repeat quarters 0, 1 (A' rows 64 .. 127), and warp w takes
            // the column quarter w / 4 + 2 (w % 4 / 2) of the tile instead of the column half w / 4
            const int rp = a.rp;
            const int q = warp & 3, g = warp >> 2;
            const int c = 16 * (rp == 2 ? (q & 1) : q) + (lane >> 1);   // this lane's child (rows 2c: Mr, 2c + 1: Mi)
            const bool odd = lane & 1;
            const bool live = c < a.C;
            const int cw = a.Nt / (NCW_ / 4) / rp;                 // columns of this warp per tile (a multiple of 8)
            const int cofs = (rp == 2 ? g + (NCW_ / 4) * (q >> 1) : g) * cw;   // this warp's first column in the tile
            const float2 *__restrict__ phc = a.ph + ((size_t)n * a.C + (live ? c : 0)) * a.P;
            __half2 *__restrict__ yc = a.y + ((size_t)n * a.C + (live ? c : 0)) * a.P * a.Kop;
            // the child's phase (c0, sl) of the current pulse, and of the next one loaded a pulse ahead
            float2 q0 = make_float2(0.f, 0.f), qn = (live && npl > 0) ? __ldg(&phc[p0]) : make_float2(0.f, 0.f);
            for (int s = 0; s < nst; ++s) {
                const int pl_i = s / a.ntile, tt = s - pl_i * a.ntile, p = p0 + pl_i;
                const int db = s & 1;
                if (tt == 0) {
                    q0 = qn;
                    if (live && pl_i + 1 < npl) qn = __ldg(&phc[p + 1]);
                }
                // warp-uniform: the accumulator loads below are warp-collective
                if (!__all_sync(0xffffffffu, mbar_wait(&dfull[db], (uint32_t)((s >> 1) & 1), 200, &s_abort, a.err))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(db * 256);
                const float2 st = cis_cycles(q0.y * (float)a.Dk), st8 = cis_cycles(q0.y * (float)(8 * a.Dk));
                // this lane's ramp at its first column of the chunk: seeded at the first chunk, then 8 columns on
                float2 wc = cis_cycles(fmaf(q0.y, (float)(a.Dk * (tt * a.Nt + cofs + (odd ? 4 : 0)) - a.plk) - a.kc, q0.x));
                wc.x *= scale;
                wc.y *= scale;
                // chunks of 8 columns; the next chunk's accumulator loads are in flight while one is processed
                float vr[8], vi[8], nr[8], ni[8];
                tmem_ld8(base + (uint32_t)cofs, vr);
                tmem_ld8(base + (uint32_t)(a.Nt + cofs), vi);
                tmem_wait_ld();
                // the accumulator is released as soon as its last chunk is in registers
                auto release = [&]() {
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&dempty[db]);
                };
                if (cw == 8) release();
                for (int k8 = 0; k8 < cw; k8 += 8) {
                    const int cb = cofs + k8;                     // first column of the chunk within the tile
                    const bool more = k8 + 8 < cw;
                    if (more) {
                        tmem_ld8(base + (uint32_t)(cb + 8), nr);
                        tmem_ld8(base + (uint32_t)(a.Nt + cb + 8), ni);
                    }
                    // even lane (Mr row) keeps columns 0..3 of the chunk, odd lane (Mi row) columns 4..7
                    float mr_r[4], mr_i[4], mi_r[4], mi_i[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const float sr = odd ? vr[i] : vr[4 + i], si = odd ? vi[i] : vi[4 + i];
                        const float rr = __shfl_xor_sync(0xffffffffu, sr, 1), ri = __shfl_xor_sync(0xffffffffu, si, 1);
                        const float orr = odd ? vr[4 + i] : vr[i], ori = odd ? vi[4 + i] : vi[i];
                        mr_r[i] = odd ? rr : orr;
                        mr_i[i] = odd ? ri : ori;
                        mi_r[i] = odd ? orr : rr;
                        mi_i[i] = odd ? ori : ri;
                    }
                    const int j0 = tt * a.Nt + cb + (odd ? 4 : 0);
                    float2 w = wc;
                    wc = cmul(wc, st8);
                    if (live && j0 < a.Ko) {
                        uint32_t outw[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const float re = mr_r[i] - mi_i[i], im = mr_i[i] + mi_r[i];
                            const float2 o = cmul(w, make_float2(re, im));
                            const __half2 hv = __floats2half2_rn(o.x, o.y);
                            outw[i] = *reinterpret_cast<const uint32_t *>(&hv);
                            w = cmul(w, st);
                        }
                        *reinterpret_cast<uint4 *>(yc + (size_t)p * a.Kop + j0) = make_uint4(outw[0], outw[1], outw[2], outw[3]);
                    }
                    tmem_wait_ld();
                    if (more && k8 + 16 >= cw) release();
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        vr[i] = nr[i];
                        vi[i] = ni[i];
                    }
                }
            }
        }
    }

    __syncthreads();
    if (warp == MMAW) {
        if (lane == 0) {
            // drain: a commit on a barrier of its own, initialized with the others, completes once every earlier MMA
            // of this thread has (a barrier initialized again here need not be visible to the tensor core's arrive)
            mma_commit(drain);
            const uint64_t t0 = global_ns();
            bool drained = false;
            while (!(drained = mbar_test(drain, 0, 0)) && global_ns() - t0 < WAIT_NS) {
            }
            if (!drained && a.err) atomicAdd(a.err, 1);              // an MMA still running: reported
        }
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" :: "r"(tmem));
    }
}

// --------------------------------------------------------------------------------------------------- pass 2
struct FirArgs {
    const __half2 *__restrict__ y;    // [rows, P, Kop]
    const float *__restrict__ tp;     // [Lp]
    float2 *__restrict__ out;         // [rows, Po, Ko]
    int *amax;
    const int *amax_in;
    int rows, P, Kop, Ko, Po, Dp, Lp, plp, SEG, nseg;
};

template <int AP>
__global__ void __launch_bounds__(128) level_fir(const FirArgs a)
{
    constexpr int APP = (AP + 3) & ~3;
    // [Dp][APP] pairs: s_tp[b APP + s] = (tp[Dp s + b], tp[Dp s + b]), a tap twice for the packed multiply-adds
    extern __shared__ __align__(16) float2 s_tp[];
    // thread -> (row, pair of columns j, j + 1), consecutive threads along a row's pairs and on into the next row;
    // blockIdx.y: the segment of output pulses
    const int t = threadIdx.x;
    for (int r = t; r < a.Dp * APP; r += 128) {
        const int b = r / APP, s = r - b * APP;
        const int tap = a.Dp * s + b;
        const float v = (s < AP && tap < a.Lp) ? (a.tp ? a.tp[tap] : 1.f) : 0.f;   // Dp = 1: one tap 1
        s_tp[r] = make_float2(v, v);
    }
    __syncthreads();
    const int npair = (a.Ko + 1) / 2;
    const long gid = (long)blockIdx.x * 128 + t;
    if (gid >= (long)a.rows * npair) return;
    const int row = (int)(gid / npair), j = 2 * (int)(gid - (long)row * npair);
    const int seg = blockIdx.y;
    const float inv = 1.f / y_scale(a.amax_in);
    const bool colok = true;
    const int i_s = seg * a.SEG, i_e = min(a.Po, i_s + a.SEG);
    const int g_end = i_e + AP - 1;
    const __half2 *__restrict__ yr = a.y + (size_t)row * a.P * a.Kop + j;
    float2 acc[2][AP];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int s = 0; s < AP; ++s) acc[h][s] = make_float2(0.f, 0.f);
    float vmax = 0.f;
    // input pulses p_start .. p_stop - 1 in chunks of U, the next chunk's loads in flight while one is filtered
    constexpr int U = 8;
    const int p_start = a.Dp * i_s - a.plp, p_stop = a.Dp * g_end - a.plp;
    auto ld = [&](int pp) -> uint2 {
        return (pp >= 0 && pp < a.P && colok) ? __ldg(reinterpret_cast<const uint2 *>(yr + (size_t)pp * a.Kop))
                                              : make_uint2(0u, 0u);
    };
    uint2 cur[U], nxt[U];
#pragma unroll
    for (int u = 0; u < U; ++u) cur[u] = ld(p_start + u);
    int b = 0, gi = i_s;
    for (int pc = p_start; pc < p_stop; pc += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) nxt[u] = ld(pc + U + u);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (pc + u >= p_stop) break;
            const float2 v0 = __half22float2(*reinterpret_cast<const __half2 *>(&cur[u].x));
            const float2 v1 = __half22float2(*reinterpret_cast<const __half2 *>(&cur[u].y));
            float2 tb[APP];
#pragma unroll
            for (int s2 = 0; s2 < APP; s2 += 2) {
                const float4 q4 = *reinterpret_cast<const float4 *>(&s_tp[b * APP + s2]);
                tb[s2] = make_float2(q4.x, q4.y);
                tb[s2 + 1] = make_float2(q4.z, q4.w);
            }
#pragma unroll
            for (int s = 0; s < AP; ++s) {
                acc[0][s] = ffma2(tb[s], v0, acc[0][s]);
                acc[1][s] = ffma2(tb[s], v1, acc[1][s]);
            }
            if (++b == a.Dp) {                                // group gi complete: output gi - (AP - 1) finished
                b = 0;
                const int i = gi - (AP - 1);
                if (i >= i_s && colok) {
                    float2 *o = a.out + ((size_t)row * a.Po + i) * a.Ko + j;
                    const float2 o0 = make_float2(acc[0][AP - 1].x * inv, acc[0][AP - 1].y * inv);
                    const float2 o1 = make_float2(acc[1][AP - 1].x * inv, acc[1][AP - 1].y * inv);
                    o[0] = o0;
                    vmax = fmaxf(vmax, fmaxf(fabsf(o0.x), fabsf(o0.y)));
                    if (j + 1 < a.Ko) {
                        o[1] = o1;
                        vmax = fmaxf(vmax, fmaxf(fabsf(o1.x), fabsf(o1.y)));
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
#pragma unroll
                    for (int s = AP - 1; s > 0; --s) acc[h][s] = acc[h][s - 1];
                    acc[h][0] = make_float2(0.f, 0.f);
                }
                ++gi;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) cur[u] = nxt[u];
    }
    if (a.amax) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if ((t & 31) == 0 && vmax > 0.f) atomicMax(a.amax, __float_as_int(vmax));
    }
}

template <int AP>
cudaError_t launch_fir(FirArgs f, cudaStream_t s)
{
    constexpr int APP = (AP + 3) & ~3;
    const long nb = ((long)f.rows * ((f.Ko + 1) / 2) + 127) / 128;
    int nseg = 1;
    while (nb * nseg < 148L * 16 && f.Po / (nseg * 2) >= 8 * AP) nseg *= 2;
    f.SEG = (f.Po + nseg - 1) / nseg;
    f.nseg = (f.Po + f.SEG - 1) / f.SEG;
    if (nb > 0x7fffffffL || f.nseg > 65535) return cudaErrorInvalidValue;
    level_fir<AP><<<dim3((unsigned)nb, (unsigned)f.nseg), 128, (size_t)f.Dp * APP * sizeof(float2), s>>>(f);
    return cudaGetLastError();
}

__global__ void amax_kernel(const float *__restrict__ v, size_t n, int *amax)
{
    float m = 0.f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 4; i += (size_t)gridDim.x * blockDim.x) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(v) + i);
        m = fmaxf(m, fmaxf(fmaxf(fabsf(q.x), fabsf(q.y)), fmaxf(fabsf(q.z), fabsf(q.w))));
    }
    for (size_t i = (n / 4) * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
    if (!isfinite(m)) m = 0.f;                                 // non-finite samples are reported by the level kernel
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(amax, __float_as_int(m));
}

}  // namespace

size_t level_tc_scratch_bytes(int Np, int C, int P, int Ko)
{
    const int Kop = (Ko + 3) & ~3;
    return (size_t)Np * C * P * Kop * sizeof(__half2);
}

// Dynamic shared memory of level_tc_gemm: both pulses' A' (hi, lo), sb stages of B' (hi, lo), the window planes, the
// taps, the staged windows and the barriers.
static size_t gemm_smem(int Lkp, int Dk, int nt, int sb, int pc)
{
    const size_t apart = (size_t)128 * Lkp * 2, bpart = (size_t)2 * nt * Lkp * 2;
    const int W = Dk * (nt - 1) + Lkp, Wp = plane_len(W, pc);
    // two stages' planes (4 planes x pc copies); barriers: afull[2], aempty[2], bfull[sb], bempty[sb], dfull[2],
    // dempty[2], pfull[2], pempty[2], drain
    return 4 * apart + (size_t)sb * 2 * bpart + (size_t)2 * 4 * pc * (Wp / 2) * 4 + (size_t)Lkp * 4 +
           (size_t)XS * Wp * 8 + (size_t)(13 + 2 * sb) * 8;
}

constexpr size_t GEMM_SMEM_MAX = 225 * 1024;                 // the opt-in limit less static shared memory and slack

bool level_tc_supported(int C, int Lk, int Dk)
{
    const int Lkp = ((Lk + 15) / 16) * 16;
    return C >= 1 && C <= 64 && Lkp <= 96 && Dk >= 1 && gemm_smem(Lkp, Dk, 32, 2, 2) <= GEMM_SMEM_MAX;
}

cudaError_t launch_amax(const float2 *x, size_t n, int *amax, cudaStream_t s)
{
    amax_kernel<<<148 * 4, 256, 0, s>>>(reinterpret_cast<const float *>(x), 2 * n, amax);
    return cudaGetLastError();
}

cudaError_t launch_level_tc_gemm(const LevelLaunch &L, const int *amax_in, void *scratch, int *err, cudaStream_t s,
                                 const char **why)
{
    *why = nullptr;
    const int Lk = L.Dk > 1 ? L.Lk : 1, plk = L.Dk > 1 ? L.plk : 0;
    if (!level_tc_supported(L.C, Lk, L.Dk)) { *why = "the tensor-core level takes C <= 64 children and Lk <= 96 taps"; return cudaErrorNotSupported; }
    GemmArgs a;
    a.x = L.x; a.ph = L.phase; a.tk = L.tk; a.wp = L.wp; a.wk = L.wk; a.bad = L.bad; a.amax_in = amax_in;
    a.y = static_cast<__half2 *>(scratch); a.err = err;
    a.Np = L.Np; a.C = L.C; a.P = L.P; a.K = L.K; a.Ko = L.Ko; a.Kop = (L.Ko + 3) & ~3; a.Dk = L.Dk; a.Lk = Lk;
    a.plk = plk; a.Lkp = ((Lk + 15) / 16) * 16; a.kc = (float)L.kc; a.test_wait_ns = L.test_wait_ns;
    int dev = 0, maxsmem = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t avail = std::min((size_t)maxsmem - 1024, GEMM_SMEM_MAX);
    // launch options (LevelLaunch::tc_*; 0 = the default): plane copies, row repeat, columns per tile, B stages
    const int pc = L.tc_pc == 4 ? 4 : 2;
    if (L.tc_pc != 0 && L.tc_pc != 2 && L.tc_pc != 4) { *why = "plane copies: 2 or 4"; return cudaErrorNotSupported; }
    a.rp = (a.Lkp > 32 && L.C <= 32 && L.tc_rp != 1) ? 2 : 1;
    if (L.tc_cw != 0 && L.tc_cw != 4 && L.tc_cw != 8 && L.tc_cw != 12) { *why = "consumer warps: 4, 8 or 12"; return cudaErrorNotSupported; }
    const int cw = L.tc_cw ? L.tc_cw : 8;
    // the consumers split a tile's columns cw / 4 ways (cw / 2 with repeated rows) in 8-column chunks; the MMA's N
    // (2 Nt) a multiple of 16
    const int unit = std::max(16, 8 * (cw / 4) * a.rp);
    auto need = [&](int nt, int sb) { return gemm_smem(a.Lkp, a.Dk, nt, sb, pc); };
    int best = 0;
    if (L.tc_nt) {
        if (L.tc_nt % unit || L.tc_nt > 128 || need(L.tc_nt, 2) > avail) {
            *why = "columns per tile: a multiple of 16 and of 8 x consumer warps / 4 (x 2 with repeated rows), up to 128, whose operands fit shared memory";
            return cudaErrorNotSupported;
        }
        best = L.tc_nt;
    } else {
        // a multiple of the unit (of 32 where the unit divides 32) up to 128 whose operands fit shared memory with two
        // B stages, the one that wastes the fewest columns on the last tile counting each tile as 32 columns of fixed
        // cost
        const int step = 32 % unit == 0 ? 32 : unit;
        int bestw = 1 << 30;
        for (int nt = (128 / step) * step; nt >= step; nt -= step) {
            if (need(nt, 2) > avail) continue;
            const int nti = (L.Ko + nt - 1) / nt, waste = nti * nt - L.Ko + nti * 32;
            if (waste < bestw) { bestw = waste; best = nt; }
        }
    }
    if (!best) { *why = "the tensor-core level's operands do not fit shared memory"; return cudaErrorNotSupported; }
    // every consumer warp's columns are whole 8-column chunks (the accumulator loads' column alignment)
    if (best % unit != 0 || (best / (cw / 4) / a.rp) % 8 != 0) {
        *why = "columns per tile do not split into the consumer warps' 8-column chunks";
        return cudaErrorNotSupported;
    }
    a.Nt = best;
    a.ntile = (L.Ko + a.Nt - 1) / a.Nt;
    a.W = a.Dk * (a.Nt - 1) + a.Lkp;
    // pulse segments: enough blocks for the device several times over
    int nseg = 1;
    while ((long)L.Np * nseg < 148L * 3 && L.P / (nseg * 2) >= 32) nseg *= 2;
    a.pseg = (L.P + nseg - 1) / nseg;
    a.nseg = (L.P + a.pseg - 1) / a.pseg;
    int SB = 4;
    if (L.tc_sb) {
        if (L.tc_sb < 2 || L.tc_sb > 4 || need(a.Nt, L.tc_sb) > avail) {
            *why = "B stages: 2 to 4 that fit shared memory";
            return cudaErrorNotSupported;
        }
        SB = L.tc_sb;
    }
    while (SB > 2 && need(a.Nt, SB) > avail) --SB;
    a.SB = SB;
    const size_t smem = need(a.Nt, SB);
    const long nb = (long)L.Np * a.nseg;
    if (nb > 0x7fffffffL) return cudaErrorInvalidValue;
    auto run = [&](auto kern) -> cudaError_t {
        cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r != cudaSuccess) return r;
        kern<<<(unsigned)nb, NTHR, smem, s>>>(a);
        return cudaGetLastError();
    };
    cudaError_t e;
#define FFBP_GEMM_RUN(N)                                                                                     \
    (cw == 4 ? (pc == 4 ? run(level_tc_gemm<N, 4, 4>) : run(level_tc_gemm<N, 2, 4>))                         \
     : cw == 12 ? (pc == 4 ? run(level_tc_gemm<N, 4, 12>) : run(level_tc_gemm<N, 2, 12>))                    \
                : (pc == 4 ? run(level_tc_gemm<N, 4, 8>) : run(level_tc_gemm<N, 2, 8>)))
    switch (a.Lkp / 8) {
        case 2: e = FFBP_GEMM_RUN(2); break;
        case 4: e = FFBP_GEMM_RUN(4); break;
        case 6: e = FFBP_GEMM_RUN(6); break;
        case 8: e = FFBP_GEMM_RUN(8); break;
        case 10: e = FFBP_GEMM_RUN(10); break;
        default: e = FFBP_GEMM_RUN(12); break;
    }
#undef FFBP_GEMM_RUN
    if (e != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t launch_level_fir_cc(const LevelLaunch &L, const int *amax_in, const void *scratch, cudaStream_t s,
                                const char **why)
{
    *why = nullptr;
    const int Lp = L.Dp > 1 ? L.Lp : 1, plp = L.Dp > 1 ? L.plp : 0;
    FirArgs f;
    f.y = static_cast<const __half2 *>(scratch); f.tp = L.tp; f.out = L.out; f.amax = L.amax; f.amax_in = amax_in;
    f.rows = L.Np * L.C; f.P = L.P; f.Kop = (L.Ko + 3) & ~3; f.Ko = L.Ko; f.Po = L.Po; f.Dp = L.Dp; f.Lp = Lp; f.plp = plp;
    const int AP = (Lp + L.Dp - 1) / L.Dp;
    switch (AP) {
        case 1: return launch_fir<1>(f, s);
        case 2: return launch_fir<2>(f, s);
        case 3: return launch_fir<3>(f, s);
        case 4: return launch_fir<4>(f, s);
        case 5: return launch_fir<5>(f, s);
        case 6: return launch_fir<6>(f, s);
        case 7: return launch_fir<7>(f, s);
        case 8: return launch_fir<8>(f, s);
        case 9: return launch_fir<9>(f, s);
        case 10: return launch_fir<10>(f, s);
        case 11: return launch_fir<11>(f, s);
        case 12: return launch_fir<12>(f, s);
        default: *why = "pulse FIR spans more than 12 output pulses"; return cudaErrorNotSupported;
    }
}

}  // namespace ffbp

namespace ffbp {

cudaError_t launch_level_tc(const LevelLaunch &L, const int *amax_in, void *scratch, int *err, cudaStream_t s,
                            const char **why)
{
    cudaError_t e = launch_level_tc_gemm(L, amax_in, scratch, err, s, why);
    if (e != cudaSuccess || *why) return e;
    return launch_level_tc_fir(L, amax_in, scratch, err, s, why);
}

cudaError_t launch_level_tc_fir(const LevelLaunch &L, const int *amax_in, const void *scratch, int *err,
                                cudaStream_t s, const char **why)
{
    // the pulse FIR on the tensor cores (a banded product per row, level_fir_tc.cu) or on the CUDA cores (level_fir);
    // by default the tensor cores where the output pulse axis fills several 128-row tiles (short axes leave most
    // of a tile's rows and the chunks' pulses empty, where the CUDA-core kernel is faster)
    const int Lp = L.Dp > 1 ? L.Lp : 1;
    const int AP = (Lp + L.Dp - 1) / L.Dp;
    const bool tc = L.tc_fir == 2 || (L.tc_fir == 0 && (L.Po >= 512 || AP > 12));
    if (L.tc_fir != 0 && L.tc_fir != 1 && L.tc_fir != 2) { *why = "pulse FIR kernel: 1 (CUDA cores) or 2 (tensor cores)"; return cudaErrorNotSupported; }
    return tc ? launch_level_fir_tc(L, amax_in, scratch, err, s, why) : launch_level_fir_cc(L, amax_in, scratch, s, why);
}

}  // namespace ffbp

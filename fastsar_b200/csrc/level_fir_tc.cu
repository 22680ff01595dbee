// The pulse FIR of a tensor-core level's second pass on the tcgen05 tensor cores (sm_100a): the reference's fir_p
// (fastsar/ffbp_cpu.cpp:262-293, fastsar/ffbp_cuda.py:200-256) on the float16 intermediate y [rows, P, Kop] that the
// first pass (level_tc_gemm) writes, as a banded product per row:
//     out[row, i, j] = sum_p H[i, p] y[row, p, j],   H[i, p] = hp[p - (Dp i - plp)]   (0 outside 0 .. Lp - 1).
// A tile is one row, MO = 128 output pulses (the accumulator's lanes) and NC complex columns (2 NC real accumulator
// columns, NC <= 128); the input pulses it needs, Dp (MO - 1) + Lp of them, are swept in chunks of KC = 64:
//   warp 4      loader: per chunk ceil(2 NC / 64) TMA loads (cp.async.bulk.tensor, 128-byte swizzle: 64 real columns
//               x 64 pulses of the tile's row each, 128 contiguous bytes per pulse) into a ring of 4 B operands, which
//               is the MN-major operand layout with the 128-byte swizzle; pulses before 0 or past the row's end and
//               columns past the intermediate's read as zeros (the copy's out-of-bounds fill), so no thread touches
//               the samples;
//   warps 6..9  per chunk the band of H as float16 hi + lo (A operand, K-major: 128 rows of output pulses, K = the
//               chunk's pulses) from shifted copies of the taps;
//   warp 5      one thread issues tcgen05.mma M = 128, N = 2 NC, K = 16, H hi and H lo times y, accumulated in float32
//               into one of two tensor-memory accumulators (a tile's chunks into the same one);
//   warps 0..3  epilogue: each reads its lane quarter of the accumulator (an output pulse per thread), undoes the
//               intermediate's power-of-two scale, writes complex64 and records the largest component.
// The MMAs do all the multiply-adds and the copy engine all the loads, so the pass runs near the bandwidth of its
// reads of the intermediate. Blocks are persistent over tiles; every wait on a barrier is bounded in time, and a wait
// that runs out sets the block's abort flag and raises *err.
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace ffbp {

namespace {

using namespace tc;

constexpr int R_NEPI = 4;                      // epilogue warps 0..3 (tensor-memory lane quarters)
constexpr int R_LDW = 4;                       // loader warp
constexpr int R_MMAW = 5;                      // MMA issuer warp
constexpr int R_TW0 = 6, R_NTW = 4;            // transposer warps 6..9
constexpr int R_NTHR = (R_TW0 + R_NTW) * 32;
constexpr int R_NTT = R_NTW * 32;
constexpr int KC = 64;                         // input pulses per chunk
constexpr int NSB = 4;                         // the ring of B operands (chunks of samples in flight)
constexpr int MO = 128;                        // output pulses per tile
constexpr uint64_t R_WAIT_NS = 2000000000ull;

struct FirTcArgs {
    const __half2 *__restrict__ y;    // [rows, P, Kop], scaled by y_scale(amax_in)
    const float *__restrict__ tp;     // [Lp] (null: Dp = 1, one tap 1)
    float2 *out;                      // [rows, Po, Ko]
    int *amax;                        // largest |component| of the output (float bits) or null
    const int *amax_in;
    int *err;
    int rows, P, Kop, Ko, Po, Dp, Lp, plp;
    int NC, ncb, nob;                 // complex columns per tile, column tiles, output-pulse tiles
    long ntiles;
    int NQ;                           // 16-byte words per shifted tap copy
};

// The power of two the first pass scaled the intermediate by (level_tc_gemm's y_scale).
__device__ __forceinline__ float fir_inv_scale(const int *amax)
{
    const float m = amax ? __int_as_float(*amax) : 0.f;
    if (!(m > 0.f) || !isfinite(m)) return 1.f;
    int ex;
    frexpf(4.f * m, &ex);
    ex = ex < -100 ? -100 : (ex > 100 ? 100 : ex);
    return ldexpf(1.f, ex - 13);
}

struct TileGeom {
    int row, i0, mo, j0;              // row; first output pulse and count; first column
    int cbase, pa, pb, c_lo, nch;     // K origin (pulse of H column 0), the row's pulses in reach, chunks
};

__device__ __forceinline__ TileGeom tile_geom(const FirTcArgs &a, long t)
{
    TileGeom g;
    const int cb = (int)(t % a.ncb);
    const long rest = t / a.ncb;
    const int ob = (int)(rest % a.nob);
    g.row = (int)(rest / a.nob);
    g.i0 = ob * MO;
    g.mo = min(MO, a.Po - g.i0);
    g.j0 = cb * a.NC;
    g.cbase = a.Dp * g.i0 - a.plp;
    g.pa = max(0, g.cbase);
    g.pb = min(a.P, a.Dp * (g.i0 + g.mo - 1) - a.plp + a.Lp);
    if (g.pa >= g.pb) {
        g.c_lo = 0;
        g.nch = 0;
    } else {
        g.c_lo = (g.pa - g.cbase) / KC;
        g.nch = (g.pb - g.cbase + KC - 1) / KC - g.c_lo;
    }
    return g;
}

// sm_100 shared-memory matrix descriptor with the 128-byte swizzle (layout type 2 at bits 61-63): start address,
// leading and stride byte offsets in 16-byte units, version 1 at bit 46; the start 1024-byte aligned
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return smem_desc(addr, lbo, sbo) | (2ull << 61);
}

// 32 consecutive columns of this thread's lane (not waited for)
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float *v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(addr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}


__global__ void __launch_bounds__(R_NTHR, 1) level_fir_tc_kernel(const FirTcArgs a, const __grid_constant__ CUtensorMap ymap)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const int N = 2 * a.NC;                                    // real accumulator columns (re, im of each column)
    const uint32_t a_part = (uint32_t)MO * KC * 2;             // one part (hi or lo) of the A operand
    const int NB = (N + 63) / 64;                              // 64-column blocks of a B operand
    const uint32_t b_bytes = (uint32_t)NB * KC * 128;          // one B operand: [NB][KC pulses][128 bytes], swizzled
    // B [NSB] | A [2 slots][hi, lo] | shifted taps [hi, lo][8 shifts][NQ] | barriers
    unsigned char *sB = smem;
    unsigned char *sA = sB + NSB * b_bytes;
    uint4 *tcp = reinterpret_cast<uint4 *>(sA + 2 * 2 * a_part);
    uint64_t *bars = reinterpret_cast<uint64_t *>(tcp + 2 * 8 * a.NQ);
    uint64_t *bfull = bars, *bempty = bars + NSB, *afull = bars + 2 * NSB, *aempty = afull + 2, *dfull = aempty + 2,
             *dempty = dfull + 2, *drain = dempty + 2;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    if (t == 0) {
        s_abort = 0;
        for (int i = 0; i < NSB; ++i) {
            mbar_init(&bfull[i], 1);
            mbar_init(&bempty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&afull[i], R_NTW);
            mbar_init(&aempty[i], 1);
            mbar_init(&dfull[i], 1);
            mbar_init(&dempty[i], R_NEPI);
        }
        mbar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // shifted copies of the taps as float16 hi and lo: copy s's word q holds taps 8 (q - 1) + s .. + 7 (zero outside
    // 0 .. Lp - 1), so that any 8 consecutive taps from t0 are one aligned 16-byte word: copy t0 & 7, word (t0 >> 3) + 1
    for (int w = t; w < 2 * 8 * a.NQ; w += R_NTHR) {
        const int part = w / (8 * a.NQ), sh = (w / a.NQ) % 8, q = w % a.NQ;
        __half h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int tap = 8 * (q - 1) + sh + e;
            const float v = (tap >= 0 && tap < a.Lp) ? (a.tp ? a.tp[tap] : 1.f) : 0.f;
            const __half hi = __float2half_rn(v);
            h[e] = part ? __float2half_rn(v - __half2float(hi)) : hi;
        }
        tcp[w] = *reinterpret_cast<const uint4 *>(h);
    }
    if (warp == R_MMAW) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" :: "r"(smem_u32(&s_tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (warp == R_LDW) {
        // ------------------------------------------------------------------ loader (one thread)
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<uint64_t>(&ymap)) : "memory");
            long g_it = 0;
            bool ok = true;
            for (long ti = blockIdx.x; ti < a.ntiles && ok; ti += gridDim.x) {
                const TileGeom g = tile_geom(a, ti);
                for (int c = 0; c < g.nch; ++c, ++g_it) {
                    const int slot = (int)(g_it % NSB);
                    const uint32_t ph = (uint32_t)((g_it / NSB) & 1);
                    if (!(ok = mbar_wait(&bempty[slot], ph ^ 1u, 200, &s_abort, a.err, R_WAIT_NS))) break;
                    const uint32_t bar = smem_u32(&bfull[slot]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(b_bytes) : "memory");
                    // box b: real columns 2 j0 + 64 b .. + 63 (16-byte aligned), pulses p0 .. p0 + 63 (negative or past
                    // P: zero fill), the tile's row
                    const int p0 = g.cbase + (g.c_lo + c) * KC;
                    for (int b = 0; b < NB; ++b)
                        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                                     "[%0], [%1, {%2, %3, %4}], [%5];"
                                     :: "r"(smem_u32(sB) + (uint32_t)slot * b_bytes + (uint32_t)b * (KC * 128)),
                                        "l"(reinterpret_cast<uint64_t>(&ymap)), "r"(2 * g.j0 + 64 * b), "r"(p0),
                                        "r"(g.row), "r"(bar) : "memory");
                }
            }
        }
        __syncwarp();
    } else if (warp >= R_TW0) {
        // ------------------------------------------------------------------ H producers (A operand)
        const int tt = t - R_TW0 * 32;
        long g_it = 0;
        bool ok = true;
        for (long ti = blockIdx.x; ti < a.ntiles && ok; ti += gridDim.x) {
            const TileGeom g = tile_geom(a, ti);
            for (int c = 0; c < g.nch; ++c, ++g_it) {
                const int aslot = (int)(g_it & 1);
                if (!(ok = mbar_wait(&aempty[aslot], (uint32_t)(((g_it >> 1) & 1) ^ 1), 200, &s_abort, a.err, R_WAIT_NS))) break;
                // row m (output pulse i0 + m), K column k (pulse p0 + k): tap (c_lo + c) KC + k - Dp m; 16-byte runs
                // of 8 columns, consecutive threads along a core matrix's rows
                unsigned char *asl = sA + (size_t)aslot * 2 * a_part;
                const int kofs = (g.c_lo + c) * KC;
                for (int it = tt; it < 2 * MO * 8; it += R_NTT) {
                    const int r8 = it & 7, u = (it >> 3) & 7, mb = (it >> 6) & 15, part = it >> 10;
                    const int t0 = kofs + 8 * u - a.Dp * (mb * 8 + r8);
                    uint4 hv = make_uint4(0u, 0u, 0u, 0u);
                    if (t0 < a.Lp && t0 > -8) hv = tcp[(part * 8 + (t0 & 7)) * a.NQ + (t0 >> 3) + 1];
                    *reinterpret_cast<uint4 *>(asl + part * a_part + (mb * 8 + u) * 128 + r8 * 16) = hv;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&afull[aslot]);
            }
        }
    } else if (warp == R_MMAW) {
        // ------------------------------------------------------------------ MMA issue
        if (lane == 0) {
            // f16 x f16 -> f32, A K-major, B MN-major (bit 16), N = 2 NC, M = 128
            const uint32_t idesc = (1u << 4) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(MO >> 4) << 24);
            // A (K-major, no swizzle): core matrices 128 bytes apart along K, 1024 along M. B (MN-major, 128-byte
            // swizzle): 8-pulse groups 1024 bytes apart along K, 64-column blocks KC x 128 bytes apart along N
            const uint32_t lbo = 128u, sbo = (uint32_t)(KC / 8) * 128u;
            const uint32_t blbo = (uint32_t)KC * 128u, bsbo = 1024u;
            long g_it = 0, t_it = 0;
            bool ok = true;
            for (long ti = blockIdx.x; ti < a.ntiles && ok; ti += gridDim.x, ++t_it) {
                const TileGeom g = tile_geom(a, ti);
                const int db = (int)(t_it & 1);
                if (!(ok = mbar_wait(&dempty[db], (uint32_t)(((t_it >> 1) & 1) ^ 1), 0, &s_abort, a.err, R_WAIT_NS))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(db * 256);
                for (int c = 0; c < g.nch; ++c, ++g_it) {
                    const int slot = (int)(g_it % NSB), aslot = (int)(g_it & 1);
                    if (!(ok = mbar_wait(&afull[aslot], (uint32_t)((g_it >> 1) & 1), 0, &s_abort, a.err, R_WAIT_NS))) break;
                    if (!(ok = mbar_wait(&bfull[slot], (uint32_t)((g_it / NSB) & 1), 0, &s_abort, a.err, R_WAIT_NS))) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ah = smem_u32(sA) + (uint32_t)aslot * 2u * a_part, al = ah + a_part;
                    const uint32_t bb = smem_u32(sB) + (uint32_t)slot * b_bytes;
#pragma unroll
                    for (int ks = 0; ks < KC / 16; ++ks) {
                        const uint32_t ko = 2u * 128u * ks;            // A: two core matrices along K per K = 16
                        const uint64_t bd = smem_desc_sw128(bb + 2048u * ks, blbo, bsbo);   // B: 16 pulse rows
                        mma_bf16(d, smem_desc(ah + ko, lbo, sbo), bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
                        mma_bf16(d, smem_desc(al + ko, lbo, sbo), bd, idesc, 1u);
                    }
                    mma_commit(&bempty[slot]);
                    mma_commit(&aempty[aslot]);
                }
                if (!ok) break;
                mma_commit(&dfull[db]);                       // a tile with no input pulses: nothing to wait for
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------------ epilogue (warps 0..3)
        const float inv = fir_inv_scale(a.amax_in);
        float vmax = 0.f;
        long t_it = 0;
        for (long ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x, ++t_it) {
            const TileGeom g = tile_geom(a, ti);
            const int db = (int)(t_it & 1);
            if (!__all_sync(0xffffffffu, mbar_wait(&dfull[db], (uint32_t)((t_it >> 1) & 1), 1000, &s_abort, a.err,
                                                    R_WAIT_NS)))
                break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m = 32 * warp + lane;
            const bool rowok = m < g.mo;
            const int ncs = min(a.NC, a.Ko - g.j0);            // columns stored
            float2 *o = a.out + ((size_t)g.row * a.Po + (g.i0 + (rowok ? m : 0))) * a.Ko + g.j0;
            const uint32_t base = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(db * 256);
            for (int cc = 0; cc < N; cc += 32) {
                float v[32];
                if (g.nch) {
                    tmem_ld32(base + (uint32_t)cc, v);
                    tmem_wait_ld();
                } else {
#pragma unroll
                    for (int e = 0; e < 32; ++e) v[e] = 0.f;
                }
                if (rowok) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const int j = cc / 2 + e;
                        if (j < ncs) {
                            const float2 w = make_float2(v[2 * e] * inv, v[2 * e + 1] * inv);
                            o[j] = w;
                            vmax = fmaxf(vmax, fmaxf(fabsf(w.x), fabsf(w.y)));
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&dempty[db]);
        }
        if (a.amax) {
#pragma unroll
            for (int s2 = 16; s2 > 0; s2 >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, s2));
            if (lane == 0 && vmax > 0.f) atomicMax(a.amax, __float_as_int(vmax));
        }
    }

    // teardown: every role is done (or aborted); the issuer drains its MMAs before the columns are freed
    __syncthreads();
    if (warp == R_MMAW && lane == 0) {
        mma_commit(drain);
        const uint64_t t0 = global_ns();
        bool drained = false;
        while (!(drained = mbar_test(drain, 0, 0)) && global_ns() - t0 < R_WAIT_NS) {
        }
        if (!drained && a.err) atomicAdd(a.err, 1);              // an MMA still running: reported
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == R_MMAW) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" :: "r"(tmem));
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (the library links the runtime only)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    }
    return fn;
}

}  // namespace

size_t level_fir_tc_smem(int Kop, int Lp)
{
    const int ncb = (Kop + 127) / 128, NC = (((Kop + ncb - 1) / ncb) + 7) & ~7;
    const int NQ = (Lp - 1) / 8 + 2;
    return (size_t)NSB * ((2 * NC + 63) / 64) * KC * 128 + (size_t)2 * 2 * MO * KC * 2 + (size_t)2 * 8 * NQ * 16 +
           (size_t)(2 * NSB + 9) * 8;
}

cudaError_t launch_level_fir_tc(const LevelLaunch &L, const int *amax_in, const void *scratch, int *err,
                                cudaStream_t s, const char **why)
{
    *why = nullptr;
    FirTcArgs a;
    a.y = static_cast<const __half2 *>(scratch); a.out = L.out; a.amax = L.amax; a.amax_in = amax_in; a.err = err;
    a.rows = L.Np * L.C; a.P = L.P; a.Kop = (L.Ko + 3) & ~3; a.Ko = L.Ko; a.Po = L.Po; a.Dp = L.Dp;
    a.Lp = L.Dp > 1 ? L.Lp : 1; a.plp = L.Dp > 1 ? L.plp : 0; a.tp = L.Dp > 1 ? L.tp : nullptr;
    a.ncb = (a.Kop + 127) / 128;
    a.NC = (((a.Kop + a.ncb - 1) / a.ncb) + 7) & ~7;
    a.nob = (a.Po + MO - 1) / MO;
    a.ntiles = (long)a.rows * a.nob * a.ncb;
    a.NQ = (a.Lp - 1) / 8 + 2;
    if (a.ntiles <= 0) return cudaSuccess;
    if (((uintptr_t)scratch & 15) != 0) { *why = "the intermediate must be 16-byte aligned"; return cudaErrorNotSupported; }
    const size_t smem = level_fir_tc_smem(a.Kop, a.Lp);
    int dev = 0, maxsmem = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem + 2048 > (size_t)maxsmem) { *why = "the pulse filter's taps do not fit shared memory"; return cudaErrorNotSupported; }
    // the intermediate as a 3-D float16 tensor: real columns (2 Kop), pulses, rows; a box is 64 columns x 64 pulses
    // of one row, 128 bytes per pulse, landing with the 128-byte swizzle
    EncodeTiledFn enc = encode_tiled();
    if (!enc) { *why = "cuTensorMapEncodeTiled is not available from the driver"; return cudaErrorNotSupported; }
    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t)(2 * a.Kop), (cuuint64_t)a.P, (cuuint64_t)a.rows};
    const cuuint64_t strides[2] = {(cuuint64_t)a.Kop * 4, (cuuint64_t)a.P * a.Kop * 4};
    const cuuint32_t box[3] = {64, (cuuint32_t)KC, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void *>(scratch), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { *why = "the intermediate's tensor map was refused by cuTensorMapEncodeTiled"; return cudaErrorNotSupported; }
    cudaError_t e = cudaFuncSetAttribute(level_fir_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)std::min<long>(a.ntiles, 148);
    level_fir_tc_kernel<<<grid, R_NTHR, smem, s>>>(a, map);
    return cudaGetLastError();
}

}  // namespace ffbp

// The fused level kernel: for every parent, each child's phase re-centring (rotation), the pulse-axis decimation
// FIR and the frequency-axis decimation FIR in one pass over the parent's samples.
//
// The reference (fastsar/ffbp_cuda.py:48-256, fastsar/ffbp_cpu.cpp:146-293) rotates and filters along frequency
// first, writes the [children, P, Ko] intermediate, and filters along pulses in a second kernel; at the 16,384-pulse
// x 8,192-sample spotlight that intermediate is 23 GB of the first level alone. The two FIRs act on different axes
// and commute, so this kernel takes the other order: rotation, then the pulse FIR, then the frequency FIR, with the
// pulse FIR held in registers and the frequency FIR applied from shared memory to each finished output row. Nothing
// at the input pulse rate reaches global memory; the output is written once.
//
// Work decomposition. A thread block owns one parent n, G consecutive children, a block of JB output columns
// (whose NK = Dk (JB - 1) + Lk input columns fit the block's NT threads, one column per thread) and a segment of
// output pulses. It sweeps the input pulses of its segment in order. Input pulse p = Dp g + b - plp (group g, phase
// b) feeds outputs i = g - s with tap r = Dp s + b for s < AP = ceil(Lp / Dp): each thread keeps those AP
// accumulators per child in registers, and after each group the oldest is finished, handed to shared memory, and
// the registers shift by one. Consecutive blocks are the child groups of one column block and segment, so the
// parent's rows they all read are served from L2.
//
// Per input sample and child the inner loop is one fused multiply-add for the phase, the hardware sine and cosine,
// a complex multiply and AP complex-by-real multiply-adds. Each thread's column of the input arrives RX rows ahead
// by asynchronous copies into a shared-memory ring that only that thread reads (so no barrier orders them); the
// child phases (c0, sl) are broadcast loads one row ahead; the pulse taps come from shared memory laid out by phase
// b with their AP values contiguous.
//
// Arithmetic: float32, the reference's. The rotation phase c0 + sl (k - kc) cycles is evaluated per sample and
// turned by the hardware sine and cosine, which are accurate to 2^-20.5 absolute over +-100 pi radians; the phases
// here stay within +-8 cycles (50 radians) at every level of the plans of record (c0 is wrapped to +-0.5 and the slope
// term is the child's range offset across half the band).
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int RX = 8;         // input rows in flight per thread (its own column, copied asynchronously)

struct LevelArgs {
    const float2 *__restrict__ x;
    const float2 *__restrict__ ph;
    const float *__restrict__ tk;
    const float *__restrict__ tp;
    const float *__restrict__ wp;
    const float *__restrict__ wk;
    float2 *__restrict__ out;
    int *bad;
    int *amax;
    int Np, C, P, K, Ko, Po, Dk, Lk, plk, Dp, Lp, plp;
    int JB, NK, ncb, ngrp, nseg, SEG;
    float kc;
};

template <int AP>
struct Taps {
    static constexpr int PAD = (AP + 3) & ~3;             // a phase's taps, padded to whole float4s
};

template <int AP, int G, int NT>
__global__ void __launch_bounds__(NT) level_kernel(const LevelArgs a)
{
    constexpr int APP = Taps<AP>::PAD;
    extern __shared__ __align__(16) float smem[];
    float *s_tp = smem;                                   // [Dp][APP]: s_tp[b APP + s] = tp[Dp s + b], zero past Lp
    float *s_tk = s_tp + a.Dp * APP;                      // [Lk] frequency taps
    const int ntk = (a.Lk + 3) & ~3;
    float2 *s_x = reinterpret_cast<float2 *>(s_tk + ntk);   // [RX][NT] the next RX input rows, one column a thread
    float2 *s_z = s_x + RX * NT;                          // [2][G][NT] finished rows before the frequency FIR

    int bid = blockIdx.x;
    const int grp = bid % a.ngrp;
    bid /= a.ngrp;
    const int cb = bid % a.ncb;
    bid /= a.ncb;
    const int seg = bid % a.nseg;
    const int n = bid / a.nseg;

    const int t = threadIdx.x;
    const int j0 = cb * a.JB;
    const int k = a.Dk * j0 - a.plk + t;
    const bool colok = (t < a.NK) && (k >= 0) && (k < a.K);
    const float kf = (float)k - a.kc;                     // exact: |k| < 2^24 and kc is a multiple of 1/2

    for (int r = t; r < a.Dp * APP; r += NT) {
        const int b = r / APP, s = r - b * APP;
        const int tap = a.Dp * s + b;
        s_tp[r] = (s < AP && tap < a.Lp) ? (a.tp ? a.tp[tap] : 1.f) : 0.f;
    }
    for (int r = t; r < a.Lk; r += NT) s_tk[r] = a.tk ? a.tk[r] : 1.f;

    const float wkk = (a.wk && colok) ? a.wk[k] : 1.f;
    const int i_s = seg * a.SEG;
    const int i_e = min(a.Po, i_s + a.SEG);
    const int c0 = grp * G;
    const int nc = min(G, a.C - c0);
    const float2 *__restrict__ phb = a.ph + ((size_t)n * a.C + c0) * a.P;
    const float2 *__restrict__ xb = a.x + (size_t)n * a.P * a.K;
    const int jbc = min(a.JB, a.Ko - j0);

    float2 acc[G][AP];
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
        for (int s = 0; s < AP; ++s) acc[c][s] = make_float2(0.f, 0.f);

    float vmax = 0.f;                                     // the largest |component| this thread writes
    const int g_end = i_e + AP - 1;
    const int p_start = a.Dp * i_s - a.plp;
    const int p_stop = a.Dp * g_end - a.plp;              // rows p_start .. p_stop - 1 are swept
    // the input ring: row p sits in slot (p - p_start) % RX of this thread's column, copied RX rows ahead
    auto issue = [&](int pr, int slot) {
        const bool ok = pr >= 0 && pr < a.P && pr < p_stop && colok;
        const float2 *src = ok ? xb + (size_t)pr * a.K + k : a.x;
        const unsigned dst = (unsigned)__cvta_generic_to_shared(s_x + slot * NT + t);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(dst), "l"(src), "r"(ok ? 8 : 0) : "memory");
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
#pragma unroll
    for (int r = 0; r < RX; ++r) issue(p_start + r, r);
    int p = p_start;
    float2 qn[G];
    {
        const bool ok = p >= 0 && p < a.P;
#pragma unroll
        for (int c = 0; c < G; ++c) qn[c] = (ok && c < nc) ? __ldg(&phb[(size_t)c * a.P + p]) : make_float2(0.f, 0.f);
    }
    int b = 0, slot = 0;
    __syncthreads();                                      // the taps
    for (int g = i_s; g < g_end;) {
        float2 q[G];
#pragma unroll
        for (int c = 0; c < G; ++c) q[c] = qn[c];
        const int pc = p;
        {
            const int pn = p + 1;
            const bool ok = pn >= 0 && pn < a.P;
#pragma unroll
            for (int c = 0; c < G; ++c) qn[c] = (ok && c < nc) ? __ldg(&phb[(size_t)c * a.P + pn]) : make_float2(0.f, 0.f);
        }
        asm volatile("cp.async.wait_group %0;\n" :: "n"(RX - 1) : "memory");
        const float2 v0 = s_x[slot * NT + t];
        if (pc >= 0 && pc < a.P) {                        // the same for every thread of the block
            float2 v = v0;
            if (a.wp) {
                const float w = a.wp[pc] * wkk;           // the reference's float32 window product
                v.x *= w;
                v.y *= w;
                if (a.bad && colok && !(isfinite(v.x) && isfinite(v.y))) atomicMin(a.bad, pc);
            }
            float tb[APP];
#pragma unroll
            for (int s4 = 0; s4 < APP; s4 += 4) {
                const float4 q4 = *reinterpret_cast<const float4 *>(&s_tp[b * APP + s4]);
                tb[s4] = q4.x; tb[s4 + 1] = q4.y; tb[s4 + 2] = q4.z; tb[s4 + 3] = q4.w;
            }
#pragma unroll
            for (int c = 0; c < G; ++c) {
                float sn, cs;
                __sincosf(TWO_PI_F * fmaf(q[c].y, kf, q[c].x), &sn, &cs);
                const float rr = fmaf(v.x, cs, -v.y * sn), ri = fmaf(v.x, sn, v.y * cs);
#pragma unroll
                for (int s = 0; s < AP; ++s) {
                    acc[c][s].x = fmaf(tb[s], rr, acc[c][s].x);
                    acc[c][s].y = fmaf(tb[s], ri, acc[c][s].y);
                }
            }
        }
        issue(pc + RX, slot);                             // refill the slot just consumed
        slot = (slot + 1 == RX) ? 0 : slot + 1;
        ++p;
        if (++b == a.Dp) {                                // group g is complete: output g - (AP - 1) is finished
            b = 0;
            const int i = g - (AP - 1);
            if (i >= i_s) {
                float2 *zb = s_z + (i & 1) * (G * NT);
#pragma unroll
                for (int c = 0; c < G; ++c) zb[c * NT + t] = acc[c][AP - 1];
                __syncthreads();
                // the frequency FIR of the finished row: outputs (c, j0 + jj), jj < jbc
                for (int w = t; w < nc * jbc; w += NT) {
                    const int c = w / jbc, jj = w - c * jbc;
                    const float2 *zr = zb + c * NT + a.Dk * jj;
                    float sr = 0.f, si = 0.f, sr2 = 0.f, si2 = 0.f;
                    int r = 0;
                    for (; r + 1 < a.Lk; r += 2) {
                        const float2 z0 = zr[r], z1 = zr[r + 1];
                        const float t0 = s_tk[r], t1 = s_tk[r + 1];
                        sr = fmaf(t0, z0.x, sr);
                        si = fmaf(t0, z0.y, si);
                        sr2 = fmaf(t1, z1.x, sr2);
                        si2 = fmaf(t1, z1.y, si2);
                    }
                    if (r < a.Lk) {
                        const float2 z0 = zr[r];
                        sr = fmaf(s_tk[r], z0.x, sr);
                        si = fmaf(s_tk[r], z0.y, si);
                    }
                    const float2 o = make_float2(sr + sr2, si + si2);
                    vmax = fmaxf(vmax, fmaxf(fabsf(o.x), fabsf(o.y)));
                    a.out[(((size_t)n * a.C + c0 + c) * a.Po + i) * a.Ko + j0 + jj] = o;
                }
            }
#pragma unroll
            for (int c = 0; c < G; ++c) {
#pragma unroll
                for (int s = AP - 1; s > 0; --s) acc[c][s] = acc[c][s - 1];
                acc[c][0] = make_float2(0.f, 0.f);
            }
            ++g;
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (a.amax) {                                         // non-negative floats order as their bits
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if ((t & 31) == 0 && vmax > 0.f) atomicMax(a.amax, __float_as_int(vmax));
    }
}

template <int AP, int G, int NT>
cudaError_t launch_t(LevelArgs a, cudaStream_t s)
{
    a.JB = (a.Dk > 1) ? (NT - a.Lk) / a.Dk + 1 : NT;
    a.NK = a.Dk * (a.JB - 1) + a.Lk;
    a.ncb = (a.Ko + a.JB - 1) / a.JB;
    a.ngrp = (a.C + G - 1) / G;
    // output segments: enough blocks to fill the device several times over, each long against its AP - 1 halo
    const long base = (long)a.Np * a.ngrp * a.ncb;
    const long target = 148L * 8 * 256 / NT;
    int nseg = 1;
    while (base * nseg < target && a.Po / (nseg * 2) >= 16 * AP) nseg *= 2;
    a.SEG = (a.Po + nseg - 1) / nseg;
    a.nseg = (a.Po + a.SEG - 1) / a.SEG;
    const long nblocks = base * a.nseg;
    if (nblocks > 0x7fffffffL) return cudaErrorInvalidValue;
    constexpr int APP = Taps<AP>::PAD;
    const size_t smem = (size_t)(a.Dp * APP + ((a.Lk + 3) & ~3)) * 4 + (size_t)RX * NT * sizeof(float2) +
                        (size_t)2 * G * NT * sizeof(float2);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(level_kernel<AP, G, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    level_kernel<AP, G, NT><<<(unsigned)nblocks, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int G, int NT>
cudaError_t launch_g(const LevelArgs &a, int ap, cudaStream_t s)
{
    switch (ap) {
        case 1: return launch_t<1, G, NT>(a, s);
        case 2: return launch_t<2, G, NT>(a, s);
        case 3: return launch_t<3, G, NT>(a, s);
        case 4: return launch_t<4, G, NT>(a, s);
        case 5: return launch_t<5, G, NT>(a, s);
        case 6: return launch_t<6, G, NT>(a, s);
        case 7: return launch_t<7, G, NT>(a, s);
        case 8: return launch_t<8, G, NT>(a, s);
        case 9: return launch_t<9, G, NT>(a, s);
        case 10: return launch_t<10, G, NT>(a, s);
        case 11: return launch_t<11, G, NT>(a, s);
        case 12: return launch_t<12, G, NT>(a, s);
        case 14: return launch_t<14, G, NT>(a, s);
        default: return launch_t<16, G, NT>(a, s);
    }
}

cudaError_t launch_g8(const LevelArgs &a, int ap, cudaStream_t s)
{
    switch (ap) {
        case 1: return launch_t<1, 8, 256>(a, s);
        case 2: return launch_t<2, 8, 256>(a, s);
        case 3: return launch_t<3, 8, 256>(a, s);
        case 4: return launch_t<4, 8, 256>(a, s);
        case 5: return launch_t<5, 8, 256>(a, s);
        case 6: return launch_t<6, 8, 256>(a, s);
        case 7: return launch_t<7, 8, 256>(a, s);
        case 8: return launch_t<8, 8, 256>(a, s);
        default: return launch_t<9, 8, 256>(a, s);
    }
}

// Whether 512 threads (input columns) per block waste clearly fewer columns on the frequency FIR's halo than 256.
bool wide_blocks(int Dk, int Lk, int Ko)
{
    auto useful = [&](int nt) {
        const int jb = (nt - Lk) / Dk + 1;
        if (jb < 1) return 0.0;
        const int nblk = (Ko + jb - 1) / jb;
        return (double)Ko * Dk / ((double)nblk * nt);
    };
    return useful(512) > 1.08 * useful(256);
}

}  // namespace

cudaError_t launch_level(const LevelLaunch &L, cudaStream_t s, const char **why)
{
    *why = nullptr;
    LevelArgs a;
    a.x = L.x; a.ph = L.phase; a.tk = L.tk; a.tp = L.tp; a.wp = L.wp; a.wk = L.wk; a.out = L.out; a.bad = L.bad;
    a.amax = L.amax;
    a.Np = L.Np; a.C = L.C; a.P = L.P; a.K = L.K; a.Ko = L.Ko; a.Po = L.Po;
    a.Dk = L.Dk; a.Lk = L.Dk > 1 ? L.Lk : 1; a.plk = L.Dk > 1 ? L.plk : 0;
    a.Dp = L.Dp; a.Lp = L.Dp > 1 ? L.Lp : 1; a.plp = L.Dp > 1 ? L.plp : 0;
    a.kc = (float)L.kc;
    const int AP = (a.Lp + a.Dp - 1) / a.Dp;
    int apt = 0;
    const int choices[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14, 16};
    for (int c : choices) if (c >= AP) { apt = c; break; }
    if (!apt) { *why = "pulse FIR spans more than 16 output pulses (Lp / Dp > 16)"; return cudaErrorInvalidValue; }
    if (a.Lk > 512) { *why = "frequency FIR longer than a block's columns (Lk > 512)"; return cudaErrorInvalidValue; }
    // 512 threads where a long frequency FIR would leave a 256-thread block little useful width. Blocks of 4
    // children by default; FFBP_LEVEL_G=8 selects 8 (one block per multiprocessor at 230 registers: measured 35%
    // slower on the 16,384-pulse spotlight, kept for other shapes)
    const bool wide = a.Lk > 256 || (a.Dk > 1 && wide_blocks(a.Dk, a.Lk, a.Ko));
    const char *gsel = getenv("FFBP_LEVEL_G");
    const int G = gsel ? atoi(gsel) : 4;
    cudaError_t e;
    if (wide) e = launch_g<4, 512>(a, apt, s);
    else if (G == 8) e = launch_g8(a, apt, s);
    else e = launch_g<4, 256>(a, apt, s);
    if (e == cudaErrorInvalidValue) *why = "too many level blocks";
    return e;
}

}  // namespace ffbp

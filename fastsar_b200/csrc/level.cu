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
// Arithmetic: float32, the reference's. The rotation phase c0 + sl (k - kc) is evaluated per sample (one fused
// multiply-add), reduced to [-0.5, 0.5] cycles and turned by the hardware sine and cosine; c0 and sl are the
// float32 phases the float64 geometry kernel computed.
#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

constexpr int NT = 256;       // threads per block = input columns per block
constexpr int G = 4;          // children per block

struct LevelArgs {
    const float2 *__restrict__ x;
    const float2 *__restrict__ ph;
    const float *__restrict__ tk;
    const float *__restrict__ tp;
    const float *__restrict__ wp;
    const float *__restrict__ wk;
    float2 *__restrict__ out;
    int *bad;
    int Np, C, P, K, Ko, Po, Dk, Lk, plk, Dp, Lp, plp;
    int JB, NK, ncb, ngrp, nseg, SEG;
    float kc;
};

template <int AP>
__global__ void __launch_bounds__(NT) level_kernel(const LevelArgs a)
{
    extern __shared__ __align__(16) float smem[];
    float *s_tp = smem;                                   // [Dp AP] pulse taps, zero past Lp, indexed Dp s + b
    const int ntp = (a.Dp * AP + 3) & ~3;
    float *s_tk = s_tp + ntp;                             // [Lk] frequency taps
    const int ntk = (a.Lk + 3) & ~3;
    float2 *s_z = reinterpret_cast<float2 *>(s_tk + ntk); // [2][G][NT] finished rows before the frequency FIR

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

    for (int r = t; r < a.Dp * AP; r += NT) s_tp[r] = (r < a.Lp) ? (a.tp ? a.tp[r] : 1.f) : 0.f;
    for (int r = t; r < a.Lk; r += NT) s_tk[r] = a.tk ? a.tk[r] : 1.f;
    __syncthreads();

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

    // the sweep: groups g = i_s .. i_e + AP - 2, rows p = Dp g + b - plp, with the next row's loads in flight
    const int g_end = i_e + AP - 1;
    int p = a.Dp * i_s - a.plp;
    float2 vn = make_float2(0.f, 0.f);
    float2 qn[G];
    {
        const bool ok = p >= 0 && p < a.P;
        if (ok && colok) vn = xb[(size_t)p * a.K + k];
#pragma unroll
        for (int c = 0; c < G; ++c) qn[c] = (ok && c < nc) ? __ldg(&phb[(size_t)c * a.P + p]) : make_float2(0.f, 0.f);
    }
    int b = 0;
    for (int g = i_s; g < g_end;) {
        const float2 v0 = vn;
        float2 q[G];
#pragma unroll
        for (int c = 0; c < G; ++c) q[c] = qn[c];
        const int pc = p;
        {
            const int pn = p + 1;
            const bool ok = pn >= 0 && pn < a.P;
            vn = (ok && colok) ? xb[(size_t)pn * a.K + k] : make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < G; ++c) qn[c] = (ok && c < nc) ? __ldg(&phb[(size_t)c * a.P + pn]) : make_float2(0.f, 0.f);
        }
        if (pc >= 0 && pc < a.P) {                        // the same for every thread of the block
            float2 v = v0;
            if (a.wp) {
                const float w = a.wp[pc] * wkk;           // the reference's float32 window product
                v.x *= w;
                v.y *= w;
            }
            if (a.bad && colok && !(isfinite(v.x) && isfinite(v.y))) atomicMin(a.bad, pc);
            float tb[AP];
#pragma unroll
            for (int s = 0; s < AP; ++s) tb[s] = s_tp[a.Dp * s + b];
#pragma unroll
            for (int c = 0; c < G; ++c) {
                float phi = fmaf(q[c].y, kf, q[c].x);
                const float2 w = cis_reduced(phi - rintf(phi));
                const float2 r = cmul(v, w);
#pragma unroll
                for (int s = 0; s < AP; ++s) {
                    acc[c][s].x = fmaf(tb[s], r.x, acc[c][s].x);
                    acc[c][s].y = fmaf(tb[s], r.y, acc[c][s].y);
                }
            }
        }
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
                    float sr = 0.f, si = 0.f;
                    for (int r = 0; r < a.Lk; ++r) {
                        const float tt = s_tk[r];
                        const float2 zz = zr[r];
                        sr = fmaf(tt, zz.x, sr);
                        si = fmaf(tt, zz.y, si);
                    }
                    a.out[(((size_t)n * a.C + c0 + c) * a.Po + i) * a.Ko + j0 + jj] = make_float2(sr, si);
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
}

template <int AP>
cudaError_t launch_ap(const LevelArgs &a, int nblocks, size_t smem, cudaStream_t s)
{
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(level_kernel<AP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    level_kernel<AP><<<nblocks, NT, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_level(const LevelLaunch &L, cudaStream_t s, const char **why)
{
    *why = nullptr;
    LevelArgs a;
    a.x = L.x; a.ph = L.phase; a.tk = L.tk; a.tp = L.tp; a.wp = L.wp; a.wk = L.wk; a.out = L.out; a.bad = L.bad;
    a.Np = L.Np; a.C = L.C; a.P = L.P; a.K = L.K; a.Ko = L.Ko; a.Po = L.Po;
    a.Dk = L.Dk; a.Lk = L.Dk > 1 ? L.Lk : 1; a.plk = L.Dk > 1 ? L.plk : 0;
    a.Dp = L.Dp; a.Lp = L.Dp > 1 ? L.Lp : 1; a.plp = L.Dp > 1 ? L.plp : 0;
    a.kc = (float)L.kc;
    if (a.Lk > NT) { *why = "frequency FIR longer than a block's columns (Lk > 256)"; return cudaErrorInvalidValue; }
    a.JB = (a.Dk > 1) ? (NT - a.Lk) / a.Dk + 1 : NT;
    a.NK = a.Dk * (a.JB - 1) + a.Lk;
    a.ncb = (a.Ko + a.JB - 1) / a.JB;
    a.ngrp = (a.C + G - 1) / G;
    const int AP = (a.Lp + a.Dp - 1) / a.Dp;
    // output segments: enough blocks to fill the device several times over, each long against its AP - 1 halo
    const long base = (long)a.Np * a.ngrp * a.ncb;
    int nseg = 1;
    while (base * nseg < 4L * 148 * 4 && a.Po / (nseg * 2) >= 16 * AP) nseg *= 2;
    a.SEG = (a.Po + nseg - 1) / nseg;
    a.nseg = (a.Po + a.SEG - 1) / a.SEG;
    const long nblocks = base * a.nseg;
    if (nblocks > 0x7fffffffL) { *why = "too many level blocks"; return cudaErrorInvalidValue; }
    int apt = 0;
    const int choices[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14, 16, 20, 24, 32};
    for (int c : choices) if (c >= AP) { apt = c; break; }
    if (!apt) { *why = "pulse FIR spans more than 32 output pulses (Lp / Dp > 32)"; return cudaErrorInvalidValue; }
    const size_t smem = (size_t)(((a.Dp * apt + 3) & ~3) + ((a.Lk + 3) & ~3)) * 4 + (size_t)2 * G * NT * sizeof(float2);
    switch (apt) {
        case 1: return launch_ap<1>(a, (int)nblocks, smem, s);
        case 2: return launch_ap<2>(a, (int)nblocks, smem, s);
        case 3: return launch_ap<3>(a, (int)nblocks, smem, s);
        case 4: return launch_ap<4>(a, (int)nblocks, smem, s);
        case 5: return launch_ap<5>(a, (int)nblocks, smem, s);
        case 6: return launch_ap<6>(a, (int)nblocks, smem, s);
        case 7: return launch_ap<7>(a, (int)nblocks, smem, s);
        case 8: return launch_ap<8>(a, (int)nblocks, smem, s);
        case 9: return launch_ap<9>(a, (int)nblocks, smem, s);
        case 10: return launch_ap<10>(a, (int)nblocks, smem, s);
        case 11: return launch_ap<11>(a, (int)nblocks, smem, s);
        case 12: return launch_ap<12>(a, (int)nblocks, smem, s);
        case 14: return launch_ap<14>(a, (int)nblocks, smem, s);
        case 16: return launch_ap<16>(a, (int)nblocks, smem, s);
        case 20: return launch_ap<20>(a, (int)nblocks, smem, s);
        case 24: return launch_ap<24>(a, (int)nblocks, smem, s);
        default: return launch_ap<32>(a, (int)nblocks, smem, s);
    }
}

}  // namespace ffbp

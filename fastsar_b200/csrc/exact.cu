// Exact backprojection and phase-history synthesis on the device: the oracle family of the former.
//
// bp_points_f64  exact backprojection at arbitrary points in float64 throughout (fastsar/bp.py:99-137's bp_points,
//                with float64 profiles as well): for every point and pulse the range offset
//                dR = |x - tx_p| (+ |x - rcv_p|, halved, bistatic) - ref_p, the range profile read at bin
//                dR inv_dr + nfft/2 by linear interpolation (circularly), turned by exp(2 pi i kcyc dR) and summed.
//                The profiles are the caller's (a zero-padded inverse FFT per pulse: cuFFT through torch).
// simulate       the phase history of point scatterers, S[p, k] += sum_n a_n exp(-2 pi i (2 f_k / c) dR_pn),
//                dR_pn = |x_n - ant_p| - |ant_p| (the CPHD convention, fastsar/sim.py:1-8): ranges and phases in
//                float64 per thread's run of 8 samples, a float32 complex recurrence along the run, the sum over
//                each chunk of 256 scatterers in float32 and over the chunks in float64.
#include "common.cuh"

namespace ffbp {

namespace {

__global__ void bp_points_f64_kernel(const double2 *__restrict__ prof, int P, int nfft, const double *__restrict__ tx,
                                     const double *__restrict__ rcv, const double *__restrict__ ref,
                                     const double *__restrict__ pts, long N, double inv_dr, double kcyc,
                                     double2 *__restrict__ out)
{
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double x = pts[3 * n], y = pts[3 * n + 1], z = pts[3 * n + 2];
    double ar = 0.0, ai = 0.0;
    for (int p = 0; p < P; ++p) {
        const double ax = x - tx[3 * p], ay = y - tx[3 * p + 1], az = z - tx[3 * p + 2];
        double dR = sqrt(ax * ax + ay * ay + az * az);
        if (rcv) {
            const double bx = x - rcv[3 * p], by = y - rcv[3 * p + 1], bz = z - rcv[3 * p + 2];
            dR = 0.5 * (dR + sqrt(bx * bx + by * by + bz * bz));
        }
        dR -= ref[p];
        const double t = dR * inv_dr + (double)(nfft / 2);
        const double fl = floor(t);
        long i = (long)fl % nfft;
        if (i < 0) i += nfft;
        const long i1 = (i + 1 == nfft) ? 0 : i + 1;
        const double w = t - fl;
        const double2 v0 = prof[(size_t)p * nfft + i], v1 = prof[(size_t)p * nfft + i1];
        const double vr = v0.x + w * (v1.x - v0.x), vi = v0.y + w * (v1.y - v0.y);
        double ph = kcyc * dR;
        ph -= rint(ph);
        double s, c;
        sincospi(2.0 * ph, &s, &c);
        ar += vr * c - vi * s;
        ai += vr * s + vi * c;
    }
    out[n] = make_double2(out[n].x + ar, out[n].y + ai);
}

constexpr int SIM_NT = 256;
constexpr int SIM_RUN = 8;                               // consecutive samples per thread

// One block: pulse p, SIM_NT * SIM_RUN consecutive samples. Per scatterer the block stages in shared memory the
// phase at its first sample (float64, reduced) and the per-sample step (float64 phase, its phasor in float32); each
// thread seeds its run's phasor from the float64 phase of its first sample and advances it by the step's phasor
// across its SIM_RUN samples (a complex recurrence of SIM_RUN - 1 steps: about 1e-6 relative).
__global__ void __launch_bounds__(SIM_NT) simulate_kernel(const double *__restrict__ ant, int P, int K, double fmin,
                                                          double df, const double *__restrict__ pos,
                                                          const double2 *__restrict__ amp, int N,
                                                          float2 *__restrict__ S)
{
    __shared__ double s_ph[SIM_NT], s_st[SIM_NT];
    __shared__ float2 s_w[SIM_NT];
    __shared__ double2 s_a[SIM_NT];
    const int span = SIM_NT * SIM_RUN;
    const int nkb = (K + span - 1) / span;
    const int p = blockIdx.x / nkb;
    const int k0 = (blockIdx.x % nkb) * span;
    const int t = threadIdx.x;
    const double ax = ant[3 * p], ay = ant[3 * p + 1], az = ant[3 * p + 2];
    const double r0 = sqrt(ax * ax + ay * ay + az * az);
    const double two_c = 2.0 / C_LIGHT;
    double sr[SIM_RUN], si[SIM_RUN];
#pragma unroll
    for (int j = 0; j < SIM_RUN; ++j) sr[j] = si[j] = 0.0;
    for (int n0 = 0; n0 < N; n0 += SIM_NT) {
        const int n = n0 + t;
        if (n < N) {
            const double dx = pos[3 * n] - ax, dy = pos[3 * n + 1] - ay, dz = pos[3 * n + 2] - az;
            const double dR = sqrt(dx * dx + dy * dy + dz * dz) - r0;
            const double ph = -two_c * (fmin + k0 * df) * dR;     // cycles at this block's first sample
            double st = -two_c * df * dR;                         // cycles per sample
            st -= rint(st);
            s_ph[t] = ph - rint(ph);
            s_st[t] = st;
            float sn, cs;
            sincospif(2.f * (float)st, &sn, &cs);
            s_w[t] = make_float2(cs, sn);
            s_a[t] = amp[n];
        } else {
            s_ph[t] = 0.0; s_st[t] = 0.0; s_w[t] = make_float2(1.f, 0.f); s_a[t] = make_double2(0.0, 0.0);
        }
        __syncthreads();
        const int nn = min(SIM_NT, N - n0);
        float cr[SIM_RUN], ci[SIM_RUN];
#pragma unroll
        for (int j = 0; j < SIM_RUN; ++j) cr[j] = ci[j] = 0.f;
        for (int m = 0; m < nn; ++m) {
            const double ph = fma((double)(SIM_RUN * t), s_st[m], s_ph[m]);
            float sn, cs;
            sincospif(2.f * (float)(ph - rint(ph)), &sn, &cs);
            const float2 st = s_w[m];
            const double2 a = s_a[m];
            float wr = (float)a.x * cs - (float)a.y * sn, wi = (float)a.x * sn + (float)a.y * cs;
#pragma unroll
            for (int j = 0; j < SIM_RUN; ++j) {
                cr[j] += wr;
                ci[j] += wi;
                const float nr = wr * st.x - wi * st.y;
                wi = wr * st.y + wi * st.x;
                wr = nr;
            }
        }
#pragma unroll
        for (int j = 0; j < SIM_RUN; ++j) { sr[j] += cr[j]; si[j] += ci[j]; }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < SIM_RUN; ++j) {
        const int k = k0 + SIM_RUN * t + j;
        if (k < K) {
            const float2 o = S[(size_t)p * K + k];
            S[(size_t)p * K + k] = make_float2(o.x + (float)sr[j], o.y + (float)si[j]);
        }
    }
}

}  // namespace

cudaError_t launch_bp_points_f64(const double2 *prof, int P, int nfft, const double *tx, const double *rcv,
                                 const double *ref, const double *pts, long N, double inv_dr, double kcyc, double2 *out,
                                 cudaStream_t s)
{
    if (N <= 0 || P <= 0) return cudaSuccess;
    const int nt = 128;
    bp_points_f64_kernel<<<(unsigned)((N + nt - 1) / nt), nt, 0, s>>>(prof, P, nfft, tx, rcv, ref, pts, N, inv_dr, kcyc, out);
    return cudaGetLastError();
}

cudaError_t launch_simulate(const double *ant, int P, int K, double fmin, double df, const double *pos,
                            const double2 *amp, int N, float2 *S, cudaStream_t s)
{
    if (P <= 0 || K <= 0 || N <= 0) return cudaSuccess;
    const long nb = (long)((K + SIM_NT * SIM_RUN - 1) / (SIM_NT * SIM_RUN)) * P;
    if (nb > 0x7fffffffL) return cudaErrorInvalidValue;
    simulate_kernel<<<(unsigned)nb, SIM_NT, 0, s>>>(ant, P, K, fmin, df, pos, amp, N, S);
    return cudaGetLastError();
}

}  // namespace ffbp

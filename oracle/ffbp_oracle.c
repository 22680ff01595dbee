/*
 * TEST INFRASTRUCTURE -- the oracle. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this
 * library, and only to check or time against it. The product (fastsar_b200) never calls it.
 *
 * A plain-C, float64 restatement of the reference's CPU factorized-backprojection kernels and of its exact point
 * backprojector, for the parity checks of the CUDA path:
 *
 *   rot_fir_k, rot_fir_k_cplx   fastsar/ffbp_cpu.cpp:146-255  rotate each parent pulse by every child's phase ramp
 *                                                            and decimate along frequency with the Kaiser FIR
 *   fir_p                       fastsar/ffbp_cpu.cpp:258-293  decimate along pulses
 *   final_tiles                 fastsar/ffbp_cpu.cpp:302-469  the separable T x T tile sum and the quadratic phase
 *   bp_points_f64               fastsar/bp.py:99-137          exact backprojection at points (here with float64
 *                                                            profiles as well: the FP64 oracle)
 *   simulate_points             fastsar/sim.py:69-90          phase history of point scatterers (the benchmark's
 *                                                            reference arm synthesizes its input with it, so that
 *                                                            arm runs no code of the product)
 *
 * The entry points keep the reference's C names and signatures (float32 inputs and outputs), so that one driver
 * (oracle/oracle.py) runs either this port or the reference's own compiled kernels. The arithmetic differs on
 * purpose: every phase is evaluated directly in float64 (no recurrences) and every sum accumulates in float64, so
 * the port is the reference's algorithm at higher precision. Its agreement with the reference's kernels and images
 * is pinned by tests/test_oracle.py against tests/golden.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static const double TWO_PI = 6.283185307179586476925286766559;

static inline void cis_cycles(double cyc, double* c, double* s)
{
    cyc -= nearbyint(cyc);
    *c = cos(TWO_PI * cyc);
    *s = sin(TWO_PI * cyc);
}

/* y_c[p, j] = sum_{r<L} taps[r] z_c[p, D j + r - pl],  z_c[p, k] = x[p, k] exp(2 pi i (c0_c[p] + sl_c[p] (k - kc))),
   x = 0 outside [0, K).  x has element stride xs (1: separate planes xr, xi; 2: interleaved, xi = xr + 1).
   c0, sl [Np, Cn, P]; y [Np Cn, P, Ko]. */
static void rot_fir(const float* xr, const float* xi, int xs, int Np, int P, int K, const float* c0, const float* sl,
                    int Cn, const float* taps, int L, int pl, int D, int Ko, double kc, float* yre, float* yim)
{
    const long total = (long)Np * Cn * P;
#pragma omp parallel
    {
        double* zr = (double*)malloc(sizeof(double) * (size_t)K);
        double* zi = (double*)malloc(sizeof(double) * (size_t)K);
#pragma omp for schedule(dynamic, 4)
        for (long idx = 0; idx < total; ++idx) {
            const int p = (int)(idx % P);
            const long nc = idx / P;                 /* n * Cn + c */
            const int n = (int)(nc / Cn);
            const double a = c0[idx], b = sl[idx];
            const float* rr = xr + ((size_t)n * P + p) * (size_t)K * xs;
            const float* ri = xi + ((size_t)n * P + p) * (size_t)K * xs;
            for (int k = 0; k < K; ++k) {
                double c, s;
                cis_cycles(a + b * ((double)k - kc), &c, &s);
                const double vr = rr[(size_t)k * xs], vi = ri[(size_t)k * xs];
                zr[k] = vr * c - vi * s;
                zi[k] = vr * s + vi * c;
            }
            float* outr = yre + ((size_t)nc * P + p) * (size_t)Ko;
            float* outi = yim + ((size_t)nc * P + p) * (size_t)Ko;
            for (int j = 0; j < Ko; ++j) {
                double ar = 0.0, ai = 0.0;
                for (int r = 0; r < L; ++r) {
                    const int k = D * j + r - pl;
                    if (k < 0 || k >= K) continue;
                    ar += (double)taps[r] * zr[k];
                    ai += (double)taps[r] * zi[k];
                }
                outr[j] = (float)ar;
                outi[j] = (float)ai;
            }
        }
        free(zr);
        free(zi);
    }
}

void rot_fir_k(const float* sre, const float* sim, int Np, int P, int K, const float* c0, const float* sl, int Cn,
               const float* taps, int L, int pl, int D, int Ko, double kc, float* yre, float* yim)
{
    rot_fir(sre, sim, 1, Np, P, K, c0, sl, Cn, taps, L, pl, D, Ko, kc, yre, yim);
}

void rot_fir_k_cplx(const float* x, int Np, int P, int K, const float* c0, const float* sl, int Cn,
                    const float* taps, int L, int pl, int D, int Ko, double kc, float* yre, float* yim)
{
    rot_fir(x, x + 1, 2, Np, P, K, c0, sl, Cn, taps, L, pl, D, Ko, kc, yre, yim);
}

/* z[b, i, j] = sum_{r<L} taps[r] y[b, D i + r - pl, j], y = 0 outside [0, P).  y [B, P, Ko]; z [B, Po, Ko]. */
void fir_p(const float* yre, const float* yim, int B, int P, int Ko, const float* taps, int L, int pl, int D, int Po,
           float* zre, float* zim)
{
#pragma omp parallel
    {
        double* ar = (double*)malloc(sizeof(double) * (size_t)Ko);
        double* ai = (double*)malloc(sizeof(double) * (size_t)Ko);
#pragma omp for schedule(dynamic, 4)
        for (long idx = 0; idx < (long)B * Po; ++idx) {
            const int b = (int)(idx / Po), i = (int)(idx % Po);
            memset(ar, 0, sizeof(double) * (size_t)Ko);
            memset(ai, 0, sizeof(double) * (size_t)Ko);
            for (int r = 0; r < L; ++r) {
                const int p = D * i + r - pl;
                if (p < 0 || p >= P) continue;
                const double t = taps[r];
                const float* a = yre + ((size_t)b * P + p) * (size_t)Ko;
                const float* c = yim + ((size_t)b * P + p) * (size_t)Ko;
                for (int j = 0; j < Ko; ++j) {
                    ar[j] += t * a[j];
                    ai[j] += t * c[j];
                }
            }
            float* orr = zre + ((size_t)b * Po + i) * (size_t)Ko;
            float* oii = zim + ((size_t)b * Po + i) * (size_t)Ko;
            for (int j = 0; j < Ko; ++j) {
                orr[j] = (float)ar[j];
                oii[j] = (float)ai[j];
            }
        }
        free(ar);
        free(ai);
    }
}

/* out[b, i, j] = e(qc_ij) sum_{p<Pf, q<Qf} d[b, p, q] wx_p(i) wy_p(j) exp(-2 pi i (ux_bp dlx_i + uy_bp dly_j)(a0 + a1 q))
   with qc_ij = (dlx_i^2 + dly_j^2 - (ucx_b dlx_i + ucy_b dly_j)^2) fc2 / (2 rc_b) cycles, and with the optional aperture
   weights wx_p(i) = w0_bp + gx_bp dlx_i, wy_p(j) = 1 + gyr_bp dly_j (both 1 when w0 is null). */
void final_tiles(const float* dre, const float* dim, int B, int Pf, int Qf, int T, const double* ux, const double* uy,
                 const double* dlx, const double* dly, double a0, double a1, const double* ucx, const double* ucy,
                 const double* rc, double fc2, float* ore, float* oim, const float* w0, const float* gx,
                 const float* gyr)
{
#pragma omp parallel
    {
        const size_t tq = (size_t)T * Qf;
        double* Axr = (double*)malloc(sizeof(double) * tq);
        double* Axi = (double*)malloc(sizeof(double) * tq);
        double* Byr = (double*)malloc(sizeof(double) * tq);
        double* Byi = (double*)malloc(sizeof(double) * tq);
        double* accr = (double*)malloc(sizeof(double) * (size_t)T * T);
        double* acci = (double*)malloc(sizeof(double) * (size_t)T * T);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < B; ++b) {
            memset(accr, 0, sizeof(double) * (size_t)T * T);
            memset(acci, 0, sizeof(double) * (size_t)T * T);
            for (int p = 0; p < Pf; ++p) {
                const size_t bp = (size_t)b * Pf + p;
                const double gxu = ux[bp], gyu = uy[bp];
                for (int i = 0; i < T; ++i) {
                    const double wx = w0 ? (double)w0[bp] + (double)gx[bp] * dlx[i] : 1.0;
                    const double wy = w0 ? 1.0 + (double)gyr[bp] * dly[i] : 1.0;
                    for (int q = 0; q < Qf; ++q) {
                        double c, s;
                        const double dr = dre[bp * Qf + q], di = dim[bp * Qf + q];
                        cis_cycles(-(gxu * dlx[i]) * (a0 + a1 * q), &c, &s);
                        Axr[(size_t)i * Qf + q] = (dr * c - di * s) * wx;
                        Axi[(size_t)i * Qf + q] = (dr * s + di * c) * wx;
                        cis_cycles(-(gyu * dly[i]) * (a0 + a1 * q), &c, &s);
                        Byr[(size_t)i * Qf + q] = c * wy;
                        Byi[(size_t)i * Qf + q] = s * wy;
                    }
                }
                for (int i = 0; i < T; ++i)
                    for (int j = 0; j < T; ++j) {
                        double sr = 0.0, si = 0.0;
                        const double* xr = Axr + (size_t)i * Qf;
                        const double* xi = Axi + (size_t)i * Qf;
                        const double* yr = Byr + (size_t)j * Qf;
                        const double* yi = Byi + (size_t)j * Qf;
                        for (int q = 0; q < Qf; ++q) {
                            sr += xr[q] * yr[q] - xi[q] * yi[q];
                            si += xr[q] * yi[q] + xi[q] * yr[q];
                        }
                        accr[(size_t)i * T + j] += sr;
                        acci[(size_t)i * T + j] += si;
                    }
            }
            const double f = fc2 / (2.0 * rc[b]);
            for (int i = 0; i < T; ++i)
                for (int j = 0; j < T; ++j) {
                    const double dx = dlx[i], dy = dly[j];
                    const double los = ucx[b] * dx + ucy[b] * dy;
                    double c, s;
                    cis_cycles((dx * dx + dy * dy - los * los) * f, &c, &s);
                    const double vr = accr[(size_t)i * T + j], vi = acci[(size_t)i * T + j];
                    ore[(size_t)b * T * T + (size_t)i * T + j] = (float)(vr * c - vi * s);
                    oim[(size_t)b * T * T + (size_t)i * T + j] = (float)(vr * s + vi * c);
                }
        }
        free(Axr); free(Axi); free(Byr); free(Byi); free(accr); free(acci);
    }
}

int ffbp_cpu_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Exact backprojection at points in float64 (fastsar/bp.py:99-137 with float64 profiles): for every point and pulse
   the range offset dR = |x - tx_p| (+ |x - rcv_p|, halved, when rcv is given) - ref_p, the profile read at bin
   dR inv_dr + nfft / 2 by linear interpolation, circularly, and turned by exp(2 pi i kcyc dR).
   prof [P, nfft] complex128 interleaved; out [N] complex128 interleaved (accumulated into). */
void bp_points_f64(const double* prof, int P, int nfft, const double* tx, const double* rcv, const double* ref,
                   const double* pts, long N, double inv_dr, double kcyc, double* out)
{
#pragma omp parallel for schedule(dynamic, 64)
    for (long n = 0; n < N; ++n) {
        const double x = pts[3 * n], y = pts[3 * n + 1], z = pts[3 * n + 2];
        double ar = 0.0, ai = 0.0;
        for (int p = 0; p < P; ++p) {
            const double* a = tx + 3 * p;
            const double ax = x - a[0], ay = y - a[1], az = z - a[2];
            double dR = sqrt(ax * ax + ay * ay + az * az);
            if (rcv) {
                const double* b = rcv + 3 * p;
                const double bx = x - b[0], by = y - b[1], bz = z - b[2];
                dR = 0.5 * (dR + sqrt(bx * bx + by * by + bz * bz));
            }
            dR -= ref[p];
            const double t = dR * inv_dr + (double)(nfft / 2);
            const double fl = floor(t);
            long i = (long)fl % nfft;
            if (i < 0) i += nfft;
            const long i1 = (i + 1 == nfft) ? 0 : i + 1;
            const double w = t - fl;
            const double* pr = prof + 2 * (size_t)p * nfft;
            const double vr = pr[2 * i] + w * (pr[2 * i1] - pr[2 * i]);
            const double vi = pr[2 * i + 1] + w * (pr[2 * i1 + 1] - pr[2 * i + 1]);
            double c, s;
            cis_cycles(kcyc * dR, &c, &s);
            ar += vr * c - vi * s;
            ai += vr * s + vi * c;
        }
        out[2 * n] += ar;
        out[2 * n + 1] += ai;
    }
}

/* Phase history of point scatterers for the reference arm of the benchmark (fastsar/sim.py:69-90 computes the same
   sum): S[p, k] += sum_n amp[n] exp(-4 pi i (fmin + k df) dR_pn / c), dR_pn = |pos[n] - ant[p]| - |ant[p]|, float64
   throughout; along k each scatterer's term is a geometric sequence, stepped by a complex product and re-seeded from
   the exact phase every 256 samples. S [P, K] complex64 interleaved (added to); amp [N] complex128 interleaved.
   Pulses in parallel. */
/* built for the host's widest vectors at run time (AVX-512, AVX2 or the x86-64 baseline) */
__attribute__((target_clones("avx512f", "avx2", "default")))
void simulate_points(const double* ant, int P, int K, double fmin, double df, const double* pos, const double* amp,
                     int N, float* S)
{
    const double C = 299792458.0;
    enum { SEG = 256, VB = 8 };
    const int NP = (N + VB - 1) / VB * VB;
#pragma omp parallel
    {
        double* dr = (double*)malloc(sizeof(double) * (size_t)NP);
        double* am = (double*)malloc(sizeof(double) * 2 * (size_t)NP);
#pragma omp for schedule(dynamic, 4)
        for (int p = 0; p < P; ++p) {
            const double* a = ant + 3 * p;
            const double ra = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
            for (int n = 0; n < NP; ++n) {
                if (n < N) {
                    const double* q = pos + 3 * (size_t)n;
                    const double dx = q[0] - a[0], dy = q[1] - a[1], dz = q[2] - a[2];
                    dr[n] = sqrt(dx * dx + dy * dy + dz * dz) - ra;
                    am[2 * n] = amp[2 * (size_t)n];
                    am[2 * n + 1] = amp[2 * (size_t)n + 1];
                } else {
                    dr[n] = am[2 * n] = am[2 * n + 1] = 0.0;
                }
            }
            float* out = S + 2 * (size_t)p * K;
            for (int k0 = 0; k0 < K; k0 += SEG) {
                const int k1 = k0 + SEG < K ? k0 + SEG : K;
                double ar[SEG], ai[SEG];
                for (int k = 0; k < k1 - k0; ++k) ar[k] = ai[k] = 0.0;
                for (int n0 = 0; n0 < NP; n0 += VB) {
                    double zr[VB], zi[VB], wr[VB], wi[VB];
                    for (int j = 0; j < VB; ++j) {
                        double c, s;
                        /* the phase in cycles, -2 (fmin + k df) dR / c, at k0; the step of one sample */
                        cis_cycles(-2.0 * (fmin + k0 * df) * dr[n0 + j] / C, &c, &s);
                        zr[j] = am[2 * (n0 + j)] * c - am[2 * (n0 + j) + 1] * s;
                        zi[j] = am[2 * (n0 + j)] * s + am[2 * (n0 + j) + 1] * c;
                        cis_cycles(-2.0 * df * dr[n0 + j] / C, &wr[j], &wi[j]);
                    }
                    for (int k = 0; k < k1 - k0; ++k) {
                        double sr = 0.0, si = 0.0;
#pragma omp simd reduction(+ : sr, si)
                        for (int j = 0; j < VB; ++j) {
                            sr += zr[j];
                            si += zi[j];
                            const double tr = zr[j] * wr[j] - zi[j] * wi[j];
                            zi[j] = zr[j] * wi[j] + zi[j] * wr[j];
                            zr[j] = tr;
                        }
                        ar[k] += sr;
                        ai[k] += si;
                    }
                }
                for (int k = k0; k < k1; ++k) {
                    out[2 * k] += (float)ar[k - k0];
                    out[2 * k + 1] += (float)ai[k - k0];
                }
            }
        }
        free(dr);
        free(am);
    }
}

// Internal launch interface between the C ABI (capi.cu) and the kernels. Not part of the public header.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace ffbp {

// One level (level.cu). Device pointers; see ffbp_level in include/ffbp_b200.h for the arithmetic.
struct LevelLaunch {
    const float2 *x;      // [Np, P, K]
    const float2 *phase;  // [Np, C, P] (c0, sl)
    const float *tk;      // [Lk] or null (Dk == 1)
    const float *tp;      // [Lp] or null (Dp == 1)
    const float *wp;      // [P] or null
    const float *wk;      // [K] or null
    float2 *out;          // [Np C, Po, Ko]
    int *bad;             // or null
    int Np, C, P, K, Ko, Po, Dk, Lk, plk, Dp, Lp, plp;
    double kc;
    int *amax = nullptr;  // or the largest |component| of the output, as float bits (atomicMax; start at 0)
    unsigned test_wait_ns = 0;   // tensor-core pass 1 only, for tests of the failure report: when nonzero the MMA
                                 // issuer first waits this long on a barrier nothing completes, as a stuck pipeline
    // tensor-core pass 1 launch options (0: the default): output columns per tile, B stages, plane copies (2 or 4),
    // row repeat (1: off), consumer warps (8, 4 or 12, 16 less them copying Hankel rows); pass 2's kernel (1: CUDA
    // cores, 2: tensor cores)
    int tc_nt = 0, tc_sb = 0, tc_pc = 0, tc_rp = 0, tc_fir = 0, tc_cw = 0;
};

// Returns cudaSuccess, or an error with *why set to a static message for shapes the kernels do not cover.
cudaError_t launch_level(const LevelLaunch &L, cudaStream_t s, const char **why);

// A level on the tensor cores (level_tc.cu): the frequency FIR of every child as one product per pulse (bfloat16
// x 3, float32 accumulation) into a float16 intermediate in `scratch` (level_tc_scratch_bytes), then the pulse FIR
// in float32. amax_in: the largest |component| of L.x (float bits), which sets the intermediate's scale; L.amax
// receives the output's. err: raised (atomicAdd) when a bounded wait runs out.
bool level_tc_supported(int C, int Lk, int Dk);
size_t level_tc_scratch_bytes(int Np, int C, int P, int Ko);
cudaError_t launch_level_tc(const LevelLaunch &L, const int *amax_in, void *scratch, int *err, cudaStream_t s,
                            const char **why);
// The same level in one pass (level_fused.cu): the pulse FIR's running sums held in tensor memory, the output
// written once as complex64 with its largest component recorded in L.amax; no intermediate. Levels of at most 64
// children, 96 frequency taps and 8 output pulses per input pulse.
bool level_fused_supported(int C, int Lk, int Dk, int Lp, int Dp);
cudaError_t launch_level_fused(const LevelLaunch &L, int *err, cudaStream_t s, const char **why);
// its two passes, for callers that time them apart
cudaError_t launch_level_tc_gemm(const LevelLaunch &L, const int *amax_in, void *scratch, int *err, cudaStream_t s,
                                 const char **why);
// the second pass: the pulse FIR of the float16 intermediate, on the kernel LevelLaunch::tc_fir selects (the tensor
// cores, level_fir_tc.cu, or the CUDA cores)
cudaError_t launch_level_tc_fir(const LevelLaunch &L, const int *amax_in, const void *scratch, int *err,
                                cudaStream_t s, const char **why);
cudaError_t launch_level_fir_tc(const LevelLaunch &L, const int *amax_in, const void *scratch, int *err,
                                cudaStream_t s, const char **why);
// The largest |component| of n complex samples into *amax (float bits, atomicMax; start at 0).
cudaError_t launch_amax(const float2 *x, size_t n, int *amax, cudaStream_t s);

// Child phases (geometry.cu).
cudaError_t launch_phases(const double *ant, int P, const double *ref, int Np, const double *cen, int C,
                          const double *range, double k0c, double k1, int cancel_free, float2 *phase, cudaStream_t s);

// Final-stage geometry (geometry.cu): per tile b and final subaperture p the direction cosines of the antenna seen
// from the tile centre along e1, e2 (ux, uy), and per tile the aperture-mean line of sight (ucx, ucy) and range (rc).
cudaError_t launch_final_geom(const double *ant_f, int Pf, const double *cen, int B, const double *e1,
                              const double *e2, double *ux, double *uy, double *ucx, double *ucy, double *rc,
                              cudaStream_t s);

// Final stage (final_fp32.cu, final_tc.cu).
struct FinalLaunch {
    const float2 *d;      // [B, Pf, Qf]
    int B, Pf, Qf, T;
    const double *ux, *uy;            // [B, Pf]
    double spx, spy, a0, a1, fc2;
    const double *ucx, *ucy, *rc;     // [B]
    const float *w;       // [3, B, Pf] (w0, gx, gyr) or null
    // output: either tiles [B, T, T] (img == null) or straight into an image with the tile origins
    float2 *tiles;
    float2 *img;          // [nx, ny]
    const int2 *first;    // [B] first pixel of each tile on the padded grid
    int nx, ny, ox, oy;
    float scale;
    int *err = nullptr;   // raised (atomicAdd) by a kernel whose bounded wait ran out (tensor-core stage), or null
    const int *amax = nullptr;   // the largest |component| of d (float bits), for the float16 operands' scale
    unsigned test_wait_ns = 0;   // tensor-core stage only, for tests of the failure report (as in LevelLaunch)
    const float4 *seeds = nullptr;   // [B, Pf] the float16 form's ramp seeds (launch_final_seeds), or null
};
cudaError_t launch_final_fp32(const FinalLaunch &F, cudaStream_t s, const char **why);
cudaError_t launch_final_tc(const FinalLaunch &F, int mode, cudaStream_t s, const char **why);
// The tensor-core final stage's ramp seeds per tile and final subaperture, reduced once in float64: (frac(ux spx a0 /
// 2), ux spx a1 / 2, frac(uy spy a0 / 2), uy spy a1 / 2), from which the float16 form's producers seed each row's
// ramp in float32 (row offset m = 2 r - (T - 1): phase -m (Y + 8 g V) at sample group g, step -m V).
cudaError_t launch_final_seeds(const double *ux, const double *uy, long n, double spx, double spy, double a0,
                               double a1, float4 *out, cudaStream_t s);

// Exact backprojection at points in float64 and the phase-history synthesis (exact.cu).
cudaError_t launch_bp_points_f64(const double2 *prof, int P, int nfft, const double *tx, const double *rcv,
                                 const double *ref, const double *pts, long N, double inv_dr, double kcyc, double2 *out,
                                 cudaStream_t s);
cudaError_t launch_simulate(const double *ant, int P, int K, double fmin, double df, const double *pos,
                            const double2 *amp, int N, float2 *S, cudaStream_t s);

// Exact backprojection onto a grid's tiles (exact_tiles.cu): the windowed, zero-padded history of a chunk of pulses
// (its fftshift folded in), and the tiled backprojection of its inverse-FFT profiles, each tile's range band of every
// profile staged by bulk copies. err: raised when a bounded wait ran out (or null).
cudaError_t launch_exact_pad(const float2 *s, int n, int K, const float *wp, const float *wk, int nfft, float2 *pad,
                             int *bad, int p_off, cudaStream_t st);
cudaError_t launch_exact_tiles(const float2 *prof, int n, int nfft, const double *ant, const double *ref,
                               const double *cen, int ntx, int nty, int tx, int ty, int nx, int ny, double spx,
                               double spy, const double *e1, const double *e2, double inv_dr, double kcyc, int cubic,
                               int along1, float2 *out, int *err, cudaStream_t st, const char **why);

// The range gate (gate.cu): pad and window a block of pulses, gather the bins about bin 0, taper the kept samples.
cudaError_t launch_gate_pad(const float2 *S, int n, int K, const float *wp, const float *wk, int npl, int Kp,
                            float2 *z, int *bad, int p_off, cudaStream_t s);
cudaError_t launch_gate_fold(const float2 *q, int n, int Kp, int N, float2 *u, cudaStream_t s);
cudaError_t launch_gate_taper(const float2 *u, int n, int N, int k0, int k1, const float *taper, float2 *out,
                              cudaStream_t s);

// The learned-tap network (mlp.cu): parameter count, work-buffer bytes for nq queries, the outputs of nq feature
// rows, and the gradient / Adam step of the decimation loss over ninst instances of S point-target pairs each.
int mlp_param_count();
int mlp_max_decimation();
size_t mlp_work_bytes(int nq);
cudaError_t mlp_taps(const float *params, const float *x, int nq, float *taps, float *work, cudaStream_t s);
cudaError_t mlp_grad(const float *params, const float *x, int nq, const float *prior, float scale, const int *inst,
                     const float *wt, int ninst, const double *f, const float2 *y, int S, float *grad, float *loss,
                     float *work, cudaStream_t s);
cudaError_t mlp_train_step(float *params, float *adam, const float *x, int nq, const float *prior, float scale,
                           const int *inst, const float *wt, int ninst, const double *f, const float2 *y, int S,
                           float lr, int t, float *loss, float *work, cudaStream_t s);

// Stack products (products.cu): box means, coherence, multilook / interferogram, the running average, tile statistics,
// the correlation's cross-spectrum, a spectrum's separable ramp and the translation's crop. kind: 0 the float as
// is, 1 |z|^2 of complex64, 2 x^2 of float.
cudaError_t launch_box_mean(const void *in, int kind, int n1, int n2, int w, int to_db, float *out, cudaStream_t s);
cudaError_t launch_coherence(const float2 *a, const float2 *b, int n1, int n2, int w1, int w2, float *out,
                             cudaStream_t s);
cudaError_t launch_multilook(const float2 *a, const float2 *b, int n1, int n2, int la, int lr, void *out,
                             cudaStream_t s);
cudaError_t launch_mean_add(const void *img, int kind, long n, float w, float weight, int first, float *sum,
                            float *wsum, cudaStream_t s);
cudaError_t launch_mean_image(const float *sum, const float *wsum, long n, float *out, cudaStream_t s);
cudaError_t launch_tile_stats(const float *x, int n1, int n2, int T, float gain, float *mean, float *var,
                              cudaStream_t s);
cudaError_t launch_cross_spectrum(const float2 *A, const float2 *B, int batch, int m1, int m2h, int nyquist,
                                  const float *e1, const float *e2, float2 *X, double *energy, cudaStream_t s);
cudaError_t launch_ramp_multiply(float2 *F, int m1, int m2, const float2 *r1, const float2 *r2, cudaStream_t s);
cudaError_t launch_window(const float *x, int batch, int n1, int n2, const float *mean, const float *w1, const float *w2,
                          float *out, cudaStream_t s);
cudaError_t launch_shift_crop(const float2 *shifted, int ld, const void *src, int src_complex, int n1, int n2, int w0,
                              int w1, void *out, cudaStream_t s);

// A patch mosaic's per-patch history (mosaic.cu): padding with the re-referencing phase, the gate's gather, and the
// gated spectrum's ramp, constant and taper.
cudaError_t launch_mosaic_pad(const float2 *S, long ldS, int rows, int K, int K2, int npl, const double *shift,
                              double f0, double df, float2 *out, cudaStream_t s);
cudaError_t launch_mosaic_gather(const float2 *Q, long ldQ, int rows, int K2, int N, const int *m, float2 *u,
                                 cudaStream_t s);
cudaError_t launch_mosaic_gate(const float2 *U, long ldU, int rows, int k0, int nk, int N, const double *d,
                               const double2 *cph, double scale, const float *taper, float2 *out, cudaStream_t s);

}  // namespace ffbp

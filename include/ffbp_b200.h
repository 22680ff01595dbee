/*
 * ffbp_b200 -- factorized backprojection (FFBP) spotlight image formation on the NVIDIA B200 (sm_100a).
 *
 * The drop-in boundary for the reference's factorized-backprojection former (saulpingerman/FastSAR 0.3.1): the
 * reference's Python former (fastsar/api.py:312-677, ImageFormer) plans on the host and hands the plan to a backend
 * (fastsar/ffbp_cuda.py:889 make_ffbp_cuda, fastsar/ffbp_cpu.py:158 make_ffbp_cpu) whose form(S) returns the image.
 * This C ABI is that backend: a plan object built from the host plan, and a form call on device buffers. The stage
 * entry points mirror the three kernels of the reference's CPU backend (fastsar/ffbp_cpu.cpp:244-260 rot_fir_k and
 * fir_p, fastsar/ffbp_cpu.cpp:458-461 final_tiles), on device pointers and a stream.
 *
 * Conventions
 *   - Every function returns 0 on success and a negative FFBP_E* code on failure; ffbp_last_error() gives the
 *     message of the last failure on the calling thread. No C++ exception crosses this boundary.
 *   - Pointers named d_* are device pointers; h_* are host pointers. Complex samples are interleaved float pairs
 *     (re, im): the layout of numpy's complex64 and of torch.complex64.
 *   - Streams are passed as void* (a cudaStream_t; NULL is the legacy default stream).
 *   - The caller owns every buffer it passes. A plan owns the device copies of its own constants (filters, float64
 *     geometry, child phases), allocated in ffbp_plan_create and freed in ffbp_plan_destroy.
 *   - A plan may be used by one thread at a time (fastsar/exact.py:412-413 states the same for a former).
 */
#ifndef FFBP_B200_H
#define FFBP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFBP_B200_ABI_VERSION 5

enum {
    FFBP_OK = 0,
    FFBP_E_ARG = -1,        /* an argument is out of range (the message names it)                         */
    FFBP_E_CUDA = -2,       /* a CUDA call failed                                                           */
    FFBP_E_NOMEM = -3,      /* a device allocation of the plan failed                                       */
    FFBP_E_WORKSPACE = -4,  /* the workspace passed to ffbp_form is smaller than ffbp_plan_workspace_bytes   */
    FFBP_E_UNSUPPORTED = -5,/* a shape the kernels do not cover (the message says which limit)              */
    FFBP_E_TRANSFER = -6    /* a history did not reach the device as it is in host memory (ffbp_form_host)  */
};

/* Final-stage arithmetic (ImageFormer's precision=, fastsar/api.py:27-31).                                     */
enum {
    FFBP_FINAL_FP32 = 0,    /* float32 on the CUDA cores: the plain path                                        */
    FFBP_FINAL_TC_F16 = 1,  /* tcgen05 tensor cores, float16 operands, float32 accumulation; ffbp_form scales  */
                            /* the samples by a power of two into float16's range, ffbp_final takes them as    */
                            /* given (each component below 2^14 in magnitude)                                   */
    FFBP_FINAL_TC_BF16X3 = 2, /* tcgen05 tensor cores, operands split x = hi + lo in bfloat16, the hi*hi, hi*lo, */
                              /* lo*hi and lo*lo products accumulated in float32                               */
    FFBP_LEVELS_TC = 0x100,   /* flag, or-ed into ffbp_plan_desc.final_mode: the levels on the tensor cores     */
                              /* (per pulse the children's modulated frequency taps times the parent row's      */
                              /* Hankel windows, three bfloat16 products accumulated in float32), in one pass:  */
                              /* the ramp and the pulse FIR follow each pulse's product on the multiprocessor,  */
                              /* the FIR's running sums in tensor memory. Levels the one-pass kernel does not   */
                              /* cover (more than 8 output pulses per input pulse) take the two-pass form below; */
                              /* levels of more than 64 children or 96 frequency taps stay on the float32 kernel */
    FFBP_LEVELS_TC2 = 0x200   /* flag, with FFBP_LEVELS_TC: every tensor-core level in two passes (the product   */
                              /* and ramp into a float16 intermediate in the workspace, then the pulse FIR in   */
                              /* float32), the form before the one-pass kernel                                    */
};

/* Launch options of a tensor-core level (level_tc_gemm, and the kernel of its pulse FIR; no counterpart in the
 * reference, whose kernels take fixed shapes). 0 in a field keeps the default. They change the schedule, not the arithmetic: the plane copies
 * and B stages leave every bit as it is; the columns per tile and the row repeat move the points where the output
 * ramp's recurrence is seeded: a rounding-level change (about 1e-7 before the float16 intermediate, whose rounding
 * it can flip by one unit: about 1e-5 relative in all). FFBP_E_UNSUPPORTED (at the form call) for a choice that
 * does not fit.                                                                                                   */
typedef struct {
    int nt;                 /* output columns per tile: a multiple of 16 (32 with repeated rows), at most 128       */
    int sb;                 /* stages of the B operand ring: 2 to 4                                                 */
    int copies;             /* shifted copies of each bfloat16 plane: 2 (4-byte loads) or 4 (8-byte loads)         */
    int repeat;             /* 1: no repeated A rows (default: repeated when more than 32 taps and at most 32 children) */
    int fir;                /* the second pass's pulse FIR: 1 on the CUDA cores, 2 on the tensor cores (a banded    */
                            /* product per row; default: the tensor cores for 512 or more output pulses)            */
    int consumers;          /* warps reading the accumulator: 8, 4 or 12 (16 less them copy Hankel rows)            */
} ffbp_tc_opts;

/* One level of the plan (fastsar/ffbp2.py:192-250, make_plan's per-level record). All pointers are host memory. */
typedef struct {
    int sx, sy;             /* children per parent along e1 and e2; C = sx * sy                                   */
    int C;
    int Dk, Dp;             /* decimation along frequency samples and along pulses (1: none)                     */
    int K, P;               /* samples and pulses of this level's input                                          */
    int Ko, Po;             /* samples and pulses of its output                                                  */
    const float *h_taps_k;  /* [Lk] frequency FIR (decimator_fir kernel), NULL when Dk == 1                      */
    int Lk, plk;
    const float *h_taps_p;  /* [Lp] pulse FIR, NULL when Dp == 1                                                 */
    int Lp, plp;
    double f0, df;          /* frequency of input sample 0 and the sample spacing (Hz)                           */
    const double *h_ant;    /* [P, 3] antenna phase centres on this level's input pulse grid (m)                 */
    const double *h_ref;    /* [B, 3] the parents' reference points (B = product of the earlier levels' C)        */
    const double *h_cen;    /* [B, C, 3] the children's centres                                                  */
    const double *h_range;  /* level 0 only, optional: [P] per-pulse one-way reference range (ImageFormer's ref=) */
    ffbp_tc_opts tc;        /* launch options when the level runs on the tensor cores in two passes (zeros: defaults) */
} ffbp_level_desc;

/* The plan of one image (make_plan's record plus the final stage and the call options). Host memory.          */
typedef struct {
    int nlev;
    const ffbp_level_desc *levels;  /* [nlev] */
    int T;                  /* final tile side, 16 or 32                                                          */
    int nx, ny;             /* the image                                                                          */
    int Nx, Ny, ox, oy;     /* the padded grid and the crop offsets                                               */
    double spx, spy;        /* pixel spacings (m) along e1, e2                                                    */
    double e1[3], e2[3];
    int Pf, Qf;             /* final stage: subapertures and frequency samples per final tile                    */
    double f0f, dff, fcf;   /* final-stage band: sample 0, spacing and centre frequency (Hz)                      */
    const double *h_ant_f;  /* [Pf, 3] antenna positions of the final subapertures                                */
    const double *h_cen_f;  /* [ntiles, 3] final tile centres, in the plan's tile order                           */
    const int *h_first_f;   /* [ntiles, 2] first pixel (x, y) of each final tile on the padded grid              */
    const float *h_wp;      /* [P0] Taylor window over pulses, or NULL (no window)                                */
    const float *h_wk;      /* [K0] Taylor window over samples, or NULL                                           */
    const float *h_wf;      /* aperture weights per (tile, final subaperture): [ntiles, Pf] (wf_ndim 2) or       */
    int wf_ndim;            /* [3, ntiles, Pf] weight and its gradients along e1, e2 (wf_ndim 3); NULL / 0 none  */
    int final_mode;         /* FFBP_FINAL_*, or-ed with FFBP_LEVELS_TC for the tensor-core levels                 */
    int partial;            /* 0: the final tiles cover the padded grid; 1: a part of it (a shard of the first     */
                            /* level's children: their descendants' tiles only; the image's other pixels untouched)*/
} ffbp_plan_desc;

typedef struct ffbp_plan ffbp_plan;

/* Last error message of the calling thread (NUL-terminated, truncated to n bytes). Returns its full length.    */
int ffbp_last_error(char *buf, int n);

/* ABI version (FFBP_B200_ABI_VERSION) and the build's target, for a loader's check.                            */
int ffbp_abi_version(void);

/* Build a plan: checks the description, uploads the filters and windows, and computes on the device, in float64,
 * every level's child phases (fastsar/ffbp2.py:313-342 for the first two levels, fastsar/ffbp_cuda.py:598-632
 * below them) and the final-stage geometry (fastsar/ffbp_cuda.py:870-886, 964-975). Runs on `stream` and returns
 * once the plan is ready. Replaces make_ffbp_cuda / make_ffbp_cpu (fastsar/ffbp_cuda.py:889, fastsar/ffbp_cpu.py:158)
 * together with collection_arrays (fastsar/ffbp2.py:313).                                                        */
int ffbp_plan_create(const ffbp_plan_desc *desc, void *stream, ffbp_plan **out);
int ffbp_plan_destroy(ffbp_plan *plan);

/* Bytes of device workspace a form call needs (the level intermediates and a status word).                     */
int ffbp_plan_workspace_bytes(const ffbp_plan *plan, size_t *bytes);

/* Form the image: d_S [P0, K0] complex64 phase history (unwindowed; the plan's window is applied here) ->
 * d_img [nx, ny] complex64. d_ws: the workspace (ffbp_plan_workspace_bytes, 256-byte aligned). The device the plan
 * was created on must be current (FFBP_E_ARG otherwise). Asynchronous on `stream`. The first non-finite sample's
 * pulse index (or -1) is written to h_bad_pulse when it is not NULL, which makes the call wait for the stream.
 * Failure reports of the tensor-core kernels: every bounded wait of theirs that runs out (a pipeline that stopped
 * making progress, which leaves that call's image incomplete) is counted in the plan. With h_bad_pulse the call
 * waits and returns FFBP_E_CUDA when its own kernels aborted; without it, the failure is returned by the plan's
 * next form call (FFBP_E_CUDA, before it launches anything) or by ffbp_plan_check. Each failure is reported once.
 * Replaces form(S) of fastsar/ffbp_cuda.py:1084-1211.                                                            */
int ffbp_form(ffbp_plan *plan, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream,
              int *h_bad_pulse);

/* Wait for `stream` and return FFBP_E_CUDA if a tensor-core kernel of an earlier form call on this plan aborted
 * (a bounded wait ran out) and that has not been reported yet. For callers of ffbp_form without h_bad_pulse, after
 * a batch of calls (the reference raises from inside form(), fastsar/ffbp_cuda.py:1084-1211).                    */
int ffbp_plan_check(ffbp_plan *plan, void *stream);

/* Test hook of the failure report above (no counterpart in the reference): from the next form call on, the MMA
 * issuers of the plan's launches of `kind` (FFBP_KIND_LEVEL_TC or FFBP_KIND_LEVEL_TC_GEMM: the tensor-core levels in
 * either form; FFBP_KIND_FINAL_TC: the tensor-core final stage) first wait on a barrier
 * that nothing completes, with a limit of limit_us microseconds (1 .. 10^6), so that the wait runs out as a stuck
 * pipeline's would and the kernel winds down without its MMAs; kind 0 turns it off. The kernels stay well-formed:
 * every wait is bounded and the block frees its tensor memory before it exits.                                 */
int ffbp_plan_test_wait(ffbp_plan *plan, int kind, unsigned limit_us);

/* Test hook of the transfer check (no counterpart in the reference): the next ffbp_form_host call leaves out the
 * upload of its image `image` (its device buffer keeps what it held), as a transfer that did not deliver would;
 * -1 turns it off. One call only.                                                                                 */
int ffbp_plan_test_transfer(ffbp_plan *plan, int image);

/* Form n images from host memory, overlapping each history's upload and each image's download with the
 * formation of its neighbours (the reference's pinned double-buffered upload, fastsar/ffbp_cuda.py:692-765,
 * carried across images): h_S[i] [P0, K0] complex64 and h_img[i] [nx, ny] complex64 in page-locked host memory
 * (pageable memory works, without the overlap). d_stage: two device histories and two device images,
 * ffbp_plan_host_bytes bytes, 256-byte aligned; d_ws: the form workspace. The formation runs on `stream`, the copies
 * on two streams of the plan. Every upload is checked (the reference's transfer check, fastsar/ffbp_cuda.py:759-764,
 * 826-863): a position-weighted float64 sum of about 2,048 x 128 sampled samples, computed by a kernel on the upload
 * stream and by the host while the device works, must agree to 1e-9 of its scale. Returns when every image is in
 * host memory; h_bad[i] is image i's first non-finite pulse (or -1); FFBP_E_CUDA when a tensor-core kernel of one of
 * the calls aborted; FFBP_E_TRANSFER, naming the first such history, when a check did not agree (that image is not
 * to be used). No counterpart in the reference's API.                                                              */
int ffbp_plan_host_bytes(const ffbp_plan *plan, size_t *bytes);
int ffbp_form_host(ffbp_plan *plan, const void *const *h_S, void *const *h_img, int n, void *d_stage,
                   size_t stage_bytes, void *d_ws, size_t ws_bytes, void *stream, int *h_bad);

/* A batch: n plans (patches of uneven sizes, of one or several collections) formed together. ffbp_batch_create
 * captures the n form calls once into a CUDA graph, each plan's launches on a branch of its own so that the kernels
 * of different plans run side by side, on the buffers given here: d_S[i] (plan i's history), d_img[i] (its image),
 * d_ws[i] (its workspace of ws_bytes[i], 256-byte aligned; one per plan, they run at once). The call runs no
 * kernel (it captures on a stream of its own; `stream` is unused). ffbp_batch_form launches the graph on `stream`
 * (the buffers' current contents are formed); with h_bad (n ints) it waits, writes each image's first non-finite
 * pulse (or -1) and returns FFBP_E_CUDA when a tensor-core kernel aborted (without h_bad: at the next launch, or by
 * ffbp_plan_check on the plan). No counterpart in the reference,
 * which forms patches one after the other (fastsar/patches.py:619-972).                                      */
typedef struct ffbp_batch ffbp_batch;
int ffbp_batch_create(ffbp_plan *const *plans, int n, const void *const *d_S, void *const *d_img, void *const *d_ws,
                      const size_t *ws_bytes, void *stream, ffbp_batch **out);
int ffbp_batch_form(ffbp_batch *batch, void *stream, int *h_bad);
int ffbp_batch_destroy(ffbp_batch *batch);

/* ffbp_form without a caller-allocated workspace, for callers that cannot allocate device memory when they form an
 * image (a device pool they do not control, a real-time loop that must not enter the CUDA allocator). No counterpart
 * in the reference. The scratch is a static device array of this library, FFBP_STATIC_WS_BYTES (64 MiB), held by
 * every GPU that loads the library until the process exits; a plan whose ffbp_plan_workspace_bytes exceeds it is
 * rejected with FFBP_E_WORKSPACE. The call allocates nothing. Its first call on a device looks the array's device
 * address up (cudaGetSymbolAddress, with that device current), so make that first call before any stream capture.
 * All calls share the array: calls whose work overlaps on the GPU race and must not be made.                    */
#define FFBP_STATIC_WS_BYTES (64u << 20)
int ffbp_form_static(ffbp_plan *plan, const void *d_S, void *d_img, void *stream, int *h_bad_pulse);

/* ffbp_form with the device time of each launch (the reference's CUDA-event stage timers, fastsar/ffbp_cuda.py:
 * 635-652 PROFILE): stage_ms[l] for level l < nlev and stage_ms[nlev] for the final stage, measured by CUDA events
 * recorded on `stream` around each launch. Waits for the stream. n_stage: the length of stage_ms (>= nlev + 1).    */
int ffbp_form_timed(ffbp_plan *plan, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream,
                    float *h_stage_ms, int n_stage);

/* ffbp_form with the device time of every launch, in launch order: h_ms[i] (ms, CUDA events recorded on `stream`
 * after each launch) and h_kind[i] = FFBP_KIND_* << 8 | level (nlev for the final stage). n >= the launch count
 * of ffbp_plan_info. Waits for the stream. No counterpart in the reference (it times stages, not launches).       */
enum {
    FFBP_KIND_AMAX = 1,            /* the history's largest component (ahead of tensor-core levels)               */
    FFBP_KIND_LEVEL = 2,           /* a float32 level kernel                                                       */
    FFBP_KIND_LEVEL_TC_GEMM = 3,   /* a tensor-core level's first pass (products, ramp, float16 intermediate)     */
    FFBP_KIND_LEVEL_TC_FIR = 4,    /* a tensor-core level's pulse FIR                                              */
    FFBP_KIND_FINAL = 5,           /* the float32 final stage                                                      */
    FFBP_KIND_FINAL_TC = 6,        /* the tensor-core final stage                                                  */
    FFBP_KIND_LEVEL_TC = 7         /* a one-pass tensor-core level                                                 */
};
int ffbp_form_profile(ffbp_plan *plan, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream,
                      float *h_ms, int *h_kind, int n);

/* Levels and launches of a plan: *nlev, and the kernels one ffbp_form launches (*launches).                  */
int ffbp_plan_info(const ffbp_plan *plan, int *nlev, int *launches);

/* ---- stage entry points (device buffers, asynchronous on `stream`) -------------------------------------- */

/* One level for Np parents: the rotation of each parent's pulses to each child's centre, the pulse FIR and the
 * frequency FIR (fastsar/ffbp_cpu.cpp:146-255 rot_fir_k then fastsar/ffbp_cpu.cpp:258-293 fir_p, fused):
 *   out[n C + c, i, j] = sum_{rp<Lp} tp[rp] sum_{rk<Lk} tk[rk] z_{n,c}[Dp i + rp - plp, Dk j + rk - plk]
 *   z_{n,c}[p, k] = w(p, k) x[n, p, k] exp(2 pi i (c0[n,c,p] + sl[n,c,p] (k - kc))),  zero outside [0,P) x [0,K)
 * d_x [Np, P, K] complex64; d_phase [Np, C, P] float pairs (c0, sl); d_tk [Lk] / d_tp [Lp] float32 (NULL with
 * Dk == 1 / Dp == 1); d_wp [P], d_wk [K] the window w(p, k) = wp[p] wk[k], or NULL; d_out [Np C, Po, Ko] complex64.
 * d_bad (optional) receives the smallest pulse index of a non-finite sample (atomic min; initialise to INT_MAX). */
int ffbp_level(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk, int plk,
               int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po, const float *d_wp,
               const float *d_wk, void *d_out, int *d_bad, void *stream);

/* The same level on the tensor cores (the arithmetic of FFBP_LEVELS_TC): per pulse the children's modulated
 * frequency taps tk[r] exp(2 pi i sl r) times the Hankel windows of the parent's row, three bfloat16 products
 * accumulated in float32; the ramp exp(2 pi i (c0 + sl (Dk j - plk - kc))); a float16 intermediate in d_scratch
 * (ffbp_level_tc_scratch_bytes, 16-byte aligned), scaled by a power of two from the input's largest component;
 * the pulse FIR in float32. C <= 64 and Lk <= 96 (FFBP_E_UNSUPPORTED otherwise). d_status: 3 ints, zeroed by the
 * caller: [0] nonzero when a bounded wait of the kernel ran out, [1] the input's largest |component| (float bits,
 * filled here), [2] the output's. No counterpart in the reference (its levels run in float32 only).            */
size_t ffbp_level_tc_scratch_bytes(int Np, int C, int P, int Ko);

/* The same level in one pass (the arithmetic of FFBP_LEVELS_TC without FFBP_LEVELS_TC2): the three bfloat16 products,
 * the ramp and the pulse FIR's running sums (tensor memory) in one kernel; the output written once as complex64. No
 * scratch. C <= 64, Lk <= 96 and ceil(Lp / Dp) <= 8 (FFBP_E_UNSUPPORTED otherwise). d_status: 3 ints, zeroed by the
 * caller: [0] nonzero when a bounded wait of the kernel ran out, [2] the output's largest |component| (float bits).
 * No counterpart in the reference (its levels run in float32 only).                                               */
int ffbp_level_fused(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk,
                     int plk, int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po,
                     const float *d_wp, const float *d_wk, void *d_out, int *d_bad, int *d_status, void *stream);
int ffbp_level_tc(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk, int plk,
                  int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po, const float *d_wp,
                  const float *d_wk, void *d_out, int *d_bad, void *d_scratch, size_t scratch_bytes, int *d_status,
                  void *stream);
/* ffbp_level_tc with launch options for its first pass (NULL: the defaults), for tuning them per level shape.      */
int ffbp_level_tc_ex(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk,
                     int plk, int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po,
                     const float *d_wp, const float *d_wk, void *d_out, int *d_bad, void *d_scratch,
                     size_t scratch_bytes, int *d_status, const ffbp_tc_opts *opts, void *stream);

/* Exact backprojection onto a grid (ExactFormer, fastsar/exact.py:404-801), in two calls per chunk of n pulses:
 * ffbp_exact_pad writes the windowed samples S[p, k] wp[p_off + p] wk[k] of d_S [n, K] complex64 into d_pad [n, nfft]
 * at bin k - K/2 (mod nfft) (fastsar/exact.py:186-194 pad_window; the other bins are the caller's, zeroed once)
 * and records in d_bad (optional, atomic min) the first pulse p_off + p with a non-finite sample; after the caller's
 * inverse FFT of length nfft (cuFFT, normalised by 1/nfft: bin 0 is zero delay), ffbp_exact_backproject adds the
 * tiled backprojection (the mathematics of fastsar/exact.py:58-162 bp_tiles) of the profiles d_prof [n, nfft]
 * complex64 (16-byte aligned, nfft even) onto d_out [nx, ny] complex64: per tile its centre's range in float64, per
 * pixel the range to third order about it, a cubic Lagrange (cubic 1, 4 samples) or linear (0) read of the profile at
 * dR inv_dr (circularly), times exp(2 pi i kcyc dR), the sum times nfft. The profiles are read in place (each tile's
 * band of bins, no cropped copy; fastsar/exact.py:196-205 crops them first). Tiles tx x ty in {32 x 32, 16 x 16,
 * 8 x 16, 8 x 8}; d_cen [ntx nty, 3] their centres (float64), tile (bx, by) at index bx nty + by; d_ant [n, 3],
 * d_ref [n] the pulses' antenna positions and reference ranges; e1, e2 host pointers to 3 doubles; along1 1 to run
 * consecutive blocks along e1. d_err (optional) is raised when a bounded wait of the kernel ran out.             */
int ffbp_exact_pad(const void *d_S, int n, int K, const float *d_wp, const float *d_wk, int nfft, void *d_pad,
                   int *d_bad, int p_off, void *stream);
int ffbp_exact_backproject(const void *d_prof, int n, int nfft, const double *d_ant, const double *d_ref,
                           const double *d_cen, int ntx, int nty, int tx, int ty, int nx, int ny, double spx, double spy,
                           const double *e1, const double *e2, double inv_dr, double kcyc, int cubic, int along1,
                           int *d_err, void *d_out, void *stream);

/* The range gate (fastsar/ffbp_cuda.py:767-864 and ImageFormer._gate fastsar/api.py:525-564), three steps around the
 * caller's two FFTs (cuFFT) per block of n pulses: ffbp_gate_pad writes d_z [n, Kp] complex64: zeros, and at
 * npl .. npl + K - 1 the pulses' samples d_S [n, K] times the window d_wp[p_off + p] d_wk[k] (both or neither), and
 * lowers *d_bad to the first pulse (p_off + p) with a non-finite sample (d_bad may be NULL); the caller takes the
 * inverse FFT of each row (scaled by 1 / Kp); ffbp_gate_fold gathers the N bins about bin 0, d_u[p, i] =
 * d_q[p, i] for i < N - N/2 and d_q[p, Kp - N + i] above; the caller takes the forward FFT of each row;
 * ffbp_gate_taper writes d_out [n, k1 - k0] = d_u[p, k0 + k] d_taper[k] (the gated history's rows).            */
int ffbp_gate_pad(const void *d_S, int n, int K, const float *d_wp, const float *d_wk, int npl, int Kp, void *d_z,
                  int *d_bad, int p_off, void *stream);
int ffbp_gate_fold(const void *d_q, int n, int Kp, int N, void *d_u, void *stream);
int ffbp_gate_taper(const void *d_u, int n, int N, int k0, int k1, const float *d_taper, void *d_out, void *stream);

/* The learned-tap network (no counterpart in the reference): an MLP 5 -> 64 -> 64 -> 64 -> 16 (GELU, bfloat16
 * weights and activations, float32 sums) that stands in for the Kaiser-sinc decimation taps of the merge stages
 * (fastsar/ffbp2.py:101-137). A query is one phase q of one axis of a stage's decimation by D: features (phase
 * phi_q, pass fraction of the axis, 1 / D, stage, axis, each scaled by the caller); outputs 0..7 correct the 8 range-axis taps of that
 * phase and 8..15 the 8 angle-axis taps (a query uses the ones of its axis): tap n, at offset phi_q - 4 + n output
 * samples, = prior + scale * output, with phi_q = (q + 1/2) / D for even D and q / D for odd D.
 * d_params: ffbp_mlp_param_count floats, per layer W [out, in] then b [out]; d_x [nq, 5] float32; d_work:
 * ffbp_mlp_work_bytes(nq) bytes. ffbp_mlp_taps writes the outputs d_out [nq, 16].
 * Training pairs: instance i of d_inst [ninst, 3] (first query, D in 1..ffbp_mlp_max_decimation(), axis 0 or 1)
 * owns queries first .. first + D - 1 with prior taps d_prior [nq, 8]; its S samples are point targets at
 * frequencies d_f [ninst, S] (float64, cycles per output sample), whose parent samples are e^{2 pi i f t}, and their
 * exact child values d_y [ninst, S] (complex64); the decimated value is v = (1 / D) sum over the instance's taps of
 * tap e^{2 pi i f t}; instance i's pairs weigh d_weight[i] (float32; NULL: all 1). ffbp_mlp_grad writes the
 * gradient of mean weight |v - y|^2 over all pairs (d_grad, param count floats, or NULL) and the sum
 * weight |v - y|^2 (*d_loss; NaN when an instance is outside the query table);
 * ffbp_mlp_train_step takes one Adam step (lr, step t >= 1, b1 0.9, b2 0.999, eps 1e-8) with d_adam (2 x param
 * count floats: first then second moments, zeroed at t = 1). */
int ffbp_mlp_param_count(void);
int ffbp_mlp_max_decimation(void);
size_t ffbp_mlp_work_bytes(int nq);
int ffbp_mlp_taps(const float *d_params, const float *d_x, int nq, float *d_out, void *d_work, void *stream);
int ffbp_mlp_grad(const float *d_params, const float *d_x, int nq, const float *d_prior, float scale,
                  const int *d_inst, const float *d_weight, int ninst, const double *d_f, const void *d_y, int S,
                  float *d_grad, float *d_loss, void *d_work, void *stream);
int ffbp_mlp_train_step(float *d_params, float *d_adam, const float *d_x, int nq, const float *d_prior, float scale,
                        const int *d_inst, const float *d_weight, int ninst, const double *d_f, const void *d_y, int S,
                        float lr, int t, float *d_loss, void *d_work, void *stream);

/* Child phases in float64 for one level (fastsar/ffbp2.py:329-339 / fastsar/ffbp_cuda.py:598-632): for parent n,
 * child c and pulse p, ddr = |cen[n,c] - ant[p]| - |ref[n] - ant[p]| (or - range[p] when d_range is given),
 * c0 = ddr k0c - rint(ddr k0c), sl = ddr k1, stored as float pairs into d_phase [Np, C, P]. cancel_free selects
 * the cancellation-free form of the difference used below the first two levels. All inputs are float64.        */
int ffbp_phases(const double *d_ant, int P, const double *d_ref, int Np, const double *d_cen, int C,
                const double *d_range, double k0c, double k1, int cancel_free, void *d_phase, void *stream);

/* The final stage for B tiles (fastsar/ffbp_cpu.cpp:302-469 final_tiles):
 *   out[b, i, j] = exp(2 pi i qc_bij) sum_{p<Pf, q<Qf} d[b,p,q] wx(b,p,i) wy(b,p,j)
 *                                      exp(-2 pi i (ux[b,p] dlx_i + uy[b,p] dly_j)(a0 + a1 q))
 *   qc_bij = (dlx_i^2 + dly_j^2 - (ucx[b] dlx_i + ucy[b] dly_j)^2) fc2 / (2 rc[b]),  dl_i = (i - (T-1)/2) sp
 * d_d [B, Pf, Qf] complex64; d_ux, d_uy [B, Pf] float64; d_ucx, d_ucy, d_rc [B] float64; d_w (NULL, or [3, B, Pf]
 * float32: w0, gx, gyr with wx = w0 + gx dlx_i, wy = 1 + gyr dly_j); d_out [B, T, T] complex64. mode: FFBP_FINAL_*.*/
int ffbp_final(const void *d_d, int B, int Pf, int Qf, int T, const double *d_ux, const double *d_uy, double spx,
               double spy, double a0, double a1, const double *d_ucx, const double *d_ucy, const double *d_rc,
               double fc2, const float *d_w, int mode, void *d_out, void *stream);

/* ---- exact backprojection and synthesis (the oracle family, on the device) ----------------------------------- */

/* Exact backprojection at N points in float64 (fastsar/bp.py:99-137 bp_points, with float64 profiles): for each point
 * and pulse p, dR = |x - tx[p]| (+ |x - rcv[p]| halved, when d_rcv is not NULL) - ref[p], the profile read at bin
 * dR inv_dr + nfft/2 by linear interpolation, circularly, times exp(2 pi i kcyc dR), accumulated into d_out.
 * d_prof [P, nfft] complex128 range profiles (fastsar/bp.py:55-63 range_compress); d_tx, d_rcv [P, 3], d_ref [P],
 * d_pts [N, 3] float64; d_out [N] complex128 (added to).                                                          */
int ffbp_bp_points_f64(const void *d_prof, int P, int nfft, const double *d_tx, const double *d_rcv,
                       const double *d_ref, const double *d_pts, long N, double inv_dr, double kcyc, void *d_out,
                       void *stream);

/* Phase history of point scatterers (fastsar/sim.py:69-90 simulate, as a direct sum): d_S [P, K] complex64 +=
 * sum_n amp[n] exp(-4 pi i (fmin + k df) dR_pn / c), dR_pn = |pos[n] - ant[p]| - |ant[p]|. Ranges and phases in
 * float64, the sum in float64 per sample. d_ant [P, 3], d_pos [N, 3] float64; d_amp [N] complex128.               */
int ffbp_simulate(const double *d_ant, int P, int K, double fmin, double df, const double *d_pos, const void *d_amp,
                  int N, void *d_S, void *stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Stack products: what the reference computes from images formed on one grid (fastsar/stack.py:485-1124 register,
 * shift_image, mean; fastsar/products.py:28-67 multilook, interferogram, coherence). Images are row-major [n1, n2]
 * device buffers; complex images complex64. A pixel kind says what a buffer holds and which intensity is taken:  */
enum {
    FFBP_PIX_AS_IS = 0,     /* float32, taken as it is (an intensity already)                                  */
    FFBP_PIX_POWER = 1,     /* complex64, intensity re*re + im*im (each product rounded to float32)            */
    FFBP_PIX_SQUARE = 2     /* float32 amplitude, intensity x*x                                                */
};

/* The mean over w x w pixels about each pixel of the intensity, the edge pixels repeated (fastsar/stack.py:493-528
 * _box of _power): the window spans (w - 1) / 2 before and w / 2 after; the w rows are summed in order and divided
 * by w in float32, then the w columns likewise, so the result equals the reference's bit for bit. to_db: 10 log10
 * of max(mean, 1e-30) instead (the registration's detected image before its clip). 1 <= w <= 33.              */
int ffbp_box_mean(const void *d_in, int kind, int n1, int n2, int w, int to_db, float *d_out, void *stream);

/* Sample coherence |<a b*>| / sqrt(<|a|^2> <|b|^2>) over w1 x w2 windows, float64 sums, the edge pixels repeated
 * (fastsar/products.py:53-67 coherence, scipy.ndimage.uniform_filter's window placement: i - w/2 .. i - w/2 + w - 1).
 * d_out [n1, n2] float32. 1 <= w1 <= 1024, 1 <= w2 <= 64.                                                        */
int ffbp_coherence(const void *d_a, const void *d_b, int n1, int n2, int w1, int w2, float *d_out, void *stream);

/* |img|^2 (d_b NULL; d_out float32) or img conj(b) (d_out complex64) averaged over la x lr boxes and decimated:
 * d_out [n1 / la, n2 / lr] (fastsar/products.py:28-32 multilook, 42-50 interferogram).                         */
int ffbp_multilook(const void *d_img, const void *d_b, int n1, int n2, int la, int lr, void *d_out, void *stream);

/* One image into a running incoherent average (fastsar/stack.py:1060-1083): with p the pixel's intensity (kind
 * FFBP_PIX_POWER or FFBP_PIX_SQUARE), d_sum = (first ? 0 : d_sum) + p w and d_wsum = (first ? 0 : d_wsum) + (p > 0 ?
 * weight : 0), each product and sum rounded to float32 once. w: the weight times the equalizing gain.           */
int ffbp_mean_add(const void *d_img, int kind, long n, float w, float weight, int first, float *d_sum, float *d_wsum,
                  void *stream);

/* The average: d_out = d_wsum > 0 ? d_sum / max(d_wsum, 1e-30) : 0, float32 (fastsar/stack.py:1092-1094).          */
int ffbp_mean_image(const float *d_sum, const float *d_wsum, long n, float *d_out, void *stream);

/* Mean and population variance of x gain over each whole T x T tile (fastsar/stack.py:1027-1034), float64 sums:
 * d_mean, d_var [(n1 / T) (n2 / T)] float32, tiles row by row.                                                     */
int ffbp_tile_stats(const float *d_x, int n1, int n2, int T, float gain, float *d_mean, float *d_var, void *stream);

/* The correlation's cross-spectra of a batch of image pairs over a real transform's half plane, d_A, d_B, d_X
 * [batch, m1, m2h] (fastsar/stack.py:570-592): X = conj(A) B hp with hp = 1 - e1[i] e2[j] (the separable factors of
 * the Gaussian the high pass removes; d_e1 NULL: no high pass), and d_energy [batch, 2] float64 = the sums of
 * |A|^2 wk hp and |B|^2 wk hp, wk 1 for the zero column and (nyquist != 0) the last, 2 for the others.           */
int ffbp_cross_spectrum(const void *d_A, const void *d_B, int batch, int m1, int m2h, int nyquist, const float *d_e1,
                        const float *d_e2, void *d_X, double *d_energy, void *stream);

/* The correlation's windowing of a batch of float32 images [batch, n1, n2] (fastsar/stack.py:565-568): d_out =
 * ((x - mean[b]) w1[i]) w2[j], each operation rounded to float32 as the reference's array operations are; d_mean
 * [batch] (each image's mean), d_w1 [n1], d_w2 [n2] float32.                                                       */
int ffbp_window(const float *d_x, int batch, int n1, int n2, const float *d_mean, const float *d_w1, const float *d_w2,
                float *d_out, void *stream);

/* d_F [m1, m2] complex64 *= r1[i] r2[j]: a separable phase ramp on a spectrum (fastsar/stack.py:700-706).           */
int ffbp_ramp_multiply(void *d_F, int m1, int m2, const void *d_r1, const void *d_r2, void *stream);

/* The translation's crop (fastsar/stack.py:712-725): d_out[i, j] = shifted[i + w0, j + w1] where that source pixel
 * lies in the image and d_src is not 0 there, else 0. d_shifted: the sub-pixel-shifted image (complex64, leading
 * dimension ld), or NULL for a whole-pixel move of d_src itself. src_complex: d_src and d_out complex64; else
 * float32, and the shifted image's real part clipped at 0.                                                       */
int ffbp_shift_crop(const void *d_shifted, int ld, const void *d_src, int src_complex, int n1, int n2, int w0, int w1,
                    void *d_out, void *stream);

/* ---------------------------------------------------------------------------------------------------------------
 * Patch mosaic: one patch's phase history re-referenced to the patch centre and gated in range to the patch
 * (fastsar/patches.py:315-500 range_profiles, patch_history), around the caller's transforms (cuFFT).            */

/* d_out [rows, K2] complex64: row p's K samples of d_S (leading dimension ldS) at columns npl .. npl + K - 1, zeros
 * elsewhere, times exp(-4 pi i f_k d_shift[p] / c) with f_k = f0 + k df (d_shift NULL: no phase; the shared range
 * profiles' padding). Phases in float64.                                                                          */
int ffbp_mosaic_pad(const void *d_S, long ldS, int rows, int K, int K2, int npl, const double *d_shift, double f0,
                    double df, void *d_out, void *stream);

/* d_u [rows, N] complex64: u[p, n] = Q[p, (j_n - m[p]) mod K2] with j_n = n for n < N / 2 and n - N otherwise (the
 * gate's bins about the centre), Q with leading dimension ldQ; d_m [rows] int32 or NULL (no offset).                */
int ffbp_mosaic_gather(const void *d_Q, long ldQ, int rows, int K2, int N, const int *d_m, void *d_u, void *stream);

/* d_out [rows, nk] complex64: U[p, k0 + k] exp(-2 pi i d[p] (k0 + k) / N) cph[p] scale taper[k] (d_d, d_cph NULL:
 * left out; d_cph complex128 [rows]; d_taper float32 [nk]); U with leading dimension ldU.                          */
int ffbp_mosaic_gate(const void *d_U, long ldU, int rows, int k0, int nk, int N, const double *d_d, const void *d_cph,
                     double scale, const float *d_taper, void *d_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FFBP_B200_H */

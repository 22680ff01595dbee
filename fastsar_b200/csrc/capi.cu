// The C ABI of include/ffbp_b200.h: plan objects, the form call and the stage entry points.
//
// A plan keeps, in device memory, everything of the reference's make_ffbp_cuda set-up (fastsar/ffbp_cuda.py:889-962)
// that depends on the geometry alone: the filters, the windows, every level's child phases (computed here in
// float64, where the reference computes the first two levels on its host, fastsar/ffbp2.py:313-342, and the rest
// per call, fastsar/ffbp_cuda.py:1016) and the final-stage geometry (computed per call in the reference,
// fastsar/ffbp_cuda.py:964-975). A form call is then one launch per level and one for the final stage, all on the
// caller's stream, over the caller's workspace: the B200 holds a whole 16,384 x 8,192 history and every level's
// intermediate at once, so the reference's first-level groups and batches (fastsar/ffbp_cuda.py:1154-1198) are not
// needed for the workloads of record and the launches cover all children of a level.
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include <vector>

#include "../../include/ffbp_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(FFBP_E_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

struct DevLevel {
    int C, Dk, Dp, K, P, Ko, Po, Lk, plk, Lp, plp, Np;
    ffbp_tc_opts tc{};
    float *tk = nullptr, *tp = nullptr;
    float2 *phase = nullptr;
    double kc;
};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// The transfer check of a history S [P, K] complex64 (the reference checks each uploaded block the same way,
// fastsar/ffbp_cuda.py:759-764,826-863): sum over the sampled pulses r (every rs-th) of (r + 1) times the sum of the
// sampled samples S[r, k] (every ks-th), in float64, on both sides of the transfer. A block that did not arrive
// (a stale or half-written buffer) changes it by about the sum's own size. About 2,048 x 128 samples.
void check_strides(int P, int K, int *rs, int *ks)
{
    *rs = P > 2048 ? P / 2048 : 1;
    *ks = K > 128 ? K / 128 : 1;
}

// out[0], out[1] += the check of S (one warp per sampled pulse; atomics, so the last bits depend on the order)
__global__ void transfer_check_kernel(const float2 *__restrict__ S, int P, int K, int rs, int ks, double *out)
{
    const int lane = threadIdx.x & 31;
    const int r = ((int)blockIdx.x * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5)) * rs;
    if (r >= P) return;
    double re = 0.0, im = 0.0;
    for (int k = lane * ks; k < K; k += 32 * ks) {
        const float2 v = S[(size_t)r * K + k];
        re += v.x;
        im += v.y;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    if (lane == 0) {
        atomicAdd(out, (r + 1.0) * re);
        atomicAdd(out + 1, (r + 1.0) * im);
    }
}

// The same check of a history in host memory, and its scale (the sum of (r + 1) (|re| + |im|) over the samples).
void host_check(const float2 *S, int P, int K, double *re, double *im, double *scale)
{
    int rs, ks;
    check_strides(P, K, &rs, &ks);
    double a = 0.0, b = 0.0, m = 0.0;
    for (int r = 0; r < P; r += rs) {
        double x = 0.0, y = 0.0, z = 0.0;
        for (int k = 0; k < K; k += ks) {
            const float2 v = S[(size_t)r * K + k];
            x += v.x;
            y += v.y;
            z += fabs((double)v.x) + fabs((double)v.y);
        }
        a += (r + 1.0) * x;
        b += (r + 1.0) * y;
        m += (r + 1.0) * z;
    }
    *re = a;
    *im = b;
    *scale = m;
}

}  // namespace

struct ffbp_plan {
    int nlev, T, nx, ny, Nx, Ny, ox, oy, Pf, Qf, ntiles, final_mode;
    double spx, spy, a0, a1, fc2;
    std::vector<DevLevel> lv;
    float *wp = nullptr, *wk = nullptr, *wf = nullptr;
    double *ux = nullptr, *uy = nullptr, *ucx = nullptr, *ucy = nullptr, *rc = nullptr;
    float4 *seeds = nullptr;          // the float16 tensor-core final stage's ramp seeds [ntiles, Pf]
    int2 *first = nullptr;
    size_t bufA = 0, bufB = 0;
    std::vector<void *> owned;
    // the host-memory pipeline of ffbp_form_host, made at its first call: an upload and a download stream, per
    // device buffer pair b the events "history b uploaded", "image b formed", "image b downloaded", and a pinned
    // array of per-image status words
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t ev_up[2] = {}, ev_formed[2] = {}, ev_down[2] = {};
    int *h_status = nullptr;
    int n_status = 0;
    // the transfer check of ffbp_form_host: per device history buffer a sampled checksum (two doubles) computed after
    // its upload, copied into h_check (page-locked, two doubles per image); test_skip_upload: the index of the image
    // whose upload the next ffbp_form_host call leaves out (ffbp_plan_test_transfer; -1 none)
    double *d_check = nullptr;
    double *h_check = nullptr;
    int n_check = 0;
    int test_skip_upload = -1;
    // the device the plan lives on, and the abort count of its tensor-core kernels: d_aborts (device memory) is
    // raised by every bounded wait that runs out and is never reset; each form call copies it into h_aborts
    // (page-locked) at its end, so that the host sees earlier calls' aborts without waiting; `reported` is the count
    // already returned as an error
    int device = -1;
    int *d_aborts = nullptr;
    int *h_aborts = nullptr;
    int reported = 0;
    // test hook (ffbp_plan_test_wait): the kind of launch whose pipeline waits on a barrier nothing completes, and
    // that wait's limit
    int test_kind = 0;
    unsigned test_ns = 0;

    template <class T_>
    cudaError_t alloc(T_ **p, size_t count)
    {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, count * sizeof(T_) + 16);
        if (e == cudaSuccess) {
            owned.push_back(q);
            *p = static_cast<T_ *>(q);
        }
        return e;
    }
    ~ffbp_plan()
    {
        for (void *q : owned) cudaFree(q);
        for (int b = 0; b < 2; ++b) {
            if (ev_up[b]) cudaEventDestroy(ev_up[b]);
            if (ev_formed[b]) cudaEventDestroy(ev_formed[b]);
            if (ev_down[b]) cudaEventDestroy(ev_down[b]);
        }
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
        if (h_status) cudaFreeHost(h_status);
        if (h_check) cudaFreeHost(h_check);
        if (h_aborts) cudaFreeHost(h_aborts);
    }
};

namespace {

const char *const WAIT_MSG = "a tensor-core kernel stopped waiting on its pipeline (a bounded wait ran out) and "
                             "left its output incomplete";

// FFBP_E_CUDA when the plan's tensor-core kernels aborted since the last report (h_aborts as last copied back).
int aborted(ffbp_plan *p, const char *when)
{
    const int n = *reinterpret_cast<volatile int *>(p->h_aborts);
    if (n == p->reported) return FFBP_OK;
    p->reported = n;
    return fail(FFBP_E_CUDA, "%s: %s", when, WAIT_MSG);
}

}  // namespace

extern "C" {

int ffbp_last_error(char *buf, int n)
{
    if (buf && n > 0) {
        strncpy(buf, g_err.c_str(), (size_t)n - 1);
        buf[n - 1] = 0;
    }
    return (int)g_err.size();
}

int ffbp_abi_version(void) { return FFBP_B200_ABI_VERSION; }

int ffbp_plan_destroy(ffbp_plan *plan)
{
    delete plan;
    return FFBP_OK;
}

int ffbp_plan_create(const ffbp_plan_desc *d, void *stream_, ffbp_plan **out)
{
    if (!d || !out) return fail(FFBP_E_ARG, "ffbp_plan_create: null argument");
    *out = nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    if (d->nlev < 1 || !d->levels) return fail(FFBP_E_ARG, "plan needs at least one level, got %d", d->nlev);
    if (d->T != 16 && d->T != 32) return fail(FFBP_E_ARG, "final tile size T must be 16 or 32, got %d", d->T);
    {
        const int fm = d->final_mode & 0xff, flags = d->final_mode & ~0xff;
        if ((fm != FFBP_FINAL_FP32 && fm != FFBP_FINAL_TC_F16 && fm != FFBP_FINAL_TC_BF16X3) ||
            (flags & ~(FFBP_LEVELS_TC | FFBP_LEVELS_TC2)))
            return fail(FFBP_E_ARG, "unknown final_mode %d", d->final_mode);
    }
    if (d->nlev > 8) return fail(FFBP_E_ARG, "%d levels, at most 8", d->nlev);
    if (d->nx < 1 || d->ny < 1 || d->Nx < d->nx || d->Ny < d->ny || d->ox < 0 || d->oy < 0)
        return fail(FFBP_E_ARG, "bad grid: nx %d ny %d Nx %d Ny %d ox %d oy %d", d->nx, d->ny, d->Nx, d->Ny, d->ox, d->oy);
    if (!d->h_ant_f || !d->h_cen_f || !d->h_first_f) return fail(FFBP_E_ARG, "final-stage geometry missing");
    ffbp_plan *p = new ffbp_plan();
    cudaGetDevice(&p->device);
    p->nlev = d->nlev; p->T = d->T; p->nx = d->nx; p->ny = d->ny; p->Nx = d->Nx; p->Ny = d->Ny;
    p->ox = d->ox; p->oy = d->oy; p->Pf = d->Pf; p->Qf = d->Qf; p->final_mode = d->final_mode;
    p->spx = d->spx; p->spy = d->spy;
    p->a0 = 2.0 * d->f0f / ffbp::C_LIGHT;
    p->a1 = 2.0 * d->dff / ffbp::C_LIGHT;
    p->fc2 = 2.0 * d->fcf / ffbp::C_LIGHT;
    cudaError_t e = cudaSuccess;
    std::vector<void *> temp;
    auto cleanup = [&](int rc) {
        for (void *q : temp) cudaFree(q);
        if (rc != FFBP_OK) delete p;
        return rc;
    };
    auto upload = [&](const void *h, size_t bytes, void **dst, bool keep) -> cudaError_t {
        void *q = nullptr;
        cudaError_t r = cudaMalloc(&q, bytes + 16);
        if (r != cudaSuccess) return r;
        (keep ? p->owned : temp).push_back(q);
        *dst = q;
        return cudaMemcpyAsync(q, h, bytes, cudaMemcpyHostToDevice, s);
    };
    int B = 1;                                            // parents of the current level
    for (int l = 0; l < d->nlev; ++l) {
        const ffbp_level_desc &L = d->levels[l];
        if (L.C != L.sx * L.sy || L.C < 1) return cleanup(fail(FFBP_E_ARG, "level %d: C %d != sx %d * sy %d", l, L.C, L.sx, L.sy));
        if (L.Dk < 1 || L.Dp < 1 || L.K < 1 || L.P < 1 || L.Ko < 1 || L.Po < 1)
            return cleanup(fail(FFBP_E_ARG, "level %d: non-positive size", l));
        if ((L.Dk > 1 && (!L.h_taps_k || L.Lk < 1)) || (L.Dp > 1 && (!L.h_taps_p || L.Lp < 1)))
            return cleanup(fail(FFBP_E_ARG, "level %d: decimating axis without taps", l));
        if (L.Dk == 1 && L.Ko != L.K) return cleanup(fail(FFBP_E_ARG, "level %d: Dk 1 needs Ko == K", l));
        if (L.Dp == 1 && L.Po != L.P) return cleanup(fail(FFBP_E_ARG, "level %d: Dp 1 needs Po == P", l));
        if (l > 0) {
            const ffbp_level_desc &Q = d->levels[l - 1];
            if (L.K != Q.Ko || L.P != Q.Po) return cleanup(fail(FFBP_E_ARG, "level %d: input %dx%d != previous output %dx%d", l, L.P, L.K, Q.Po, Q.Ko));
        }
        if (!L.h_ant || !L.h_ref || !L.h_cen) return cleanup(fail(FFBP_E_ARG, "level %d: geometry missing", l));
        DevLevel v;
        v.C = L.C; v.Dk = L.Dk; v.Dp = L.Dp; v.K = L.K; v.P = L.P; v.Ko = L.Ko; v.Po = L.Po;
        v.Lk = L.Dk > 1 ? L.Lk : 1; v.plk = L.Dk > 1 ? L.plk : 0;
        v.Lp = L.Dp > 1 ? L.Lp : 1; v.plp = L.Dp > 1 ? L.plp : 0;
        v.Np = B;
        v.kc = (L.K - 1) / 2.0;
        v.tc = L.tc;
        void *q;
        if (L.Dk > 1) {
            if ((e = upload(L.h_taps_k, sizeof(float) * L.Lk, &q, true)) != cudaSuccess) return cleanup(cuda_fail(e, "upload taps"));
            v.tk = (float *)q;
        }
        if (L.Dp > 1) {
            if ((e = upload(L.h_taps_p, sizeof(float) * L.Lp, &q, true)) != cudaSuccess) return cleanup(cuda_fail(e, "upload taps"));
            v.tp = (float *)q;
        }
        if ((e = p->alloc(&v.phase, (size_t)B * L.C * L.P)) != cudaSuccess) return cleanup(cuda_fail(e, "allocate phases"));
        // geometry to the device (temporary), then the phases in float64
        void *dant, *dref, *dcen, *drange = nullptr;
        const bool cancel_free = l >= 2;                  // the reference's host levels take the plain difference
        if ((e = upload(L.h_ant, sizeof(double) * 3 * L.P, &dant, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload antenna"));
        if ((e = upload(L.h_ref, sizeof(double) * 3 * B, &dref, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload refs"));
        if (cancel_free) {
            // the children's offsets from their parent's reference, those of the first parent (fastsar/ffbp2.py:239 d)
            std::vector<double> off(3 * (size_t)L.C);
            for (int c = 0; c < L.C; ++c)
                for (int k = 0; k < 3; ++k) off[3 * c + k] = L.h_cen[3 * c + k] - L.h_ref[k];
            if ((e = upload(off.data(), sizeof(double) * off.size(), &dcen, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload offsets"));
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cleanup(cuda_fail(e, "upload"));
        } else {
            if ((e = upload(L.h_cen, sizeof(double) * 3 * (size_t)B * L.C, &dcen, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload centres"));
        }
        if (l == 0 && L.h_range) {
            if ((e = upload(L.h_range, sizeof(double) * L.P, &drange, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload ranges"));
        }
        const double k0c = 2.0 * (L.f0 + v.kc * L.df) / ffbp::C_LIGHT;
        const double k1 = 2.0 * L.df / ffbp::C_LIGHT;
        e = ffbp::launch_phases((const double *)dant, L.P, (const double *)dref, B, (const double *)dcen, L.C,
                                (const double *)drange, k0c, k1, cancel_free ? 1 : 0, v.phase, s);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "phases kernel"));
        const size_t outn = (size_t)B * L.C * L.Po * L.Ko;
        if (l % 2 == 0) p->bufA = std::max(p->bufA, outn); else p->bufB = std::max(p->bufB, outn);
        p->lv.push_back(v);
        B *= L.C;
    }
    p->ntiles = B;
    const ffbp_level_desc &last = d->levels[d->nlev - 1];
    if (p->Pf != last.Po || p->Qf != last.Ko) return cleanup(fail(FFBP_E_ARG, "final stage %dx%d != last level output %dx%d", p->Pf, p->Qf, last.Po, last.Ko));
    if (d->partial ? (long)B * d->T * d->T > (long)d->Nx * d->Ny : (long)B * d->T * d->T != (long)d->Nx * d->Ny)
        return cleanup(fail(FFBP_E_ARG, "tiles %d of %d^2 do not %s %dx%d", B, d->T, d->partial ? "fit" : "cover", d->Nx, d->Ny));
    void *q;
    if (d->h_wp) {
        if ((e = upload(d->h_wp, sizeof(float) * d->levels[0].P, &q, true)) != cudaSuccess) return cleanup(cuda_fail(e, "upload window"));
        p->wp = (float *)q;
    }
    if (d->h_wk) {
        if ((e = upload(d->h_wk, sizeof(float) * d->levels[0].K, &q, true)) != cudaSuccess) return cleanup(cuda_fail(e, "upload window"));
        p->wk = (float *)q;
    }
    if (d->h_wf) {
        if (d->wf_ndim != 3) return cleanup(fail(FFBP_E_UNSUPPORTED, "aperture weights: pass the [3, ntiles, Pf] form (weight and gradients)"));
        if ((e = upload(d->h_wf, sizeof(float) * 3 * (size_t)B * d->Pf, &q, true)) != cudaSuccess) return cleanup(cuda_fail(e, "upload weights"));
        p->wf = (float *)q;
    }
    if ((e = upload(d->h_first_f, sizeof(int) * 2 * (size_t)B, &q, true)) != cudaSuccess) return cleanup(cuda_fail(e, "upload tile origins"));
    p->first = (int2 *)q;
    void *dantf, *dcenf;
    if ((e = upload(d->h_ant_f, sizeof(double) * 3 * d->Pf, &dantf, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload final antenna"));
    if ((e = upload(d->h_cen_f, sizeof(double) * 3 * (size_t)B, &dcenf, false)) != cudaSuccess) return cleanup(cuda_fail(e, "upload tile centres"));
    if ((e = p->alloc(&p->ux, (size_t)B * d->Pf)) != cudaSuccess || (e = p->alloc(&p->uy, (size_t)B * d->Pf)) != cudaSuccess ||
        (e = p->alloc(&p->ucx, (size_t)B)) != cudaSuccess || (e = p->alloc(&p->ucy, (size_t)B)) != cudaSuccess ||
        (e = p->alloc(&p->rc, (size_t)B)) != cudaSuccess)
        return cleanup(cuda_fail(e, "allocate final geometry"));
    e = ffbp::launch_final_geom((const double *)dantf, d->Pf, (const double *)dcenf, B, d->e1, d->e2, p->ux, p->uy,
                                p->ucx, p->ucy, p->rc, s);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "final geometry kernel"));
    if ((d->final_mode & 0xff) == FFBP_FINAL_TC_F16) {
        if ((e = p->alloc(&p->seeds, (size_t)B * d->Pf)) != cudaSuccess) return cleanup(cuda_fail(e, "allocate final seeds"));
        e = ffbp::launch_final_seeds(p->ux, p->uy, (long)B * d->Pf, p->spx, p->spy, p->a0, p->a1, p->seeds, s);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "final seeds kernel"));
    }
    if ((e = p->alloc(&p->d_aborts, 1)) != cudaSuccess || (e = cudaMemsetAsync(p->d_aborts, 0, sizeof(int), s)) != cudaSuccess)
        return cleanup(cuda_fail(e, "allocate the abort count"));
    if ((e = cudaHostAlloc(reinterpret_cast<void **>(&p->h_aborts), sizeof(int), cudaHostAllocDefault)) != cudaSuccess)
        return cleanup(cuda_fail(e, "allocate the abort count"));
    *p->h_aborts = 0;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cleanup(cuda_fail(e, "plan set-up"));
    *out = p;
    return cleanup(FFBP_OK);
}

// How level l runs: 0 the float32 kernel; 1 the one-pass tensor-core kernel (FFBP_LEVELS_TC, a shape it covers,
// FFBP_LEVELS_TC2 not set); 2 the two-pass tensor-core kernels (FFBP_LEVELS_TC2, or a shape only they cover).
static int level_form(const ffbp_plan *p, int l)
{
    if (!(p->final_mode & FFBP_LEVELS_TC)) return 0;
    const DevLevel &v = p->lv[l];
    const int Lk = v.Dk > 1 ? v.Lk : 1, Lp = v.Dp > 1 ? v.Lp : 1;
    if (!(p->final_mode & FFBP_LEVELS_TC2) && ffbp::level_fused_supported(v.C, Lk, v.Dk, Lp, v.Dp)) return 1;
    return ffbp::level_tc_supported(v.C, Lk, v.Dk) ? 2 : 0;
}

// The float16 intermediate of the two-pass tensor-core levels: the largest any of them needs.
static size_t tc_scratch(const ffbp_plan *p)
{
    size_t m = 0;
    for (int l = 0; l < p->nlev; ++l) {
        if (level_form(p, l) != 2) continue;
        const DevLevel &v = p->lv[l];
        m = std::max(m, ffbp::level_tc_scratch_bytes(v.Np, v.C, v.P, v.Ko));
    }
    return m;
}

// Whether any level runs the two-pass kernels, whose intermediate is scaled from the input's largest component
// (the history's is found by a scan ahead of the first level).
static bool any_two_pass(const ffbp_plan *p)
{
    for (int l = 0; l < p->nlev; ++l)
        if (level_form(p, l) == 2) return true;
    return false;
}

int ffbp_plan_workspace_bytes(const ffbp_plan *p, size_t *bytes)
{
    if (!p || !bytes) return fail(FFBP_E_ARG, "null argument");
    *bytes = 256 + align256(p->bufA * sizeof(float2)) + align256(p->bufB * sizeof(float2)) + align256(tc_scratch(p));
    return FFBP_OK;
}

// One form call. When `prof` is given, an event is recorded after every launch (and one before the first):
// prof->kind[i] = FFBP_KIND_* << 8 | level of launch i.
struct FormProfile {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    ~FormProfile() { for (auto &x : ev) cudaEventDestroy(x); }
};

static int form_impl(ffbp_plan *p, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream_, int *h_bad,
                     FormProfile *prof)
{
    if (!p || !d_S || !d_img || !d_ws) return fail(FFBP_E_ARG, "ffbp_form: null argument");
    {
        int dev = -1;
        cudaGetDevice(&dev);
        if (dev != p->device) return fail(FFBP_E_ARG, "the plan lives on device %d, but device %d is current", p->device, dev);
    }
    // an abort of an earlier call that the host has not been told of yet (no wait: the count as last copied back)
    if (int rc = aborted(p, "an earlier form call on this plan")) return rc;
    size_t need;
    ffbp_plan_workspace_bytes(p, &need);
    if (ws_bytes < need) return fail(FFBP_E_WORKSPACE, "workspace of %zu bytes, %zu needed", ws_bytes, need);
    if (((uintptr_t)d_ws & 255) != 0) return fail(FFBP_E_ARG, "workspace must be 256-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    char *ws = static_cast<char *>(d_ws);
    int *bad = reinterpret_cast<int *>(ws);
    float2 *bufA = reinterpret_cast<float2 *>(ws + 256);
    float2 *bufB = reinterpret_cast<float2 *>(ws + 256 + align256(p->bufA * sizeof(float2)));
    void *scratch = ws + 256 + align256(p->bufA * sizeof(float2)) + align256(p->bufB * sizeof(float2));
    // status words: bad[0] the first non-finite pulse (0x7f7f7f7f: none), bad[1] unused, bad[2 + l] the largest
    // |component| of level l's input (float bits; l = nlev: the final stage's). The tensor-core kernels count the
    // bounded waits that ran out in the plan's d_aborts.
    int *amax = bad + 2;
    cudaError_t e = cudaMemsetAsync(bad, 0x7f, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad + 1, 0, (size_t)(p->nlev + 2) * sizeof(int), s);
    if (e != cudaSuccess) return cuda_fail(e, "status reset");
    auto mark = [&](int kind) {
        if (!prof) return;
        cudaEvent_t x;
        cudaEventCreate(&x);
        cudaEventRecord(x, s);
        prof->ev.push_back(x);
        prof->kind.push_back(kind);
    };
    mark(0);
    const float2 *in = static_cast<const float2 *>(d_S);
    if (level_form(p, 0) == 2) {
        if ((e = ffbp::launch_amax(in, (size_t)p->lv[0].P * p->lv[0].K, amax, s)) != cudaSuccess) return cuda_fail(e, "history scan");
        mark(FFBP_KIND_AMAX << 8);
    }
    for (int l = 0; l < p->nlev; ++l) {
        const DevLevel &v = p->lv[l];
        float2 *outp = (l % 2 == 0) ? bufA : bufB;
        ffbp::LevelLaunch L;
        L.x = in; L.phase = v.phase; L.tk = v.tk; L.tp = v.tp;
        L.wp = l == 0 ? p->wp : nullptr; L.wk = l == 0 ? p->wk : nullptr;
        L.out = outp; L.bad = l == 0 ? bad : nullptr;
        L.Np = v.Np; L.C = v.C; L.P = v.P; L.K = v.K; L.Ko = v.Ko; L.Po = v.Po; L.Dk = v.Dk; L.Lk = v.Lk; L.plk = v.plk;
        L.Dp = v.Dp; L.Lp = v.Lp; L.plp = v.plp; L.kc = v.kc;
        L.amax = amax + l + 1;
        L.test_wait_ns = p->test_kind == FFBP_KIND_LEVEL_TC ? p->test_ns : 0u;
        L.tc_nt = v.tc.nt; L.tc_sb = v.tc.sb; L.tc_pc = v.tc.copies; L.tc_rp = v.tc.repeat; L.tc_fir = v.tc.fir;
        L.tc_cw = v.tc.consumers;
        const char *why = nullptr;
        const int form = level_form(p, l);
        if (form == 1) {
            e = ffbp::launch_level_fused(L, p->d_aborts, s, &why);
            if (!why && e == cudaSuccess) mark(FFBP_KIND_LEVEL_TC << 8 | l);
        } else if (form == 2) {
            e = ffbp::launch_level_tc_gemm(L, amax + l, scratch, p->d_aborts, s, &why);
            if (!why && e == cudaSuccess) {
                mark(FFBP_KIND_LEVEL_TC_GEMM << 8 | l);
                e = ffbp::launch_level_tc_fir(L, amax + l, scratch, p->d_aborts, s, &why);
                if (!why && e == cudaSuccess) mark(FFBP_KIND_LEVEL_TC_FIR << 8 | l);
            }
        } else {
            e = ffbp::launch_level(L, s, &why);
            if (!why && e == cudaSuccess) mark(FFBP_KIND_LEVEL << 8 | l);
        }
        if (why) return fail(FFBP_E_UNSUPPORTED, "level %d: %s", l, why);
        if (e != cudaSuccess) return cuda_fail(e, "level kernel");
        in = outp;
    }
    ffbp::FinalLaunch F;
    F.d = in; F.B = p->ntiles; F.Pf = p->Pf; F.Qf = p->Qf; F.T = p->T; F.ux = p->ux; F.uy = p->uy; F.seeds = p->seeds;
    F.spx = p->spx; F.spy = p->spy; F.a0 = p->a0; F.a1 = p->a1; F.fc2 = p->fc2; F.ucx = p->ucx; F.ucy = p->ucy;
    F.rc = p->rc; F.w = p->wf; F.tiles = nullptr; F.img = static_cast<float2 *>(d_img); F.first = p->first;
    F.nx = p->nx; F.ny = p->ny; F.ox = p->ox; F.oy = p->oy; F.scale = 1.f; F.err = p->d_aborts;
    F.amax = amax + p->nlev;
    F.test_wait_ns = p->test_kind == FFBP_KIND_FINAL_TC ? p->test_ns : 0u;
    const int fm = p->final_mode & 0xff;
    const char *why = nullptr;
    e = fm == FFBP_FINAL_FP32 ? ffbp::launch_final_fp32(F, s, &why) : ffbp::launch_final_tc(F, fm, s, &why);
    if (why) return fail(FFBP_E_UNSUPPORTED, "final stage: %s", why);
    if (e != cudaSuccess) return cuda_fail(e, "final kernel");
    mark((fm == FFBP_FINAL_FP32 ? FFBP_KIND_FINAL : FFBP_KIND_FINAL_TC) << 8 | p->nlev);
    // the abort count back to the host once this call's kernels are done (read by the next call, or below)
    if ((e = cudaMemcpyAsync(p->h_aborts, p->d_aborts, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "status read");
    if (prof) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "form");
        if (int rc = aborted(p, "ffbp_form")) return rc;
    }
    if (h_bad) {
        int v = 0;
        if ((e = cudaMemcpyAsync(&v, bad, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_fail(e, "status read");
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "form");
        *h_bad = (v == 0x7f7f7f7f) ? -1 : v;
        if (int rc = aborted(p, "ffbp_form")) return rc;
    }
    return FFBP_OK;
}

int ffbp_plan_host_bytes(const ffbp_plan *p, size_t *bytes)
{
    if (!p || !bytes) return fail(FFBP_E_ARG, "ffbp_plan_host_bytes: null argument");
    *bytes = 2 * align256((size_t)p->lv[0].P * p->lv[0].K * sizeof(float2)) +
             2 * align256((size_t)p->nx * p->ny * sizeof(float2));
    return FFBP_OK;
}

int ffbp_form_host(ffbp_plan *p, const void *const *h_S, void *const *h_img, int n, void *d_stage,
                   size_t stage_bytes, void *d_ws, size_t ws_bytes, void *stream, int *h_bad)
{
    if (!p || !h_S || !h_img || !d_stage || !d_ws || !h_bad || n < 1) return fail(FFBP_E_ARG, "ffbp_form_host: bad arguments");
    for (int i = 0; i < n; ++i)
        if (!h_S[i] || !h_img[i]) return fail(FFBP_E_ARG, "ffbp_form_host: null host buffer %d", i);
    size_t need;
    ffbp_plan_host_bytes(p, &need);
    if (stage_bytes < need) return fail(FFBP_E_WORKSPACE, "staging buffer of %zu bytes, %zu needed", stage_bytes, need);
    if (((uintptr_t)d_stage & 255) != 0) return fail(FFBP_E_ARG, "staging buffer must be 256-byte aligned");
    cudaError_t e = cudaSuccess;
    if (!p->up) {
        if ((e = cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "ffbp_form_host: streams");
        for (int b = 0; b < 2; ++b)
            if ((e = cudaEventCreateWithFlags(&p->ev_up[b], cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&p->ev_formed[b], cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&p->ev_down[b], cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "ffbp_form_host: events");
    }
    if (p->n_status < 2 * n) {
        if (p->h_status) cudaFreeHost(p->h_status);
        p->h_status = nullptr;
        p->n_status = 0;
        if ((e = cudaHostAlloc(reinterpret_cast<void **>(&p->h_status), 2 * (size_t)n * sizeof(int), cudaHostAllocDefault)) != cudaSuccess)
            return cuda_fail(e, "ffbp_form_host: status array");
        p->n_status = 2 * n;
    }
    if (!p->d_check && (e = p->alloc(&p->d_check, 4)) != cudaSuccess) return cuda_fail(e, "ffbp_form_host: check sums");
    if (p->n_check < 2 * n) {
        if (p->h_check) cudaFreeHost(p->h_check);
        p->h_check = nullptr;
        p->n_check = 0;
        if ((e = cudaHostAlloc(reinterpret_cast<void **>(&p->h_check), 2 * (size_t)n * sizeof(double), cudaHostAllocDefault)) != cudaSuccess)
            return cuda_fail(e, "ffbp_form_host: check sums");
        p->n_check = 2 * n;
    }
    const int skip = p->test_skip_upload;
    p->test_skip_upload = -1;
    const int P0 = p->lv[0].P, K0 = p->lv[0].K;
    int crs, cks;
    check_strides(P0, K0, &crs, &cks);
    const int nrows = (P0 + crs - 1) / crs;
    std::vector<double> sent(3 * (size_t)n, 0.0);           // per image: the host's check (re, im) and its scale
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t sb = (size_t)p->lv[0].P * p->lv[0].K * sizeof(float2), ib = (size_t)p->nx * p->ny * sizeof(float2);
    char *st = static_cast<char *>(d_stage);
    void *dS[2] = {st, st + align256(sb)};
    void *dI[2] = {st + 2 * align256(sb), st + 2 * align256(sb) + align256(ib)};
    const int *bad = static_cast<const int *>(d_ws);           // form_impl's status words
    int rc = FFBP_OK;
    // image i: upload on `up` once image i - 2 no longer reads history buffer i % 2; form on `stream` once the upload
    // is done and image i - 2 has left image buffer i % 2; download on `down` once formed. Up to two images are in
    // flight, so the uploads and downloads of one image overlap the formation of its neighbours.
    for (int i = 0; i < n && rc == FFBP_OK; ++i) {
        const int b = i & 1;
        if (i >= 2 && (e = cudaStreamWaitEvent(p->up, p->ev_formed[b], 0)) != cudaSuccess) { rc = cuda_fail(e, "ffbp_form_host"); break; }
        // the upload, then the check of what arrived, computed on the upload stream and copied back
        if ((i != skip && (e = cudaMemcpyAsync(dS[b], h_S[i], sb, cudaMemcpyHostToDevice, p->up)) != cudaSuccess) ||
            (e = cudaMemsetAsync(p->d_check + 2 * b, 0, 2 * sizeof(double), p->up)) != cudaSuccess) { rc = cuda_fail(e, "ffbp_form_host"); break; }
        transfer_check_kernel<<<(nrows + 7) / 8, 256, 0, p->up>>>(static_cast<const float2 *>(dS[b]), P0, K0, crs, cks,
                                                                 p->d_check + 2 * b);
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(p->h_check + 2 * i, p->d_check + 2 * b, 2 * sizeof(double), cudaMemcpyDeviceToHost, p->up)) != cudaSuccess ||
            (e = cudaEventRecord(p->ev_up[b], p->up)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(s, p->ev_up[b], 0)) != cudaSuccess ||
            (i >= 2 && (e = cudaStreamWaitEvent(s, p->ev_down[b], 0)) != cudaSuccess)) { rc = cuda_fail(e, "ffbp_form_host"); break; }
        if ((rc = form_impl(p, dS[b], dI[b], d_ws, ws_bytes, stream, nullptr, nullptr)) != FFBP_OK) break;
        if ((e = cudaMemcpyAsync(p->h_status + 2 * i, bad, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaEventRecord(p->ev_formed[b], s)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(p->down, p->ev_formed[b], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_img[i], dI[b], ib, cudaMemcpyDeviceToHost, p->down)) != cudaSuccess ||
            (e = cudaEventRecord(p->ev_down[b], p->down)) != cudaSuccess) { rc = cuda_fail(e, "ffbp_form_host"); break; }
        // the host side of image i's check, while the device works
        host_check(static_cast<const float2 *>(h_S[i]), P0, K0, &sent[3 * i], &sent[3 * i + 1], &sent[3 * i + 2]);
    }
    // wait for everything queued (the host buffers are in use until then), also after an error
    const cudaError_t e1 = cudaStreamSynchronize(p->up), e2 = cudaStreamSynchronize(s), e3 = cudaStreamSynchronize(p->down);
    if (rc != FFBP_OK) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
        return cuda_fail(e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3, "ffbp_form_host");
    for (int i = 0; i < n; ++i) h_bad[i] = p->h_status[2 * i] == 0x7f7f7f7f ? -1 : p->h_status[2 * i];
    for (int i = 0; i < n; ++i) {
        const double dr = p->h_check[2 * i] - sent[3 * i], di = p->h_check[2 * i + 1] - sent[3 * i + 1];
        if (!(fabs(dr) + fabs(di) <= 1e-9 * sent[3 * i + 2]))
            return fail(FFBP_E_TRANSFER, "ffbp_form_host: history %d did not reach the device as it is in host memory "
                        "(check sums %.9g%+.9gi sent, %.9g%+.9gi received): its image is not to be used", i, sent[3 * i],
                        sent[3 * i + 1], p->h_check[2 * i], p->h_check[2 * i + 1]);
    }
    return aborted(p, "ffbp_form_host");
}

}  // extern "C"

// A batch: the form calls of n plans captured once into a CUDA graph, each plan's launches on a branch of its own
// (forked from and joined to the capturing stream), so that the kernels of different plans run side by side and one
// graph launch replaces them all.
struct ffbp_batch {
    int n = 0;
    std::vector<const int *> status;     // each plan's workspace status word (first non-finite pulse)
    std::vector<ffbp_plan *> plans;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int *h_status = nullptr;             // page-locked, 2 n ints
    ~ffbp_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (h_status) cudaFreeHost(h_status);
    }
};

extern "C" {

int ffbp_batch_create(ffbp_plan *const *plans, int n, const void *const *d_S, void *const *d_img, void *const *d_ws,
                      const size_t *ws_bytes, void *stream, ffbp_batch **out)
{
    if (!plans || !d_S || !d_img || !d_ws || !ws_bytes || !out || n < 1) return fail(FFBP_E_ARG, "ffbp_batch_create: bad arguments");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!plans[i] || !d_S[i] || !d_img[i] || !d_ws[i]) return fail(FFBP_E_ARG, "ffbp_batch_create: null entry %d", i);
        size_t need;
        ffbp_plan_workspace_bytes(plans[i], &need);
        if (ws_bytes[i] < need) return fail(FFBP_E_WORKSPACE, "plan %d: workspace of %zu bytes, %zu needed", i, ws_bytes[i], need);
        if (((uintptr_t)d_ws[i] & 255) != 0) return fail(FFBP_E_ARG, "plan %d: workspace must be 256-byte aligned", i);
    }
    (void)stream;                        // nothing runs here: the graph is captured on a stream of the call's own
    ffbp_batch *b = new ffbp_batch;
    b->n = n;
    cudaStream_t s = nullptr;            // the capturing stream (the legacy default stream cannot capture)
    std::vector<cudaStream_t> br(n, nullptr);
    std::vector<cudaEvent_t> joined(n, nullptr);
    cudaEvent_t fork = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&joined[i], cudaEventDisableTiming);
    }
    auto cleanup = [&]() {
        for (int i = 0; i < n; ++i) {
            if (joined[i]) cudaEventDestroy(joined[i]);
            if (br[i]) cudaStreamDestroy(br[i]);
        }
        if (fork) cudaEventDestroy(fork);
        if (s) cudaStreamDestroy(s);
    };
    if (e != cudaSuccess) { cleanup(); delete b; return cuda_fail(e, "ffbp_batch_create: streams"); }
    int rc = FFBP_OK;
    // capture: relaxed, since the tensor-core launchers set their kernels' shared-memory attribute as they launch
    if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed)) != cudaSuccess) { cleanup(); delete b; return cuda_fail(e, "ffbp_batch_create: capture"); }
    e = cudaEventRecord(fork, s);
    for (int i = 0; i < n && e == cudaSuccess && rc == FFBP_OK; ++i) {
        if ((e = cudaStreamWaitEvent(br[i], fork, 0)) != cudaSuccess) break;
        rc = form_impl(plans[i], d_S[i], d_img[i], d_ws[i], ws_bytes[i], br[i], nullptr, nullptr);
        if (rc != FFBP_OK) break;
        if ((e = cudaEventRecord(joined[i], br[i])) != cudaSuccess) break;
        e = cudaStreamWaitEvent(s, joined[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (rc == FFBP_OK && e == cudaSuccess && e2 == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
    b->graph = g;
    cleanup();
    if (rc != FFBP_OK) { delete b; return rc; }
    if (e != cudaSuccess || e2 != cudaSuccess) { delete b; return cuda_fail(e != cudaSuccess ? e : e2, "ffbp_batch_create: graph"); }
    for (int i = 0; i < n; ++i) {
        b->status.push_back(static_cast<const int *>(d_ws[i]));
        b->plans.push_back(plans[i]);
    }
    if ((e = cudaHostAlloc(reinterpret_cast<void **>(&b->h_status), 2 * (size_t)n * sizeof(int), cudaHostAllocDefault)) != cudaSuccess) {
        delete b;
        return cuda_fail(e, "ffbp_batch_create: status array");
    }
    *out = b;
    return FFBP_OK;
}

int ffbp_batch_form(ffbp_batch *b, void *stream, int *h_bad)
{
    if (!b) return fail(FFBP_E_ARG, "ffbp_batch_form: null batch");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // aborts of earlier launches that the host has not been told of (the counts as last copied back)
    for (int i = 0; i < b->n; ++i)
        if (aborted(b->plans[i], "an earlier batch launch") != FFBP_OK) return fail(FFBP_E_CUDA, "image %d: %s", i, WAIT_MSG);
    cudaError_t e = cudaGraphLaunch(b->exec, s);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_batch_form");
    if (!h_bad) return FFBP_OK;
    for (int i = 0; i < b->n && e == cudaSuccess; ++i)
        e = cudaMemcpyAsync(b->h_status + 2 * i, b->status[i], sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_batch_form");
    for (int i = 0; i < b->n; ++i) h_bad[i] = b->h_status[2 * i] == 0x7f7f7f7f ? -1 : b->h_status[2 * i];
    for (int i = 0; i < b->n; ++i)
        if (aborted(b->plans[i], "ffbp_batch_form") != FFBP_OK) return fail(FFBP_E_CUDA, "image %d: %s", i, WAIT_MSG);
    return FFBP_OK;
}

int ffbp_batch_destroy(ffbp_batch *b)
{
    delete b;
    return FFBP_OK;
}

int ffbp_form(ffbp_plan *p, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream, int *h_bad)
{
    return form_impl(p, d_S, d_img, d_ws, ws_bytes, stream, h_bad, nullptr);
}

int ffbp_plan_check(ffbp_plan *p, void *stream)
{
    if (!p) return fail(FFBP_E_ARG, "ffbp_plan_check: null plan");
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_plan_check");
    return aborted(p, "a form call on this plan");
}

int ffbp_plan_test_transfer(ffbp_plan *p, int image)
{
    if (!p) return fail(FFBP_E_ARG, "ffbp_plan_test_transfer: null plan");
    if (image < -1) return fail(FFBP_E_ARG, "ffbp_plan_test_transfer: image %d < -1", image);
    p->test_skip_upload = image;
    return FFBP_OK;
}

int ffbp_plan_test_wait(ffbp_plan *p, int kind, unsigned limit_us)
{
    if (!p) return fail(FFBP_E_ARG, "ffbp_plan_test_wait: null plan");
    if (kind != 0 && kind != FFBP_KIND_LEVEL_TC_GEMM && kind != FFBP_KIND_LEVEL_TC && kind != FFBP_KIND_FINAL_TC)
        return fail(FFBP_E_ARG, "ffbp_plan_test_wait: kind %d is neither 0, FFBP_KIND_LEVEL_TC, FFBP_KIND_LEVEL_TC_GEMM "
                    "nor FFBP_KIND_FINAL_TC", kind);
    if (kind == FFBP_KIND_LEVEL_TC_GEMM) kind = FFBP_KIND_LEVEL_TC;              // both tensor-core level forms
    if (kind != 0 && (limit_us < 1 || limit_us > 1000000))
        return fail(FFBP_E_ARG, "ffbp_plan_test_wait: limit of %u us outside 1 .. 1000000", limit_us);
    p->test_kind = kind;
    p->test_ns = kind ? limit_us * 1000u : 0u;
    return FFBP_OK;
}

int ffbp_form_timed(ffbp_plan *p, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream,
                    float *h_stage_ms, int n_stage)
{
    if (!h_stage_ms) return fail(FFBP_E_ARG, "ffbp_form_timed: null stage_ms");
    if (!p) return fail(FFBP_E_ARG, "ffbp_form_timed: null plan");
    if (n_stage < p->nlev + 1) return fail(FFBP_E_ARG, "stage_ms holds %d entries, %d needed", n_stage, p->nlev + 1);
    FormProfile prof;
    const int rc = form_impl(p, d_S, d_img, d_ws, ws_bytes, stream, nullptr, &prof);
    if (rc != FFBP_OK) return rc;
    // a stage runs from the event before its first launch to the one after its last (the history scan goes to
    // level 0)
    for (int l = 0; l <= p->nlev; ++l) h_stage_ms[l] = 0.f;
    size_t i0 = 0;
    for (size_t i = 1; i < prof.ev.size(); ++i) {
        const int lv = prof.kind[i] & 0xff, k = prof.kind[i] >> 8;
        const int next = i + 1 < prof.ev.size() ? (prof.kind[i + 1] & 0xff) : -1;
        if (k == FFBP_KIND_AMAX) continue;
        if (next != lv) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, prof.ev[i0], prof.ev[i]);
            h_stage_ms[lv] = ms;
            i0 = i;
        }
    }
    return FFBP_OK;
}

int ffbp_form_profile(ffbp_plan *p, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream,
                      float *h_ms, int *h_kind, int n)
{
    if (!p || !h_ms || !h_kind) return fail(FFBP_E_ARG, "ffbp_form_profile: null argument");
    int nl = 0, nk = 0;
    ffbp_plan_info(p, &nl, &nk);
    if (n < nk) return fail(FFBP_E_ARG, "ffbp_form_profile: %d entries, %d launches", n, nk);
    FormProfile prof;
    const int rc = form_impl(p, d_S, d_img, d_ws, ws_bytes, stream, nullptr, &prof);
    if (rc != FFBP_OK) return rc;
    for (int i = 0; i < n; ++i) { h_ms[i] = 0.f; h_kind[i] = 0; }
    for (size_t i = 1; i < prof.ev.size() && (int)i <= n; ++i) {
        cudaEventElapsedTime(&h_ms[i - 1], prof.ev[i - 1], prof.ev[i]);
        h_kind[i - 1] = prof.kind[i];
    }
    return FFBP_OK;
}

int ffbp_plan_info(const ffbp_plan *p, int *nlev, int *launches)
{
    if (!p) return fail(FFBP_E_ARG, "ffbp_plan_info: null plan");
    if (nlev) *nlev = p->nlev;
    if (launches) {
        int n = 1;
        for (int l = 0; l < p->nlev; ++l) n += level_form(p, l) == 2 ? 2 : 1;
        if (any_two_pass(p) && level_form(p, 0) == 2) n += 1;      // the history scan
        *launches = n;
    }
    return FFBP_OK;
}

int ffbp_level(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk, int plk,
               int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po, const float *d_wp,
               const float *d_wk, void *d_out, int *d_bad, void *stream)
{
    if (!d_x || !d_phase || !d_out) return fail(FFBP_E_ARG, "ffbp_level: null buffer");
    if (Np < 1 || P < 1 || K < 1 || C < 1 || Dk < 1 || Dp < 1 || Ko < 1 || Po < 1) return fail(FFBP_E_ARG, "ffbp_level: non-positive size");
    if ((Dk > 1 && (!d_tk || Lk < 1)) || (Dp > 1 && (!d_tp || Lp < 1))) return fail(FFBP_E_ARG, "ffbp_level: taps missing");
    ffbp::LevelLaunch L;
    L.x = static_cast<const float2 *>(d_x); L.phase = static_cast<const float2 *>(d_phase); L.tk = d_tk; L.tp = d_tp;
    L.wp = d_wp; L.wk = d_wk; L.out = static_cast<float2 *>(d_out); L.bad = d_bad;
    L.Np = Np; L.C = C; L.P = P; L.K = K; L.Ko = Ko; L.Po = Po; L.Dk = Dk; L.Lk = Lk; L.plk = plk; L.Dp = Dp;
    L.Lp = Lp; L.plp = plp; L.kc = kc;
    const char *why = nullptr;
    cudaError_t e = ffbp::launch_level(L, static_cast<cudaStream_t>(stream), &why);
    if (why) return fail(FFBP_E_UNSUPPORTED, "ffbp_level: %s", why);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_level");
    return FFBP_OK;
}

size_t ffbp_level_tc_scratch_bytes(int Np, int C, int P, int Ko)
{
    if (Np < 1 || C < 1 || P < 1 || Ko < 1) return 0;
    return ffbp::level_tc_scratch_bytes(Np, C, P, Ko);
}

int ffbp_level_tc(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk, int plk,
                  int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po, const float *d_wp,
                  const float *d_wk, void *d_out, int *d_bad, void *d_scratch, size_t scratch_bytes, int *d_status,
                  void *stream)
{
    return ffbp_level_tc_ex(d_x, Np, P, K, d_phase, C, d_tk, Lk, plk, Dk, Ko, kc, d_tp, Lp, plp, Dp, Po, d_wp, d_wk,
                            d_out, d_bad, d_scratch, scratch_bytes, d_status, nullptr, stream);
}

int ffbp_level_tc_ex(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk,
                     int plk, int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po,
                     const float *d_wp, const float *d_wk, void *d_out, int *d_bad, void *d_scratch,
                     size_t scratch_bytes, int *d_status, const ffbp_tc_opts *opts, void *stream)
{
    if (!d_x || !d_phase || !d_out || !d_scratch || !d_status) return fail(FFBP_E_ARG, "ffbp_level_tc: null buffer");
    if (Np < 1 || P < 1 || K < 1 || C < 1 || Dk < 1 || Dp < 1 || Ko < 1 || Po < 1) return fail(FFBP_E_ARG, "ffbp_level_tc: non-positive size");
    if ((Dk > 1 && (!d_tk || Lk < 1)) || (Dp > 1 && (!d_tp || Lp < 1))) return fail(FFBP_E_ARG, "ffbp_level_tc: taps missing");
    if (((uintptr_t)d_scratch & 15) != 0) return fail(FFBP_E_ARG, "ffbp_level_tc: scratch must be 16-byte aligned");
    const size_t need = ffbp::level_tc_scratch_bytes(Np, C, P, Ko);
    if (scratch_bytes < need) return fail(FFBP_E_WORKSPACE, "ffbp_level_tc: scratch of %zu bytes, %zu needed", scratch_bytes, need);
    ffbp::LevelLaunch L;
    L.x = static_cast<const float2 *>(d_x); L.phase = static_cast<const float2 *>(d_phase); L.tk = d_tk; L.tp = d_tp;
    L.wp = d_wp; L.wk = d_wk; L.out = static_cast<float2 *>(d_out); L.bad = d_bad;
    L.Np = Np; L.C = C; L.P = P; L.K = K; L.Ko = Ko; L.Po = Po; L.Dk = Dk; L.Lk = Lk; L.plk = plk; L.Dp = Dp;
    L.Lp = Lp; L.plp = plp; L.kc = kc; L.amax = d_status + 2;
    if (opts) {
        L.tc_nt = opts->nt; L.tc_sb = opts->sb; L.tc_pc = opts->copies; L.tc_rp = opts->repeat; L.tc_fir = opts->fir;
        L.tc_cw = opts->consumers;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = ffbp::launch_amax(L.x, (size_t)Np * P * K, d_status + 1, s);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_level_tc");
    const char *why = nullptr;
    e = ffbp::launch_level_tc(L, d_status + 1, d_scratch, d_status, s, &why);
    if (why) return fail(FFBP_E_UNSUPPORTED, "ffbp_level_tc: %s", why);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_level_tc");
    return FFBP_OK;
}

int ffbp_level_fused(const void *d_x, int Np, int P, int K, const void *d_phase, int C, const float *d_tk, int Lk,
                     int plk, int Dk, int Ko, double kc, const float *d_tp, int Lp, int plp, int Dp, int Po,
                     const float *d_wp, const float *d_wk, void *d_out, int *d_bad, int *d_status, void *stream)
{
    if (!d_x || !d_phase || !d_out || !d_status) return fail(FFBP_E_ARG, "ffbp_level_fused: null buffer");
    if (Np < 1 || P < 1 || K < 1 || C < 1 || Dk < 1 || Dp < 1 || Ko < 1 || Po < 1) return fail(FFBP_E_ARG, "ffbp_level_fused: non-positive size");
    if ((Dk > 1 && (!d_tk || Lk < 1)) || (Dp > 1 && (!d_tp || Lp < 1))) return fail(FFBP_E_ARG, "ffbp_level_fused: taps missing");
    ffbp::LevelLaunch L;
    L.x = static_cast<const float2 *>(d_x); L.phase = static_cast<const float2 *>(d_phase); L.tk = d_tk; L.tp = d_tp;
    L.wp = d_wp; L.wk = d_wk; L.out = static_cast<float2 *>(d_out); L.bad = d_bad;
    L.Np = Np; L.C = C; L.P = P; L.K = K; L.Ko = Ko; L.Po = Po; L.Dk = Dk; L.Lk = Lk; L.plk = plk; L.Dp = Dp;
    L.Lp = Lp; L.plp = plp; L.kc = kc; L.amax = d_status + 2;
    const char *why = nullptr;
    cudaError_t e = ffbp::launch_level_fused(L, d_status, static_cast<cudaStream_t>(stream), &why);
    if (why) return fail(FFBP_E_UNSUPPORTED, "ffbp_level_fused: %s", why);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_level_fused");
    return FFBP_OK;
}

int ffbp_exact_pad(const void *d_S, int n, int K, const float *d_wp, const float *d_wk, int nfft, void *d_pad,
                   int *d_bad, int p_off, void *stream)
{
    if (!d_S || !d_pad) return fail(FFBP_E_ARG, "ffbp_exact_pad: null buffer");
    if (n < 0 || K < 2 || nfft < K || p_off < 0) return fail(FFBP_E_ARG, "ffbp_exact_pad: bad sizes");
    cudaError_t e = ffbp::launch_exact_pad(static_cast<const float2 *>(d_S), n, K, d_wp, d_wk, nfft,
                                           static_cast<float2 *>(d_pad), d_bad, p_off, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_exact_pad");
    return FFBP_OK;
}

int ffbp_exact_backproject(const void *d_prof, int n, int nfft, const double *d_ant, const double *d_ref,
                           const double *d_cen, int ntx, int nty, int tx, int ty, int nx, int ny, double spx, double spy,
                           const double *e1, const double *e2, double inv_dr, double kcyc, int cubic, int along1,
                           int *d_err, void *d_out, void *stream)
{
    if (!d_prof || !d_ant || !d_ref || !d_cen || !e1 || !e2 || !d_out)
        return fail(FFBP_E_ARG, "ffbp_exact_backproject: null buffer");
    if (n < 0 || ntx < 1 || nty < 1 || nx < 1 || ny < 1 || (long)ntx * tx < nx || (long)nty * ty < ny ||
        !(inv_dr > 0.0) || !std::isfinite(kcyc))
        return fail(FFBP_E_ARG, "ffbp_exact_backproject: bad sizes");
    const char *why = nullptr;
    cudaError_t e = ffbp::launch_exact_tiles(static_cast<const float2 *>(d_prof), n, nfft, d_ant, d_ref, d_cen, ntx, nty,
                                             tx, ty, nx, ny, spx, spy, e1, e2, inv_dr, kcyc, cubic, along1,
                                             static_cast<float2 *>(d_out), d_err, static_cast<cudaStream_t>(stream),
                                             &why);
    if (why) return fail(FFBP_E_ARG, "ffbp_exact_backproject: %s", why);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_exact_backproject");
    return FFBP_OK;
}

int ffbp_gate_pad(const void *d_S, int n, int K, const float *d_wp, const float *d_wk, int npl, int Kp, void *d_z,
                  int *d_bad, int p_off, void *stream)
{
    if (!d_S || !d_z || n < 0 || K < 1 || npl < 0 || Kp < K + npl || (!d_wp) != (!d_wk) || p_off < 0)
        return fail(FFBP_E_ARG, "ffbp_gate_pad: bad arguments");
    cudaError_t e = ffbp::launch_gate_pad(static_cast<const float2 *>(d_S), n, K, d_wp, d_wk, npl, Kp,
                                          static_cast<float2 *>(d_z), d_bad, p_off, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_gate_pad");
    return FFBP_OK;
}

int ffbp_gate_fold(const void *d_q, int n, int Kp, int N, void *d_u, void *stream)
{
    if (!d_q || !d_u || n < 0 || N < 2 || N > Kp) return fail(FFBP_E_ARG, "ffbp_gate_fold: bad arguments");
    cudaError_t e = ffbp::launch_gate_fold(static_cast<const float2 *>(d_q), n, Kp, N, static_cast<float2 *>(d_u),
                                           static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_gate_fold");
    return FFBP_OK;
}

int ffbp_gate_taper(const void *d_u, int n, int N, int k0, int k1, const float *d_taper, void *d_out, void *stream)
{
    if (!d_u || !d_taper || !d_out || n < 0 || k0 < 0 || k1 <= k0 || k1 > N) return fail(FFBP_E_ARG, "ffbp_gate_taper: bad arguments");
    cudaError_t e = ffbp::launch_gate_taper(static_cast<const float2 *>(d_u), n, N, k0, k1, d_taper,
                                            static_cast<float2 *>(d_out), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_gate_taper");
    return FFBP_OK;
}

int ffbp_mlp_param_count(void) { return ffbp::mlp_param_count(); }

int ffbp_mlp_max_decimation(void) { return ffbp::mlp_max_decimation(); }

size_t ffbp_mlp_work_bytes(int nq) { return nq > 0 ? ffbp::mlp_work_bytes(nq) : 0; }

int ffbp_mlp_taps(const float *d_params, const float *d_x, int nq, float *d_out, void *d_work, void *stream)
{
    if (!d_params || !d_x || !d_out || !d_work || nq < 1) return fail(FFBP_E_ARG, "ffbp_mlp_taps: bad arguments");
    cudaError_t e = ffbp::mlp_taps(d_params, d_x, nq, d_out, static_cast<float *>(d_work), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_mlp_taps");
    return FFBP_OK;
}

static bool mlp_pairs_ok(const float *d_x, int nq, const float *d_prior, float scale, const int *d_inst, int ninst,
                         const double *d_f, const void *d_y, int S)
{
    return d_x && d_prior && d_inst && d_f && d_y && nq >= 1 && ninst >= 1 && ninst <= 65535 && S >= 1 &&
           (long long)ninst * S <= (1LL << 31) && std::isfinite(scale);
}

int ffbp_mlp_grad(const float *d_params, const float *d_x, int nq, const float *d_prior, float scale,
                  const int *d_inst, const float *d_weight, int ninst, const double *d_f, const void *d_y, int S,
                  float *d_grad, float *d_loss, void *d_work, void *stream)
{
    if (!d_params || !d_loss || !d_work || !mlp_pairs_ok(d_x, nq, d_prior, scale, d_inst, ninst, d_f, d_y, S))
        return fail(FFBP_E_ARG, "ffbp_mlp_grad: bad arguments");
    cudaError_t e = ffbp::mlp_grad(d_params, d_x, nq, d_prior, scale, d_inst, d_weight, ninst, d_f, static_cast<const float2 *>(d_y),
                                   S, d_grad, d_loss, static_cast<float *>(d_work), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_mlp_grad");
    return FFBP_OK;
}

int ffbp_mlp_train_step(float *d_params, float *d_adam, const float *d_x, int nq, const float *d_prior, float scale,
                        const int *d_inst, const float *d_weight, int ninst, const double *d_f, const void *d_y, int S,
                        float lr, int t, float *d_loss, void *d_work, void *stream)
{
    if (!d_params || !d_adam || !d_loss || !d_work || t < 1 || !std::isfinite(lr) ||
        !mlp_pairs_ok(d_x, nq, d_prior, scale, d_inst, ninst, d_f, d_y, S))
        return fail(FFBP_E_ARG, "ffbp_mlp_train_step: bad arguments");
    cudaError_t e = ffbp::mlp_train_step(d_params, d_adam, d_x, nq, d_prior, scale, d_inst, d_weight, ninst, d_f,
                                         static_cast<const float2 *>(d_y), S, lr, t, d_loss, static_cast<float *>(d_work),
                                         static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_mlp_train_step");
    return FFBP_OK;
}

int ffbp_phases(const double *d_ant, int P, const double *d_ref, int Np, const double *d_cen, int C,
                const double *d_range, double k0c, double k1, int cancel_free, void *d_phase, void *stream)
{
    if (!d_ant || !d_ref || !d_cen || !d_phase) return fail(FFBP_E_ARG, "ffbp_phases: null buffer");
    if (P < 1 || Np < 1 || C < 1) return fail(FFBP_E_ARG, "ffbp_phases: non-positive size");
    cudaError_t e = ffbp::launch_phases(d_ant, P, d_ref, Np, d_cen, C, d_range, k0c, k1, cancel_free,
                                        static_cast<float2 *>(d_phase), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_phases");
    return FFBP_OK;
}

int ffbp_final(const void *d_d, int B, int Pf, int Qf, int T, const double *d_ux, const double *d_uy, double spx,
               double spy, double a0, double a1, const double *d_ucx, const double *d_ucy, const double *d_rc,
               double fc2, const float *d_w, int mode, void *d_out, void *stream)
{
    if (!d_d || !d_ux || !d_uy || !d_ucx || !d_ucy || !d_rc || !d_out) return fail(FFBP_E_ARG, "ffbp_final: null buffer");
    if (B < 1 || Pf < 1 || Qf < 1) return fail(FFBP_E_ARG, "ffbp_final: non-positive size");
    ffbp::FinalLaunch F;
    F.d = static_cast<const float2 *>(d_d); F.B = B; F.Pf = Pf; F.Qf = Qf; F.T = T; F.ux = d_ux; F.uy = d_uy;
    F.spx = spx; F.spy = spy; F.a0 = a0; F.a1 = a1; F.fc2 = fc2; F.ucx = d_ucx; F.ucy = d_ucy; F.rc = d_rc; F.w = d_w;
    F.tiles = static_cast<float2 *>(d_out); F.img = nullptr; F.first = nullptr; F.nx = F.ny = F.ox = F.oy = 0;
    F.scale = 1.f;
    const char *why = nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = mode == FFBP_FINAL_FP32 ? ffbp::launch_final_fp32(F, s, &why) : ffbp::launch_final_tc(F, mode, s, &why);
    if (why) return fail(FFBP_E_UNSUPPORTED, "ffbp_final: %s", why);
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_final");
    return FFBP_OK;
}

int ffbp_bp_points_f64(const void *d_prof, int P, int nfft, const double *d_tx, const double *d_rcv,
                       const double *d_ref, const double *d_pts, long N, double inv_dr, double kcyc, void *d_out,
                       void *stream)
{
    if (!d_prof || !d_tx || !d_ref || !d_pts || !d_out) return fail(FFBP_E_ARG, "ffbp_bp_points_f64: null buffer");
    if (P < 0 || nfft < 2 || N < 0) return fail(FFBP_E_ARG, "ffbp_bp_points_f64: bad size");
    cudaError_t e = ffbp::launch_bp_points_f64(static_cast<const double2 *>(d_prof), P, nfft, d_tx, d_rcv, d_ref, d_pts,
                                               N, inv_dr, kcyc, static_cast<double2 *>(d_out),
                                               static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_bp_points_f64");
    return FFBP_OK;
}

int ffbp_simulate(const double *d_ant, int P, int K, double fmin, double df, const double *d_pos, const void *d_amp,
                  int N, void *d_S, void *stream)
{
    if (!d_ant || !d_pos || !d_amp || !d_S) return fail(FFBP_E_ARG, "ffbp_simulate: null buffer");
    if (P < 1 || K < 1 || N < 0) return fail(FFBP_E_ARG, "ffbp_simulate: bad size");
    cudaError_t e = ffbp::launch_simulate(d_ant, P, K, fmin, df, d_pos, static_cast<const double2 *>(d_amp), N,
                                          static_cast<float2 *>(d_S), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "ffbp_simulate");
    return FFBP_OK;
}

// ------------------------------------------------------------------------------------------------ stack products
static int image_args(const char *who, const void *p, int n1, int n2)
{
    if (!p) return fail(FFBP_E_ARG, "%s: null buffer", who);
    if (n1 < 1 || n2 < 1) return fail(FFBP_E_ARG, "%s: image of %d x %d pixels", who, n1, n2);
    if ((long long)n1 * n2 >= (1LL << 40)) return fail(FFBP_E_ARG, "%s: image of %d x %d pixels", who, n1, n2);
    return FFBP_OK;
}

static int done(cudaError_t e, const char *who) { return e == cudaSuccess ? FFBP_OK : cuda_fail(e, who); }

int ffbp_box_mean(const void *d_in, int kind, int n1, int n2, int w, int to_db, float *d_out, void *stream)
{
    if (int r = image_args("ffbp_box_mean", d_in, n1, n2)) return r;
    if (!d_out) return fail(FFBP_E_ARG, "ffbp_box_mean: null output");
    if (kind < FFBP_PIX_AS_IS || kind > FFBP_PIX_SQUARE) return fail(FFBP_E_ARG, "ffbp_box_mean: pixel kind %d", kind);
    if (w < 1 || w > 33) return fail(FFBP_E_UNSUPPORTED, "ffbp_box_mean: window %d (1 to 33 pixels)", w);
    return done(ffbp::launch_box_mean(d_in, kind, n1, n2, w, to_db, d_out, static_cast<cudaStream_t>(stream)),
                "ffbp_box_mean");
}

int ffbp_coherence(const void *d_a, const void *d_b, int n1, int n2, int w1, int w2, float *d_out, void *stream)
{
    if (int r = image_args("ffbp_coherence", d_a, n1, n2)) return r;
    if (!d_b || !d_out) return fail(FFBP_E_ARG, "ffbp_coherence: null buffer");
    if (w1 < 1 || w1 > 1024 || w2 < 1 || w2 > 64)
        return fail(FFBP_E_UNSUPPORTED, "ffbp_coherence: window %d x %d (1 to 1024 rows, 1 to 64 columns)", w1, w2);
    return done(ffbp::launch_coherence(static_cast<const float2 *>(d_a), static_cast<const float2 *>(d_b), n1, n2, w1,
                                       w2, d_out, static_cast<cudaStream_t>(stream)),
                "ffbp_coherence");
}

int ffbp_multilook(const void *d_img, const void *d_b, int n1, int n2, int la, int lr, void *d_out, void *stream)
{
    if (int r = image_args("ffbp_multilook", d_img, n1, n2)) return r;
    if (!d_out) return fail(FFBP_E_ARG, "ffbp_multilook: null output");
    if (la < 1 || lr < 1) return fail(FFBP_E_ARG, "ffbp_multilook: looks %d x %d", la, lr);
    return done(ffbp::launch_multilook(static_cast<const float2 *>(d_img), static_cast<const float2 *>(d_b), n1, n2,
                                       la, lr, d_out, static_cast<cudaStream_t>(stream)),
                "ffbp_multilook");
}

int ffbp_mean_add(const void *d_img, int kind, long n, float w, float weight, int first, float *d_sum, float *d_wsum,
                  void *stream)
{
    if (!d_img || !d_sum || !d_wsum) return fail(FFBP_E_ARG, "ffbp_mean_add: null buffer");
    if (n < 0) return fail(FFBP_E_ARG, "ffbp_mean_add: %ld pixels", n);
    if (kind != FFBP_PIX_POWER && kind != FFBP_PIX_SQUARE) return fail(FFBP_E_ARG, "ffbp_mean_add: pixel kind %d", kind);
    return done(ffbp::launch_mean_add(d_img, kind, n, w, weight, first, d_sum, d_wsum, static_cast<cudaStream_t>(stream)),
                "ffbp_mean_add");
}

int ffbp_mean_image(const float *d_sum, const float *d_wsum, long n, float *d_out, void *stream)
{
    if (!d_sum || !d_wsum || !d_out) return fail(FFBP_E_ARG, "ffbp_mean_image: null buffer");
    if (n < 0) return fail(FFBP_E_ARG, "ffbp_mean_image: %ld pixels", n);
    return done(ffbp::launch_mean_image(d_sum, d_wsum, n, d_out, static_cast<cudaStream_t>(stream)), "ffbp_mean_image");
}

int ffbp_tile_stats(const float *d_x, int n1, int n2, int T, float gain, float *d_mean, float *d_var, void *stream)
{
    if (int r = image_args("ffbp_tile_stats", d_x, n1, n2)) return r;
    if (!d_mean || !d_var) return fail(FFBP_E_ARG, "ffbp_tile_stats: null output");
    if (T < 1) return fail(FFBP_E_ARG, "ffbp_tile_stats: tile %d", T);
    if ((long long)(n1 / T) * (n2 / T) >= (1LL << 31) || n1 / T > 65535) return fail(FFBP_E_ARG, "ffbp_tile_stats: too many tiles");
    return done(ffbp::launch_tile_stats(d_x, n1, n2, T, gain, d_mean, d_var, static_cast<cudaStream_t>(stream)),
                "ffbp_tile_stats");
}

int ffbp_cross_spectrum(const void *d_A, const void *d_B, int batch, int m1, int m2h, int nyquist, const float *d_e1,
                        const float *d_e2, void *d_X, double *d_energy, void *stream)
{
    if (int r = image_args("ffbp_cross_spectrum", d_A, m1, m2h)) return r;
    if (!d_B || !d_X || !d_energy || (!d_e1 != !d_e2)) return fail(FFBP_E_ARG, "ffbp_cross_spectrum: null buffer");
    if (batch < 1 || batch > 65535) return fail(FFBP_E_ARG, "ffbp_cross_spectrum: batch of %d", batch);
    return done(ffbp::launch_cross_spectrum(static_cast<const float2 *>(d_A), static_cast<const float2 *>(d_B), batch,
                                            m1, m2h, nyquist, d_e1, d_e2, static_cast<float2 *>(d_X), d_energy,
                                            static_cast<cudaStream_t>(stream)),
                "ffbp_cross_spectrum");
}

int ffbp_window(const float *d_x, int batch, int n1, int n2, const float *d_mean, const float *d_w1, const float *d_w2,
                float *d_out, void *stream)
{
    if (int r = image_args("ffbp_window", d_x, n1, n2)) return r;
    if (!d_mean || !d_w1 || !d_w2 || !d_out) return fail(FFBP_E_ARG, "ffbp_window: null buffer");
    if (batch < 1 || batch > 65535) return fail(FFBP_E_ARG, "ffbp_window: batch of %d", batch);
    return done(ffbp::launch_window(d_x, batch, n1, n2, d_mean, d_w1, d_w2, d_out, static_cast<cudaStream_t>(stream)),
                "ffbp_window");
}

int ffbp_ramp_multiply(void *d_F, int m1, int m2, const void *d_r1, const void *d_r2, void *stream)
{
    if (int r = image_args("ffbp_ramp_multiply", d_F, m1, m2)) return r;
    if (!d_r1 || !d_r2) return fail(FFBP_E_ARG, "ffbp_ramp_multiply: null ramp");
    return done(ffbp::launch_ramp_multiply(static_cast<float2 *>(d_F), m1, m2, static_cast<const float2 *>(d_r1),
                                           static_cast<const float2 *>(d_r2), static_cast<cudaStream_t>(stream)),
                "ffbp_ramp_multiply");
}

int ffbp_mosaic_pad(const void *d_S, long ldS, int rows, int K, int K2, int npl, const double *d_shift, double f0,
                    double df, void *d_out, void *stream)
{
    if (!d_S || !d_out) return fail(FFBP_E_ARG, "ffbp_mosaic_pad: null buffer");
    if (rows < 0 || K < 1 || K2 < 1 || npl < 0 || npl + K > K2 || ldS < K)
        return fail(FFBP_E_ARG, "ffbp_mosaic_pad: %d samples at %d of %d (leading dimension %ld)", K, npl, K2, ldS);
    return done(ffbp::launch_mosaic_pad(static_cast<const float2 *>(d_S), ldS, rows, K, K2, npl, d_shift, f0, df,
                                        static_cast<float2 *>(d_out), static_cast<cudaStream_t>(stream)),
                "ffbp_mosaic_pad");
}

int ffbp_mosaic_gather(const void *d_Q, long ldQ, int rows, int K2, int N, const int *d_m, void *d_u, void *stream)
{
    if (!d_Q || !d_u) return fail(FFBP_E_ARG, "ffbp_mosaic_gather: null buffer");
    if (rows < 0 || K2 < 1 || N < 1 || ldQ < K2)
        return fail(FFBP_E_ARG, "ffbp_mosaic_gather: %d bins of %d (leading dimension %ld)", N, K2, ldQ);
    return done(ffbp::launch_mosaic_gather(static_cast<const float2 *>(d_Q), ldQ, rows, K2, N, d_m,
                                           static_cast<float2 *>(d_u), static_cast<cudaStream_t>(stream)),
                "ffbp_mosaic_gather");
}

int ffbp_mosaic_gate(const void *d_U, long ldU, int rows, int k0, int nk, int N, const double *d_d, const void *d_cph,
                     double scale, const float *d_taper, void *d_out, void *stream)
{
    if (!d_U || !d_taper || !d_out) return fail(FFBP_E_ARG, "ffbp_mosaic_gate: null buffer");
    if (rows < 0 || k0 < 0 || nk < 0 || N < 1 || k0 + nk > ldU)
        return fail(FFBP_E_ARG, "ffbp_mosaic_gate: samples %d .. %d of rows of %ld", k0, k0 + nk, ldU);
    return done(ffbp::launch_mosaic_gate(static_cast<const float2 *>(d_U), ldU, rows, k0, nk, N, d_d,
                                         static_cast<const double2 *>(d_cph), scale, d_taper,
                                         static_cast<float2 *>(d_out), static_cast<cudaStream_t>(stream)),
                "ffbp_mosaic_gate");
}

int ffbp_shift_crop(const void *d_shifted, int ld, const void *d_src, int src_complex, int n1, int n2, int w0, int w1,
                    void *d_out, void *stream)
{
    if (int r = image_args("ffbp_shift_crop", d_src, n1, n2)) return r;
    if (!d_out) return fail(FFBP_E_ARG, "ffbp_shift_crop: null output");
    if (d_shifted && ld < n2) return fail(FFBP_E_ARG, "ffbp_shift_crop: leading dimension %d below %d", ld, n2);
    return done(ffbp::launch_shift_crop(static_cast<const float2 *>(d_shifted), ld, d_src, src_complex, n1, n2, w0, w1,
                                        d_out, static_cast<cudaStream_t>(stream)),
                "ffbp_shift_crop");
}

}  // extern "C"

namespace ffbp {

// ffbp_form on a workspace the caller names, for the entry points of other translation units.
int form_on_workspace(ffbp_plan *p, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream, int *h_bad)
{
    return form_impl(p, d_S, d_img, d_ws, ws_bytes, stream, h_bad, nullptr);
}

int set_error(int code, const char *msg)
{
    return fail(code, "%s", msg);
}

}  // namespace ffbp

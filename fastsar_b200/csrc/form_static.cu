// ffbp_form_static: the form call with its scratch in a fixed device array of this library instead of a workspace
// the caller allocates.
//
// Who needs it: a caller that cannot allocate device memory at the time it forms an image -- a process whose
// device memory is handed out by a pool it does not control, a real-time loop that must not enter the CUDA
// allocator (cudaMalloc can synchronise the device and take milliseconds), or code running where no allocator is
// reachable. Such a caller builds its plan during set-up and then forms images of plans whose workspace fits here.
//
// The scratch is g_static_ws below, FFBP_STATIC_WS_BYTES (64 MiB): every GPU that loads this library holds it
// until the process exits. Host code only sees a stand-in for that array, not a device address, so its device
// address is looked up with cudaGetSymbolAddress once per device, with that device current, on the first call made
// on that device; that first call should therefore come before any stream capture. Every call shares the array
// and it keeps the last call's contents: the form call resets the status word at its start and every level writes
// all of its output before the next level reads it, so nothing else needs clearing. Calls whose work overlaps on the
// GPU (two streams, or two host threads) race on the array and must not be made.
#include <cstdio>
#include <mutex>

#include "../../include/ffbp_b200.h"
#include "kernels.h"

struct ffbp_plan;

namespace ffbp {
int form_on_workspace(ffbp_plan *p, const void *d_S, void *d_img, void *d_ws, size_t ws_bytes, void *stream, int *h_bad);
int set_error(int code, const char *msg);
}  // namespace ffbp

static __device__ __align__(256) unsigned char g_static_ws[FFBP_STATIC_WS_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_lock;
void *g_addr[MAX_DEVICES] = {};

// The device address of g_static_ws on the current device (looked up on first use, with that device current).
int static_workspace(void **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ffbp::set_error(FFBP_E_CUDA, "ffbp_form_static: cudaGetDevice failed");
    if (dev < 0 || dev >= MAX_DEVICES) return ffbp::set_error(FFBP_E_UNSUPPORTED, "ffbp_form_static: device ordinal beyond 64");
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_addr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_static_ws);
        if (e != cudaSuccess || !ptr)
            return ffbp::set_error(FFBP_E_CUDA, "ffbp_form_static: cudaGetSymbolAddress of the static workspace failed");
        g_addr[dev] = ptr;
    }
    *out = g_addr[dev];
    return FFBP_OK;
}

}  // namespace

extern "C" int ffbp_form_static(ffbp_plan *plan, const void *d_S, void *d_img, void *stream, int *h_bad_pulse)
{
    if (!plan || !d_S || !d_img) return ffbp::set_error(FFBP_E_ARG, "ffbp_form_static: null argument");
    size_t need = 0;
    int rc = ffbp_plan_workspace_bytes(plan, &need);
    if (rc != FFBP_OK) return rc;
    if (need > (size_t)FFBP_STATIC_WS_BYTES) {
        char msg[256];
        snprintf(msg, sizeof msg, "ffbp_form_static: the plan needs %zu bytes of workspace, more than the %zu of the "
                 "static workspace; use ffbp_form with a workspace of ffbp_plan_workspace_bytes", need,
                 (size_t)FFBP_STATIC_WS_BYTES);
        return ffbp::set_error(FFBP_E_WORKSPACE, msg);
    }
    void *ws = nullptr;
    if ((rc = static_workspace(&ws)) != FFBP_OK) return rc;
    return ffbp::form_on_workspace(plan, d_S, d_img, ws, (size_t)FFBP_STATIC_WS_BYTES, stream, h_bad_pulse);
}

// pyfwi_gradient_static: a whole gradient evaluation that allocates no
// device memory.
//
// Who needs it: callers that cannot call cudaMalloc themselves -- a host
// program that drives this library from another language without a CUDA
// allocator of its own, or an application whose memory pool owns every
// byte of the device and forbids side allocations.  The regular entry points
// take a caller-allocated workspace; this one uses a fixed array that the
// library itself carries in device memory (PYFWI_STATIC_SCRATCH_BYTES per
// GPU, held by every GPU that loads the library until the process exits).
//
// Contract (also in include/pyfwi_b200.h):
//   * the survey's workspace + traces + residuals must fit the array; larger
//     plans are rejected with PYFWI_E_WORKSPACE and a message giving the
//     bytes needed;
//   * the first call on each device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture on the device.  The address is kept for the
//     life of the process, so the entry point must not be used again after
//     a cudaDeviceReset of that device (the module, and the array with it,
//     would be loaded afresh at another address);
//   * every call on a device reuses the same array and leaves its contents
//     behind; the call clears what must start from zero itself.  Calls whose
//     work overlaps on the GPU (other streams, other host threads) race on
//     the array.
#include "pyfwi_b200.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

// Defined in pyfwi_b200.cu: the message pyfwi_last_error() returns, the
// trace dimensions of a plan, and the notice that its workspace was cleared.
void pyfwi_set_error(const char *msg);
void pyfwi_plan_trace_dims(const pyfwi_plan *p, int *nt_ext, int *ns, int *nr);
void pyfwi_plan_workspace_cleared(pyfwi_plan *p);

namespace {

// The scratch array.  In host code `g_static_scratch` names a host-side
// stand-in, not device memory: its device address comes from
// cudaGetSymbolAddress below and is the only pointer passed to kernels.
static __device__ __align__(256) unsigned char g_static_scratch[PYFWI_STATIC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_lock;
void *g_addr[MAX_DEVICES] = {};

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

// Device address of the array on the current device (looked up once per device).
int scratch_address(void **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        pyfwi_set_error((std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
        return PYFWI_E_CUDA;
    }
    if (dev < 0 || dev >= MAX_DEVICES) {
        pyfwi_set_error("device index out of range");
        return PYFWI_E_INVALID;
    }
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            pyfwi_set_error((std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
            return PYFWI_E_CUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return PYFWI_OK;
}

}  // namespace

extern "C" int pyfwi_gradient_static(pyfwi_plan *plan, const float *vp, const float *vs, const float *rho,
                                     const float *damp_x, const float *damp_z, const float *src_vals, int32_t n_src,
                                     const float *const *observed, int32_t parameterization, float *grad,
                                     double *misfit, void *stream)
{
    if (!plan || !observed || !grad || !misfit) {
        pyfwi_set_error("pyfwi_gradient_static: NULL argument");
        return PYFWI_E_INVALID;
    }
    int nt_ext = 0, ns = 0, nr = 0;
    pyfwi_plan_trace_dims(plan, &nt_ext, &ns, &nr);
    size_t ws_bytes = 0;
    int rc = pyfwi_workspace_size(plan, &ws_bytes);
    if (rc) return rc;
    const size_t comp = (size_t)nt_ext * ns * nr * sizeof(float);
    int n_obs = 0;
    for (int c = 0; c < 5; ++c) n_obs += observed[c] != nullptr;
    // [workspace | traces (5 components) | residuals of the observed
    // components | reduction scratch]
    const size_t o_traces = up256(ws_bytes), o_res = o_traces + up256(5 * comp);
    const size_t o_red = o_res + (size_t)n_obs * up256(comp);
    const size_t need = o_red + up256(PYFWI_REDUCE_SLOTS * sizeof(double));
    if (need > (size_t)PYFWI_STATIC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof msg, "this survey needs %zu bytes of scratch; the library's static array holds %zu "
                 "(use pyfwi_gradient with a workspace, or smaller segment / shot_batch options)",
                 need, (size_t)PYFWI_STATIC_SCRATCH_BYTES);
        pyfwi_set_error(msg);
        return PYFWI_E_WORKSPACE;
    }
    void *base = nullptr;
    rc = scratch_address(&base);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the array holds whatever the previous call (any plan) left: start from zero
    cudaError_t e = cudaMemsetAsync(base, 0, need, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(misfit, 0, sizeof(double), st);
    if (e != cudaSuccess) {
        pyfwi_set_error((std::string("cudaMemsetAsync: ") + cudaGetErrorString(e)).c_str());
        return PYFWI_E_CUDA;
    }
    pyfwi_plan_workspace_cleared(plan);
    char *b = static_cast<char *>(base);
    float *traces = reinterpret_cast<float *>(b + o_traces);
    if ((rc = pyfwi_set_model(plan, base, ws_bytes, vp, vs, rho, damp_x, damp_z, stream))) return rc;
    if ((rc = pyfwi_forward(plan, base, ws_bytes, src_vals, n_src, traces, stream))) return rc;
    const float *res[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int q = 0;
    for (int c = 0; c < 5; ++c) {
        if (!observed[c]) continue;
        float *r = reinterpret_cast<float *>(b + o_res + (size_t)q++ * up256(comp));
        const float *est = reinterpret_cast<const float *>(reinterpret_cast<const char *>(traces) + c * comp);
        if ((rc = pyfwi_l2_residual(est, observed[c], r, (int64_t)nt_ext * ns * nr,
                                    reinterpret_cast<double *>(b + o_red), misfit, stream)))
            return rc;
        res[c] = r;
    }
    return pyfwi_gradient(plan, base, ws_bytes, res, parameterization, grad, nullptr, stream);
}

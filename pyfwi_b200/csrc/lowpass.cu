// Low-pass filtering of trace planes for the multiscale misfit
// (lowpass / adj_lowpass, PyFWI src/PyFWI/fwi_tools.py:1188-1258, applied by
// cost_preparation / adj_cost_preparation, :1153-1273).
//
// The reference pads every trace with 512 zeros, takes its FFT, multiplies
// it by h and by conj(h) (h the frequency response of a Butterworth design)
// and keeps the first nt samples of the real inverse FFT; its "adjoint"
// applies conj(h) and h, the same product.  That operator is linear along
// time, so it is the matrix K[t][s] = g[(t - s) mod (nt + 512)] with g the
// real inverse FFT of conj(h) h: the host builds K once per cutoff and this
// entry point applies it to every trace as a plain FP32 GEMM (cuBLAS, FP32
// arithmetic, no tensor-core rounding).
#include "pyfwi_b200.h"

#include <climits>
#include <cstdio>
#include <cublas_v2.h>
#include <cuda_runtime.h>

void pyfwi_set_error(const char *msg);

namespace {

constexpr int MAX_DEVICES = 64;

int fail(int code, const char *msg)
{
    pyfwi_set_error(msg);
    return code;
}

// One handle per thread and device: a handle binds one stream at a time.
int handle_for_current_device(cublasHandle_t *out)
{
    thread_local cublasHandle_t handles[MAX_DEVICES] = {};
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail(PYFWI_E_CUDA, "pyfwi_lowpass: no current CUDA device");
    if (!handles[dev]) {
        if (cublasCreate(&handles[dev]) != CUBLAS_STATUS_SUCCESS) return fail(PYFWI_E_CUDA, "cublasCreate failed");
        if (cublasSetMathMode(handles[dev], CUBLAS_PEDANTIC_MATH) != CUBLAS_STATUS_SUCCESS)
            return fail(PYFWI_E_CUDA, "cublasSetMathMode failed");
    }
    *out = handles[dev];
    return PYFWI_OK;
}

}  // namespace

extern "C" int pyfwi_lowpass(const float *response, const float *in, float *out, int32_t nt, int64_t ncols,
                             int32_t n_planes, void *stream)
{
    if (!response || !in || !out || nt < 1 || ncols < 0 || n_planes < 0)
        return fail(PYFWI_E_INVALID, "pyfwi_lowpass: bad argument");
    if (ncols > INT_MAX) return fail(PYFWI_E_INVALID, "pyfwi_lowpass: more than 2^31-1 traces per plane");
    const long long plane = (long long)nt * ncols;
    if (out < in + plane * n_planes && in < out + plane * n_planes)
        return fail(PYFWI_E_INVALID, "pyfwi_lowpass: in and out overlap");
    if (ncols == 0 || n_planes == 0) return PYFWI_OK;
    cublasHandle_t h;
    int rc = handle_for_current_device(&h);
    if (rc) return rc;
    if (cublasSetStream(h, static_cast<cudaStream_t>(stream)) != CUBLAS_STATUS_SUCCESS)
        return fail(PYFWI_E_CUDA, "cublasSetStream failed");
    const float one = 1.f, zero = 0.f;
    for (int p = 0; p < n_planes; ++p) {
        // row-major planes [nt][ncols]: out^T = in^T K^T in cuBLAS's column-major terms (K is symmetric)
        cublasStatus_t s = cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)ncols, nt, nt, &one, in + p * plane,
                                       (int)ncols, response, nt, &zero, out + p * plane, (int)ncols);
        if (s != CUBLAS_STATUS_SUCCESS) {
            char msg[96];
            snprintf(msg, sizeof msg, "pyfwi_lowpass: cublasSgemm failed (%d)", (int)s);
            return fail(PYFWI_E_CUDA, msg);
        }
    }
    return PYFWI_OK;
}

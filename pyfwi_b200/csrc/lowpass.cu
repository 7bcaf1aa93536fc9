// Low-pass filtering of trace planes for the multiscale misfit
// (lowpass / adj_lowpass, PyFWI src/PyFWI/fwi_tools.py:1188-1258, applied by
// cost_preparation / adj_cost_preparation, :1153-1273).
//
// The reference pads every trace with 512 zeros, takes its FFT, multiplies
// it by h and by conj(h) (h the frequency response of a Butterworth design)
// and keeps the first nt samples of the real inverse FFT; its "adjoint"
// applies conj(h) and h, the same product.  Along time that is the
// symmetric Toeplitz operator y[t] = sum_s g[|t - s|] x[s] (t, s < nt), g the
// real inverse FFT of conj(h) h on nt + 512 points.  Embedded in a circulant
// of nfft >= 2 nt - 1 points (a power of two) the operator is diagonal in
// Fourier space with a real spectrum C (the response is real and even), so
// each trace is filtered by one forward FFT, a product with C and one inverse
// FFT.  The host builds C (with the 1/nfft of the inverse folded in) and the
// twiddle table once per cutoff.
//
// One CTA filters PAIRS pairs of adjacent traces of one plane: trace 2p goes
// in the real part and trace 2p+1 in the imaginary part of one complex
// signal (C is real and even, so the two stay apart).  Each signal lives in
// shared memory: loaded in bit-reversed order, a radix-2 decimation-in-time
// FFT leaves it in natural order, the product with C, then a radix-2
// decimation-in-frequency inverse FFT (conjugate twiddles) leaves it in
// bit-reversed order, from which the first nt samples are stored.  FP32
// arithmetic throughout.
#include "pyfwi_b200.h"

#include <cuda_runtime.h>

void pyfwi_set_error(const char *msg);

namespace {

constexpr int LOWPASS_THREADS = 512;
constexpr int MAX_SIGNAL = 1 << 14;  // complex points of shared memory per CTA (128 KB)

int fail(int code, const char *msg)
{
    pyfwi_set_error(msg);
    return code;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmulc(float2 a, float2 b)  // a * conj(b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// filter: [0, nfft) the real spectrum C, then nfft/2 twiddles
// exp(-2 pi i j / nfft) as (cos, sin) pairs.
__global__ void __launch_bounds__(LOWPASS_THREADS) lowpass_fft_kernel(const float *filter, int nfft, int logn,
                                                                      int pairs, const float *in, float *out, int nt,
                                                                      long long ncols)
{
    extern __shared__ float2 sig[];  // [pairs][nfft]
    const float *spec = filter;
    const float2 *tw = reinterpret_cast<const float2 *>(filter + nfft);
    const long long plane = (long long)nt * ncols;
    const float *src = in + blockIdx.y * plane;
    float *dst = out + blockIdx.y * plane;
    const long long c0 = (long long)blockIdx.x * 2 * pairs;  // first trace of this CTA
    const int width = 2 * pairs;                             // traces per CTA
    const int total = pairs * nfft;
    const int shift = 32 - logn;

    for (int e = threadIdx.x; e < total; e += blockDim.x) sig[e] = make_float2(0.f, 0.f);
    __syncthreads();
    // rows of `width` adjacent traces: consecutive threads read consecutive columns
    for (int e = threadIdx.x; e < nt * width; e += blockDim.x) {
        const int t = e / width, q = e - t * width;
        if (c0 + q >= ncols) continue;
        const float v = __ldg(src + (long long)t * ncols + c0 + q);
        float2 *slot = &sig[(q >> 1) * nfft + (__brev((unsigned)t) >> shift)];
        if (q & 1)
            slot->y = v;
        else
            slot->x = v;
    }
    __syncthreads();

    const int half_n = nfft >> 1;
    // forward FFT, decimation in time: spans 1, 2, 4, ... nfft/2
    for (int s = 1; s <= logn; ++s) {
        const int half = 1 << (s - 1), step = nfft >> s;
        for (int e = threadIdx.x; e < pairs * half_n; e += blockDim.x) {
            const int p = e / half_n, b = e - p * half_n;
            const int j = b & (half - 1), k = ((b >> (s - 1)) << s) + j;
            float2 *a = sig + p * nfft;
            const float2 u = a[k], v = cmul(a[k + half], __ldg(tw + j * step));
            a[k] = make_float2(u.x + v.x, u.y + v.y);
            a[k + half] = make_float2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
    // the filter: real spectrum, 1/nfft included
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const float c = __ldg(spec + (e & (nfft - 1)));
        sig[e] = make_float2(sig[e].x * c, sig[e].y * c);
    }
    __syncthreads();
    // inverse FFT, decimation in frequency: spans nfft/2, ... 2, 1
    for (int s = logn; s >= 1; --s) {
        const int half = 1 << (s - 1), step = nfft >> s;
        for (int e = threadIdx.x; e < pairs * half_n; e += blockDim.x) {
            const int p = e / half_n, b = e - p * half_n;
            const int j = b & (half - 1), k = ((b >> (s - 1)) << s) + j;
            float2 *a = sig + p * nfft;
            const float2 u = a[k], v = a[k + half];
            a[k] = make_float2(u.x + v.x, u.y + v.y);
            a[k + half] = cmulc(make_float2(u.x - v.x, u.y - v.y), __ldg(tw + j * step));
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < nt * width; e += blockDim.x) {
        const int t = e / width, q = e - t * width;
        if (c0 + q >= ncols) continue;
        const float2 v = sig[(q >> 1) * nfft + (__brev((unsigned)t) >> shift)];
        dst[(long long)t * ncols + c0 + q] = (q & 1) ? v.y : v.x;
    }
}

}  // namespace

extern "C" int pyfwi_lowpass(const float *filter, int32_t nfft, const float *in, float *out, int32_t nt,
                             int64_t ncols, int32_t n_planes, void *stream)
{
    if (!filter || !in || !out || nt < 1 || ncols < 0 || n_planes < 0)
        return fail(PYFWI_E_INVALID, "pyfwi_lowpass: bad argument");
    if (nfft < 2 || (nfft & (nfft - 1)) || nfft > MAX_SIGNAL || nfft < 2 * nt - 1)
        return fail(PYFWI_E_INVALID, "pyfwi_lowpass: nfft must be a power of two with 2*nt - 1 <= nfft <= 16384");
    const long long plane = (long long)nt * ncols;
    if (out < in + plane * n_planes && in < out + plane * n_planes)
        return fail(PYFWI_E_INVALID, "pyfwi_lowpass: in and out overlap");
    if (ncols == 0 || n_planes == 0) return PYFWI_OK;
    if (n_planes > 65535) return fail(PYFWI_E_INVALID, "pyfwi_lowpass: more than 65535 planes");
    int logn = 0;
    while ((1 << logn) < nfft) ++logn;
    // up to 4 pairs (8 adjacent traces, one 32-byte sector per row) while the signals fit
    int pairs = MAX_SIGNAL / nfft;
    if (pairs > 4) pairs = 4;
    const long long ctas = (ncols + 2 * pairs - 1) / (2 * pairs);
    if (ctas > 0x7fffffffLL) return fail(PYFWI_E_INVALID, "pyfwi_lowpass: too many traces per plane");
    const size_t smem = (size_t)pairs * nfft * sizeof(float2);
    // the largest shared-memory request, on the current device (a host call per filtering)
    if (cudaFuncSetAttribute(lowpass_fft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(MAX_SIGNAL * sizeof(float2))) != cudaSuccess)
        return fail(PYFWI_E_CUDA, "pyfwi_lowpass: cudaFuncSetAttribute failed");
    lowpass_fft_kernel<<<dim3((unsigned)ctas, (unsigned)n_planes), LOWPASS_THREADS, smem,
                         static_cast<cudaStream_t>(stream)>>>(filter, nfft, logn, pairs, in, out, nt, ncols);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PYFWI_E_CUDA, cudaGetErrorString(e));
    return PYFWI_OK;
}

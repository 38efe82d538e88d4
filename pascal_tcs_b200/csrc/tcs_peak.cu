// tcs_peak.cu -- device measurements behind the reported numbers:
//  * the FP64 arithmetic peak of the device: the denominator of the FP64-pipe
//    roofline of the line-solver kernels, whose stencil builds and
//    eliminations are FP64 arithmetic at 5-9 FLOP per byte of compulsory HBM
//    traffic (at or above the B200's FP64 ridge point);
//  * the accuracy of the line solver's FP64 reciprocal (qrcp) against the
//    correctly rounded quotient.
#include "tcs_kernels.h"
#include "tcs.h"

#include <vector>

namespace tcs {

// Eight independent FMA chains per thread, ITERS steps each: 16 * ITERS FP64
// FLOP per thread.  x -> x * a + b with |a| < 1 stays bounded.
constexpr int PEAK_ITERS = 2048;

__global__ void __launch_bounds__(256) fp64_fma_kernel(double a, double b, double *out)
{
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = 1e-3 * (threadIdx.x + q);
    for (int it = 0; it < PEAK_ITERS; it++) {
#pragma unroll
        for (int q = 0; q < 8; q++) x[q] = fma(x[q], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; q++) s += x[q];
    if (s == 12345.678) out[0] = s;   // keeps the chains live; never true for these inputs
}

// |qrcp(b) - 1/b| / ulp(1/b) over n values b = +-10^x, x evenly spaced in [-6, 6]
// and both signs; out[i] holds the error of value i in ulps of the correctly
// rounded 1/b.
template <class R>
__global__ void rcp_check_kernel(int n, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = -6.0 + 12.0 * (double)(i >> 1) / (double)((n >> 1) > 1 ? (n >> 1) - 1 : 1);
    const R b = (R)(((i & 1) ? -1.0 : 1.0) * exp10(x));
    const R q = R(1) / b, r = qrcp(b);
    const double ulp = fabs((double)nextafter(q, R(2) * q) - (double)q);
    out[i] = fabs((double)r - (double)q) / ulp;
}

} // namespace tcs

extern "C" int tcs_check_reciprocal(int n, int fp32, double *max_ulp)
{
    using namespace tcs;
    if (!max_ulp || n < 2) return set_error(TCS_ERR_ARG, "tcs_check_reciprocal: need n >= 2 and a result pointer");
    *max_ulp = -1.0;
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * (size_t)n) != cudaSuccess) return set_error(TCS_ERR_NOMEM, "tcs_check_reciprocal: allocation");
    if (fp32) rcp_check_kernel<float><<<(n + 255) / 256, 256>>>(n, d);
    else rcp_check_kernel<double><<<(n + 255) / 256, 256>>>(n, d);
    int rc = record_launch_error("rcp_check") ? TCS_ERR_CUDA : TCS_OK;
    std::vector<double> h(n);
    if (rc == TCS_OK && cudaMemcpy(h.data(), d, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = set_error(TCS_ERR_CUDA, "tcs_check_reciprocal: copy");
    cudaFree(d);
    if (rc == TCS_OK) {
        double m = 0.0;
        for (double v : h) m = v > m ? v : m;
        *max_ulp = m;
    }
    return rc;
}

extern "C" int tcs_measure_fp64_peak(int device, double *tflops)
{
    using namespace tcs;
    if (!tflops) return set_error(TCS_ERR_ARG, "tcs_measure_fp64_peak: null result pointer");
    *tflops = 0.0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();   // leave no error behind for the next launch check
        return set_error(TCS_ERR_ARG, "tcs_measure_fp64_peak: no such device");
    }
    int prev = 0;
    cudaGetDevice(&prev);   // the caller's current device is put back at the end
    if (cudaSetDevice(device) != cudaSuccess) return set_error(TCS_ERR_CUDA, "tcs_measure_fp64_peak: cudaSetDevice failed");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t s = nullptr;
    bool ok = cudaMalloc(&out, sizeof(double)) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
              cudaEventCreate(&e1) == cudaSuccess && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    const int grid = sms * 8, block = 256;
    float best = 0.f;
    for (int rep = 0; ok && rep < 6; rep++) {
        cudaEventRecord(e0, s);
        fp64_fma_kernel<<<grid, block, 0, s>>>(0.999999, 1e-7, out);
        cudaEventRecord(e1, s);
        ok = record_launch_error("fp64_fma") == 0 && cudaEventSynchronize(e1) == cudaSuccess;
        float ms = 0.f;
        if (ok) cudaEventElapsedTime(&ms, e0, e1);
        if (ok && rep > 0 && (best == 0.f || ms < best)) best = ms;   // the first launch warms up
    }
    if (ok && best > 0.f) *tflops = (double)grid * block * 16.0 * PEAK_ITERS / (best * 1e-3) / 1e12;
    if (s) cudaStreamDestroy(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (out) cudaFree(out);
    cudaSetDevice(prev);
    return ok ? TCS_OK : set_error(TCS_ERR_CUDA, "tcs_measure_fp64_peak: the timing kernel failed");
}

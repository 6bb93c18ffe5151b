// FP64 fused multiply-add throughput of the current GPU, measured with CUDA
// events (no counterpart in the reference).  It is the denominator of the
// FP64 roofline fraction the benchmark reports for the propagator sweeps,
// whose FFT work is above B200's HBM ridge point.
//
// Every thread runs eight independent FMA chains a <- a * b + c (b just below
// one, so the values stay bounded); eight CTAs of 256 threads per SM keep
// every FP64 pipe busy.  The sum of the chains is written out so that no
// chain is dead code.
#include <cuda_runtime.h>

#include "polystring_b200.h"
#include "ps_internal.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) dfma_peak_kernel(double* out, int iters, double b, double c) {
    double a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = 1e-3 * (threadIdx.x + j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = fma(a[j], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int fail(int code, const char* msg) {
    ps::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int ps_measure_fp64_peak(double* tflops) {
    if (!tflops) return fail(PS_ERR_INVALID, "ps_measure_fp64_peak: null output");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return fail(PS_ERR_CUDA, "ps_measure_fp64_peak: no device");
    const int threads = 256, blocks = sms * 8, iters = 1 << 15, reps = 5;
    double* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    int rc = PS_OK;
    float ms = 0.f;
    if (cudaMalloc(&out, sizeof(double) * (size_t)blocks * threads) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = fail(PS_ERR_CUDA, "ps_measure_fp64_peak: allocation failed");
    } else {
        for (int w = 0; w < 2; ++w) dfma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.9999999, 1e-7);
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps; ++r) dfma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.9999999, 1e-7);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
            cudaGetLastError() != cudaSuccess)
            rc = fail(PS_ERR_CUDA, "ps_measure_fp64_peak: kernel failed");
        else
            *tflops = 2.0 * kChains * (double)iters * blocks * threads * reps / (ms * 1e-3) / 1e12;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (out) cudaFree(out);
    return rc;
}

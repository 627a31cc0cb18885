// FP64 throughput of the device's CUDA cores, measured by this library's own
// kernel: the denominator of the complex128 tile kernel's FP64 roofline.
//
// Every thread runs eight independent chains of dependent FP64 fused
// multiply-adds (x <- x * a + b with a just below 1, so the values settle and
// never overflow or go subnormal); 2 FLOPs per FMA, timed with CUDA events over
// a grid of several resident blocks per SM.
#include <algorithm>
#include <string>

#include "common.hpp"

namespace dq {
namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;
constexpr int kThreadsPerBlock = 256;

__global__ void __launch_bounds__(kThreadsPerBlock) k_fp64_fma(double* out, double a, double b) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s != s) out[0] = s;  // never true (the chains settle near 1); keeps them live
}

}  // namespace

double fp64_fma_tflops(int device) {
    int prev = 0;
    cudaGetDevice(&prev);
    auto check = [](cudaError_t e, const char* what) {
        if (e != cudaSuccess) fail(kCudaError, std::string(what) + ": " + cudaGetErrorString(e));
    };
    check(cudaSetDevice(device), "cudaSetDevice");
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    const int blocks = std::max(1, sms) * 8;
    cudaStream_t s;
    cudaEvent_t e0, e1;
    double* sink = nullptr;
    check(cudaMalloc(&sink, sizeof(double)), "probe buffer");
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreate(&e0), "cudaEventCreate");
    check(cudaEventCreate(&e1), "cudaEventCreate");
    double best_ms = 1e30;
    for (int rep = 0; rep < 4; rep++) {  // the first launch also warms the clocks
        check(cudaEventRecord(e0, s), "cudaEventRecord");
        k_fp64_fma<<<blocks, kThreadsPerBlock, 0, s>>>(sink, 0.9999999, 1e-7);
        check(cudaGetLastError(), "fp64 probe launch");
        check(cudaEventRecord(e1, s), "cudaEventRecord");
        check(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        if (rep > 0) best_ms = std::min(best_ms, double(ms));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    cudaFree(sink);
    cudaSetDevice(prev);
    const double flops = 2.0 * kChains * double(kIters) * double(blocks) * kThreadsPerBlock;
    return flops / (best_ms * 1e-3) / 1e12;
}

}  // namespace dq

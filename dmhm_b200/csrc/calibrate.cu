// FP64 arithmetic peak of this GPU, measured by the library's own kernels.
//
// The FP64 H x dense product runs on the FP64 tensor cores (mma.sync .f64);
// its roofline needs the throughput those instructions reach on this part
// and clock, which no vendor figure states for the running clock.  Each
// form below keeps eight independent accumulators per thread in registers
// and issues one instruction shape in a loop (no memory traffic inside the
// loop); the result is 2 * m * n * k per MMA (2 per FMA) over the CUDA-event
// time of the launch.  The accumulators are written to a device sink only
// when a run-time flag that is always 0 says so, which keeps the compiler
// from removing the loop without adding stores to it.
//
// Forms: 0 mma.sync m8n8k4 .f64, 1 mma.sync m16n8k4 .f64, 2 m16n8k8 .f64,
// 3 m16n8k16 .f64, 4 scalar fma.rn.f64.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "common.h"
#include "engine.h"

namespace hmb {
namespace {

constexpr int kCalThreads = 256;
constexpr int kCalAcc = 8;

__device__ __forceinline__ void mma_m8n8k4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}
__device__ __forceinline__ void mma_m16n8k4(double (&d)[4], const double (&a)[2], double b) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
        "{%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(b));
}
__device__ __forceinline__ void mma_m16n8k8(double (&d)[4], const double (&a)[4],
                                            const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
__device__ __forceinline__ void mma_m16n8k16(double (&d)[4], const double (&a)[8],
                                             const double (&b)[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, "
        "{%4, %5, %6, %7, %8, %9, %10, %11}, {%12, %13, %14, %15}, {%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
          "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

template <int FORM>
__global__ void __launch_bounds__(kCalThreads)
fp64_peak_kernel(int iters, int write_flag, double* sink) {
    const double seed = 1e-3 * (threadIdx.x + 1);
    double s = 0.0;
    if constexpr (FORM == 0) {
        double d[kCalAcc][2] = {};
        const double a = seed, b = 1.0 - seed;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int q = 0; q < kCalAcc; ++q) mma_m8n8k4(d[q], a, b);
#pragma unroll
        for (int q = 0; q < kCalAcc; ++q) s += d[q][0] + d[q][1];
    } else if constexpr (FORM == 1) {
        double d[kCalAcc][4] = {};
        const double a[2] = {seed, 2.0 * seed};
        const double b = 1.0 - seed;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int q = 0; q < kCalAcc; ++q) mma_m16n8k4(d[q], a, b);
#pragma unroll
        for (int q = 0; q < kCalAcc; ++q) s += d[q][0] + d[q][1] + d[q][2] + d[q][3];
    } else if constexpr (FORM == 2) {
        double d[kCalAcc][4] = {};
        const double a[4] = {seed, 2.0 * seed, 3.0 * seed, 4.0 * seed};
        const double b[2] = {1.0 - seed, 1.0 + seed};
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int q = 0; q < kCalAcc; ++q) mma_m16n8k8(d[q], a, b);
#pragma unroll
        for (int q = 0; q < kCalAcc; ++q) s += d[q][0] + d[q][1] + d[q][2] + d[q][3];
    } else if constexpr (FORM == 3) {
        double d[kCalAcc][4] = {};
        double a[8], b[4];
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = (q + 1) * seed;
#pragma unroll
        for (int q = 0; q < 4; ++q) b[q] = 1.0 - q * seed;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int q = 0; q < kCalAcc; ++q) mma_m16n8k16(d[q], a, b);
#pragma unroll
        for (int q = 0; q < kCalAcc; ++q) s += d[q][0] + d[q][1] + d[q][2] + d[q][3];
    } else {
        double d[kCalAcc];
#pragma unroll
        for (int q = 0; q < kCalAcc; ++q) d[q] = q * seed;
        const double a = 1.0 - seed, b = seed;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int q = 0; q < kCalAcc; ++q) d[q] = fma(d[q], a, b);
#pragma unroll
        for (int q = 0; q < kCalAcc; ++q) s += d[q];
    }
    if (write_flag) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// flops of one instruction of the form, per warp (MMA) or per thread (FMA)
constexpr double form_flops(int form) {
    return form == 0 ? 2.0 * 8 * 8 * 4
         : form == 1 ? 2.0 * 16 * 8 * 4
         : form == 2 ? 2.0 * 16 * 8 * 8
         : form == 3 ? 2.0 * 16 * 8 * 16
                     : 2.0;
}

}  // namespace
}  // namespace hmb

using namespace hmb;

extern "C" int hm_measure_fp64_peak(int device, int form, int iterations, double* tflops,
                                    double* ms) {
    try {
        HMB_REQUIRE(tflops != nullptr, HM_ERR_ARGUMENT, "tflops is NULL");
        HMB_REQUIRE(form >= 0 && form <= 4, HM_ERR_ARGUMENT, "form must be 0..4");
        HMB_REQUIRE(iterations > 0 && iterations <= (1 << 24), HM_ERR_ARGUMENT,
                    "iterations must be in 1..2^24");
        HMB_CUDA(cudaSetDevice(device));
        int sms = 0;
        HMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        const int blocks = sms * 4;   // 32 warps per SM
        cudaStream_t s;
        HMB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        auto launch = [&](int it) {
            g_launches.fetch_add(1, std::memory_order_relaxed);
            switch (form) {
                case 0: fp64_peak_kernel<0><<<blocks, kCalThreads, 0, s>>>(it, 0, nullptr); break;
                case 1: fp64_peak_kernel<1><<<blocks, kCalThreads, 0, s>>>(it, 0, nullptr); break;
                case 2: fp64_peak_kernel<2><<<blocks, kCalThreads, 0, s>>>(it, 0, nullptr); break;
                case 3: fp64_peak_kernel<3><<<blocks, kCalThreads, 0, s>>>(it, 0, nullptr); break;
                default: fp64_peak_kernel<4><<<blocks, kCalThreads, 0, s>>>(it, 0, nullptr); break;
            }
        };
        launch(iterations / 8 + 1);                 // warm-up (clocks, code load)
        cudaEventRecord(e0, s);
        launch(iterations);
        cudaEventRecord(e1, s);
        cudaError_t err = cudaEventSynchronize(e1);
        float t = 0.f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
        if (err == cudaSuccess) err = cudaGetLastError();
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(s);
        HMB_CUDA(err);
        const double per_inst = form_flops(form);
        const double units = form == 4 ? (double)blocks * kCalThreads
                                       : (double)blocks * (kCalThreads / 32);
        const double flops = per_inst * units * kCalAcc * (double)iterations;
        *tflops = flops / (t * 1e-3) / 1e12;
        if (ms) *ms = t;
        return HM_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return HM_ERR_INTERNAL;
    }
}

// Shared device helpers for the tractor_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tractor_b200.h"

#define TB_LOG2E 1.4426950408889634
#define TB_PI 3.14159265358979323846

namespace tb {

// 2^x on the SFU (MUFU.EX2), flushing denormal results to zero.
// exp(e) in FP64 for -50 <= e <= 0 (the Gaussian exponents of the model
// evaluations), relative error below 3e-13: e = k ln 2 + g with k =
// rint(e / ln 2) and |g| <= ln 2 / 2 (|k| <= 73, so k ln 2 rounds to within
// 6e-15), exp(g) by its Taylor series to degree 10 (remainder below
// 0.347^11 / 11! = 2.3e-13) in Horner form, and 2^k written into the
// exponent field (a normal double for k >= -1022).
__device__ __forceinline__ double exp_taylor(double e) {
    const double k = rint(e * 1.4426950408889634);
    const double g = fma(k, -0.6931471805599453, e);
    double p = 1.0 / 3628800.0;
    p = fma(p, g, 1.0 / 362880.0);
    p = fma(p, g, 1.0 / 40320.0);
    p = fma(p, g, 1.0 / 5040.0);
    p = fma(p, g, 1.0 / 720.0);
    p = fma(p, g, 1.0 / 120.0);
    p = fma(p, g, 1.0 / 24.0);
    p = fma(p, g, 1.0 / 6.0);
    p = fma(p, g, 0.5);
    p = fma(p, g, 1.0);
    p = fma(p, g, 1.0);
    const long long bits = (long long)((int)k + 1023) << 52;
    return p * __longlong_as_double(bits);
}

__device__ __forceinline__ float ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Records the first failure of a launch in a device status word.
__device__ __forceinline__ void report(tb_status* st, int code, int item, int detail) {
    if (st == nullptr) return;
    if (atomicCAS(&st->code, 0, code) == 0) {
        st->item = item;
        st->detail = detail;
    }
    atomicAdd(&st->count, 1);
}

// Dynamic work distribution for persistent kernels: thread 0 takes the next
// unit from a global counter and broadcasts it through shared memory.
__device__ __forceinline__ int64_t next_unit(int32_t* counter, int64_t* slot) {
    __syncthreads();
    if (threadIdx.x == 0) *slot = (int64_t)atomicAdd(counter, 1);
    __syncthreads();
    return *slot;
}

inline int num_sms() {
    int n = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

}  // namespace tb

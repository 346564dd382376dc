// Test infrastructure: runs the shared transcendental functions
// (include/phiray_math.h) on the device beside CUDA's own exp2f, log2f,
// sinf, cosf, powf and expf, so a test can check that the device computes
// the same bits as the host build of the header and measure how far both
// are from CUDA's library. Built with the library's flags (no contraction).
#include <cuda_runtime.h>
#include <stdint.h>

#include "phiray_math.h"

__global__ void k_probe(int fn, const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ ours,
                        float* __restrict__ cuda, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float a = x[i], b = y[i];
    float o, c;
    switch (fn) {
        case 0: o = pm_exp2(a); c = exp2f(a); break;
        case 1: o = pm_log2(a); c = log2f(a); break;
        case 2: o = pm_sin(a); c = sinf(a); break;
        case 3: o = pm_cos(a); c = cosf(a); break;
        case 4: o = pm_pow(a, b); c = powf(a, b); break;
        default: o = pm_exp(a); c = expf(a); break;
    }
    ours[i] = o;
    cuda[i] = c;
}

// x, y, ours, cuda: device arrays of n floats. Returns a cudaError_t.
extern "C" int phx_test_math_probe(int fn, const float* x, const float* y, float* ours, float* cuda, int n) {
    if (n <= 0) return 0;
    k_probe<<<(n + 255) / 256, 256>>>(fn, x, y, ours, cuda, n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

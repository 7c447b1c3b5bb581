// g3x_peak.cu -- integer-pipe throughput probe used as the roofline denominator.
//
// The extension's cell recurrence is integer max/add work on the ALU pipe; there is no
// published B200 figure for it, so the library measures it: many independent chains of the
// 3-input DPX maximum (VIMNMX3, one 32-bit op per lane per instruction), enough warps to fill
// every SM, timed with CUDA events.  Result: 32-bit integer ops per second.
#include <cuda_runtime.h>
#include "g3x_internal.h"

namespace g3x {

__global__ void __launch_bounds__(256) int_peak_kernel(const int* __restrict__ in, int* out,
                                                       int iters, int d) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = in[(t * 8 + i) & 255];
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = __vimax3_s32(a[i], a[(i + 1) & 7], d);
        }
    }
    int s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s ^= a[i];
    if (s == 0x7F3A5C11) out[t] = s;   // keeps the chains live; practically never true
}

int measure_int_peak(int device, double* ops_per_s) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return G3X_ERR_CUDA;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    int *in = nullptr, *out = nullptr;
    if (cudaMalloc(&in, 256 * sizeof(int)) != cudaSuccess) return G3X_ERR_NOMEM;
    if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(int)) != cudaSuccess) { cudaFree(in); return G3X_ERR_NOMEM; }
    cudaMemset(in, 1, 256 * sizeof(int));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int rc = G3X_OK;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        int_peak_kernel<<<blocks, threads>>>(in, out, iters, 3);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = G3X_ERR_CUDA; break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;   // first launch is a warm-up
    }
    if (rc == G3X_OK) *ops_per_s = (double)blocks * threads * iters * 32.0 / (best * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(in);
    cudaFree(out);
    return rc;
}

}  // namespace g3x

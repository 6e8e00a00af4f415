// probe.cu -- FP32 FMA throughput probe: the denominator of the forward kernel's
// roofline (the path's bound is FP32 FMA issue, not HBM or tensor cores).  Each thread
// runs 16 independent FFMA chains, so the FMA pipes stay saturated at any occupancy
// above a few warps per scheduler.  FLOPs = blocks * threads * iters * 16 * 2.
#include "bp_kernels.cuh"

namespace mmn {

__global__ void __launch_bounds__(256) fma_probe_kernel(float *out, int iters, float a, float b) {
    float x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = 1.0f + 1e-3f * (float)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += x[k];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace mmn

extern "C" int mmn_fp32_peak_probe(int blocks, int iters, float *out, cudaStream_t stream) {
    if (blocks < 1 || iters < 1) return MMN_ERR_INVALID_ARGUMENT;
    if (!out) return MMN_ERR_NULL_POINTER;
    mmn::fma_probe_kernel<<<blocks, 256, 0, stream>>>(out, iters, 0.99999f, 1e-5f);
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

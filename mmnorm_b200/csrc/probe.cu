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

namespace mmn {

// One warp waits, with the copy pipelines' bounded wait, on the first phase of an mbarrier
// that expects one arrival.  With `arrive` set, lane 0 arrives (no transaction bytes) and
// the phase completes; otherwise nothing arrives, every lane gives up after `limit_ns` and
// MMN_ERR_TIMEOUT lands in the status word.  No copy is ever in flight.
__global__ void __launch_bounds__(32) wait_probe_kernel(int32_t *status, uint64_t limit_ns,
                                                        int arrive) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 0);
    mbar_wait_bounded(&bar, 0, status, limit_ns);
}

}  // namespace mmn

extern "C" int mmn_wait_timeout_probe(uint32_t limit_us, int arrive, void *workspace,
                                      cudaStream_t stream) {
    if (!workspace) return MMN_ERR_NULL_POINTER;
    if (limit_us > 10000000u) return MMN_ERR_INVALID_ARGUMENT;  // at most 10 s
    mmn::wait_probe_kernel<<<1, 32, 0, stream>>>(static_cast<int32_t *>(workspace),
                                                  (uint64_t)limit_us * 1000ull, arrive);
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

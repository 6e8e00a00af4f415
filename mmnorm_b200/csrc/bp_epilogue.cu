// bp_epilogue.cu -- voxel mask and unit normals from the fused (image, vote) output.
//
//   mask(v)  = |I(v)| > filter_percent * max_v |I(v)|      (py_sn_est_gpu.py:326)
//   raw(v)   = Re(conj(I(v)) * W(v)) / |I(v)|              (surface_normal_est.cu:138-144)
//   unit(v)  = raw(v) / |raw(v)|, NaN outside the mask     (image_processor.py:396,
//                                                           py_sn_est_gpu.py:374-376)
//
// Pass 1 reduces max|I| (warp shuffles, then one atomicMax on the float's bit pattern --
// exact and order-independent because |I| >= 0).  Pass 2 is one thread per voxel.
#include "bp_kernels.cuh"

namespace mmn {

__global__ void max_abs_kernel(const float2 *__restrict__ image, int64_t n,
                               unsigned int *__restrict__ max_bits) {
    float m = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float2 c = image[i];
        m = fmaxf(m, sqrtf(c.x * c.x + c.y * c.y));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wm[warp] = m;
    __syncthreads();
    if (warp == 0) {
        m = lane < (int)(blockDim.x >> 5) ? wm[lane] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) atomicMax(max_bits, __float_as_uint(m));
    }
}

__global__ void normals_kernel(const float2 *__restrict__ image, const float2 *__restrict__ vote,
                               int64_t n, float filter_percent,
                               const unsigned int *__restrict__ max_bits,
                               float *__restrict__ normals, uint8_t *__restrict__ mask,
                               float *__restrict__ raw) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const float thr = __uint_as_float(*max_bits) * filter_percent;
    const float2 c = image[v];
    const float mag = sqrtf(c.x * c.x + c.y * c.y);
    const bool in = mag > thr;
    float r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 w = vote[k * n + v];
        r[k] = (c.x * w.x + c.y * w.y) / mag;
    }
    const float nrm = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const float qnan = __int_as_float(0x7fc00000);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (normals) normals[3 * v + k] = in ? r[k] / nrm : qnan;
        if (raw) raw[3 * v + k] = in ? r[k] : qnan;
    }
    if (mask) mask[v] = in ? 1 : 0;
}

cudaError_t launch_max_abs(int64_t nvox, const float2 *image, unsigned int *max_bits,
                           cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(max_bits, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int nt = 256;
    int64_t blocks = (nvox + nt - 1) / nt;
    if (blocks > 4 * sms) blocks = 4 * sms;
    if (blocks < 1) blocks = 1;
    max_abs_kernel<<<(unsigned)blocks, nt, 0, stream>>>(image, nvox, max_bits);
    return cudaGetLastError();
}

cudaError_t launch_normals_from_max(int64_t nvox, const float2 *image, const float2 *vote,
                                    float filter_percent, float *normals, uint8_t *mask,
                                    float *raw, const unsigned int *max_bits,
                                    cudaStream_t stream) {
    const int nt = 256;
    const int64_t b2 = (nvox + nt - 1) / nt;
    normals_kernel<<<(unsigned)b2, nt, 0, stream>>>(image, vote, nvox, filter_percent, max_bits,
                                                    normals, mask, raw);
    return cudaGetLastError();
}

cudaError_t launch_normals(int64_t nvox, const float2 *image, const float2 *vote,
                           float filter_percent, float *normals, uint8_t *mask, float *raw,
                           unsigned int *max_bits, cudaStream_t stream) {
    cudaError_t e = launch_max_abs(nvox, image, max_bits, stream);
    if (e != cudaSuccess) return e;
    return launch_normals_from_max(nvox, image, vote, filter_percent, normals, mask, raw,
                                   max_bits, stream);
}

}  // namespace mmn

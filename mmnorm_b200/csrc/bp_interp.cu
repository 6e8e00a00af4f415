// bp_interp.cu -- interpolated-mode backprojection and normal vote (the reference's
// shipped default, src/utils/params.json:4 "use_interpolated_processing": true).
//
// Per (voxel, virtual antenna) the reference takes ONE sample -- the range-FFT bin
// floor(d/fft_spacing/2) -- and ONE phasor exp(-j*2*pi*d/lambda) evaluated in FP64
// (imaging_gpu.cu:90-105; surface_normal_est.cu:99-124).  These kernels keep that
// arithmetic expression for expression (FP32 distance, FP64 phase and cos/sin, FP32
// accumulation in antenna order), so their outputs reproduce the reference's
// kernels; what changes is the structure around it: the antenna geometry streams
// through shared memory in chunks instead of being re-read from global memory by
// every thread, the measurement gather is a single 8-byte load of the complex bin,
// and the image pass can fuse the vote vector W = sum_i c_i (tx_i + o_i/2 - v).
#include "bp_kernels.cuh"

namespace mmn {

namespace {
constexpr int kInterpThreads = 256;
constexpr int kInterpChunk = 256;  // antennas staged per shared-memory chunk
const double kRefPi = 3.1415926535897932384626433832795028841971693993751058209749445923078164062862089986280348253421170679;

struct RefContrib {
    float sum_r, sum_i;
    bool valid;
};

__device__ __forceinline__ void load_meas(const InterpParams &p, unsigned idx, float &mr,
                                          float &mi) {
    if (p.meas) {
        const float2 m = __ldg(p.meas + idx);
        mr = m.x;
        mi = m.y;
    } else {
        mr = __ldg(p.meas_r + idx);
        mi = __ldg(p.meas_i + idx);
    }
}

// imaging_gpu.cu:70-105 -- the per-antenna contribution, same expressions.
__device__ __forceinline__ RefContrib image_contrib(const InterpParams &p, unsigned i,
                                                    float x_loc, float y_loc, float z_loc,
                                                    float x_antenna_loc, float y_antenna_loc,
                                                    float z_antenna_loc, float rx_offset_x,
                                                    float rx_offset_y, float rx_offset_z) {
    RefContrib r;
    r.valid = false;
    float antenna_x_diff = x_loc - x_antenna_loc;
    float antenna_y_diff = y_loc - y_antenna_loc;
    float antenna_z_diff = z_loc - z_antenna_loc;
    float forward_dist = sqrtf(antenna_x_diff * antenna_x_diff +
                               antenna_y_diff * antenna_y_diff +
                               antenna_z_diff * antenna_z_diff);
    float back_dist = sqrtf((antenna_x_diff - rx_offset_x) * (antenna_x_diff - rx_offset_x) +
                            (antenna_y_diff - rx_offset_y) * (antenna_y_diff - rx_offset_y) +
                            (antenna_z_diff - rx_offset_z) * (antenna_z_diff - rx_offset_z));
    float distance = forward_dist + back_dist;
    if (p.is_ti != 0) {
        distance += 0.15;
    }
    if (distance < 0 || distance > p.fft_spacing * p.nbins) {
        return r;
    }
    int dist_bin = floorf(distance / p.fft_spacing / 2);
    float real_meas, imag_meas;
    load_meas(p, i * p.nbins + dist_bin, real_meas, imag_meas);
    float real_phase = cos(-2 * kRefPi * distance / p.wavelength);
    float imag_phase = sin(-2 * kRefPi * distance / p.wavelength);
    r.sum_r = (real_meas * real_phase - imag_meas * imag_phase);
    r.sum_i = (real_meas * imag_phase + imag_meas * real_phase);
    r.valid = true;
    return r;
}

__device__ __forceinline__ void stage_chunk(const InterpParams &p, int a0, int n, float *sh) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int i = a0 + j;
        const int rx = i % p.num_rx;
        sh[6 * j + 0] = p.ant[3 * i + 0];
        sh[6 * j + 1] = p.ant[3 * i + 1];
        sh[6 * j + 2] = p.ant[3 * i + 2];
        sh[6 * j + 3] = p.rxo[3 * rx + 0];
        sh[6 * j + 4] = p.rxo[3 * rx + 1];
        sh[6 * j + 5] = p.rxo[3 * rx + 2];
    }
}
}  // namespace

// Image pass (cuda_image, interpolated branch), optionally fusing the vote vector.
__global__ void __launch_bounds__(kInterpThreads) interp_image_kernel(const InterpParams p) {
    __shared__ float sh[6 * kInterpChunk];
    const int64_t rel = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ind = rel + p.start;
    const bool active = rel < p.count && ind < p.nvox;
    const int64_t v = active ? ind : 0;
    const int64_t nyz = (int64_t)p.ny * p.nz;
    const int x = (int)(v / nyz);
    const int y = (int)((v - (int64_t)x * nyz) / p.nz);
    const int z = (int)(v - (int64_t)x * nyz - (int64_t)y * p.nz);
    const float x_loc = p.x_locs[x];
    const float y_loc = p.y_locs[y];
    const float z_loc = p.z_locs[z];
    float sum_r = 0;
    float sum_i = 0;
    float w[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_chunk(p, a0, n, sh);
        __syncthreads();
        if (!active) continue;
        for (int j = 0; j < n; ++j) {
            const float *g = sh + 6 * j;
            const RefContrib c = image_contrib(p, (unsigned)(a0 + j), x_loc, y_loc, z_loc, g[0],
                                               g[1], g[2], g[3], g[4], g[5]);
            if (!c.valid) continue;
            sum_r += c.sum_r;
            sum_i += c.sum_i;
            if (p.vote) {
                const float vec_x = (g[0] + g[3] / 2) - x_loc;
                const float vec_y = (g[1] + g[4] / 2) - y_loc;
                const float vec_z = (g[2] + g[5] / 2) - z_loc;
                w[0] = fmaf(c.sum_r, vec_x, w[0]);
                w[1] = fmaf(c.sum_i, vec_x, w[1]);
                w[2] = fmaf(c.sum_r, vec_y, w[2]);
                w[3] = fmaf(c.sum_i, vec_y, w[3]);
                w[4] = fmaf(c.sum_r, vec_z, w[4]);
                w[5] = fmaf(c.sum_i, vec_z, w[5]);
            }
        }
    }
    if (!active) return;
    if (p.out_r) {
        p.out_r[v] = sum_r;
        p.out_i[v] = sum_i;
    }
    if (p.image) p.image[v] = make_float2(sum_r, sum_i);
    if (p.vote) {
        p.vote[v] = make_float2(w[0], w[1]);
        p.vote[p.nvox + v] = make_float2(w[2], w[3]);
        p.vote[2 * p.nvox + v] = make_float2(w[4], w[5]);
    }
}

// Normal pass (cuda_sn_est, surface_normal_est.cu:63-149) over a valid-voxel list.
__global__ void __launch_bounds__(kInterpThreads) interp_normals_kernel(const InterpParams p) {
    __shared__ float sh[6 * kInterpChunk];
    const int64_t rel = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ind64 = rel + p.start;
    const bool active = rel < p.count && ind64 < p.num_valid && ind64 >= 0;
    const int ind = active ? (int)ind64 : 0;
    int x = 0, y = 0, z = 0;
    if (active) {
        x = p.vidx_x[ind];
        y = p.vidx_y[ind];
        z = p.vidx_z[ind];
    }
    const float x_loc = p.x_locs[x];
    const float y_loc = p.y_locs[y];
    const float z_loc = p.z_locs[z];
    const float image_r = active ? p.img_r[x * p.ny * p.nz + y * p.nz + z] : 1.f;
    const float image_i = active ? p.img_i[x * p.ny * p.nz + y * p.nz + z] : 0.f;
    const float image_mag = sqrtf(image_r * image_r + image_i * image_i);
    float sn_x = 0;
    float sn_y = 0;
    float sn_z = 0;
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_chunk(p, a0, n, sh);
        __syncthreads();
        if (!active) continue;
        for (int j = 0; j < n; ++j) {
            const float *g = sh + 6 * j;
            const float x_antenna_loc = g[0], y_antenna_loc = g[1], z_antenna_loc = g[2];
            const float rx_offset_x = g[3], rx_offset_y = g[4], rx_offset_z = g[5];
            const RefContrib c = image_contrib(p, (unsigned)(a0 + j), x_loc, y_loc, z_loc,
                                               x_antenna_loc, y_antenna_loc, z_antenna_loc,
                                               rx_offset_x, rx_offset_y, rx_offset_z);
            if (!c.valid) continue;
            float sum_r = c.sum_r;
            float sum_i = c.sum_i;
            float virtual_antenna_x = x_antenna_loc + rx_offset_x / 2;
            float virtual_antenna_y = y_antenna_loc + rx_offset_y / 2;
            float virtual_antenna_z = z_antenna_loc + rx_offset_z / 2;
            float vec_x = virtual_antenna_x - x_loc;
            float vec_y = virtual_antenna_y - y_loc;
            float vec_z = virtual_antenna_z - z_loc;
            float weight = (sum_r * image_r) + (sum_i * image_i);
            weight /= image_mag;
            sn_x += (vec_x * weight);
            sn_y += (vec_y * weight);
            sn_z += (vec_z * weight);
        }
    }
    if (!active) return;
    p.n_x[ind] = sn_x;
    p.n_y[ind] = sn_y;
    p.n_z[ind] = sn_z;
}

cudaError_t launch_interp_image(const InterpParams &p, cudaStream_t stream) {
    if (p.count <= 0) return cudaSuccess;
    const int64_t blocks = (p.count + kInterpThreads - 1) / kInterpThreads;
    interp_image_kernel<<<(unsigned)blocks, kInterpThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_interp_normals(const InterpParams &p, cudaStream_t stream) {
    if (p.count <= 0) return cudaSuccess;
    const int64_t blocks = (p.count + kInterpThreads - 1) / kInterpThreads;
    interp_normals_kernel<<<(unsigned)blocks, kInterpThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace mmn

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
#include <atomic>

#include "bp_kernels.cuh"

namespace mmn {

// Form of the fast passes: 0 packed voxel pairs (default), 1 scalar.
std::atomic<int> g_interp_fast_form{0};

namespace {
constexpr int kInterpThreads = 256;
constexpr int kInterpChunk = 256;  // antennas staged per shared-memory chunk

struct Contrib {
    float re, im;
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

// One (voxel, virtual antenna) term of imaging_gpu.cu:70-105 with the same floating-point
// operations in the same order (FP32 legs and path, FP64 phase and cos/sin, FP32 complex
// product), so the sums reproduce the reference kernel's bits.
__device__ __forceinline__ Contrib pair_contrib(const InterpParams &p, unsigned i, float vx,
                                                float vy, float vz, float tx, float ty,
                                                float tz, float ox, float oy, float oz) {
    Contrib r;
    r.valid = false;
    float dx = vx - tx;
    float dy = vy - ty;
    float dz = vz - tz;
    float leg_out = sqrtf(dx * dx +
                          dy * dy +
                          dz * dz);
    float leg_back = sqrtf((dx - ox) * (dx - ox) +
                           (dy - oy) * (dy - oy) +
                           (dz - oz) * (dz - oz));
    float path = leg_out + leg_back;
    if (p.is_ti != 0) {
        path += 0.15;
    }
    if (path < 0 || path > p.fft_spacing * p.nbins) {
        return r;
    }
    int bin = floorf(path / p.fft_spacing / 2);
    float m_re, m_im;
    load_meas(p, i * p.nbins + bin, m_re, m_im);
    float ph_re = cos(-2 * kPi * path / p.wavelength);
    float ph_im = sin(-2 * kPi * path / p.wavelength);
    r.re = (m_re * ph_re - m_im * ph_im);
    r.im = (m_re * ph_im + m_im * ph_re);
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
    const float vx = p.x_locs[x];
    const float vy = p.y_locs[y];
    const float vz = p.z_locs[z];
    float acc_re = 0;
    float acc_im = 0;
    float w[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_chunk(p, a0, n, sh);
        __syncthreads();
        if (!active) continue;
        for (int j = 0; j < n; ++j) {
            const float *g = sh + 6 * j;
            const Contrib c = pair_contrib(p, (unsigned)(a0 + j), vx, vy, vz, g[0], g[1], g[2],
                                           g[3], g[4], g[5]);
            if (!c.valid) continue;
            acc_re += c.re;
            acc_im += c.im;
            if (p.vote) {
                const float ex = (g[0] + g[3] / 2) - vx;
                const float ey = (g[1] + g[4] / 2) - vy;
                const float ez = (g[2] + g[5] / 2) - vz;
                w[0] = fmaf(c.re, ex, w[0]);
                w[1] = fmaf(c.im, ex, w[1]);
                w[2] = fmaf(c.re, ey, w[2]);
                w[3] = fmaf(c.im, ey, w[3]);
                w[4] = fmaf(c.re, ez, w[4]);
                w[5] = fmaf(c.im, ez, w[5]);
            }
        }
    }
    if (!active) return;
    if (p.out_r) {
        p.out_r[v] = acc_re;
        p.out_i[v] = acc_im;
    }
    if (p.image) p.image[v] = make_float2(acc_re, acc_im);
    if (p.vote) {
        p.vote[v] = make_float2(w[0], w[1]);
        p.vote[p.nvox + v] = make_float2(w[2], w[3]);
        p.vote[2 * p.nvox + v] = make_float2(w[4], w[5]);
    }
}

// Normal pass (cuda_sn_est, surface_normal_est.cu:63-149) over a valid-voxel list; the
// weight and the virtual-antenna direction use the reference's operations in order.
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
    const float vx = p.x_locs[x];
    const float vy = p.y_locs[y];
    const float vz = p.z_locs[z];
    const float i_re = active ? p.img_r[x * p.ny * p.nz + y * p.nz + z] : 1.f;
    const float i_im = active ? p.img_i[x * p.ny * p.nz + y * p.nz + z] : 0.f;
    const float mag = sqrtf(i_re * i_re + i_im * i_im);
    float acc_x = 0;
    float acc_y = 0;
    float acc_z = 0;
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_chunk(p, a0, n, sh);
        __syncthreads();
        if (!active) continue;
        for (int j = 0; j < n; ++j) {
            const float *g = sh + 6 * j;
            const float tx = g[0], ty = g[1], tz = g[2];
            const float ox = g[3], oy = g[4], oz = g[5];
            const Contrib c = pair_contrib(p, (unsigned)(a0 + j), vx, vy, vz, tx, ty, tz, ox,
                                           oy, oz);
            if (!c.valid) continue;
            float c_re = c.re;
            float c_im = c.im;
            float ux = tx + ox / 2;
            float uy = ty + oy / 2;
            float uz = tz + oz / 2;
            float ex = ux - vx;
            float ey = uy - vy;
            float ez = uz - vz;
            float wgt = (c_re * i_re) + (c_im * i_im);
            wgt /= mag;
            acc_x += (ex * wgt);
            acc_y += (ey * wgt);
            acc_z += (ez * wgt);
        }
    }
    if (!active) return;
    p.n_x[ind] = acc_x;
    p.n_y[ind] = acc_y;
    p.n_z[ind] = acc_z;
}

// ---------------------------------------------------------------------------------
// Fast form.  The path length and the range bin are the reference's (same FP32
// operations, so the same bin is gathered); only the phasor exp(-j 2 pi path/lambda) is
// formed differently: instead of an FP64 cos and sin of the ~1e3-radian phase, the turn
// count path/lambda is formed as a double-float product (1/lambda = hi + lo, both FP32;
// the rounding error of path*hi recovered exactly by an FMA), its integer part removed
// exactly, and the hardware sine/cosine (__sincosf, absolute error about 2^-21.4 on
// [-pi, pi]) evaluated on the wrapped angle.  Phase error ~2e-7 turns + 4e-7 absolute in
// each phasor component: about 5e-7 relative per term against the reference's phasor.
// ---------------------------------------------------------------------------------
namespace {
constexpr int kFastT = 2;                  // voxels per thread
constexpr float kRoundMagic = 12582912.f;  // 1.5 * 2^23: (x + M) - M rounds |x| < 2^22

// Range antenna record of the fast kernels: TX, RX offset and the vote anchor TX + o/2
// (formed in FP32 as surface_normal_est.cu:128-130 does).
struct __align__(16) FastAnt {
    float4 t, o, u;
};

__device__ __forceinline__ void stage_fast_chunk(const InterpParams &p, int a0, int n,
                                                 FastAnt *sh) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int i = a0 + j;
        const int rx = i % p.num_rx;
        const float tx = p.ant[3 * i + 0], ty = p.ant[3 * i + 1], tz = p.ant[3 * i + 2];
        const float ox = p.rxo[3 * rx + 0], oy = p.rxo[3 * rx + 1], oz = p.rxo[3 * rx + 2];
        FastAnt a;
        a.t = make_float4(tx, ty, tz, 0.f);
        a.o = make_float4(ox, oy, oz, 0.f);
        a.u = make_float4(tx + ox / 2, ty + oy / 2, tz + oz / 2, 0.f);
        sh[j] = a;
    }
}

// floor(RN(path / fsp) / 2), the reference's range bin (imaging_gpu.cu:100), for
// 0 <= path <= fsp * nbins.  h = path * (1/(2 fsp)) is within 2e-7 h of the rounded
// quotient's half, so floor(h) is that bin unless h lies within 1.2e-6 h of an integer;
// then the reference's own division decides.  The floor comes from the rounding constant
// (no conversion instruction): bits(h + M) - bits(M) = rint(h) for 0 <= h < 2^22.
__device__ __forceinline__ int fast_bin(float path, float fsp, float half_inv) {
    const float h = path * half_inv;
    const float hm = h + kRoundMagic;
    const float r = hm - kRoundMagic;
    const bool above = r > h;
    const float fr = h - (above ? r - 1.f : r);
    const float tol = fmaxf(h, 1.f) * 1.2e-6f;
    if (fr < tol || fr > 1.f - tol) return (int)floorf(path / fsp / 2);
    return __float_as_int(hm) - __float_as_int(kRoundMagic) - (above ? 1 : 0);
}

// (cos, sin) of -2 pi path / lambda with 1/lambda = hi + lo.
__device__ __forceinline__ void fast_phasor(float path, float hi, float lo, float &c,
                                            float &s) {
    const float q = path * hi;
    const float e = fmaf(path, hi, -q);        // exact: path*hi = q + e
    const float n = (q + kRoundMagic) - kRoundMagic;
    const float f = (q - n) + fmaf(path, lo, e);  // path/lambda - n; |f| <= 0.5 + ulp(q)
    __sincosf(-6.28318530717958647692f * f, &s, &c);
}

template <bool MONO>
__device__ __forceinline__ float2 fast_contrib(const InterpParams &p, size_t row, float vx,
                                               float vy, float vz, const FastAnt &a,
                                               float range_max) {
    const float dx = vx - a.t.x;
    const float dy = vy - a.t.y;
    const float dz = vz - a.t.z;
    const float leg_out = sqrtf(dx * dx +
                                dy * dy +
                                dz * dz);
    float path;
    if (MONO) {
        path = leg_out + leg_out;  // the return leg with a zero offset is the same value
    } else {
        const float leg_back = sqrtf((dx - a.o.x) * (dx - a.o.x) +
                                     (dy - a.o.y) * (dy - a.o.y) +
                                     (dz - a.o.z) * (dz - a.o.z));
        path = leg_out + leg_back;
    }
    if (p.is_ti != 0) {
        path += 0.15;
    }
    const bool valid = !(path < 0 || path > range_max);
    const int bin = valid ? fast_bin(path, p.fft_spacing, p.half_inv_fsp) : 0;
    float m_re, m_im;
    if (p.meas) {
        const float2 m = __ldg(p.meas + row + bin);
        m_re = m.x;
        m_im = m.y;
    } else {
        m_re = __ldg(p.meas_r + row + bin);
        m_im = __ldg(p.meas_i + row + bin);
    }
    float c, s;
    fast_phasor(path, p.inv_lambda_hi, p.inv_lambda_lo, c, s);
    const float re = fmaf(m_re, c, -m_im * s);
    const float im = fmaf(m_re, s, m_im * c);
    return valid ? make_float2(re, im) : make_float2(0.f, 0.f);
}

// Does any staged antenna of this chunk have a non-zero RX offset?  (Uniform per CTA.)
__device__ __forceinline__ bool chunk_has_offsets(const FastAnt *sh, int n) {
    bool any = false;
    for (int j = threadIdx.x; j < n; j += blockDim.x)
        any |= (sh[j].o.x != 0.f) | (sh[j].o.y != 0.f) | (sh[j].o.z != 0.f);
    return __syncthreads_or(any) != 0;
}

template <bool MONO, bool VOTE>
__device__ __forceinline__ void fast_image_chunk(const InterpParams &p, const FastAnt *sh,
                                                 int a0, int n, float range_max,
                                                 const float (&vx)[kFastT],
                                                 const float (&vy)[kFastT],
                                                 const float (&vz)[kFastT],
                                                 float (&acc)[kFastT][8]) {
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        const FastAnt a = sh[j];
        const size_t row = (size_t)(a0 + j) * (size_t)p.nbins;
#pragma unroll
        for (int k = 0; k < kFastT; ++k) {
            const float2 c = fast_contrib<MONO>(p, row, vx[k], vy[k], vz[k], a, range_max);
            acc[k][0] += c.x;
            acc[k][1] += c.y;
            if (VOTE) {
                const float ex = a.u.x - vx[k], ey = a.u.y - vy[k], ez = a.u.z - vz[k];
                acc[k][2] = fmaf(c.x, ex, acc[k][2]);
                acc[k][3] = fmaf(c.y, ex, acc[k][3]);
                acc[k][4] = fmaf(c.x, ey, acc[k][4]);
                acc[k][5] = fmaf(c.y, ey, acc[k][5]);
                acc[k][6] = fmaf(c.x, ez, acc[k][6]);
                acc[k][7] = fmaf(c.y, ez, acc[k][7]);
            }
        }
    }
}
}  // namespace

// Image pass in fast form, kFastT voxels per thread (strided by the block size so loads
// and stores coalesce), optionally fusing the vote vector.
__global__ void __launch_bounds__(kInterpThreads) interp_image_fast_kernel(const InterpParams p) {
    __shared__ FastAnt sh[kInterpChunk];
    const int64_t nyz = (int64_t)p.ny * p.nz;
    const float range_max = p.fft_spacing * p.nbins;
    int64_t vox[kFastT];
    bool active[kFastT];
    float vx[kFastT], vy[kFastT], vz[kFastT];
    float acc[kFastT][8];
#pragma unroll
    for (int k = 0; k < kFastT; ++k) {
        const int64_t rel = ((int64_t)blockIdx.x * kFastT + k) * blockDim.x + threadIdx.x;
        active[k] = rel < p.count && rel + p.start < p.nvox;
        const int64_t v = active[k] ? rel + p.start : 0;
        vox[k] = v;
        const int x = (int)(v / nyz);
        const int y = (int)((v - (int64_t)x * nyz) / p.nz);
        const int z = (int)(v - (int64_t)x * nyz - (int64_t)y * p.nz);
        vx[k] = p.x_locs[x];
        vy[k] = p.y_locs[y];
        vz[k] = p.z_locs[z];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[k][q] = 0.f;
    }
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_fast_chunk(p, a0, n, sh);
        __syncthreads();
        const bool offsets = chunk_has_offsets(sh, n);
        if (p.vote) {
            if (offsets) fast_image_chunk<false, true>(p, sh, a0, n, range_max, vx, vy, vz, acc);
            else fast_image_chunk<true, true>(p, sh, a0, n, range_max, vx, vy, vz, acc);
        } else {
            if (offsets) fast_image_chunk<false, false>(p, sh, a0, n, range_max, vx, vy, vz, acc);
            else fast_image_chunk<true, false>(p, sh, a0, n, range_max, vx, vy, vz, acc);
        }
    }
#pragma unroll
    for (int k = 0; k < kFastT; ++k) {
        if (!active[k]) continue;
        const int64_t v = vox[k];
        if (p.out_r) {
            p.out_r[v] = acc[k][0];
            p.out_i[v] = acc[k][1];
        }
        if (p.image) p.image[v] = make_float2(acc[k][0], acc[k][1]);
        if (p.vote) {
            p.vote[v] = make_float2(acc[k][2], acc[k][3]);
            p.vote[p.nvox + v] = make_float2(acc[k][4], acc[k][5]);
            p.vote[2 * p.nvox + v] = make_float2(acc[k][6], acc[k][7]);
        }
    }
}

// Normal pass in fast form over a valid-voxel list (one voxel per thread).
__global__ void __launch_bounds__(kInterpThreads) interp_normals_fast_kernel(const InterpParams p) {
    __shared__ FastAnt sh[kInterpChunk];
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
    const float vx = p.x_locs[x], vy = p.y_locs[y], vz = p.z_locs[z];
    const int64_t v = ((int64_t)x * p.ny + y) * p.nz + z;
    const float i_re = active ? p.img_r[v] : 1.f;
    const float i_im = active ? p.img_i[v] : 0.f;
    const float inv_mag = 1.f / sqrtf(i_re * i_re + i_im * i_im);
    const float range_max = p.fft_spacing * p.nbins;
    float acc_x = 0.f, acc_y = 0.f, acc_z = 0.f;
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_fast_chunk(p, a0, n, sh);
        __syncthreads();
        const bool offsets = chunk_has_offsets(sh, n);
        if (!active) continue;
#pragma unroll 2
        for (int j = 0; j < n; ++j) {
            const FastAnt a = sh[j];
            const size_t row = (size_t)(a0 + j) * (size_t)p.nbins;
            const float2 c = offsets ? fast_contrib<false>(p, row, vx, vy, vz, a, range_max)
                                     : fast_contrib<true>(p, row, vx, vy, vz, a, range_max);
            const float wgt = fmaf(c.x, i_re, c.y * i_im) * inv_mag;
            acc_x = fmaf(a.u.x - vx, wgt, acc_x);
            acc_y = fmaf(a.u.y - vy, wgt, acc_y);
            acc_z = fmaf(a.u.z - vz, wgt, acc_z);
        }
    }
    if (!active) return;
    p.n_x[ind] = acc_x;
    p.n_y[ind] = acc_y;
    p.n_z[ind] = acc_z;
}

// ---------------------------------------------------------------------------------
// Fast form, packed: each thread's two voxels ride in the two halves of Blackwell's packed
// FP32 instructions (FADD2 / FMUL2 / FFMA2; each half rounds exactly like the scalar
// instruction), so the per-pair arithmetic -- differences, squared range, range bin,
// turn count, complex product, vote -- issues once per voxel pair.  The square roots, the
// sine/cosine and the gathers stay per voxel.  The squared range must reproduce the
// reference's FP32 value bit for bit (its path length selects the bin and sets the phase
// to ~1e-4 rad per ulp): nvcc contracts the reference's dx*dx + dy*dy + dz*dz into
// fma(dz, dz, fma(dx, dx, dy*dy)), which sumsq2 repeats.  (Measured: that order gives the
// bit-exact kernel's bins and phases, 7.5e-7 from it at the 128^3 / 16384-antenna
// workload; the order fma(dz, dz, fma(dy, dy, dx*dx)) is 2.5e-4 away.)
// ---------------------------------------------------------------------------------
namespace {
// Staged antenna of the packed form: values pre-negated and duplicated in both halves, so
// one 16-byte shared load feeds a packed instruction directly.
struct __align__(16) PackAnt {
    float2 ntx, nty, ntz, pad0;  // -TX
    float2 nox, noy, noz, pad1;  // -RX offset
    float2 ux, uy, uz, pad2;     // TX + o/2 (vote anchor)
};

__device__ __forceinline__ float2 dup(float a) { return make_float2(a, a); }

__device__ __forceinline__ void stage_pack_chunk(const InterpParams &p, int a0, int n,
                                                 PackAnt *sh) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int i = a0 + j;
        const int rx = i % p.num_rx;
        const float tx = p.ant[3 * i + 0], ty = p.ant[3 * i + 1], tz = p.ant[3 * i + 2];
        const float ox = p.rxo[3 * rx + 0], oy = p.rxo[3 * rx + 1], oz = p.rxo[3 * rx + 2];
        PackAnt a;
        a.ntx = dup(-tx);
        a.nty = dup(-ty);
        a.ntz = dup(-tz);
        a.nox = dup(-ox);
        a.noy = dup(-oy);
        a.noz = dup(-oz);
        a.ux = dup(tx + ox / 2);
        a.uy = dup(ty + oy / 2);
        a.uz = dup(tz + oz / 2);
        a.pad0 = a.pad1 = a.pad2 = dup(0.f);
        sh[j] = a;
    }
}

__device__ __forceinline__ bool pack_chunk_has_offsets(const PackAnt *sh, int n) {
    bool any = false;
    for (int j = threadIdx.x; j < n; j += blockDim.x)
        any |= (sh[j].nox.x != 0.f) | (sh[j].noy.x != 0.f) | (sh[j].noz.x != 0.f);
    return __syncthreads_or(any) != 0;
}

__device__ __forceinline__ float2 sumsq2(float2 dx, float2 dy, float2 dz) {
    return __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
}

// The two voxels' FP32 path lengths, as imaging_gpu.cu:70-89 forms them.
template <bool MONO>
__device__ __forceinline__ float2 path2(float2 vx, float2 vy, float2 vz, const PackAnt &a,
                                        bool ti) {
    const float2 dx = __fadd2_rn(vx, a.ntx);
    const float2 dy = __fadd2_rn(vy, a.nty);
    const float2 dz = __fadd2_rn(vz, a.ntz);
    const float2 s = sumsq2(dx, dy, dz);
    const float2 leg = make_float2(sqrtf(s.x), sqrtf(s.y));
    float2 path;
    if (MONO) {
        path = __fadd2_rn(leg, leg);
    } else {
        const float2 bx = __fadd2_rn(dx, a.nox);
        const float2 by = __fadd2_rn(dy, a.noy);
        const float2 bz = __fadd2_rn(dz, a.noz);
        const float2 sb = sumsq2(bx, by, bz);
        path = __fadd2_rn(leg, make_float2(sqrtf(sb.x), sqrtf(sb.y)));
    }
    if (ti) {  // float += double, as the reference adds its 0.15 m
        path.x += 0.15;
        path.y += 0.15;
    }
    return path;
}

// fast_bin for two paths (the arithmetic packed, the rare division fallback per voxel).
__device__ __forceinline__ int2 bin2(float2 path, float fsp, float half_inv) {
    const float2 h = __fmul2_rn(path, dup(half_inv));
    const float2 hm = __fadd2_rn(h, dup(kRoundMagic));
    const float2 r = __fadd2_rn(hm, dup(-kRoundMagic));
    const bool ax = r.x > h.x, ay = r.y > h.y;
    const float2 fr = __fadd2_rn(__fadd2_rn(h, make_float2(-r.x, -r.y)),
                                 make_float2(ax ? 1.f : 0.f, ay ? 1.f : 0.f));
    const float2 tol = __fmul2_rn(make_float2(fmaxf(h.x, 1.f), fmaxf(h.y, 1.f)), dup(1.2e-6f));
    int2 b = make_int2(__float_as_int(hm.x) - __float_as_int(kRoundMagic) - (ax ? 1 : 0),
                       __float_as_int(hm.y) - __float_as_int(kRoundMagic) - (ay ? 1 : 0));
    if (fr.x < tol.x || fr.x > 1.f - tol.x) b.x = (int)floorf(path.x / fsp / 2);
    if (fr.y < tol.y || fr.y > 1.f - tol.y) b.y = (int)floorf(path.y / fsp / 2);
    return b;
}

// fast_phasor for two paths: returns (cos, sin) of -2 pi path / lambda per half.
__device__ __forceinline__ void phasor2(float2 path, float hi, float lo, float2 &c,
                                        float2 &s) {
    const float2 qn = __fmul2_rn(path, dup(-hi));               // -q
    const float2 e = __ffma2_rn(path, dup(hi), qn);             // path*hi - q, exact
    const float2 nn = __fadd2_rn(__fadd2_rn(qn, dup(kRoundMagic)), dup(-kRoundMagic));  // -n
    const float2 g = __ffma2_rn(nn, dup(-1.f), qn);             // -(q - n), exact
    const float2 w = __ffma2_rn(path, dup(lo), e);              // path*lo + e
    const float2 f = __ffma2_rn(g, dup(-1.f), w);               // (q - n) + w
    const float2 ang = __fmul2_rn(f, dup(-6.28318530717958647692f));
    __sincosf(ang.x, &s.x, &c.x);
    __sincosf(ang.y, &s.y, &c.y);
}

template <bool MONO, bool VOTE, bool SOA>
__device__ __forceinline__ void pack_image_chunk(const InterpParams &p, const PackAnt *sh,
                                                 int a0, int n, float range_max, bool ti,
                                                 float2 vx, float2 vy, float2 vz, float2 nvx,
                                                 float2 nvy, float2 nvz, float2 (&acc)[8]) {
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        const PackAnt &a = sh[j];
        const size_t row = (size_t)(a0 + j) * (size_t)p.nbins;
        const float2 path = path2<MONO>(vx, vy, vz, a, ti);
        const bool v0 = !(path.x < 0 || path.x > range_max);
        const bool v1 = !(path.y < 0 || path.y > range_max);
        int2 b = bin2(path, p.fft_spacing, p.half_inv_fsp);
        b.x = v0 ? b.x : 0;
        b.y = v1 ? b.y : 0;
        float2 mre, mim;
        if (SOA) {
            mre = make_float2(__ldg(p.meas_r + row + b.x), __ldg(p.meas_r + row + b.y));
            mim = make_float2(__ldg(p.meas_i + row + b.x), __ldg(p.meas_i + row + b.y));
        } else {
            const float2 m0 = __ldg(p.meas + row + b.x), m1 = __ldg(p.meas + row + b.y);
            mre = make_float2(m0.x, m1.x);
            mim = make_float2(m0.y, m1.y);
        }
        float2 c, s;
        phasor2(path, p.inv_lambda_hi, p.inv_lambda_lo, c, s);
        float2 re = __ffma2_rn(mre, c, __fmul2_rn(mim, make_float2(-s.x, -s.y)));
        float2 im = __ffma2_rn(mre, s, __fmul2_rn(mim, c));
        re = make_float2(v0 ? re.x : 0.f, v1 ? re.y : 0.f);
        im = make_float2(v0 ? im.x : 0.f, v1 ? im.y : 0.f);
        acc[0] = __fadd2_rn(acc[0], re);
        acc[1] = __fadd2_rn(acc[1], im);
        if (VOTE) {
            const float2 ex = __fadd2_rn(a.ux, nvx);
            const float2 ey = __fadd2_rn(a.uy, nvy);
            const float2 ez = __fadd2_rn(a.uz, nvz);
            acc[2] = __ffma2_rn(re, ex, acc[2]);
            acc[3] = __ffma2_rn(im, ex, acc[3]);
            acc[4] = __ffma2_rn(re, ey, acc[4]);
            acc[5] = __ffma2_rn(im, ey, acc[5]);
            acc[6] = __ffma2_rn(re, ez, acc[6]);
            acc[7] = __ffma2_rn(im, ez, acc[7]);
        }
    }
}

template <bool VOTE, bool SOA>
__device__ __forceinline__ void pack_image_dispatch(const InterpParams &p, const PackAnt *sh,
                                                    int a0, int n, float range_max, bool ti,
                                                    bool offsets, float2 vx, float2 vy,
                                                    float2 vz, float2 nvx, float2 nvy,
                                                    float2 nvz, float2 (&acc)[8]) {
    if (offsets)
        pack_image_chunk<false, VOTE, SOA>(p, sh, a0, n, range_max, ti, vx, vy, vz, nvx,
                                                  nvy, nvz, acc);
    else
        pack_image_chunk<true, VOTE, SOA>(p, sh, a0, n, range_max, ti, vx, vy, vz, nvx,
                                                 nvy, nvz, acc);
}
}  // namespace

// Image pass in packed fast form: voxels rel and rel + blockDim of each 2*blockDim tile
// (coalesced stores), optionally fusing the vote vector.
__global__ void __launch_bounds__(kInterpThreads) interp_image_pack_kernel(const InterpParams p) {
    __shared__ PackAnt sh[kInterpChunk];
    const int64_t nyz = (int64_t)p.ny * p.nz;
    const float range_max = p.fft_spacing * p.nbins;
    const bool ti = p.is_ti != 0;
    int64_t vox[2];
    bool active[2];
    float px[2], py[2], pz[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int64_t rel = ((int64_t)blockIdx.x * 2 + k) * blockDim.x + threadIdx.x;
        active[k] = rel < p.count && rel + p.start < p.nvox;
        const int64_t v = active[k] ? rel + p.start : 0;
        vox[k] = v;
        const int x = (int)(v / nyz);
        const int y = (int)((v - (int64_t)x * nyz) / p.nz);
        const int z = (int)(v - (int64_t)x * nyz - (int64_t)y * p.nz);
        px[k] = p.x_locs[x];
        py[k] = p.y_locs[y];
        pz[k] = p.z_locs[z];
    }
    const float2 vx = make_float2(px[0], px[1]), vy = make_float2(py[0], py[1]),
                 vz = make_float2(pz[0], pz[1]);
    const float2 nvx = make_float2(-px[0], -px[1]), nvy = make_float2(-py[0], -py[1]),
                 nvz = make_float2(-pz[0], -pz[1]);
    float2 acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = dup(0.f);
    const bool soa = p.meas == nullptr;
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_pack_chunk(p, a0, n, sh);
        __syncthreads();
        const bool offsets = pack_chunk_has_offsets(sh, n);
        if (p.vote) {
            if (soa) pack_image_dispatch<true, true>(p, sh, a0, n, range_max, ti, offsets,
                                                            vx, vy, vz, nvx, nvy, nvz, acc);
            else pack_image_dispatch<true, false>(p, sh, a0, n, range_max, ti, offsets,
                                                         vx, vy, vz, nvx, nvy, nvz, acc);
        } else {
            if (soa) pack_image_dispatch<false, true>(p, sh, a0, n, range_max, ti,
                                                             offsets, vx, vy, vz, nvx, nvy, nvz,
                                                             acc);
            else pack_image_dispatch<false, false>(p, sh, a0, n, range_max, ti, offsets,
                                                          vx, vy, vz, nvx, nvy, nvz, acc);
        }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (!active[k]) continue;
        const int64_t v = vox[k];
        const float re = k ? acc[0].y : acc[0].x, im = k ? acc[1].y : acc[1].x;
        if (p.out_r) {
            p.out_r[v] = re;
            p.out_i[v] = im;
        }
        if (p.image) p.image[v] = make_float2(re, im);
        if (p.vote) {
            p.vote[v] = make_float2(k ? acc[2].y : acc[2].x, k ? acc[3].y : acc[3].x);
            p.vote[p.nvox + v] = make_float2(k ? acc[4].y : acc[4].x, k ? acc[5].y : acc[5].x);
            p.vote[2 * p.nvox + v] = make_float2(k ? acc[6].y : acc[6].x,
                                                 k ? acc[7].y : acc[7].x);
        }
    }
}

namespace {
template <bool MONO, bool SOA>
__device__ __forceinline__ void pack_normals_chunk(const InterpParams &p, const PackAnt *sh,
                                                   int a0, int n, float range_max, bool ti,
                                                   float2 vx, float2 vy, float2 vz, float2 nvx,
                                                   float2 nvy, float2 nvz, float2 ire,
                                                   float2 iim, float2 inv_mag,
                                                   float2 (&acc)[3]) {
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        const PackAnt &a = sh[j];
        const size_t row = (size_t)(a0 + j) * (size_t)p.nbins;
        const float2 path = path2<MONO>(vx, vy, vz, a, ti);
        const bool v0 = !(path.x < 0 || path.x > range_max);
        const bool v1 = !(path.y < 0 || path.y > range_max);
        int2 b = bin2(path, p.fft_spacing, p.half_inv_fsp);
        b.x = v0 ? b.x : 0;
        b.y = v1 ? b.y : 0;
        float2 mre, mim;
        if (SOA) {
            mre = make_float2(__ldg(p.meas_r + row + b.x), __ldg(p.meas_r + row + b.y));
            mim = make_float2(__ldg(p.meas_i + row + b.x), __ldg(p.meas_i + row + b.y));
        } else {
            const float2 m0 = __ldg(p.meas + row + b.x), m1 = __ldg(p.meas + row + b.y);
            mre = make_float2(m0.x, m1.x);
            mim = make_float2(m0.y, m1.y);
        }
        float2 c, s;
        phasor2(path, p.inv_lambda_hi, p.inv_lambda_lo, c, s);
        const float2 re = __ffma2_rn(mre, c, __fmul2_rn(mim, make_float2(-s.x, -s.y)));
        const float2 im = __ffma2_rn(mre, s, __fmul2_rn(mim, c));
        // weight Re(c conj(I)) / |I| (surface_normal_est.cu:138-139); zero for a skipped pair
        float2 w = __fmul2_rn(__ffma2_rn(re, ire, __fmul2_rn(im, iim)), inv_mag);
        w = make_float2(v0 ? w.x : 0.f, v1 ? w.y : 0.f);
        acc[0] = __ffma2_rn(__fadd2_rn(a.ux, nvx), w, acc[0]);
        acc[1] = __ffma2_rn(__fadd2_rn(a.uy, nvy), w, acc[1]);
        acc[2] = __ffma2_rn(__fadd2_rn(a.uz, nvz), w, acc[2]);
    }
}
}  // namespace

// Normal pass in packed fast form over a valid-voxel list: entries ind and ind + blockDim
// of each 2*blockDim tile per thread.
__global__ void __launch_bounds__(kInterpThreads) interp_normals_pack_kernel(const InterpParams p) {
    __shared__ PackAnt sh[kInterpChunk];
    const float range_max = p.fft_spacing * p.nbins;
    const bool ti = p.is_ti != 0;
    int ind[2];
    bool active[2];
    float px[2], py[2], pz[2], pr[2], pi[2], pm[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int64_t rel = ((int64_t)blockIdx.x * 2 + k) * blockDim.x + threadIdx.x;
        const int64_t i64 = rel + p.start;
        active[k] = rel < p.count && i64 < p.num_valid && i64 >= 0;
        ind[k] = active[k] ? (int)i64 : 0;
        int x = 0, y = 0, z = 0;
        if (active[k]) {
            x = p.vidx_x[ind[k]];
            y = p.vidx_y[ind[k]];
            z = p.vidx_z[ind[k]];
        }
        px[k] = p.x_locs[x];
        py[k] = p.y_locs[y];
        pz[k] = p.z_locs[z];
        const int64_t v = ((int64_t)x * p.ny + y) * p.nz + z;
        pr[k] = active[k] ? p.img_r[v] : 1.f;
        pi[k] = active[k] ? p.img_i[v] : 0.f;
        pm[k] = 1.f / sqrtf(pr[k] * pr[k] + pi[k] * pi[k]);
    }
    const float2 vx = make_float2(px[0], px[1]), vy = make_float2(py[0], py[1]),
                 vz = make_float2(pz[0], pz[1]);
    const float2 nvx = make_float2(-px[0], -px[1]), nvy = make_float2(-py[0], -py[1]),
                 nvz = make_float2(-pz[0], -pz[1]);
    const float2 ire = make_float2(pr[0], pr[1]), iim = make_float2(pi[0], pi[1]),
                 inv_mag = make_float2(pm[0], pm[1]);
    float2 acc[3] = {dup(0.f), dup(0.f), dup(0.f)};
    const bool soa = p.meas == nullptr;
    for (int a0 = 0; a0 < p.num_ant; a0 += kInterpChunk) {
        const int n = min(kInterpChunk, p.num_ant - a0);
        __syncthreads();
        stage_pack_chunk(p, a0, n, sh);
        __syncthreads();
        const bool offsets = pack_chunk_has_offsets(sh, n);
        if (!active[0] && !active[1]) continue;
        if (offsets) {
            if (soa) pack_normals_chunk<false, true>(p, sh, a0, n, range_max, ti, vx, vy, vz,
                                                     nvx, nvy, nvz, ire, iim, inv_mag, acc);
            else pack_normals_chunk<false, false>(p, sh, a0, n, range_max, ti, vx, vy, vz, nvx,
                                                  nvy, nvz, ire, iim, inv_mag, acc);
        } else {
            if (soa) pack_normals_chunk<true, true>(p, sh, a0, n, range_max, ti, vx, vy, vz,
                                                    nvx, nvy, nvz, ire, iim, inv_mag, acc);
            else pack_normals_chunk<true, false>(p, sh, a0, n, range_max, ti, vx, vy, vz, nvx,
                                                 nvy, nvz, ire, iim, inv_mag, acc);
        }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (!active[k]) continue;
        p.n_x[ind[k]] = k ? acc[0].y : acc[0].x;
        p.n_y[ind[k]] = k ? acc[1].y : acc[1].x;
        p.n_z[ind[k]] = k ? acc[2].y : acc[2].x;
    }
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

cudaError_t launch_interp_image_fast(const InterpParams &p, cudaStream_t stream) {
    if (p.count <= 0) return cudaSuccess;
    const int64_t per = (int64_t)kInterpThreads * 2;  // kFastT == 2 in every form
    const int64_t blocks = (p.count + per - 1) / per;
    if (g_interp_fast_form.load() == 1)
        interp_image_fast_kernel<<<(unsigned)blocks, kInterpThreads, 0, stream>>>(p);
    else
        interp_image_pack_kernel<<<(unsigned)blocks, kInterpThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_interp_normals_fast(const InterpParams &p, cudaStream_t stream) {
    if (p.count <= 0) return cudaSuccess;
    if (g_interp_fast_form.load() == 1) {
        const int64_t blocks = (p.count + kInterpThreads - 1) / kInterpThreads;
        interp_normals_fast_kernel<<<(unsigned)blocks, kInterpThreads, 0, stream>>>(p);
    } else {
        const int64_t per = (int64_t)kInterpThreads * 2;
        const int64_t blocks = (p.count + per - 1) / per;
        interp_normals_pack_kernel<<<(unsigned)blocks, kInterpThreads, 0, stream>>>(p);
    }
    return cudaGetLastError();
}

}  // namespace mmn

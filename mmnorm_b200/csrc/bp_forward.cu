// bp_forward.cu -- fused full matched-filter backprojection + surface-normal vote.
//
// What one launch computes, for every voxel v of a tile and every virtual antenna i
// of an antenna range (the reference's cuda_image full mode, imaging_gpu.cu:65-117,
// fused with the vote of cuda_sn_est, surface_normal_est.cu:128-145):
//
//   c_i(v) = sum_j m[i,j] * exp(-j * d_i(v) * kappa_j),   kappa_j = 2*pi*(1/lambda + j*slope/c)
//   I(v)  += c_i(v)
//   W(v)  += c_i(v) * (tx_i + o_i/2 - v)                  (complex 3-vector)
//
// The reference recomputes every c_i in a second kernel to form the vote
// sum_i Re(c_i conj(I))/|I| * u_i; that equals Re(conj(I) * W)/|I|, so one pass
// with 8 FP32 accumulators per voxel gives the image and the un-normalised normal.
//
// MIXED form (default).  Per (voxel, antenna): d in FP64; the sample sum is split
// into blocks of 32 samples, each evaluated by Horner's rule in FP32,
//     h_b = sum_{t<32} m[i, 32b+t] * z^t,   z = exp(-j d kappa_step)   (4 FFMA / sample)
// i.e. the rotation recurrence is applied to the running partial sum instead of to a
// separate phasor, and every block is re-anchored with the exact FP64-wrapped phase
//     c_i += exp(-j d kappa_{32b}) * h_b.
// The per-sample work is one complex multiply-add (4 FFMA), no SFU.
//
// PLAIN form.  FP32 distance and FP32 phase -d*kappa_j with one sincosf per sample,
// then a complex multiply-add -- the straightforward FP32 kernel.
//
// Work item = (voxel tile, antenna split).  A CTA of NT threads owns NT*T voxels (T
// per thread, strided by NT so stores coalesce).  Antenna records and measurement
// rows stream through a double-buffered shared-memory stage filled by one elected
// thread with bulk TMA copies (cp.async.bulk) completing on an mbarrier; every
// thread reads the samples as broadcast float4 loads (two complex samples).  With
// one split per tile the CTA writes the final image/vote; otherwise it writes an
// 8-float partial per voxel that bp_reduce_partials sums in split order
// (deterministic).
#include "bp_kernels.cuh"

namespace mmn {

template <int T>
__device__ __forceinline__ void horner_step(float (&hr)[T], float (&hi)[T],
                                            const float (&zr)[T], const float (&zi)[T],
                                            const float (&nzi)[T], float mr, float mi) {
#pragma unroll
    for (int k = 0; k < T; ++k) {
        float a = fmaf(hr[k], zr[k], mr);
        float b = fmaf(hr[k], zi[k], mi);
        hr[k] = fmaf(hi[k], nzi[k], a);
        hi[k] = fmaf(hi[k], zr[k], b);
    }
}

template <int T, int NT, bool PLAIN>
__global__ void __launch_bounds__(NT) bp_fwd_kernel(const FwdParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    const int fp = p.fp;
    const int nas = p.ant_per_stage;
    const size_t stage_bytes = (size_t)nas * sizeof(AntRec) + (size_t)nas * fp * sizeof(float2);
    unsigned char *stage_base = smem + 128;
    float *kappa_tab = reinterpret_cast<float *>(stage_base + 2 * stage_bytes);  // PLAIN only

    const int tile = blockIdx.x % p.num_tiles;
    const int split = blockIdx.x / p.num_tiles;
    const int a_begin = split * p.ant_per_split;
    const int a_end = min(p.num_ant, a_begin + p.ant_per_split);
    const int n_chunks = a_end > a_begin ? (a_end - a_begin + nas - 1) / nas : 0;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    if (PLAIN) {
        for (int j = threadIdx.x; j < fp; j += NT)
            kappa_tab[j] = (float)fma((double)j, p.kd, p.k0);
    }
    __syncthreads();

    auto issue = [&](int c) {
        const int s = c & 1;
        const int a0 = a_begin + c * nas;
        const int na = min(nas, a_end - a0);
        unsigned char *st = stage_base + s * stage_bytes;
        const uint32_t ant_bytes = (uint32_t)(na * sizeof(AntRec));
        const uint32_t meas_bytes = (uint32_t)((size_t)na * fp * sizeof(float2));
        mbar_arrive_expect_tx(&bars[s], ant_bytes + meas_bytes);
        bulk_g2s(st, p.ant + a0, ant_bytes, &bars[s]);
        bulk_g2s(st + (size_t)nas * sizeof(AntRec), p.meas + (size_t)a0 * fp, meas_bytes,
                 &bars[s]);
    };
    if (threadIdx.x == 0) {
        if (n_chunks > 0) issue(0);
        if (n_chunks > 1) issue(1);
    }

    // voxels of this thread: rel = tile*NT*T + tid + k*NT, voxel = vox_start + rel
    const int64_t rbase = (int64_t)tile * (NT * T) + threadIdx.x;
    float vx[T], vy[T], vz[T];
    double vxd[T], vyd[T], vzd[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        const int64_t rel = rbase + (int64_t)k * NT;
        const int64_t v = rel < p.vox_count ? p.vox_start + rel : p.vox_start;
        const int64_t nyz = (int64_t)p.ny * p.nz;
        const int ix = (int)(v / nyz);
        const int64_t rem = v - (int64_t)ix * nyz;
        const int iy = (int)(rem / p.nz);
        const int iz = (int)(rem - (int64_t)iy * p.nz);
        vx[k] = __ldg(p.x_locs + ix);
        vy[k] = __ldg(p.y_locs + iy);
        vz[k] = __ldg(p.z_locs + iz);
        vxd[k] = vx[k];
        vyd[k] = vy[k];
        vzd[k] = vz[k];
    }
    float acc[T][8];
#pragma unroll
    for (int k = 0; k < T; ++k)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[k][q] = 0.f;

    const bool mono = *p.mono_flag != 0;
    const int nblk = fp / kBlockF;

    for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        bool ok = mbar_wait_bounded(&bars[s], (uint32_t)((c >> 1) & 1), p.status);
        if (!__syncthreads_and(ok)) return;
        const AntRec *ants = reinterpret_cast<const AntRec *>(stage_base + s * stage_bytes);
        const float4 *meas4 = reinterpret_cast<const float4 *>(
            stage_base + s * stage_bytes + (size_t)nas * sizeof(AntRec));
        const int na = min(nas, a_end - (a_begin + c * nas));

        for (int a = 0; a < na; ++a) {
            const AntRec &ar = ants[a];
            const float4 *m4 = meas4 + (size_t)a * (fp / 2);
            float cr[T], ci[T];
#pragma unroll
            for (int k = 0; k < T; ++k) cr[k] = ci[k] = 0.f;

            if (!PLAIN) {
                double d[T];
                float zr[T], zi[T], nzi[T];
#pragma unroll
                for (int k = 0; k < T; ++k) {
                    d[k] = range_fp64(vxd[k], vyd[k], vzd[k], ar, mono, p.ti);
                    float2 z = cis_fp64_phase(-d[k] * p.kd);
                    zr[k] = z.x;
                    zi[k] = z.y;
                    nzi[k] = -z.y;
                }
                for (int b = 0; b < nblk; ++b) {
                    const float4 *mb = m4 + b * (kBlockF / 2);
                    float hr[T], hi[T];
                    const float4 top = mb[kBlockF / 2 - 1];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        hr[k] = top.z;
                        hi[k] = top.w;
                    }
                    horner_step<T>(hr, hi, zr, zi, nzi, top.x, top.y);
#pragma unroll
                    for (int q = kBlockF / 2 - 2; q >= 0; --q) {
                        const float4 mm = mb[q];
                        horner_step<T>(hr, hi, zr, zi, nzi, mm.z, mm.w);
                        horner_step<T>(hr, hi, zr, zi, nzi, mm.x, mm.y);
                    }
                    const double kap = fma((double)(b * kBlockF), p.kd, p.k0);
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        const float2 an = cis_fp64_phase(-d[k] * kap);
                        cr[k] = fmaf(an.x, hr[k], fmaf(-an.y, hi[k], cr[k]));
                        ci[k] = fmaf(an.x, hi[k], fmaf(an.y, hr[k], ci[k]));
                    }
                }
            } else {
                // FP32 distance as the reference computes it (imaging_gpu.cu:67-88)
                float df[T];
                const float tx = (float)ar.tx[0], ty = (float)ar.tx[1], tz = (float)ar.tx[2];
                const float ox = (float)(ar.rx[0] - ar.tx[0]), oy = (float)(ar.rx[1] - ar.tx[1]),
                            oz = (float)(ar.rx[2] - ar.tx[2]);
#pragma unroll
                for (int k = 0; k < T; ++k) {
                    const float ax = vx[k] - tx, ay = vy[k] - ty, az = vz[k] - tz;
                    const float f = sqrtf(ax * ax + ay * ay + az * az);
                    const float bx = ax - ox, by = ay - oy, bz = az - oz;
                    df[k] = f + sqrtf(bx * bx + by * by + bz * bz) + (float)p.ti;
                }
                const float2 *kap2 = reinterpret_cast<const float2 *>(kappa_tab);
                for (int b = 0; b < nblk; ++b) {
#pragma unroll 4
                    for (int q = 0; q < kBlockF / 2; ++q) {
                        const float4 mm = m4[b * (kBlockF / 2) + q];
                        const float2 kk = kap2[b * (kBlockF / 2) + q];
#pragma unroll
                        for (int k = 0; k < T; ++k) {
                            float sn, cs;
                            sincosf(-df[k] * kk.x, &sn, &cs);
                            cr[k] = fmaf(mm.x, cs, fmaf(-mm.y, sn, cr[k]));
                            ci[k] = fmaf(mm.x, sn, fmaf(mm.y, cs, ci[k]));
                            sincosf(-df[k] * kk.y, &sn, &cs);
                            cr[k] = fmaf(mm.z, cs, fmaf(-mm.w, sn, cr[k]));
                            ci[k] = fmaf(mm.z, sn, fmaf(mm.w, cs, ci[k]));
                        }
                    }
                }
            }
            // image + vote accumulation
            const float ux0 = ar.virt[0], uy0 = ar.virt[1], uz0 = ar.virt[2];
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float ux = ux0 - vx[k], uy = uy0 - vy[k], uz = uz0 - vz[k];
                acc[k][0] += cr[k];
                acc[k][1] += ci[k];
                acc[k][2] = fmaf(cr[k], ux, acc[k][2]);
                acc[k][3] = fmaf(ci[k], ux, acc[k][3]);
                acc[k][4] = fmaf(cr[k], uy, acc[k][4]);
                acc[k][5] = fmaf(ci[k], uy, acc[k][5]);
                acc[k][6] = fmaf(cr[k], uz, acc[k][6]);
                acc[k][7] = fmaf(ci[k], uz, acc[k][7]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + 2 < n_chunks) issue(c + 2);
    }

#pragma unroll
    for (int k = 0; k < T; ++k) {
        const int64_t rel = rbase + (int64_t)k * NT;
        if (rel >= p.vox_count) continue;
        const int64_t v = p.vox_start + rel;
        if (p.num_splits == 1) {
            if (p.image) p.image[v] = make_float2(acc[k][0], acc[k][1]);
            if (p.out_r) {
                p.out_r[v] = acc[k][0];
                p.out_i[v] = acc[k][1];
            }
            if (p.vote) {
                p.vote[v] = make_float2(acc[k][2], acc[k][3]);
                p.vote[p.nvox + v] = make_float2(acc[k][4], acc[k][5]);
                p.vote[2 * p.nvox + v] = make_float2(acc[k][6], acc[k][7]);
            }
        } else {
            float4 *dst = p.partial + 2 * ((size_t)split * p.vox_count + rel);
            dst[0] = make_float4(acc[k][0], acc[k][1], acc[k][2], acc[k][3]);
            dst[1] = make_float4(acc[k][4], acc[k][5], acc[k][6], acc[k][7]);
        }
    }
}

__global__ void bp_reduce_partials(const FwdParams p) {
    const int64_t rel = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (rel >= p.vox_count) return;
    const int64_t v = p.vox_start + rel;
    float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
    for (int sp = 0; sp < p.num_splits; ++sp) {
        const float4 *src = p.partial + 2 * ((size_t)sp * p.vox_count + rel);
        const float4 a = src[0], b = src[1];
        s0.x += a.x; s0.y += a.y; s0.z += a.z; s0.w += a.w;
        s1.x += b.x; s1.y += b.y; s1.z += b.z; s1.w += b.w;
    }
    if (p.image) p.image[v] = make_float2(s0.x, s0.y);
    if (p.out_r) {
        p.out_r[v] = s0.x;
        p.out_i[v] = s0.y;
    }
    if (p.vote) {
        p.vote[v] = make_float2(s0.z, s0.w);
        p.vote[p.nvox + v] = make_float2(s1.x, s1.y);
        p.vote[2 * p.nvox + v] = make_float2(s1.z, s1.w);
    }
}

// Builds the 64-byte antenna records: TX (+ optional per-antenna offset), RX = TX +
// rx_offsets[i % R], and the float32 vote anchor TX + o/2 computed as the reference
// does (surface_normal_est.cu:128-130).
__global__ void prep_antennas(const float *__restrict__ ant, const float *__restrict__ rxo,
                              int R, const float *__restrict__ pos_off, int A,
                              AntRec *__restrict__ out, int32_t *__restrict__ mono_flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        int mono = 1;
        for (int q = 0; q < 3 * R; ++q) mono &= (rxo[q] == 0.f);
        *mono_flag = mono;
    }
    if (i >= A) return;
    AntRec r;
    const int q = i % R;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float a = ant[3 * i + k];
        double ad = a;
        if (pos_off) {
            ad += (double)pos_off[3 * i + k];
            a = a + pos_off[3 * i + k];
        }
        const float o = rxo[3 * q + k];
        r.tx[k] = ad;
        r.rx[k] = ad + (double)o;
        r.virt[k] = a + o / 2;
    }
    r.pad = 0.f;
    out[i] = r;
}

// Copies [A, F] complex64 rows into [A, Fp] rows zero-padded to Fp (Fp % 32 == 0).
// Zero samples at the top of a Horner block contribute exactly nothing.
__global__ void pad_meas(const float2 *__restrict__ src, int A, int F, float2 *__restrict__ dst,
                         int Fp) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)A * Fp) return;
    const int64_t a = idx / Fp;
    const int j = (int)(idx - a * Fp);
    dst[idx] = j < F ? src[a * F + j] : make_float2(0.f, 0.f);
}

// Interleaves SoA measurement planes (the reference's meas_r / meas_i layout,
// py_image_gpu.py:261-262) into padded complex64 rows.
__global__ void interleave_pad_meas(const float *__restrict__ re, const float *__restrict__ im,
                                    int A, int F, float2 *__restrict__ dst, int Fp) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)A * Fp) return;
    const int64_t a = idx / Fp;
    const int j = (int)(idx - a * Fp);
    dst[idx] = j < F ? make_float2(re[a * F + j], im[a * F + j]) : make_float2(0.f, 0.f);
}

// ------------------------------------------------------------------ instantiations
template <int T, int NT, bool PLAIN>
static const void *fwd_ptr() {
    return reinterpret_cast<const void *>(&bp_fwd_kernel<T, NT, PLAIN>);
}

const FwdVariant *fwd_variants(int *count) {
    static const FwdVariant v[] = {
        {4, 128, false, fwd_ptr<4, 128, false>()},
        {2, 128, false, fwd_ptr<2, 128, false>()},
        {4, 256, false, fwd_ptr<4, 256, false>()},
        {2, 256, false, fwd_ptr<2, 256, false>()},
        {2, 128, true, fwd_ptr<2, 128, true>()},
        {1, 128, true, fwd_ptr<1, 128, true>()},
        {2, 256, true, fwd_ptr<2, 256, true>()},
    };
    *count = (int)(sizeof(v) / sizeof(v[0]));
    return v;
}

cudaError_t launch_fwd(const FwdVariant &var, const FwdParams &p, size_t smem,
                       cudaStream_t stream) {
    void *args[] = {const_cast<FwdParams *>(&p)};
    const int grid = p.num_tiles * p.num_splits;
    return cudaLaunchKernel(var.fn, dim3(grid), dim3(var.nt), args, smem, stream);
}

cudaError_t launch_reduce(const FwdParams &p, cudaStream_t stream) {
    const int nt = 256;
    const int64_t blocks = (p.vox_count + nt - 1) / nt;
    bp_reduce_partials<<<(unsigned)blocks, nt, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_prep_antennas(const float *ant, const float *rxo, int R, const float *pos_off,
                                 int A, AntRec *out, int32_t *mono_flag, cudaStream_t stream) {
    const int nt = 256;
    prep_antennas<<<(A + nt) / nt, nt, 0, stream>>>(ant, rxo, R, pos_off, A, out, mono_flag);
    return cudaGetLastError();
}

cudaError_t launch_pad_meas(const float2 *src, int A, int F, float2 *dst, int Fp,
                            cudaStream_t stream) {
    const int nt = 256;
    const int64_t n = (int64_t)A * Fp;
    pad_meas<<<(unsigned)((n + nt - 1) / nt), nt, 0, stream>>>(src, A, F, dst, Fp);
    return cudaGetLastError();
}

cudaError_t launch_interleave_pad(const float *re, const float *im, int A, int F, float2 *dst,
                                  int Fp, cudaStream_t stream) {
    const int nt = 256;
    const int64_t n = (int64_t)A * Fp;
    interleave_pad_meas<<<(unsigned)((n + nt - 1) / nt), nt, 0, stream>>>(re, im, A, F, dst, Fp);
    return cudaGetLastError();
}

}  // namespace mmn

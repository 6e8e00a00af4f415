// bp_backward.cu -- adjoint of the fused backprojection + vote (mixed precision).
//
// Forward (per voxel v, virtual antenna a, sample j):
//   c_a(v) = sum_j m[a,j] p_aj(v),  p_aj = exp(-j d_a(v) kappa_j),  kappa_j = 2pi(1/lambda + j slope/c)
//   I(v) = sum_a c_a(v),  W(v) = sum_a c_a(v) u_a(v),  u_a = tx_a + o_a/2 - v,
//   with d_a(v) = |v - tx_a| + |v - rx_a| (+0.15), tx_a = antenna_a + delta_a, rx_a = tx_a + o_a.
// Upstream gradients gI = dL/dI, gW = dL/dW in torch's convention (dL/dRe + i dL/dIm);
// G_a(v) = gI(v) + sum_k gW_k(v) u_ak(v) is dL/dc_a(v).
//
//   dL/dm[a,j]   = sum_v G_a(v) conj(p_aj(v))                      (measurement pass)
//   dL/ddelta_a  = sum_v [ Im(conj(G) c'_a) * (-(e_tx + e_rx)) + Re(conj(gW) c_a) ]
//                  c'_a(v) = sum_j kappa_j m[a,j] p_aj(v),  e = unit vectors antenna -> voxel
//                                                                  (position pass)
// Phasors are recomputed, nothing per (voxel, antenna) is stored.
//
// Position pass: the forward's tiling and antenna staging; per (voxel, antenna) two Horner
// chains ride in the two halves of every FFMA2 -- (kappa_j m_j) and (m_j), staged as
// (kappa*re, re, kappa*im, im) -- with the forward's fixed-point block anchors.  Per-antenna
// sums over a CTA's voxels (warp shuffles, then shared memory) go to per-tile partials
// that a second kernel adds in tile order (deterministic).
// Measurement pass: one thread per (antenna, 32-sample block); voxels stream through
// shared memory; per voxel the block's 32 outputs receive G * conj(p) generated by an
// FP32 rotation from an exact FP64-wrapped anchor (re-anchored per voxel and block).
#include "bp_stage.cuh"

namespace mmn {

// Rows padded to Fp (antenna rows past A and samples past F are zero):
//   layout 0: (kappa_j re, re, kappa_j im, im)  -- the two chains of one voxel
//   layout 1: (kappa_j re, kappa_j re, kappa_j im, kappa_j im)  -- one chain, voxel pairs
__global__ void bwd_stage_kernel(const float2 *__restrict__ meas, int A, int F, int Fp,
                                 int rows, double k0, double kd, int layout,
                                 float4 *__restrict__ dst) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)rows * Fp) return;
    const int64_t a = idx / Fp;
    const int j = (int)(idx - a * Fp);
    float2 m = make_float2(0.f, 0.f);
    if (a < A && j < F) m = meas[a * F + j];
    const float kap = (float)fma((double)j, kd, k0);
    dst[idx] = layout == 0 ? make_float4(kap * m.x, m.x, kap * m.y, m.y)
                           : make_float4(kap * m.x, kap * m.x, kap * m.y, kap * m.y);
}

__global__ void bwd_vox_rec_kernel(const BwdParams bp, float4 *__restrict__ dst) {
    const FwdParams &p = bp.f;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= p.nvox) return;
    const int64_t nyz = (int64_t)p.ny * p.nz;
    const int ix = (int)(v / nyz);
    const int64_t rem = v - (int64_t)ix * nyz;
    const int iy = (int)(rem / p.nz);
    const int iz = (int)(rem - (int64_t)iy * p.nz);
    const float2 gi = bp.grad_image ? bp.grad_image[v] : make_float2(0.f, 0.f);
    float2 gw[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    if (bp.grad_vote)
        for (int k = 0; k < 3; ++k) gw[k] = bp.grad_vote[k * p.nvox + v];
    dst[3 * v + 0] = make_float4(p.x_locs[ix], p.y_locs[iy], p.z_locs[iz], 0.f);
    dst[3 * v + 1] = make_float4(gi.x, gi.y, gw[0].x, gw[0].y);
    dst[3 * v + 2] = make_float4(gw[1].x, gw[1].y, gw[2].x, gw[2].y);
}

// ------------------------------------------------------------------ position pass
template <int T, int NT>
__global__ void __launch_bounds__(NT) bp_bwd_pos_kernel(const BwdParams bp) {
    const FwdParams &p = bp.f;
    extern __shared__ __align__(128) unsigned char smem[];
    Stage st;
    st.bars = reinterpret_cast<uint64_t *>(smem);
    st.base = smem + 128;
    st.nas = p.ant_per_stage;
    st.esz = 16;
    st.fp = p.fp;
    st.stage_bytes = (size_t)st.nas * sizeof(AntRec) + (size_t)st.nas * st.fp * st.esz;
    float *wsum = reinterpret_cast<float *>(st.base + 2 * st.stage_bytes);  // [NT/32][nas][3]
    constexpr int NW = NT / 32;
    const int fp = p.fp;
    const int tile = blockIdx.x % p.num_tiles;
    const int split = blockIdx.x / p.num_tiles;
    const int a_begin = split * p.ant_per_split;
    const int a_end = min(p.num_ant, a_begin + p.ant_per_split);
    const int n_chunks = a_end > a_begin ? (a_end - a_begin + st.nas - 1) / st.nas : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        mbar_init(&st.bars[0], 1);
        mbar_init(&st.bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n_chunks > 0) st.issue(p, 0, a_begin, a_end);
        if (n_chunks > 1) st.issue(p, 1, a_begin, a_end);
    }

    const int64_t rbase = (int64_t)tile * (NT * T) + threadIdx.x;
    float vx[T], vy[T], vz[T];
    float2 gi[T], gw[T][3];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        const int64_t rel = rbase + (int64_t)k * NT;
        decode_voxel(p, rel, vx[k], vy[k], vz[k]);
        const bool ok = rel < p.vox_count;
        const int64_t v = p.vox_start + (ok ? rel : 0);
        gi[k] = (ok && bp.grad_image) ? bp.grad_image[v] : make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            gw[k][q] = (ok && bp.grad_vote) ? bp.grad_vote[q * p.nvox + v] : make_float2(0.f, 0.f);
    }
    const bool mono = *p.mono_flag != 0;
    const int nblk = fp / kBlockF;

    int c_failed = -1;  // chunk whose wait gave up; the drain runs after the loop
    for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        bool ok = mbar_wait_bounded(&st.bars[s], (uint32_t)((c >> 1) & 1), p.status);
        if (!__syncthreads_and(ok)) {
            c_failed = c;
            break;
        }
        const AntRec *ants = st.ants(s);
        const float4 *mstage = reinterpret_cast<const float4 *>(st.meas(s));
        const int a0 = a_begin + c * st.nas;
        const int na = min(st.nas, a_end - a0);

        for (int a = 0; a < na; ++a) {
            const AntRec &ar = ants[a];
            const float4 *m4 = mstage + (size_t)a * fp;
            float e3[T][3];
            unsigned long long ph[T], stp[T];
            float2 zr[T], zi[T], nzi[T], cr[T], ci[T];
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const double x = vx[k], y = vy[k], z = vz[k];
                const double dx = x - ar.tx[0], dy = y - ar.tx[1], dz = z - ar.tx[2];
                const double f = sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
                double b = f, bx = dx, by = dy, bz = dz;
                if (!mono) {
                    bx = x - ar.rx[0];
                    by = y - ar.rx[1];
                    bz = z - ar.rx[2];
                    b = sqrt(fma(bx, bx, fma(by, by, bz * bz)));
                }
                const double d = f + b + p.ti;
                // -(e_tx + e_rx): derivative of d with respect to the antenna offset (a
                // direction: FP32 is ample)
                const float rf = 1.f / (float)f, rb = mono ? rf : 1.f / (float)b;
                e3[k][0] = -fmaf((float)dx, rf, (float)bx * rb);
                e3[k][1] = -fmaf((float)dy, rf, (float)by * rb);
                e3[k][2] = -fmaf((float)dz, rf, (float)bz * rb);
                const float2 zz = cis_fp64_phase(-d * p.kd);
                zr[k] = make_float2(zz.x, zz.x);
                zi[k] = make_float2(zz.y, zz.y);
                nzi[k] = make_float2(-zz.y, -zz.y);
                ph[k] = turns_to_fixed(-d * p.t0);
                stp[k] = turns_to_fixed(-d * p.tblk);
                cr[k] = ci[k] = make_float2(0.f, 0.f);
            }
            for (int b = 0; b < nblk; ++b) {
                const float4 *mb = m4 + b * kBlockF;
                float2 hr[T], hi[T];
                const float4 top = mb[kBlockF - 1];
#pragma unroll
                for (int k = 0; k < T; ++k) {
                    hr[k] = make_float2(top.x, top.y);
                    hi[k] = make_float2(top.z, top.w);
                }
#pragma unroll
                for (int t = kBlockF - 2; t >= 0; --t) {
                    const float4 mm = mb[t];
                    const float2 mr = make_float2(mm.x, mm.y), mi = make_float2(mm.z, mm.w);
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        const float2 u = __ffma2_rn(hr[k], zr[k], mr);
                        const float2 w = __ffma2_rn(hr[k], zi[k], mi);
                        hr[k] = __ffma2_rn(hi[k], nzi[k], u);
                        hi[k] = __ffma2_rn(hi[k], zr[k], w);
                    }
                }
#pragma unroll
                for (int k = 0; k < T; ++k) {
                    float ac, as;
                    fixed_cis(ph[k], ac, as);
                    ph[k] += stp[k];
                    const float2 anr = make_float2(ac, ac), ani = make_float2(as, as),
                                 nani = make_float2(-as, -as);
                    cr[k] = __ffma2_rn(anr, hr[k], __ffma2_rn(nani, hi[k], cr[k]));
                    ci[k] = __ffma2_rn(anr, hi[k], __ffma2_rn(ani, hr[k], ci[k]));
                }
            }
            // lane .x carries c' = sum kappa m p, lane .y carries c = sum m p
            float g3[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float u[3] = {ar.virt[0] - vx[k], ar.virt[1] - vy[k], ar.virt[2] - vz[k]};
                float Gr = gi[k].x, Gi = gi[k].y;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    Gr = fmaf(gw[k][q].x, u[q], Gr);
                    Gi = fmaf(gw[k][q].y, u[q], Gi);
                }
                const float s1 = Gr * ci[k].x - Gi * cr[k].x;  // Im(conj(G) c')
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    g3[q] += fmaf(s1, e3[k][q], gw[k][q].x * cr[k].y + gw[k][q].y * ci[k].y);
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) g3[q] += __shfl_xor_sync(0xffffffffu, g3[q], o);
            }
            if (lane == 0) {
                wsum[(warp * st.nas + a) * 3 + 0] = g3[0];
                wsum[(warp * st.nas + a) * 3 + 1] = g3[1];
                wsum[(warp * st.nas + a) * 3 + 2] = g3[2];
            }
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < na * 3; idx += NT) {
            float sum = 0.f;
#pragma unroll
            for (int w = 0; w < NW; ++w) sum += wsum[w * st.nas * 3 + idx];
            bp.pos_partial[((size_t)tile * p.num_ant + a0) * 3 + idx] = sum;
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + 2 < n_chunks) st.issue(p, c + 2, a_begin, a_end);
    }
    if (c_failed >= 0) {
        st.drain_after_timeout((uint32_t)c_failed, c_failed + 1 < n_chunks, p.status);
        return;
    }
}

__global__ void bwd_pos_reduce_kernel(const BwdParams bp) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= bp.num_ant_real * 3) return;
    float s = 0.f;
    for (int t = 0; t < bp.f.num_tiles; ++t)
        s += bp.pos_partial[(size_t)t * bp.f.num_ant * 3 + idx];
    bp.grad_pos[idx] = s;
}

// Position pass when the loss has no vote term (dL/dW = 0): only c' = sum kappa m p is
// needed, so the FFMA2 halves carry two voxels' chains (staging layout 1), the forward's
// voxel-pair arrangement -- half the two-chain kernel's FMA work.
template <int T, int NT>
__global__ void __launch_bounds__(NT) bp_bwd_pos_img_kernel(const BwdParams bp) {
    static_assert(T % 2 == 0, "voxel pairs");
    constexpr int P = T / 2;
    const FwdParams &p = bp.f;
    extern __shared__ __align__(128) unsigned char smem[];
    Stage st;
    st.bars = reinterpret_cast<uint64_t *>(smem);
    st.base = smem + 128;
    st.nas = p.ant_per_stage;
    st.esz = 16;
    st.fp = p.fp;
    st.stage_bytes = (size_t)st.nas * sizeof(AntRec) + (size_t)st.nas * st.fp * st.esz;
    float *wsum = reinterpret_cast<float *>(st.base + 2 * st.stage_bytes);  // [NT/32][nas][3]
    constexpr int NW = NT / 32;
    const int fp = p.fp;
    const int tile = blockIdx.x % p.num_tiles;
    const int split = blockIdx.x / p.num_tiles;
    const int a_begin = split * p.ant_per_split;
    const int a_end = min(p.num_ant, a_begin + p.ant_per_split);
    const int n_chunks = a_end > a_begin ? (a_end - a_begin + st.nas - 1) / st.nas : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        mbar_init(&st.bars[0], 1);
        mbar_init(&st.bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n_chunks > 0) st.issue(p, 0, a_begin, a_end);
        if (n_chunks > 1) st.issue(p, 1, a_begin, a_end);
    }

    const int64_t rbase = (int64_t)tile * (NT * T) + threadIdx.x;
    float vx[T], vy[T], vz[T];
    float2 gi[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        const int64_t rel = rbase + (int64_t)k * NT;
        decode_voxel(p, rel, vx[k], vy[k], vz[k]);
        const bool ok = rel < p.vox_count;
        gi[k] = ok ? bp.grad_image[p.vox_start + rel] : make_float2(0.f, 0.f);
    }
    const bool mono = *p.mono_flag != 0;
    const int nblk = fp / kBlockF;

    int c_failed = -1;  // chunk whose wait gave up; the drain runs after the loop
    for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        bool ok = mbar_wait_bounded(&st.bars[s], (uint32_t)((c >> 1) & 1), p.status);
        if (!__syncthreads_and(ok)) {
            c_failed = c;
            break;
        }
        const AntRec *ants = st.ants(s);
        const float4 *mstage = reinterpret_cast<const float4 *>(st.meas(s));
        const int a0 = a_begin + c * st.nas;
        const int na = min(st.nas, a_end - a0);

        for (int a = 0; a < na; ++a) {
            const AntRec &ar = ants[a];
            const float4 *m4 = mstage + (size_t)a * fp;
            float e3[T][3];
            double d[T];
            unsigned long long ph[T], stp[T];
            float2 zr[P], zi[P], nzi[P], cr[P], ci[P];
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const double x = vx[k], y = vy[k], z = vz[k];
                const double dx = x - ar.tx[0], dy = y - ar.tx[1], dz = z - ar.tx[2];
                const double f = sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
                double b = f, bx = dx, by = dy, bz = dz;
                if (!mono) {
                    bx = x - ar.rx[0];
                    by = y - ar.rx[1];
                    bz = z - ar.rx[2];
                    b = sqrt(fma(bx, bx, fma(by, by, bz * bz)));
                }
                d[k] = f + b + p.ti;
                const float rf = 1.f / (float)f, rb = mono ? rf : 1.f / (float)b;
                e3[k][0] = -fmaf((float)dx, rf, (float)bx * rb);
                e3[k][1] = -fmaf((float)dy, rf, (float)by * rb);
                e3[k][2] = -fmaf((float)dz, rf, (float)bz * rb);
                ph[k] = turns_to_fixed(-d[k] * p.t0);
                stp[k] = turns_to_fixed(-d[k] * p.tblk);
            }
#pragma unroll
            for (int q = 0; q < P; ++q) {
                cis_fp64_phase_pair(-d[2 * q] * p.kd, -d[2 * q + 1] * p.kd, zr[q], zi[q], nzi[q]);
                cr[q] = ci[q] = make_float2(0.f, 0.f);
            }
            for (int b = 0; b < nblk; ++b) {
                const float4 *mb = m4 + b * kBlockF;
                float2 hr[P], hi[P];
                const float4 top = mb[kBlockF - 1];
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    hr[q] = make_float2(top.x, top.y);
                    hi[q] = make_float2(top.z, top.w);
                }
#pragma unroll
                for (int t = kBlockF - 2; t >= 0; --t) {
                    const float4 mm = mb[t];
                    const float2 mr = make_float2(mm.x, mm.y), mi = make_float2(mm.z, mm.w);
#pragma unroll
                    for (int q = 0; q < P; ++q) {
                        const float2 u = __ffma2_rn(hr[q], zr[q], mr);
                        const float2 w = __ffma2_rn(hr[q], zi[q], mi);
                        hr[q] = __ffma2_rn(hi[q], nzi[q], u);
                        hi[q] = __ffma2_rn(hi[q], zr[q], w);
                    }
                }
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    float2 anr, ani;
                    fixed_cis(ph[2 * q], anr.x, ani.x);
                    fixed_cis(ph[2 * q + 1], anr.y, ani.y);
                    const float2 nani = make_float2(-ani.x, -ani.y);
                    ph[2 * q] += stp[2 * q];
                    ph[2 * q + 1] += stp[2 * q + 1];
                    cr[q] = __ffma2_rn(anr, hr[q], __ffma2_rn(nani, hi[q], cr[q]));
                    ci[q] = __ffma2_rn(anr, hi[q], __ffma2_rn(ani, hr[q], ci[q]));
                }
            }
            float g3[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float cpr = (k & 1) ? cr[k / 2].y : cr[k / 2].x;
                const float cpi = (k & 1) ? ci[k / 2].y : ci[k / 2].x;
                const float s1 = gi[k].x * cpi - gi[k].y * cpr;  // Im(conj(gI) c')
#pragma unroll
                for (int q = 0; q < 3; ++q) g3[q] = fmaf(s1, e3[k][q], g3[q]);
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) g3[q] += __shfl_xor_sync(0xffffffffu, g3[q], o);
            }
            if (lane == 0) {
                wsum[(warp * st.nas + a) * 3 + 0] = g3[0];
                wsum[(warp * st.nas + a) * 3 + 1] = g3[1];
                wsum[(warp * st.nas + a) * 3 + 2] = g3[2];
            }
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < na * 3; idx += NT) {
            float sum = 0.f;
#pragma unroll
            for (int w = 0; w < NW; ++w) sum += wsum[w * st.nas * 3 + idx];
            bp.pos_partial[((size_t)tile * p.num_ant + a0) * 3 + idx] = sum;
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + 2 < n_chunks) st.issue(p, c + 2, a_begin, a_end);
    }
    if (c_failed >= 0) {
        st.drain_after_timeout((uint32_t)c_failed, c_failed + 1 < n_chunks, p.status);
        return;
    }
}

// --------------------------------------------------------------- measurement pass
constexpr int kMeasThreads = 128;
constexpr int kVoxChunk = 256;  // voxel records per shared-memory chunk (12 KB)

__global__ void __launch_bounds__(kMeasThreads) bp_bwd_meas_kernel(const BwdParams bp) {
    const FwdParams &p = bp.f;
    __shared__ float4 vrec[kVoxChunk * 3];
    const int nblk = p.fp / kBlockF;
    const int item = blockIdx.x * kMeasThreads + threadIdx.x;
    const bool active = item < bp.num_items;
    const int it = active ? item : 0;
    const int a = it / nblk;
    const int b = it - a * nblk;
    const AntRec ar = p.ant[a];
    const bool mono = *p.mono_flag != 0;
    const double kap = fma((double)(b * kBlockF), p.kd, p.k0);
    float accr[kBlockF], acci[kBlockF];
#pragma unroll
    for (int t = 0; t < kBlockF; ++t) accr[t] = acci[t] = 0.f;

    for (int64_t v0 = 0; v0 < p.nvox; v0 += kVoxChunk) {
        const int nv = (int)min((int64_t)kVoxChunk, p.nvox - v0);
        __syncthreads();
        for (int q = threadIdx.x; q < nv * 3; q += kMeasThreads) vrec[q] = bp.vox_rec[v0 * 3 + q];
        __syncthreads();
        if (!active) continue;
        for (int j = 0; j < nv; ++j) {
            const float4 r0 = vrec[3 * j], r1 = vrec[3 * j + 1], r2 = vrec[3 * j + 2];
            const double d = range_fp64((double)r0.x, (double)r0.y, (double)r0.z, ar, mono, p.ti);
            const float2 z = cis_fp64_phase(d * p.kd);   // conj of the forward step
            const float2 an = cis_fp64_phase(d * kap);   // conj of the forward block anchor
            const float ux = ar.virt[0] - r0.x, uy = ar.virt[1] - r0.y, uz = ar.virt[2] - r0.z;
            const float Gr = fmaf(r2.z, uz, fmaf(r2.x, uy, fmaf(r1.z, ux, r1.x)));
            const float Gi = fmaf(r2.w, uz, fmaf(r2.y, uy, fmaf(r1.w, ux, r1.y)));
            float qr = Gr * an.x - Gi * an.y;
            float qi = Gr * an.y + Gi * an.x;
#pragma unroll
            for (int t = 0; t < kBlockF; ++t) {
                accr[t] += qr;
                acci[t] += qi;
                const float nr = fmaf(qr, z.x, -qi * z.y);
                qi = fmaf(qr, z.y, qi * z.x);
                qr = nr;
            }
        }
    }
    if (!active) return;
#pragma unroll
    for (int t = 0; t < kBlockF; ++t) {
        const int j = b * kBlockF + t;
        if (j < bp.num_samples) bp.grad_meas[(size_t)a * bp.num_samples + j] = make_float2(accr[t], acci[t]);
    }
}

// ------------------------------------------------- measurement pass, warp per antenna
// A CTA of NW warps covers NW consecutive antennas (one per warp); all warps stream the
// same voxel records through shared memory.  Lane l takes voxel (chunk + 32i + l).  For
// each 32-sample block the lane needs G*conj(p_t) for t = 0..31; it keeps the value of
// sample t = i XOR l in register slot i.  Then a recursive-halving transpose-reduce over
// the warp is select-free -- at every level each lane keeps slots [0, half) and sends
// slots [half, 2*half) -- and slot 0 of lane l ends with the warp's sum for sample l.
// Slot 0 is G * exp(+j d kappa_{32b + l}) (fixed-point phase, exact wrap); slot i is slot
// (i - 2^k) times conj(z)^(+-2^k), 2^k the top bit of i, so every value is at most five
// FP32 complex multiplies from its anchor.  Per (antenna, sample) the sum runs in a fixed
// order: deterministic, no partial buffers.
constexpr int kMeas2Warps = 8;
constexpr int kMeas2Chunk = 512;  // voxel records per shared-memory chunk (24 KB)

__device__ __forceinline__ void warp_transpose_reduce32(float (&v)[kBlockF], int first_level = 0) {
#pragma unroll
    for (int level = first_level; level < 5; ++level) {
        const int half = 16 >> level;
#pragma unroll
        for (int i = 0; i < half; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i + half], half);
    }
}

template <int MAXB>
__global__ void __launch_bounds__(kMeas2Warps * 32) bp_bwd_meas2_kernel(const BwdParams bp) {
    const FwdParams &p = bp.f;
    __shared__ float4 vrec[kMeas2Chunk * 3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int a = blockIdx.x * kMeas2Warps + warp;
    const bool active = a < bp.num_ant_real;
    const AntRec ar = p.ant[active ? a : 0];
    const bool mono = *p.mono_flag != 0;
    const int nblk = p.fp / kBlockF;
    const double t1 = p.tblk / kBlockF;  // turns per metre per sample step
    float accr[MAXB], acci[MAXB];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) accr[b] = acci[b] = 0.f;

    for (int64_t v0 = 0; v0 < p.nvox; v0 += kMeas2Chunk) {
        const int nv = (int)min((int64_t)kMeas2Chunk, p.nvox - v0);
        __syncthreads();
        for (int q = threadIdx.x; q < nv * 3; q += kMeas2Warps * 32) vrec[q] = bp.vox_rec[v0 * 3 + q];
        __syncthreads();
        if (!active) continue;
        for (int base = 0; base < nv; base += 32) {
            const int j = base + lane;
            const bool vok = j < nv;
            const float4 r0 = vrec[3 * (vok ? j : 0)];
            const float4 r1 = vrec[3 * (vok ? j : 0) + 1];
            const float4 r2 = vrec[3 * (vok ? j : 0) + 2];
            const double d = range_fp64((double)r0.x, (double)r0.y, (double)r0.z, ar, mono, p.ti);
            // conj(z)^(2^k), and its conjugate where lane bit k is set
            float wr[5], wi[5];
            {
                const float2 z = cis_fp64_phase(d * p.kd);  // conj of the forward step
                wr[0] = z.x;
                wi[0] = z.y;
#pragma unroll
                for (int k = 1; k < 5; ++k) {
                    wr[k] = wr[k - 1] * wr[k - 1] - wi[k - 1] * wi[k - 1];
                    wi[k] = 2.f * wr[k - 1] * wi[k - 1];
                }
#pragma unroll
                for (int k = 0; k < 5; ++k)
                    if (lane & (1 << k)) wi[k] = -wi[k];
            }
            const float ux = ar.virt[0] - r0.x, uy = ar.virt[1] - r0.y, uz = ar.virt[2] - r0.z;
            float Gr = fmaf(r2.z, uz, fmaf(r2.x, uy, fmaf(r1.z, ux, r1.x)));
            float Gi = fmaf(r2.w, uz, fmaf(r2.y, uy, fmaf(r1.w, ux, r1.y)));
            if (!vok) Gr = Gi = 0.f;
            // phase of sample (32b + lane): turns d*(1/lambda + (32b + lane)*slope/c)
            unsigned long long ph = turns_to_fixed(d * p.t0) +
                                    (unsigned long long)lane * turns_to_fixed(d * t1);
            const unsigned long long stp = turns_to_fixed(d * p.tblk);
#pragma unroll 1
            for (int b = 0; b < nblk; ++b) {
                float ac, as;
                fixed_cis(ph, ac, as);
                ph += stp;
                float qr[kBlockF], qi[kBlockF];
                qr[0] = Gr * ac - Gi * as;
                qi[0] = Gr * as + Gi * ac;
#pragma unroll
                for (int i = 1; i < kBlockF; ++i) {
                    const int k = 31 - __clz(i);  // top bit of i (compile-time after unrolling)
                    const int par = i - (1 << k);
                    qr[i] = fmaf(qr[par], wr[k], -qi[par] * wi[k]);
                    qi[i] = fmaf(qr[par], wi[k], qi[par] * wr[k]);
                }
                warp_transpose_reduce32(qr);
                warp_transpose_reduce32(qi);
#pragma unroll
                for (int bb = 0; bb < MAXB; ++bb)
                    if (bb == b) {
                        accr[bb] += qr[0];
                        acci[bb] += qi[0];
                    }
            }
        }
    }
    if (!active) return;
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int j = b * kBlockF + lane;
        if (b < nblk && j < bp.num_samples)
            bp.grad_meas[(size_t)a * bp.num_samples + j] = make_float2(accr[b], acci[b]);
    }
}

// Two voxels per lane (FFMA2 halves).  Slots are generated depth-first (parent =
// slot - lowest set bit), so only the ancestor path is live; each pair is folded into one
// scalar slot (the two voxels' sum) as soon as it exists, and one transpose-reduce then
// serves 64 voxels.
template <int G>
struct PairSteps {
    // per voxel pair g and half: step conj(z)^(2^k), conjugated where lane bit k is set
    float2 wr[G][5], wi[G][5], nwi[G][5];
};

__host__ __device__ constexpr int dfs_child_bits(int i) { return i == 0 ? 5 : (i & 1 ? 0 : 1 + dfs_child_bits(i >> 1)); }

template <int I, int G>
__device__ __forceinline__ void meas_dfs(const float2 (&r)[G], const float2 (&m)[G],
                                         const PairSteps<G> &w, float (&sr)[kBlockF],
                                         float (&si)[kBlockF]);

// children of slot I are I + 2^k for k below I's lowest set bit, visited from the top bit down
template <int I, int K, int G>
__device__ __forceinline__ void meas_dfs_children(const float2 (&r)[G], const float2 (&m)[G],
                                                  const PairSteps<G> &w, float (&sr)[kBlockF],
                                                  float (&si)[kBlockF]) {
    if constexpr (K > 0) {
        constexpr int k = K - 1;
        float2 cr[G], cm[G];
#pragma unroll
        for (int g = 0; g < G; ++g) {
            cr[g] = __ffma2_rn(m[g], w.nwi[g][k], __fmul2_rn(r[g], w.wr[g][k]));
            cm[g] = __ffma2_rn(r[g], w.wi[g][k], __fmul2_rn(m[g], w.wr[g][k]));
        }
        meas_dfs<I + (1 << k), G>(cr, cm, w, sr, si);
        meas_dfs_children<I, K - 1, G>(r, m, w, sr, si);
    }
}

// slot I of every pair folded into one scalar (the sum over the lane's 2G voxels), and the
// transpose-reduce's first level (slot i += the xor-16 partner's slot i+16) done as soon as
// both slots exist: the depth-first order makes slot i+16 before slot i (i > 0), and slot
// 16 right after slot 0, so at most 17 slots per component are live at a time
template <int I, int G>
__device__ __forceinline__ void meas_dfs(const float2 (&r)[G], const float2 (&m)[G],
                                         const PairSteps<G> &w, float (&sr)[kBlockF],
                                         float (&si)[kBlockF]) {
    float2 tr = r[0], tm = m[0];
#pragma unroll
    for (int g = 1; g < G; ++g) {
        tr = __fadd2_rn(tr, r[g]);
        tm = __fadd2_rn(tm, m[g]);
    }
    const float vr = tr.x + tr.y, vi = tm.x + tm.y;
    if constexpr (I == 16) {
        sr[0] += __shfl_xor_sync(0xffffffffu, vr, 16);
        si[0] += __shfl_xor_sync(0xffffffffu, vi, 16);
    } else if constexpr (I > 0 && I < 16) {
        sr[I] = vr + __shfl_xor_sync(0xffffffffu, sr[I + 16], 16);
        si[I] = vi + __shfl_xor_sync(0xffffffffu, si[I + 16], 16);
    } else {
        sr[I] = vr;
        si[I] = vi;
    }
    meas_dfs_children<I, dfs_child_bits(I), G>(r, m, w, sr, si);
}

// Grid: (antennas / NW) x meas_splits; CTA (x, s) covers voxel range s, and with several
// ranges writes its sums to the range's partial buffer (reduced in range order after).
// Every lane takes G voxel pairs (2G voxels) per pass: one transpose-reduce serves 64G.
template <int MAXB, int NW, int G>
__global__ void __launch_bounds__(NW * 32, 16 / NW) bp_bwd_meas3_kernel(const BwdParams bp) {
    const FwdParams &p = bp.f;
    __shared__ float4 vrec[kMeas2Chunk * 3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int a = blockIdx.x * NW + warp;
    const int64_t v_begin = (int64_t)blockIdx.y * bp.vox_per_split;
    const int64_t v_end = min(p.nvox, v_begin + bp.vox_per_split);
    const bool active = a < bp.num_ant_real;
    const AntRec ar = p.ant[active ? a : 0];
    const bool mono = *p.mono_flag != 0;
    const int nblk = p.fp / kBlockF;
    const double t1 = p.tblk / kBlockF;
    float accr[MAXB], acci[MAXB];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) accr[b] = acci[b] = 0.f;

    for (int64_t v0 = v_begin; v0 < v_end; v0 += kMeas2Chunk) {
        const int nv = (int)min((int64_t)kMeas2Chunk, v_end - v0);
        __syncthreads();
        for (int q = threadIdx.x; q < nv * 3; q += NW * 32) vrec[q] = bp.vox_rec[v0 * 3 + q];
        __syncthreads();
        if (!active) continue;
        for (int base = 0; base < nv; base += 64 * G) {
            PairSteps<G> w;
            float2 gr[G], gi[G];
            unsigned long long ph[G][2], stp[G][2];
#pragma unroll
            for (int g = 0; g < G; ++g) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int j = base + 64 * g + 32 * h + lane;
                    const bool vok = j < nv;
                    const float4 r0 = vrec[3 * (vok ? j : 0)];
                    const float4 r1 = vrec[3 * (vok ? j : 0) + 1];
                    const float4 r2 = vrec[3 * (vok ? j : 0) + 2];
                    const double d =
                        range_fp64((double)r0.x, (double)r0.y, (double)r0.z, ar, mono, p.ti);
                    const float2 z = cis_fp64_phase(d * p.kd);  // conj of the forward step
                    float zr = z.x, zi = z.y;
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        const float si = (lane & (1 << k)) ? -zi : zi;
                        (h ? w.wr[g][k].y : w.wr[g][k].x) = zr;
                        (h ? w.wi[g][k].y : w.wi[g][k].x) = si;
                        (h ? w.nwi[g][k].y : w.nwi[g][k].x) = -si;
                        const float nr = zr * zr - zi * zi;
                        zi = 2.f * zr * zi;
                        zr = nr;
                    }
                    const float ux = ar.virt[0] - r0.x, uy = ar.virt[1] - r0.y,
                                uz = ar.virt[2] - r0.z;
                    float Gr = fmaf(r2.z, uz, fmaf(r2.x, uy, fmaf(r1.z, ux, r1.x)));
                    float Gi = fmaf(r2.w, uz, fmaf(r2.y, uy, fmaf(r1.w, ux, r1.y)));
                    if (!vok) Gr = Gi = 0.f;
                    (h ? gr[g].y : gr[g].x) = Gr;
                    (h ? gi[g].y : gi[g].x) = Gi;
                    ph[g][h] = turns_to_fixed(d * p.t0) +
                               (unsigned long long)lane * turns_to_fixed(d * t1);
                    stp[g][h] = turns_to_fixed(d * p.tblk);
                }
            }
#pragma unroll 1
            for (int b = 0; b < nblk; ++b) {
                float2 r[G], m[G];
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    float2 ac, as;
                    fixed_cis(ph[g][0], ac.x, as.x);
                    fixed_cis(ph[g][1], ac.y, as.y);
                    ph[g][0] += stp[g][0];
                    ph[g][1] += stp[g][1];
                    // slot 0: G * anchor (both halves)
                    r[g] = __ffma2_rn(gr[g], ac, __fmul2_rn(gi[g], make_float2(-as.x, -as.y)));
                    m[g] = __ffma2_rn(gr[g], as, __fmul2_rn(gi[g], ac));
                }
                float sr[kBlockF], si[kBlockF];
                meas_dfs<0, G>(r, m, w, sr, si);  // the depth-first slot tree, level 0 folded
                warp_transpose_reduce32(sr, 1);
                warp_transpose_reduce32(si, 1);
#pragma unroll
                for (int bb = 0; bb < MAXB; ++bb)
                    if (bb == b) {
                        accr[bb] += sr[0];
                        acci[bb] += si[0];
                    }
            }
        }
    }
    if (!active) return;
    float2 *dst = bp.meas_splits > 1
                      ? bp.meas_partial + ((size_t)blockIdx.y * bp.num_ant_real + a) * bp.num_samples
                      : bp.grad_meas + (size_t)a * bp.num_samples;
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int j = b * kBlockF + lane;
        if (b < nblk && j < bp.num_samples) dst[j] = make_float2(accr[b], acci[b]);
    }
}

// grad_meas = the voxel ranges' partial sums, added in range order (deterministic)
__global__ void bwd_meas_reduce_kernel(const BwdParams bp) {
    const int64_t n = (int64_t)bp.num_ant_real * bp.num_samples;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 s = bp.meas_partial[i];
    for (int k = 1; k < bp.meas_splits; ++k) {
        const float2 v = bp.meas_partial[(size_t)k * n + i];
        s.x += v.x;
        s.y += v.y;
    }
    bp.grad_meas[i] = s;
}

// -------------------------------------------------------------------- launchers
const void *bwd_pos_img_kernel_ptr(int *threads, int *voxels_per_thread) {
    *threads = 256;
    *voxels_per_thread = 2;
    return reinterpret_cast<const void *>(&bp_bwd_pos_img_kernel<2, 256>);
}

const void *bwd_pos_kernel_ptr(int variant, int *threads, int *voxels_per_thread) {
    if (variant == 1) {
        *threads = 128;
        *voxels_per_thread = 2;
        return reinterpret_cast<const void *>(&bp_bwd_pos_kernel<2, 128>);
    }
    *threads = 256;
    *voxels_per_thread = 1;
    return reinterpret_cast<const void *>(&bp_bwd_pos_kernel<1, 256>);
}

cudaError_t launch_bwd_stage(const float *meas, int A, int F, int Fp, double k0, double kd,
                             int layout, void *dst, cudaStream_t stream) {
    const int nt = 256;
    const int rows = A;
    const int64_t n = (int64_t)rows * Fp;
    bwd_stage_kernel<<<(unsigned)((n + nt - 1) / nt), nt, 0, stream>>>(
        reinterpret_cast<const float2 *>(meas), A, F, Fp, rows, k0, kd, layout,
        reinterpret_cast<float4 *>(dst));
    return cudaGetLastError();
}

cudaError_t launch_bwd_vox_rec(const BwdParams &bp, float4 *dst, cudaStream_t stream) {
    const int nt = 256;
    bwd_vox_rec_kernel<<<(unsigned)((bp.f.nvox + nt - 1) / nt), nt, 0, stream>>>(bp, dst);
    return cudaGetLastError();
}

cudaError_t launch_bwd_pos(const BwdParams &bp, int variant, size_t smem, cudaStream_t stream) {
    int nt = 0, t = 0;
    const void *fn = variant < 0 ? bwd_pos_img_kernel_ptr(&nt, &t)
                                 : bwd_pos_kernel_ptr(variant, &nt, &t);
    void *args[] = {const_cast<BwdParams *>(&bp)};
    return cudaLaunchKernel(fn, dim3(bp.f.num_tiles * bp.f.num_splits), dim3(nt), args, smem,
                            stream);
}

cudaError_t launch_bwd_pos_reduce(const BwdParams &bp, cudaStream_t stream) {
    const int nt = 256;
    const int n = bp.num_ant_real * 3;
    bwd_pos_reduce_kernel<<<(n + nt - 1) / nt, nt, 0, stream>>>(bp);
    return cudaGetLastError();
}

constexpr int kMeas3Warps = 4;  // 4 warps per CTA: three CTAs per SM at ~150 registers
// voxel pairs per lane and pass: 2 halves the transposes per update but needs ~254
// registers (two CTAs, 8 warps per SM) and measured no faster than 1 (38.6 vs 38.3 ms)
constexpr int kMeasPairs = 1;

int bwd_meas_splits(int num_ant, int fp, int64_t nvox) {
    const int nblk = fp / kBlockF;
    if (nblk > 8 || num_ant < 1 || nvox < 1) return 1;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void *fn = nblk <= 4 ? reinterpret_cast<const void *>(&bp_bwd_meas3_kernel<4, kMeas3Warps, kMeasPairs>)
                               : reinterpret_cast<const void *>(&bp_bwd_meas3_kernel<8, kMeas3Warps, kMeasPairs>);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kMeas3Warps * 32, 0) !=
            cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int64_t slots = (int64_t)sms * per_sm;
    const int64_t bx = (num_ant + kMeas3Warps - 1) / kMeas3Warps;
    const int64_t chunks = (nvox + kMeas2Chunk - 1) / kMeas2Chunk;
    // time ~ rounds of CTAs x work per CTA (1/S of the voxels), +0.5 % per extra range
    int best = 1;
    double best_cost = 1e300;
    for (int s = 1; s <= 64 && s <= chunks; ++s) {
        const double rounds = (double)((bx * s + slots - 1) / slots);
        const double cost = rounds / s * (1.0 + 0.005 * (s - 1));
        if (cost < best_cost - 1e-12) {
            best_cost = cost;
            best = s;
        }
    }
    return best;
}

cudaError_t launch_bwd_meas(const BwdParams &bp, cudaStream_t stream) {
    const int nblk = bp.f.fp / kBlockF;
    const int blocks2 = (bp.num_ant_real + kMeas2Warps - 1) / kMeas2Warps;
    const dim3 grid3((bp.num_ant_real + kMeas3Warps - 1) / kMeas3Warps, bp.meas_splits);
    if (nblk <= 8) {
        if (nblk <= 4)
            bp_bwd_meas3_kernel<4, kMeas3Warps, kMeasPairs><<<grid3, kMeas3Warps * 32, 0, stream>>>(bp);
        else
            bp_bwd_meas3_kernel<8, kMeas3Warps, kMeasPairs><<<grid3, kMeas3Warps * 32, 0, stream>>>(bp);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess || bp.meas_splits <= 1) return e;
        const int64_t n = (int64_t)bp.num_ant_real * bp.num_samples;
        bwd_meas_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(bp);
    } else if (nblk <= 16) {
        bp_bwd_meas2_kernel<16><<<blocks2, kMeas2Warps * 32, 0, stream>>>(bp);
    } else {
        const int blocks = (bp.num_items + kMeasThreads - 1) / kMeasThreads;
        bp_bwd_meas_kernel<<<blocks, kMeasThreads, 0, stream>>>(bp);
    }
    return cudaGetLastError();
}

}  // namespace mmn

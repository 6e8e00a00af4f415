// bp_pos_nufft.cu -- position pass of the adjoint in interpolation form.
//
// The position gradient needs, per (voxel v, antenna a), the two sample sums
//   c_a(v)  = sum_j m[a,j] p_aj(v),   c'_a(v) = sum_j kappa_j m[a,j] p_aj(v),
//   p_aj = exp(-i d kappa_j),  kappa_j = 2pi(1/lambda + j slope/c).
// Both are one antenna's discrete-time Fourier sum evaluated at the point
// u = d slope / c (turns per sample):  c = e^{-2pi i d (1/lambda + J0 slope/c)} M(u) with
// M(u) = sum_j' m[J0+j'] e^{-2pi i j' u},  j' = j - J0 centred on J0 = F/2.  M is
// evaluated as a type-2 non-uniform FFT: on a grid of N = 2F cells,
//   M(u) ~= sum_k phi(N u - k) G_k,   G_k = sum_j' (m / phihat(j'/N)) e^{-2pi i j' k / N},
// with phi the exponential-of-semicircle kernel exp(beta (sqrt(1 - (2z/W)^2) - 1)),
// W = 8 cells, beta = 2.3 W, and phihat its Fourier transform.  Per (voxel, antenna) that
// is eight taps -- weights from degree-8 polynomials in the fractional cell offset
// (es_taps.cuh; mirror taps share one even and one odd part), one 16-byte shared load of
// (G'.re, G.re, G'.im, G.im) and two FFMA2 each -- in place of two F-step Horner chains.
// Accuracy ~1e-7 relative (the FP32 Horner chains' level).
//
// Kernels: nufft_tables_kernel (1/phihat by midpoint quadrature in FP64, twiddles),
// nufft_grid_kernel (per-antenna grids by a direct FP64 transform: F x (N + W - 1) per
// antenna, small next to the voxel work), bp_bwd_pos_nufft_kernel (the forward's tiling and
// double-buffered antenna staging, rows of N + W - 1 cells so no tap wraps; per-antenna
// sums over a CTA's voxels go to the same per-tile partials as the Horner form).
#include <algorithm>

#include "bp_stage.cuh"
#include "es_taps.cuh"

namespace mmn {

namespace {

constexpr double kNuBeta = 2.30 * kNuW;
constexpr int kNuQuad = 256;  // midpoint nodes on [0, W/2]: 1/phihat to ~1e-11

__device__ __forceinline__ double es_kernel(double z) {
    const double t = 2.0 * z / kNuW;
    const double q = 1.0 - t * t;
    return q > 0.0 ? exp(kNuBeta * (sqrt(q) - 1.0)) : 0.0;
}

}  // namespace

// Per (voxel, antenna) geometry of the interpolation form.
//   d      round-trip range in FP64.  Each leg's square root starts from an FP32 rsqrt of the
//          FP32 difference vector and takes one FP64 Newton step (relative error ~1e-13, far
//          below what the phase needs), which avoids the IEEE FP64 square root's slow path.
//   e3     -(unit(v - tx) + unit(v - rx)) in FP32 (the derivative of d with respect to an
//          antenna offset; a direction needs no more).
//   ix, s  grid cell and fractional offset of N * (u mod 1), u = d slope/c, reduced with the
//          1.5*2^52 rounding constant (no conversion instructions); clamped so that a NaN or a
//          fraction that rounds up to 1 still reads inside the row.
//   w[8]   tap weights (es_taps.cuh): P_i(t) and P_i(-t) from one even and one odd part.
struct NuPair {
    double d;
    float e3[3];
    int ix;
    float w[kNuW];
};

__device__ __forceinline__ void nufft_pair(double vxd, double vyd, double vzd, float vx, float vy,
                                           float vz, const AntRec &ar, const float (&txf)[3],
                                           const float (&rxf)[3], bool mono, double ti, double uq,
                                           int n, NuPair &o) {
    const float ax = vx - txf[0], ay = vy - txf[1], az = vz - txf[2];
    const float rf = rsqrtf(fmaf(ax, ax, fmaf(ay, ay, az * az)));
    const double dx = vxd - ar.tx[0], dy = vyd - ar.tx[1], dz = vzd - ar.tx[2];
    const double D = fma(dx, dx, fma(dy, dy, dz * dz));
    const double r = (double)rf;
    double f = D * r;
    f = fma(fma(-f, f, D), 0.5 * r, f);
    double b = f;
    float bx = ax, by = ay, bz = az, rb = rf;
    if (!mono) {
        bx = vx - rxf[0];
        by = vy - rxf[1];
        bz = vz - rxf[2];
        rb = rsqrtf(fmaf(bx, bx, fmaf(by, by, bz * bz)));
        const double ex = vxd - ar.rx[0], ey = vyd - ar.rx[1], ez = vzd - ar.rx[2];
        const double B = fma(ex, ex, fma(ey, ey, ez * ez));
        const double rr = (double)rb;
        b = B * rr;
        b = fma(fma(-b, b, B), 0.5 * rr, b);
    }
    o.d = f + b + ti;
    o.e3[0] = -fmaf(ax, rf, bx * rb);
    o.e3[1] = -fmaf(ay, rf, by * rb);
    o.e3[2] = -fmaf(az, rf, bz * rb);

    const double kRound = 6755399441055744.0;  // 1.5 * 2^52
    const double u = o.d * uq;
    double uf = u - ((u + kRound) - kRound);  // [-1/2, 1/2]
    uf = uf < 0.0 ? uf + 1.0 : uf;            // [0, 1]
    const double x = uf * (double)n;
    const double xt = x + kRound;
    int ix = __double2loint(xt);
    double fr = x - (xt - kRound);             // [-1/2, 1/2]
    ix = fr < 0.0 ? ix - 1 : ix;
    fr = fr < 0.0 ? fr + 1.0 : fr;
    float sfr = (float)fr;
    const bool lo = !(ix >= 0), hi = ix >= n;
    ix = lo ? 0 : (hi ? n - 1 : ix);
    sfr = lo ? 0.f : (hi ? 1.f : sfr);
    o.ix = ix;

    const float t = sfr - 0.5f, t2 = t * t;
#pragma unroll
    for (int i = 0; i < kNuW / 2; ++i) {
        float e = kEsEven[i][kEsEvenTerms - 1];
#pragma unroll
        for (int q = kEsEvenTerms - 2; q >= 0; --q) e = fmaf(e, t2, kEsEven[i][q]);
        float od = kEsOdd[i][kEsOddTerms - 1];
#pragma unroll
        for (int q = kEsOddTerms - 2; q >= 0; --q) od = fmaf(od, t2, kEsOdd[i][q]);
        o.w[i] = fmaf(t, od, e);
        o.w[kNuW - 1 - i] = fmaf(-t, od, e);
    }
}

// sc[j] = 1 / phihat((j - J0) / N) for j < F (one warp per j), tw[k] = e^{-2pi i k/N}.
__global__ void nufft_tables_kernel(int F, int N, int J0, double *__restrict__ sc,
                                    double2 *__restrict__ tw) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gw = gid >> 5;
    const int lane = threadIdx.x & 31;
    if (gw < F) {
        const double xi = (double)(gw - J0) / N;
        const double h = 0.5 * kNuW / kNuQuad;
        double s = 0.0;
        for (int q = lane; q < kNuQuad; q += 32) {
            const double z = (q + 0.5) * h;
            s += es_kernel(z) * cospi(2.0 * xi * z);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sc[gw] = 1.0 / (2.0 * h * s);
    }
    if (gid < N) {
        double sn, cs;
        sincospi(2.0 * (double)gid / N, &sn, &cs);
        tw[gid] = make_double2(cs, -sn);
    }
}

// rows[a][jj] = (G'_k.re, G_k.re, G'_k.im, G_k.im) for cell k = (jj - (W/2 - 1)) mod N,
// jj < N + W - 1: a tap run starting at any cell reads W consecutive entries.
__global__ void nufft_grid_kernel(const float2 *__restrict__ meas, int F, int N, int J0, int row,
                                  double k0, double kd, const double *__restrict__ sc,
                                  const double2 *__restrict__ tw, float4 *__restrict__ rows,
                                  int blocks_per_row) {
    const int a = blockIdx.x / blocks_per_row;
    const int jj = (blockIdx.x - a * blocks_per_row) * blockDim.x + threadIdx.x;
    if (jj >= row) return;
    const int k = ((jj - (kNuW / 2 - 1)) % N + N) % N;
    int idx = (int)((((int64_t)(-J0) * k) % N + N) % N);  // (j - J0) k mod N at j = 0
    const float2 *m = meas + (size_t)a * F;
    double gr = 0.0, gi = 0.0, hr = 0.0, hi = 0.0;
    for (int j = 0; j < F; ++j) {
        const float2 mv = __ldg(m + j);
        const double s = __ldg(sc + j);
        const double2 t = __ldg(tw + idx);
        const double ar = s * (double)mv.x, ai = s * (double)mv.y;
        const double pr = fma(ar, t.x, -ai * t.y), pi = fma(ar, t.y, ai * t.x);
        const double kap = fma((double)j, kd, k0);
        gr += pr;
        gi += pi;
        hr = fma(kap, pr, hr);
        hi = fma(kap, pi, hi);
        idx += k;
        if (idx >= N) idx -= N;
    }
    rows[(size_t)a * row + jj] = make_float4((float)hr, (float)gr, (float)hi, (float)gi);
}

// Position pass, interpolation form.  VOTE: the loss has a vote term (grad_vote set).
template <int T, int NT, bool VOTE>
__global__ void __launch_bounds__(NT) bp_bwd_pos_nufft_kernel(const BwdParams bp) {
    const FwdParams &p = bp.f;
    extern __shared__ __align__(128) unsigned char smem[];
    Stage st;
    st.bars = reinterpret_cast<uint64_t *>(smem);
    st.base = smem + 128;
    st.nas = p.ant_per_stage;
    st.esz = 16;
    st.fp = p.fp;  // grid row length N + W - 1
    st.stage_bytes = (size_t)st.nas * sizeof(AntRec) + (size_t)st.nas * st.fp * st.esz;
    float *wsum = reinterpret_cast<float *>(st.base + 2 * st.stage_bytes);  // [NT/32][nas][3]
    constexpr int NW = NT / 32;
    const int row_len = p.fp;
    const int n = bp.nu_n;
    const double uq = bp.nu_u, k0c = bp.nu_k0c;
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
    double vxd[T], vyd[T], vzd[T];
    float2 gi[T], gw[T][3];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        const int64_t rel = rbase + (int64_t)k * NT;
        decode_voxel(p, rel, vx[k], vy[k], vz[k]);
        vxd[k] = vx[k];
        vyd[k] = vy[k];
        vzd[k] = vz[k];
        const bool ok = rel < p.vox_count;
        const int64_t v = p.vox_start + (ok ? rel : 0);
        gi[k] = (ok && bp.grad_image) ? bp.grad_image[v] : make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            gw[k][q] = (VOTE && ok) ? bp.grad_vote[q * p.nvox + v] : make_float2(0.f, 0.f);
    }
    const bool mono = *p.mono_flag != 0;

    for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        bool ok = mbar_wait_bounded(&st.bars[s], (uint32_t)((c >> 1) & 1), p.status);
        if (!__syncthreads_and(ok)) return;
        const AntRec *ants = st.ants(s);
        const float4 *mstage = reinterpret_cast<const float4 *>(st.meas(s));
        const int a0 = a_begin + c * st.nas;
        const int na = min(st.nas, a_end - a0);

        for (int a = 0; a < na; ++a) {
            const AntRec &ar = ants[a];
            const float4 *row = mstage + (size_t)a * row_len;
            // FP32 antenna positions for the gradient directions (a direction needs no more)
            const float txf[3] = {(float)ar.tx[0], (float)ar.tx[1], (float)ar.tx[2]};
            const float rxf[3] = {(float)ar.rx[0], (float)ar.rx[1], (float)ar.rx[2]};
            float g3[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < T; ++k) {
                NuPair g;
                nufft_pair(vxd[k], vyd[k], vzd[k], vx[k], vy[k], vz[k], ar, txf, rxf, mono, p.ti,
                           uq, n, g);
                const double d = g.d;
                const float *e3 = g.e3;
                float2 acc_r = make_float2(0.f, 0.f), acc_i = make_float2(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < kNuW; ++i) {
                    const float4 e = row[g.ix + i];
                    acc_r = __ffma2_rn(make_float2(g.w[i], g.w[i]), make_float2(e.x, e.y), acc_r);
                    acc_i = __ffma2_rn(make_float2(g.w[i], g.w[i]), make_float2(e.z, e.w), acc_i);
                }
                // rotate by the anchor e^{-2pi i d (1/lambda + J0 slope/c)}: .x c', .y c
                const float2 an = cis_fp64_phase(-d * k0c);
                const float2 anr = make_float2(an.x, an.x), ani = make_float2(an.y, an.y);
                const float2 cr = __ffma2_rn(anr, acc_r, __fmul2_rn(make_float2(-an.y, -an.y), acc_i));
                const float2 ci = __ffma2_rn(anr, acc_i, __fmul2_rn(ani, acc_r));

                float Gr = gi[k].x, Gi = gi[k].y;
                if (VOTE) {
                    const float uu[3] = {ar.virt[0] - vx[k], ar.virt[1] - vy[k],
                                         ar.virt[2] - vz[k]};
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        Gr = fmaf(gw[k][q].x, uu[q], Gr);
                        Gi = fmaf(gw[k][q].y, uu[q], Gi);
                    }
                }
                const float s1 = Gr * ci.x - Gi * cr.x;  // Im(conj(G) c')
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    g3[q] += VOTE ? fmaf(s1, e3[q], gw[k][q].x * cr.y + gw[k][q].y * ci.y)
                                  : s1 * e3[q];
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
}

// Launch shapes (voxels per thread, threads per CTA, cap on one shared-memory stage).
struct NuVariant {
    int t, nt, stage_cap;
    const void *fn_vote, *fn_img;
    const char *name;
};

#define MMN_NU_VARIANT(T, NT, CAP)                                                         \
    {T, NT, CAP, reinterpret_cast<const void *>(&bp_bwd_pos_nufft_kernel<T, NT, true>),     \
     reinterpret_cast<const void *>(&bp_bwd_pos_nufft_kernel<T, NT, false>),               \
     "interp_t" #T "_n" #NT "_s" #CAP}

// At 64^3 voxels, 4096 antennas, 128 samples (position pass alone; with vote term / image
// loss only): 9.00/8.43, 9.64/8.16, 11.1/11.8, 10.7/9.85 ms in this order; the first is the
// default.
const NuVariant kNuVariants[] = {
    MMN_NU_VARIANT(2, 128, 24),
    MMN_NU_VARIANT(2, 256, 24),
    MMN_NU_VARIANT(1, 256, 48),
    MMN_NU_VARIANT(1, 128, 16),
};
#undef MMN_NU_VARIANT

int bwd_pos_nufft_num_variants() { return (int)(sizeof(kNuVariants) / sizeof(kNuVariants[0])); }

const char *bwd_pos_nufft_variant_name(int variant) {
    return variant >= 0 && variant < bwd_pos_nufft_num_variants() ? kNuVariants[variant].name
                                                                   : nullptr;
}

const void *bwd_pos_nufft_kernel_ptr(int variant, bool vote, int *threads, int *voxels_per_thread,
                                     int *stage_cap_bytes) {
    if (variant < 0 || variant >= bwd_pos_nufft_num_variants()) variant = 0;
    const NuVariant &v = kNuVariants[variant];
    *threads = v.nt;
    *voxels_per_thread = v.t;
    *stage_cap_bytes = v.stage_cap * 1024;
    return vote ? v.fn_vote : v.fn_img;
}

cudaError_t launch_nufft_grid(const float *meas, int A, int F, int N, int J0, double k0,
                              double kd, double *sc, double2 *tw, float4 *rows,
                              cudaStream_t stream) {
    const int nt = 256;
    const int64_t tthreads = std::max<int64_t>((int64_t)F * 32, N);
    nufft_tables_kernel<<<(unsigned)((tthreads + nt - 1) / nt), nt, 0, stream>>>(F, N, J0, sc,
                                                                                 tw);
    const int row = nufft_row(N);
    const int bpr = (row + nt - 1) / nt;
    nufft_grid_kernel<<<(unsigned)((int64_t)A * bpr), nt, 0, stream>>>(
        reinterpret_cast<const float2 *>(meas), F, N, J0, row, k0, kd, sc, tw, rows, bpr);
    return cudaGetLastError();
}

}  // namespace mmn

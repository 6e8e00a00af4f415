// bp_nufft.cu -- the adjoint's two passes in interpolation form.
//
// Position pass.  The position gradient needs, per (voxel v, antenna a), the two sums
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
// Measurement pass.  dL/dm[a, J0+j'] = sum_v G_a(v) conj(p) = sum_v h_v e^{2pi i j' u_v} with
// h_v = G_a(v) conj(anchor): the transposed (type-1) transform.  Each voxel spreads
// h_v phi(N u_v - k) onto the same 8 cells it would read, the cells are summed over all
// voxels into the antenna's grid S_k, and dL/dm[a, J0+j'] = sum_k S_k e^{2pi i j' k/N} /
// phihat(j'/N) per antenna.  The spread is summed without atomics (deterministic): a warp
// owns one antenna's grid row; each lane writes its 8 weighted cells into its own
// 16-cell window in shared memory (cell-major across the lanes: conflict-free) at its
// offset from the warp's lowest cell, and one
// XOR-permuted transpose-reduce (31 shuffles) leaves cell j/2 of the window summed over
// the warp in lane j.  Lanes whose cells fall outside a 16-cell window wait for the next
// round, so any spread of distances is handled.
//
// Kernels: nufft_tables_kernel (1/phihat by midpoint quadrature in FP64, twiddles),
// nufft_grid_kernel (per-antenna grids by a direct FP64 transform: F x (N + W - 1) per
// antenna, small next to the voxel work), bp_bwd_pos_nufft_kernel (the forward's tiling and
// double-buffered antenna staging, rows of N + W - 1 cells so no tap wraps; per-antenna
// sums over a CTA's voxels go to the same per-tile partials as the Horner form),
// nufft_vox_kernel + bp_bwd_meas_nufft_kernel + nufft_meas_out_kernel (measurement pass).
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
// jj < N + W - 1: a tap run starting at any cell reads W consecutive entries.  FWD_ONLY:
// the forward reads only G, so its rows are (G_k.re, G_k.im) -- 8 bytes a cell -- and the
// G' sums are not formed; those rows carry one more cell (never read) to an even length,
// which keeps them multiples of 16 bytes for the bulk copies.
template <bool FWD_ONLY>
__global__ void nufft_grid_kernel(const float2 *__restrict__ meas, int F, int N, int J0, int row,
                                  double k0, double kd, const double *__restrict__ sc,
                                  const double2 *__restrict__ tw, void *__restrict__ rows,
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
        gr += pr;
        gi += pi;
        if (!FWD_ONLY) {
            const double kap = fma((double)j, kd, k0);
            hr = fma(kap, pr, hr);
            hi = fma(kap, pi, hi);
        }
        idx += k;
        if (idx >= N) idx -= N;
    }
    if (FWD_ONLY)
        static_cast<float2 *>(rows)[(size_t)a * row + jj] = make_float2((float)gr, (float)gi);
    else
        static_cast<float4 *>(rows)[(size_t)a * row + jj] =
            make_float4((float)hr, (float)gr, (float)hi, (float)gi);
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
    if (c_failed >= 0) {
        st.drain_after_timeout((uint32_t)c_failed, c_failed + 1 < n_chunks, p.status);
        return;
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

// ---------------------------------------------------------------- forward pass
// The forward's per-(voxel, antenna) sum c = sum_j m_j p_j by the same 8-tap gather as the
// position pass (the rows' G cells), accumulated as I += c, W += c (virt - v) per voxel
// over the CTA's antennas; results go through store_voxel (direct or per-split partials).
template <int T, int NT>
__global__ void __launch_bounds__(NT) bp_fwd_nufft_kernel(const BwdParams bp) {
    const FwdParams &p = bp.f;
    extern __shared__ __align__(128) unsigned char smem[];
    Stage st;
    st.bars = reinterpret_cast<uint64_t *>(smem);
    st.base = smem + 128;
    st.nas = p.ant_per_stage;
    st.esz = 8;    // (G.re, G.im) cells
    st.fp = p.fp;  // grid row length N + W - 1
    st.stage_bytes = (size_t)st.nas * sizeof(AntRec) + (size_t)st.nas * st.fp * st.esz;
    const int row_len = p.fp;
    const int n = bp.nu_n;
    const double uq = bp.nu_u, k0c = bp.nu_k0c;
    const int tile = blockIdx.x % p.num_tiles;
    const int split = blockIdx.x / p.num_tiles;
    const int a_begin = split * p.ant_per_split;
    const int a_end = min(p.num_ant, a_begin + p.ant_per_split);
    const int n_chunks = a_end > a_begin ? (a_end - a_begin + st.nas - 1) / st.nas : 0;

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
    float acc[T][8];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        decode_voxel(p, rbase + (int64_t)k * NT, vx[k], vy[k], vz[k]);
        vxd[k] = vx[k];
        vyd[k] = vy[k];
        vzd[k] = vz[k];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[k][q] = 0.f;
    }
    const bool mono = *p.mono_flag != 0;

    int c_failed = -1;  // chunk whose wait gave up; the drain runs after the loop
    for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        bool ok = mbar_wait_bounded(&st.bars[s], (uint32_t)((c >> 1) & 1), p.status);
        if (!__syncthreads_and(ok)) {
            c_failed = c;
            break;
        }
        const AntRec *ants = st.ants(s);
        const float2 *mstage = reinterpret_cast<const float2 *>(st.meas(s));
        const int a0 = a_begin + c * st.nas;
        const int na = min(st.nas, a_end - a0);
        for (int a = 0; a < na; ++a) {
            const AntRec &ar = ants[a];
            const float2 *row = mstage + (size_t)a * row_len;
            const float txf[3] = {(float)ar.tx[0], (float)ar.tx[1], (float)ar.tx[2]};
            const float rxf[3] = {(float)ar.rx[0], (float)ar.rx[1], (float)ar.rx[2]};
#pragma unroll
            for (int k = 0; k < T; ++k) {
                NuPair g;
                nufft_pair(vxd[k], vyd[k], vzd[k], vx[k], vy[k], vz[k], ar, txf, rxf, mono, p.ti,
                           uq, n, g);
                float2 h = make_float2(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < kNuW; ++i)
                    h = __ffma2_rn(make_float2(g.w[i], g.w[i]), row[g.ix + i], h);
                const float2 an = cis_fp64_phase(-g.d * k0c);
                const float cr = fmaf(an.x, h.x, -an.y * h.y), ci = fmaf(an.x, h.y, an.y * h.x);
                const float u0 = ar.virt[0] - vx[k], u1 = ar.virt[1] - vy[k],
                            u2 = ar.virt[2] - vz[k];
                acc[k][0] += cr;
                acc[k][1] += ci;
                acc[k][2] = fmaf(cr, u0, acc[k][2]);
                acc[k][3] = fmaf(ci, u0, acc[k][3]);
                acc[k][4] = fmaf(cr, u1, acc[k][4]);
                acc[k][5] = fmaf(ci, u1, acc[k][5]);
                acc[k][6] = fmaf(cr, u2, acc[k][6]);
                acc[k][7] = fmaf(ci, u2, acc[k][7]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + 2 < n_chunks) st.issue(p, c + 2, a_begin, a_end);
    }
    if (c_failed >= 0) {
        st.drain_after_timeout((uint32_t)c_failed, c_failed + 1 < n_chunks, p.status);
        return;
    }
#pragma unroll
    for (int k = 0; k < T; ++k) store_voxel(p, split, rbase + (int64_t)k * NT, acc[k]);
}

constexpr int kNuFwdT = 2, kNuFwdNT = 128;

const void *fwd_nufft_kernel_ptr(int *threads, int *voxels_per_thread) {
    *threads = kNuFwdNT;
    *voxels_per_thread = kNuFwdT;
    return reinterpret_cast<const void *>(&bp_fwd_nufft_kernel<kNuFwdT, kNuFwdNT>);
}

// ------------------------------------------------------------- measurement pass

// Voxel records of the measurement pass, 5 x 16 bytes: (x, y) and (z, 0) in FP64, (x, y, z)
// in FP32, (gI, gW_x), (gW_y, gW_z).
__global__ void nufft_vox_kernel(const FwdParams p, const float2 *__restrict__ grad_image,
                                 const float2 *__restrict__ grad_vote, float4 *__restrict__ rec) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= p.nvox) return;
    const int64_t nyz = (int64_t)p.ny * p.nz;
    const int ix = (int)(v / nyz);
    const int64_t rem = v - (int64_t)ix * nyz;
    const int iy = (int)(rem / p.nz);
    const int iz = (int)(rem - (int64_t)iy * p.nz);
    const float x = p.x_locs[ix], y = p.y_locs[iy], z = p.z_locs[iz];
    const float2 gi = grad_image ? grad_image[v] : make_float2(0.f, 0.f);
    float2 gw[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    if (grad_vote)
        for (int k = 0; k < 3; ++k) gw[k] = grad_vote[k * p.nvox + v];
    float4 *r = rec + 5 * v;
    reinterpret_cast<double2 *>(r)[0] = make_double2(x, y);
    reinterpret_cast<double2 *>(r)[1] = make_double2(z, 0.0);
    r[2] = make_float4(x, y, z, 0.f);
    r[3] = make_float4(gi.x, gi.y, gw[0].x, gw[0].y);
    r[4] = make_float4(gw[1].x, gw[1].y, gw[2].x, gw[2].y);
}

constexpr int kNuMeasWarps = 4;
constexpr int kNuWin = 16;  // window cells per round

// blockIdx.x = antenna group (one antenna per warp) + groups * voxel range.
template <int NW>
__global__ void __launch_bounds__(NW * 32) bp_bwd_meas_nufft_kernel(const NuMeasParams q) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int groups = (q.num_ant + NW - 1) / NW;
    const int g = blockIdx.x % groups;
    const int range = blockIdx.x / groups;
    const int a = g * NW + warp;
    if (a >= q.num_ant) return;  // warps are independent: no block-wide barrier below
    // per warp: its antenna's grid row, then the lanes' windows cell-major (cell * 32 + lane:
    // every access of a half-warp falls in 16 different banks, whatever the cells)
    float2 *row = reinterpret_cast<float2 *>(smem) + (size_t)warp * (q.mrow + 32 * kNuWin);
    float2 *win = row + q.mrow + lane;
    float *rowf = reinterpret_cast<float *>(row);
    for (int c = lane; c < q.mrow; c += 32) row[c] = make_float2(0.f, 0.f);
    __syncwarp();

    const AntRec ar = q.ant[a];
    const float txf[3] = {(float)ar.tx[0], (float)ar.tx[1], (float)ar.tx[2]};
    const float rxf[3] = {(float)ar.rx[0], (float)ar.rx[1], (float)ar.rx[2]};
    const bool mono = *q.mono_flag != 0;
    const bool odd = lane & 1;
    const int64_t v0 = (int64_t)range * q.vox_per_range;
    const int64_t v1 = min(q.nvox, v0 + q.vox_per_range);

    for (int64_t vb = v0; vb < v1; vb += 32) {
        const int64_t v = vb + lane;
        const bool ok = v < v1;
        const float4 *r = q.vox + 5 * (ok ? v : v0);
        const double2 xy = reinterpret_cast<const double2 *>(r)[0];
        const double2 zz = reinterpret_cast<const double2 *>(r)[1];
        const float4 fx = r[2], g0 = r[3], g1 = r[4];
        NuPair pr;
        nufft_pair(xy.x, xy.y, zz.x, fx.x, fx.y, fx.z, ar, txf, rxf, mono, q.ti, q.uq, q.n, pr);
        const float2 an = cis_fp64_phase(-pr.d * q.k0c);
        // G = gI + gW . (virt - v);  h = G conj(anchor), stored (re, im) on even lanes and
        // (im, re) on odd lanes, the order the transpose-reduce reads them in
        const float u0 = ar.virt[0] - fx.x, u1 = ar.virt[1] - fx.y, u2 = ar.virt[2] - fx.z;
        float Gr = fmaf(g0.z, u0, g0.x), Gi = fmaf(g0.w, u0, g0.y);
        Gr = fmaf(g1.x, u1, Gr);
        Gi = fmaf(g1.y, u1, Gi);
        Gr = fmaf(g1.z, u2, Gr);
        Gi = fmaf(g1.w, u2, Gi);
        const float hr = fmaf(Gr, an.x, Gi * an.y), hi = fmaf(Gi, an.x, -Gr * an.y);
        const float h0 = odd ? hi : hr, h1 = odd ? hr : hi;
        const int ix = pr.ix;

        unsigned pending = __ballot_sync(0xffffffffu, ok);
        while (pending) {
            const bool mine_p = (pending >> lane) & 1u;
            const int base = __reduce_min_sync(0xffffffffu, mine_p ? ix : 0x7fffffff);
            const int off = ix - base;
            const bool mine = mine_p && off <= 8;
            if (mine) {
#pragma unroll
                for (int i = 0; i < kNuW; ++i)
                    win[(off + i) * 32] = make_float2(h0 * pr.w[i], h1 * pr.w[i]);
            }
            __syncwarp();
            // slot s holds window component s ^ lane: component c = cell c/2, re/im c&1
            float vv[32];
#pragma unroll
            for (int s2 = 0; s2 < 16; ++s2) {
                const int cell = s2 ^ (lane >> 1);
                const int i = cell - off;
                float2 t = make_float2(0.f, 0.f);
                if (mine && i >= 0 && i < kNuW) t = win[cell * 32];
                vv[2 * s2] = t.x;
                vv[2 * s2 + 1] = t.y;
            }
            __syncwarp();
#pragma unroll
            for (int h = 16; h >= 1; h >>= 1) {
#pragma unroll
                for (int i = 0; i < h; ++i) vv[i] += __shfl_xor_sync(0xffffffffu, vv[i + h], h);
            }
            rowf[2 * (base + (lane >> 1)) + (lane & 1)] += vv[0];
            __syncwarp();
            pending &= ~__ballot_sync(0xffffffffu, mine);
        }
    }
    float2 *dst = q.part + ((size_t)range * q.num_ant + a) * q.mrow;
    for (int c = lane; c < q.mrow; c += 32) dst[c] = row[c];
}

// Per antenna (one block): S_k = sum over voxel ranges and over the row cells that wrap
// onto cell k, then dL/dm[a, j] = sc[j] sum_k S_k e^{2pi i (j - J0) k / N} in FP64.
__global__ void nufft_meas_out_kernel(const NuMeasParams q) {
    extern __shared__ __align__(16) unsigned char smem_out[];
    double2 *S = reinterpret_cast<double2 *>(smem_out);
    const int a = blockIdx.x;
    const int n = q.n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double sr = 0.0, si = 0.0;
        for (int r = 0; r < q.ranges; ++r) {
            const float2 *row = q.part + ((size_t)r * q.num_ant + a) * q.mrow;
            for (int jj = (k + kNuW / 2 - 1) % n; jj < q.mrow; jj += n) {
                sr += row[jj].x;
                si += row[jj].y;
            }
        }
        S[k] = make_double2(sr, si);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < q.F; j += blockDim.x) {
        const int step = ((j - q.J0) % n + n) % n;
        int idx = 0;
        double er = 0.0, ei = 0.0;
        for (int k = 0; k < n; ++k) {
            const double2 t = q.tw[idx];  // e^{-2pi i idx/N}; the transform needs its conjugate
            const double2 sk = S[k];
            er = fma(sk.x, t.x, fma(sk.y, t.y, er));
            ei = fma(sk.y, t.x, fma(-sk.x, t.y, ei));
            idx += step;
            if (idx >= n) idx -= n;
        }
        const double sc = q.sc[j];
        q.grad_meas[(size_t)a * q.F + j] = make_float2((float)(er * sc), (float)(ei * sc));
    }
}

size_t nufft_meas_smem(int mrow) {
    return (size_t)kNuMeasWarps * (mrow + 32 * kNuWin) * sizeof(float2);
}

int nufft_meas_warps() { return kNuMeasWarps; }

const void *nufft_meas_kernel_ptr() {
    return reinterpret_cast<const void *>(&bp_bwd_meas_nufft_kernel<kNuMeasWarps>);
}

cudaError_t launch_nufft_meas(const NuMeasParams &q, const FwdParams &p,
                              const float2 *grad_image, const float2 *grad_vote, float4 *rec,
                              cudaStream_t stream) {
    const int nt = 256;
    nufft_vox_kernel<<<(unsigned)((p.nvox + nt - 1) / nt), nt, 0, stream>>>(p, grad_image,
                                                                             grad_vote, rec);
    const size_t smem = nufft_meas_smem(q.mrow);
    const void *fn = nufft_meas_kernel_ptr();
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int groups = (q.num_ant + kNuMeasWarps - 1) / kNuMeasWarps;
    void *args[] = {const_cast<NuMeasParams *>(&q)};
    cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)((int64_t)groups * q.ranges)),
                                     dim3(kNuMeasWarps * 32), args, smem, stream);
    if (e != cudaSuccess) return e;
    const size_t osmem = (size_t)q.n * sizeof(double2);
    if (osmem > 48 * 1024)
        cudaFuncSetAttribute(reinterpret_cast<const void *>(&nufft_meas_out_kernel),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)osmem);
    nufft_meas_out_kernel<<<q.num_ant, 256, osmem, stream>>>(q);
    return cudaGetLastError();
}

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

cudaError_t launch_nufft_tables(int F, int N, int J0, double *sc, double2 *tw,
                                cudaStream_t stream) {
    const int nt = 256;
    const int64_t tthreads = std::max<int64_t>((int64_t)F * 32, N);
    nufft_tables_kernel<<<(unsigned)((tthreads + nt - 1) / nt), nt, 0, stream>>>(F, N, J0, sc,
                                                                                 tw);
    return cudaGetLastError();
}

cudaError_t launch_nufft_grid(const float *meas, int A, int F, int N, int J0, double k0,
                              double kd, const double *sc, const double2 *tw, void *rows,
                              bool fwd_only, cudaStream_t stream) {
    const int nt = 256;
    const int row = fwd_only ? nufft_row_fwd(N) : nufft_row(N);
    const int bpr = (row + nt - 1) / nt;
    const unsigned grid = (unsigned)((int64_t)A * bpr);
    const float2 *m = reinterpret_cast<const float2 *>(meas);
    if (fwd_only)
        nufft_grid_kernel<true><<<grid, nt, 0, stream>>>(m, F, N, J0, row, k0, kd, sc, tw, rows,
                                                         bpr);
    else
        nufft_grid_kernel<false><<<grid, nt, 0, stream>>>(m, F, N, J0, row, k0, kd, sc, tw, rows,
                                                          bpr);
    return cudaGetLastError();
}

}  // namespace mmn

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
// MIXED form.  Per (voxel, antenna): d in FP64; the sample sum is split into blocks of
// L = 32 (or 64) samples, each summed in FP32 by a rotation recurrence with
// z = exp(-j d kappa_step), and every block is re-anchored with the exact FP64-wrapped
// phase
//     c_i += exp(-j d kappa_{L b}) * h_b,   h_b = sum_{t<L} m[i, L b + t] * z^t.
// The per-sample work is 4 FP32 lane operations, no SFU, in one of two recurrences:
//  * second-order (Clenshaw) -- the autotuner's usual pick:
//    b_t = m_t + 2 cos(theta) b_{t+1} - b_{t+2}, h_b = b_0 - conj(z) b_1.  The multiplier
//    is real, so a (voxel, antenna) chain is one (re, im) register pair: one FADD2 + one
//    FFMA2 (Blackwell's packed FP32) per sample on plain (re, im) samples, one 16-byte
//    shared load feeding two samples to each of the thread's voxels.  The default variant
//    splits each 64-sample block into even and odd chains in z^2 (clen_block_eo), which
//    keeps the second-order form's extra error small at a few per cent of its speed;
//  * first-order Horner, h <- h z + m_t (one complex multiply-add): voxel pairs or
//    antenna pairs in the halves of FFMA2 (the sample duplicated into (re, re, im, im)
//    or antenna-pair records), or scalar FFMA.
//
// PLAIN form.  FP32 distance and FP32 phase -d*kappa_j with one sincosf per sample,
// then a complex multiply-add -- the straightforward FP32 kernel.
//
// Work item = (voxel tile, antenna split).  A CTA of NT threads owns NT*T voxels (T
// per thread, strided by NT so stores coalesce).  Antenna records and measurement
// rows stream through a double-buffered shared-memory stage filled by one elected
// thread with bulk TMA copies (cp.async.bulk) completing on an mbarrier.  With one
// split per tile the CTA writes the final image/vote; otherwise it writes an 8-float
// partial per voxel that bp_reduce_partials sums in split order (deterministic).
#include "bp_stage.cuh"

namespace mmn {


// Kernel forms
constexpr int kFormMixedPair = 0;    // FFMA2 voxel pairs, (re,re,im,im) samples
constexpr int kFormMixedScalar = 1;  // scalar FFMA, (re,im) samples
constexpr int kFormPlain = 2;        // FP32 sincosf per sample, (re,im) samples
constexpr int kFormMixedAntPair = 3; // FFMA2 antenna pairs, (re_a,re_a',im_a,im_a') samples
// voxel pairs as kFormMixedPair, each 32-sample block evaluated as two independent 16-step
// Horner chains joined by one multiply with z^16 (two dependency chains per thread)
constexpr int kFormMixedPairSplit = 4;
// second-order (Clenshaw) form of the block sum, (re, im) samples: see fwd_item
constexpr int kFormMixedClen = 5;
constexpr int kFormMixedClen64 = 6;  // the same with 64-sample blocks
// 64-sample blocks as two interleaved second-order chains in z^2 (clen_block_eo)
constexpr int kFormMixedClenEO = 7;
// The second-order form is used for a warp's (voxels, antenna) pairs when every lane's
// per-sample rotation z = e^{-i theta} has |cos theta| <= kClenMaxCos (theta in
// [0.2, pi - 0.2]); otherwise that antenna's blocks run the first-order Horner form.
constexpr float kClenMaxCos = 0.98f;

// Block anchors: kAnchorPoly recomputes exp(-j d kappa_{32b}) per block from the FP64
// phase (FP64 quarter-turn reduction + FP32 Taylor polynomials); kAnchorFixed steps a
// 64-bit fixed-point phase accumulator per block and evaluates the hardware sine/cosine
// on the wrapped angle.
constexpr int kAnchorPoly = 0;
constexpr int kAnchorFixed = 1;
// kAnchorFixed2: the fixed-point anchors of kAnchorFixed with a cheaper prologue -- the
// FP64 range from an FP32 rsqrt seed and one Newton step, the per-sample turn count
// u = -d slope/c as 64-bit fixed point from the FP64 rounding constant (no 64-bit
// conversion), the rotation z from u's top word (integer quarter turns + FP32 Taylor),
// the block step as u << 5 and the start phase rounded to 2^-33 turns.
constexpr int kAnchorFixed2 = 2;

// One block of the second-order form (see fwd_item): the sums h_k = sum_{t<L} m_t z_k^t of
// the thread's T voxels against one antenna, from L samples (re, im) at mb (two per
// 16-byte load), by Clenshaw's recurrence when `clen`, else by first-order Horner.
template <int T, int L>
__device__ __forceinline__ void clen_block(const float4 *mb, bool clen, const float2 (&c2)[T],
                                           const float (&zr)[T], const float (&zi)[T],
                                           float (&sr)[T], float (&si)[T]) {
    const float4 top = mb[L / 2 - 1];  // samples L-2, L-1
    if (clen) {
        float2 b1[T], b2[T];
#pragma unroll
        for (int k = 0; k < T; ++k) {
            b2[k] = make_float2(top.z, top.w);  // b_{L-1} = m_{L-1}
            b1[k] = __ffma2_rn(c2[k], b2[k], make_float2(top.x, top.y));  // b_{L-2}
        }
#pragma unroll
        for (int q = L / 2 - 2; q >= 0; --q) {
            const float4 mm = mb[q];
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float2 dd = __fadd2_rn(make_float2(mm.z, mm.w),
                                             make_float2(-b2[k].x, -b2[k].y));
                b2[k] = b1[k];
                b1[k] = __ffma2_rn(c2[k], b1[k], dd);
            }
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float2 dd = __fadd2_rn(make_float2(mm.x, mm.y),
                                             make_float2(-b2[k].x, -b2[k].y));
                b2[k] = b1[k];
                b1[k] = __ffma2_rn(c2[k], b1[k], dd);
            }
        }
        // h = b_0 - conj(z) b_1   (b1 = b_0, b2 = b_1)
#pragma unroll
        for (int k = 0; k < T; ++k) {
            sr[k] = fmaf(-zr[k], b2[k].x, fmaf(-zi[k], b2[k].y, b1[k].x));
            si[k] = fmaf(-zr[k], b2[k].y, fmaf(zi[k], b2[k].x, b1[k].y));
        }
    } else {
        // first-order Horner, h <- h z + m_t, voxel pairs in the halves of FFMA2 (each half
        // rounds as the scalar FMA: the same bits as the scalar form)
        constexpr int P = T / 2;
        float2 hr[P], hi[P], zr2[P], zi2[P], nzi2[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            zr2[q] = make_float2(zr[2 * q], zr[2 * q + 1]);
            zi2[q] = make_float2(zi[2 * q], zi[2 * q + 1]);
            nzi2[q] = make_float2(-zi[2 * q], -zi[2 * q + 1]);
            hr[q] = make_float2(top.z, top.z);
            hi[q] = make_float2(top.w, top.w);
            const float2 u = __ffma2_rn(hr[q], zr2[q], make_float2(top.x, top.x));
            const float2 w = __ffma2_rn(hr[q], zi2[q], make_float2(top.y, top.y));
            hr[q] = __ffma2_rn(hi[q], nzi2[q], u);
            hi[q] = __ffma2_rn(hi[q], zr2[q], w);
        }
#pragma unroll 1
        for (int q2 = L / 2 - 2; q2 >= 0; --q2) {
            const float4 mm = mb[q2];
            const float2 m1r = make_float2(mm.z, mm.z), m1i = make_float2(mm.w, mm.w);
            const float2 m0r = make_float2(mm.x, mm.x), m0i = make_float2(mm.y, mm.y);
#pragma unroll
            for (int q = 0; q < P; ++q) {
                float2 u = __ffma2_rn(hr[q], zr2[q], m1r);
                float2 w = __ffma2_rn(hr[q], zi2[q], m1i);
                hr[q] = __ffma2_rn(hi[q], nzi2[q], u);
                hi[q] = __ffma2_rn(hi[q], zr2[q], w);
                u = __ffma2_rn(hr[q], zr2[q], m0r);
                w = __ffma2_rn(hr[q], zi2[q], m0i);
                hr[q] = __ffma2_rn(hi[q], nzi2[q], u);
                hi[q] = __ffma2_rn(hi[q], zr2[q], w);
            }
        }
#pragma unroll
        for (int q = 0; q < P; ++q) {
            sr[2 * q] = hr[q].x;
            sr[2 * q + 1] = hr[q].y;
            si[2 * q] = hi[q].x;
            si[2 * q + 1] = hi[q].y;
        }
    }
}

// A 64-sample block of the split second-order form (kFormMixedClenEO): the even and the
// odd samples as two chains in w = z^2, E = sum_k m_{2k} w^k and O = sum_k m_{2k+1} w^k,
// each by Clenshaw's recurrence with the real multiplier c2w = 2 cos(2 phi), and
// h = E + z O.  One 16-byte load (samples 2k, 2k+1) feeds one step of both chains; the
// chains are half as long and their modes e^{+-2 i phi} twice as far from 0, which keeps
// the growth of b and the effect of the FP32 multiplier's rounding several times smaller
// than one chain over the whole block.
template <int T>
__device__ __forceinline__ void clen_block_eo(const float4 *mb, const float (&zr)[T],
                                              const float (&zi)[T], const float (&wr)[T],
                                              const float (&wi)[T], float (&sr)[T],
                                              float (&si)[T]) {
    const float4 top = mb[31];  // samples 62 (even k = 31), 63 (odd k = 31)
    float2 be1[T], be2[T], bo1[T], bo2[T], c2[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        c2[k] = make_float2(2.f * wr[k], 2.f * wr[k]);
        be1[k] = make_float2(top.x, top.y);  // b_31 of each chain
        bo1[k] = make_float2(top.z, top.w);
        be2[k] = bo2[k] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q = 30; q >= 0; --q) {
        const float4 mm = mb[q];
#pragma unroll
        for (int k = 0; k < T; ++k) {
            const float2 de = __fadd2_rn(make_float2(mm.x, mm.y),
                                         make_float2(-be2[k].x, -be2[k].y));
            const float2 dd = __fadd2_rn(make_float2(mm.z, mm.w),
                                         make_float2(-bo2[k].x, -bo2[k].y));
            be2[k] = be1[k];
            bo2[k] = bo1[k];
            be1[k] = __ffma2_rn(c2[k], be1[k], de);
            bo1[k] = __ffma2_rn(c2[k], bo1[k], dd);
        }
    }
#pragma unroll
    for (int k = 0; k < T; ++k) {
        // E = b0 - conj(w) b1 for each chain, then h = E + z O
        const float er = fmaf(-wr[k], be2[k].x, fmaf(-wi[k], be2[k].y, be1[k].x));
        const float ei = fmaf(-wr[k], be2[k].y, fmaf(wi[k], be2[k].x, be1[k].y));
        const float orr = fmaf(-wr[k], bo2[k].x, fmaf(-wi[k], bo2[k].y, bo1[k].x));
        const float oi = fmaf(-wr[k], bo2[k].y, fmaf(wi[k], bo2[k].x, bo1[k].y));
        sr[k] = fmaf(zr[k], orr, fmaf(-zi[k], oi, er));
        si[k] = fmaf(zr[k], oi, fmaf(zi[k], orr, ei));
    }
}

// The last rem (< L) valid samples of a row, as clen_block with a runtime length: the
// recurrence starts at b_rem = b_{rem+1} = 0, which is where the padded zeros above them
// would have left it.
template <int T>
__device__ __forceinline__ void clen_partial(const float2 *m2, int rem, bool clen,
                                             const float2 (&c2)[T], const float (&zr)[T],
                                             const float (&zi)[T], float (&sr)[T],
                                             float (&si)[T]) {
    if (clen) {
        float2 b1[T], b2[T];
#pragma unroll
        for (int k = 0; k < T; ++k) b1[k] = b2[k] = make_float2(0.f, 0.f);
#pragma unroll 2
        for (int t = rem - 1; t >= 0; --t) {
            const float2 m = m2[t];
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float2 dd = __fadd2_rn(m, make_float2(-b2[k].x, -b2[k].y));
                b2[k] = b1[k];
                b1[k] = __ffma2_rn(c2[k], b1[k], dd);
            }
        }
#pragma unroll
        for (int k = 0; k < T; ++k) {
            sr[k] = fmaf(-zr[k], b2[k].x, fmaf(-zi[k], b2[k].y, b1[k].x));
            si[k] = fmaf(-zr[k], b2[k].y, fmaf(zi[k], b2[k].x, b1[k].y));
        }
    } else {
#pragma unroll
        for (int k = 0; k < T; ++k) sr[k] = si[k] = 0.f;
#pragma unroll 1
        for (int t = rem - 1; t >= 0; --t) {
            const float2 m = m2[t];
#pragma unroll
            for (int k = 0; k < T; ++k) {
                const float u = fmaf(sr[k], zr[k], m.x);
                const float w = fmaf(sr[k], zi[k], m.y);
                sr[k] = fmaf(-si[k], zi[k], u);
                si[k] = fmaf(si[k], zr[k], w);
            }
        }
    }
}

// One work item: voxel tile `tile` of p against antenna split `split`.  The two stage
// buffers' mbarriers are initialised by the caller; `gchunk` counts the chunks this CTA
// has consumed so far (stage = gchunk & 1, phase parity = (gchunk >> 1) & 1), so a
// persistent CTA can run item after item on the same barriers.  Returns -1, or, if a
// bounded wait gave up (the status word is set), 2 * (global chunk index) + (1 if the
// next chunk's copy was issued): the caller then drains the stages (drain_stages) after
// its own loop, which keeps that path out of the loops' register allocation.
template <int T, int NT, int FORM, int ANCHOR, bool PERSISTENT>
__device__ __forceinline__ int fwd_item(const FwdParams &p, int tile, int split,
                                        unsigned char *smem, uint32_t &gchunk) {
    static_assert((FORM != kFormMixedPair && FORM != kFormMixedPairSplit) || T % 2 == 0,
                  "pair form needs an even T");
    constexpr bool kPairRows = FORM == kFormMixedPair || FORM == kFormMixedPairSplit;
    Stage st;
    st.bars = reinterpret_cast<uint64_t *>(smem);
    st.base = smem + 128;
    st.nas = p.ant_per_stage;
    st.esz = kPairRows ? 16 : 8;  // antenna pairs: 16 B per pair = 8 B per antenna
    st.fp = p.fp;
    st.stage_bytes = (size_t)st.nas * sizeof(AntRec) + (size_t)st.nas * st.fp * st.esz;
    float *kappa_tab = reinterpret_cast<float *>(st.base + 2 * st.stage_bytes);  // PLAIN only
    const int fp = p.fp;

    const int a_begin = split * p.ant_per_split;
    const int a_end = min(p.num_ant, a_begin + p.ant_per_split);
    const int n_chunks = a_end > a_begin ? (a_end - a_begin + st.nas - 1) / st.nas : 0;
    const uint32_t g0 = PERSISTENT ? gchunk : 0u;

    if (!PERSISTENT && threadIdx.x == 0) {
        mbar_init(&st.bars[0], 1);
        mbar_init(&st.bars[1], 1);
        fence_mbar_init();
    }
    if constexpr (FORM == kFormPlain) {
        for (int j = threadIdx.x; j < fp; j += NT)
            kappa_tab[j] = (float)fma((double)j, p.kd, p.k0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n_chunks > 0) st.issue(p, 0, (int)(g0 & 1), a_begin, a_end);
        if (n_chunks > 1) st.issue(p, 1, (int)((g0 + 1) & 1), a_begin, a_end);
    }

    const int64_t rbase = (int64_t)tile * (NT * T) + threadIdx.x;
    float vx[T], vy[T], vz[T];
#pragma unroll
    for (int k = 0; k < T; ++k) decode_voxel(p, rbase + (int64_t)k * NT, vx[k], vy[k], vz[k]);
    float acc[T][8];
#pragma unroll
    for (int k = 0; k < T; ++k)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[k][q] = 0.f;

    const bool mono = *p.mono_flag != 0;
    const int nblk = fp / kBlockF;

    int c_failed = -1;  // chunk whose wait gave up; the drain runs after the loop
    for (int c = 0; c < n_chunks; ++c) {
        const uint32_t gc = g0 + (uint32_t)c;
        const int s = (int)(gc & 1);
        bool ok = mbar_wait_bounded(&st.bars[s], (gc >> 1) & 1, p.status);
        if (!__syncthreads_and(ok)) {
            c_failed = c;
            break;
        }
        const AntRec *ants = st.ants(s);
        const unsigned char *mstage = st.meas(s);
        const int na = min(st.nas, a_end - (a_begin + c * st.nas));

        if constexpr (FORM == kFormMixedAntPair) {
            // antennas (2pp, 2pp+1) ride in the two halves of every FFMA2
            const float4 *m4base = reinterpret_cast<const float4 *>(mstage);
            for (int pp = 0; pp < na / 2; ++pp) {
                const AntRec &a0r = ants[2 * pp];
                const AntRec &a1r = ants[2 * pp + 1];
                const float4 *m4 = m4base + (size_t)pp * fp;
                double d0[T], d1[T];
                unsigned long long ph0[T], ph1[T], st0[T], st1[T];
                float2 zr[T], zi[T], nzi[T], c2r[T], c2i[T];
#pragma unroll
                for (int k = 0; k < T; ++k) {
                    const double x = vx[k], y = vy[k], z = vz[k];
                    c2r[k] = c2i[k] = make_float2(0.f, 0.f);
                    if constexpr (ANCHOR == kAnchorFixed2) {
                        d0[k] = range_fp64_newton(x, y, z, a0r, mono, p.ti);
                        d1[k] = range_fp64_newton(x, y, z, a1r, mono, p.ti);
                        const unsigned long long u0 = turns_fixed64(-d0[k] * p.tsmp);
                        const unsigned long long u1 = turns_fixed64(-d1[k] * p.tsmp);
                        cis_turns_pair((int32_t)(u0 >> 32), (int32_t)(u1 >> 32), zr[k], zi[k],
                                       nzi[k]);
                        st0[k] = u0 << 5;
                        st1[k] = u1 << 5;
                        ph0[k] = turns_fixed_top(-d0[k] * p.t0);
                        ph1[k] = turns_fixed_top(-d1[k] * p.t0);
                    } else {
                        d0[k] = range_fp64(x, y, z, a0r, mono, p.ti);
                        d1[k] = range_fp64(x, y, z, a1r, mono, p.ti);
                        cis_fp64_phase_pair(-d0[k] * p.kd, -d1[k] * p.kd, zr[k], zi[k], nzi[k]);
                        if constexpr (ANCHOR == kAnchorFixed) {
                            ph0[k] = turns_to_fixed(-d0[k] * p.t0);
                            ph1[k] = turns_to_fixed(-d1[k] * p.t0);
                            st0[k] = turns_to_fixed(-d0[k] * p.tblk);
                            st1[k] = turns_to_fixed(-d1[k] * p.tblk);
                        }
                    }
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
                        float2 anr, ani, nani;
                        if constexpr (ANCHOR != kAnchorPoly) {
                            fixed_cis(ph0[k], anr.x, ani.x);
                            fixed_cis(ph1[k], anr.y, ani.y);
                            nani = make_float2(-ani.x, -ani.y);
                            ph0[k] += st0[k];
                            ph1[k] += st1[k];
                        } else {
                            const double kap = fma((double)(b * kBlockF), p.kd, p.k0);
                            cis_fp64_phase_pair(-d0[k] * kap, -d1[k] * kap, anr, ani, nani);
                        }
                        c2r[k] = __ffma2_rn(anr, hr[k], __ffma2_rn(nani, hi[k], c2r[k]));
                        c2i[k] = __ffma2_rn(anr, hi[k], __ffma2_rn(ani, hr[k], c2i[k]));
                    }
                }
                // image + vote, antenna 2pp then 2pp+1 (the scalar kernels' order)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const AntRec &ar = h ? a1r : a0r;
                    const float ux0 = ar.virt[0], uy0 = ar.virt[1], uz0 = ar.virt[2];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        const float cr = h ? c2r[k].y : c2r[k].x;
                        const float ci = h ? c2i[k].y : c2i[k].x;
                        const float ux = ux0 - vx[k], uy = uy0 - vy[k], uz = uz0 - vz[k];
                        acc[k][0] += cr;
                        acc[k][1] += ci;
                        acc[k][2] = fmaf(cr, ux, acc[k][2]);
                        acc[k][3] = fmaf(ci, ux, acc[k][3]);
                        acc[k][4] = fmaf(cr, uy, acc[k][4]);
                        acc[k][5] = fmaf(ci, uy, acc[k][5]);
                        acc[k][6] = fmaf(cr, uz, acc[k][6]);
                        acc[k][7] = fmaf(ci, uz, acc[k][7]);
                    }
                }
            }
        } else
        for (int a = 0; a < na; ++a) {
            const AntRec &ar = ants[a];
            float cr[T], ci[T];
            if constexpr (kPairRows) {
                constexpr int P = T / 2;
                constexpr bool kSplit = FORM == kFormMixedPairSplit;
                const float4 *m4 = reinterpret_cast<const float4 *>(mstage) + (size_t)a * fp;
                double d[T];
                unsigned long long ph[T], stp[T];
                float2 zr[P], zi[P], nzi[P], c2r[P], c2i[P];
                if constexpr (ANCHOR == kAnchorFixed2) {
                    int32_t za[T];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        d[k] = range_fp64_newton((double)vx[k], (double)vy[k], (double)vz[k], ar,
                                                 mono, p.ti);
                        const unsigned long long u = turns_fixed64(-d[k] * p.tsmp);
                        za[k] = (int32_t)(u >> 32);
                        stp[k] = u << 5;
                        ph[k] = turns_fixed_top(-d[k] * p.t0);
                    }
#pragma unroll
                    for (int q = 0; q < P; ++q) {
                        cis_turns_pair(za[2 * q], za[2 * q + 1], zr[q], zi[q], nzi[q]);
                        c2r[q] = c2i[q] = make_float2(0.f, 0.f);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        d[k] = range_fp64((double)vx[k], (double)vy[k], (double)vz[k], ar, mono,
                                          p.ti);
                        if constexpr (ANCHOR == kAnchorFixed) {
                            ph[k] = turns_to_fixed(-d[k] * p.t0);
                            stp[k] = turns_to_fixed(-d[k] * p.tblk);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < P; ++q) {
                        cis_fp64_phase_pair(-d[2 * q] * p.kd, -d[2 * q + 1] * p.kd, zr[q], zi[q],
                                            nzi[q]);
                        c2r[q] = c2i[q] = make_float2(0.f, 0.f);
                    }
                }
                // z^16 by four complex squarings (split form only)
                float2 z16r[P], z16i[P], nz16i[P];
                if constexpr (kSplit) {
#pragma unroll
                    for (int q = 0; q < P; ++q) {
                        float2 ar2 = zr[q], ai2 = zi[q];
#pragma unroll
                        for (int k2 = 0; k2 < 4; ++k2) {
                            const float2 nr = __ffma2_rn(ar2, ar2, __fmul2_rn(ai2, make_float2(-ai2.x, -ai2.y)));
                            ai2 = __fmul2_rn(__fadd2_rn(ar2, ar2), ai2);
                            ar2 = nr;
                        }
                        z16r[q] = ar2;
                        z16i[q] = ai2;
                        nz16i[q] = make_float2(-ai2.x, -ai2.y);
                    }
                }
                for (int b = 0; b < nblk; ++b) {
                    const float4 *mb = m4 + b * kBlockF;
                    float2 hr[P], hi[P];
                    if constexpr (kSplit) {
                        constexpr int H = kBlockF / 2;
                        float2 hrb[P], hib[P];
                        const float4 topa = mb[H - 1], topb = mb[kBlockF - 1];
#pragma unroll
                        for (int q = 0; q < P; ++q) {
                            hr[q] = make_float2(topa.x, topa.y);
                            hi[q] = make_float2(topa.z, topa.w);
                            hrb[q] = make_float2(topb.x, topb.y);
                            hib[q] = make_float2(topb.z, topb.w);
                        }
#pragma unroll
                        for (int t = H - 2; t >= 0; --t) {
                            const float4 ma = mb[t], mbb = mb[H + t];
                            const float2 mra = make_float2(ma.x, ma.y), mia = make_float2(ma.z, ma.w);
                            const float2 mrb = make_float2(mbb.x, mbb.y), mib = make_float2(mbb.z, mbb.w);
#pragma unroll
                            for (int q = 0; q < P; ++q) {
                                const float2 ua = __ffma2_rn(hr[q], zr[q], mra);
                                const float2 wa = __ffma2_rn(hr[q], zi[q], mia);
                                const float2 ub = __ffma2_rn(hrb[q], zr[q], mrb);
                                const float2 wb = __ffma2_rn(hrb[q], zi[q], mib);
                                hr[q] = __ffma2_rn(hi[q], nzi[q], ua);
                                hi[q] = __ffma2_rn(hi[q], zr[q], wa);
                                hrb[q] = __ffma2_rn(hib[q], nzi[q], ub);
                                hib[q] = __ffma2_rn(hib[q], zr[q], wb);
                            }
                        }
                        // h = h_low + z^16 h_high
#pragma unroll
                        for (int q = 0; q < P; ++q) {
                            const float2 r2 = __ffma2_rn(z16r[q], hrb[q], __ffma2_rn(nz16i[q], hib[q], hr[q]));
                            hi[q] = __ffma2_rn(z16r[q], hib[q], __ffma2_rn(z16i[q], hrb[q], hi[q]));
                            hr[q] = r2;
                        }
                    } else {
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
                    }
#pragma unroll
                    for (int q = 0; q < P; ++q) {
                        float2 anr, ani, nani;
                        if constexpr (ANCHOR != kAnchorPoly) {
                            fixed_cis(ph[2 * q], anr.x, ani.x);
                            fixed_cis(ph[2 * q + 1], anr.y, ani.y);
                            nani = make_float2(-ani.x, -ani.y);
                            ph[2 * q] += stp[2 * q];
                            ph[2 * q + 1] += stp[2 * q + 1];
                        } else {
                            const double kap = fma((double)(b * kBlockF), p.kd, p.k0);
                            cis_fp64_phase_pair(-d[2 * q] * kap, -d[2 * q + 1] * kap, anr, ani,
                                                nani);
                        }
                        c2r[q] = __ffma2_rn(anr, hr[q], __ffma2_rn(nani, hi[q], c2r[q]));
                        c2i[q] = __ffma2_rn(anr, hi[q], __ffma2_rn(ani, hr[q], c2i[q]));
                    }
                }
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    cr[2 * q] = c2r[q].x;
                    cr[2 * q + 1] = c2r[q].y;
                    ci[2 * q] = c2i[q].x;
                    ci[2 * q + 1] = c2i[q].y;
                }
            } else if constexpr (FORM == kFormMixedClen || FORM == kFormMixedClen64) {
                // Second-order form.  With z = e^{i phi}, z^{t+1} = 2 cos(phi) z^t - z^{t-1},
                // so the block sum h = sum_{t<L} m_t z^t follows from the backward recurrence
                //     b_t = m_t + c2 b_{t+1} - b_{t+2},  c2 = 2 cos(phi),  b_L = b_{L+1} = 0,
                //     h = b_0 - conj(z) b_1
                // (Clenshaw's summation for a three-term recurrence).  The multiplier is real,
                // so each (voxel, antenna) chain keeps its complex b as one (re, im) register
                // pair: one FADD2 + one FFMA2 per sample (4 lane operations, as the Horner step),
                // and one 16-byte shared load feeds two samples to every voxel of the thread.
                // Blocks are L = 32 or 64 samples long (kFormMixedClen64: half the re-anchoring);
                // a row's last block runs over its remaining valid samples only.
                // Error: a rounding error made at step t reaches b_0 scaled by at most
                // min(t + 1, 1 / |sin phi|), and for rows dominated by a few scatterers (input
                // near the recurrence's own modes e^{+-i phi t}) |b| grows to ~L|m| / sin phi,
                // so each block sum carries several times the Horner form's error (measured on
                // the 128^3 workload: 6.9e-6 (L = 32) and 8.8e-6 (L = 64) image relative L2
                // against FP64, Horner 2.6e-6).  The form is kept away from phi near 0 and pi
                // (kClenMaxCos); there the same blocks run the first-order Horner form.
                static_assert(T % 2 == 0, "the second-order form takes voxels in pairs");
                constexpr int L = FORM == kFormMixedClen64 ? 64 : kBlockF;
                constexpr int LSH = FORM == kFormMixedClen64 ? 6 : 5;
                const int ns = p.nsmp > 0 ? min(p.nsmp, fp) : fp;  // valid samples per row
                const int nblk_c = ns / L;
                const float4 *m4 = reinterpret_cast<const float4 *>(mstage) + (size_t)a * (fp / 2);
                unsigned long long ph[T], stp[T];
                float zr[T], zi[T];
                float2 c2[T];
                bool clen = true;
                {
                    int32_t za[T];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        const double d = range_fp64_newton((double)vx[k], (double)vy[k],
                                                           (double)vz[k], ar, mono, p.ti);
                        const unsigned long long u = turns_fixed64(-d * p.tsmp);
                        za[k] = (int32_t)(u >> 32);
                        stp[k] = u << 5;  // 32 samples; an L-block steps stp << (LSH - 5)
                        ph[k] = turns_fixed_top(-d * p.t0);
                        cr[k] = ci[k] = 0.f;
                    }
#pragma unroll
                    for (int q = 0; q < T / 2; ++q) {
                        float2 c, s, nsn;
                        cis_turns_pair(za[2 * q], za[2 * q + 1], c, s, nsn);
                        zr[2 * q] = c.x;
                        zr[2 * q + 1] = c.y;
                        zi[2 * q] = s.x;
                        zi[2 * q + 1] = s.y;
                    }
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        c2[k] = make_float2(2.f * zr[k], 2.f * zr[k]);
                        clen = clen && fabsf(zr[k]) <= kClenMaxCos;
                    }
                }
                clen = __all_sync(0xffffffffu, clen);
                // whole L-sample blocks, then one block of the row's rem < L remaining valid
                // samples, whose padded zeros are skipped (they add exactly nothing: the
                // recurrence from the top of a zero run stays at zero)
                auto anchor = [&](const float (&sr)[T], const float (&si)[T], int shift) {
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        float anr, ani;
                        fixed_cis(ph[k], anr, ani);
                        ph[k] += stp[k] << shift;
                        cr[k] = fmaf(anr, sr[k], fmaf(-ani, si[k], cr[k]));
                        ci[k] = fmaf(anr, si[k], fmaf(ani, sr[k], ci[k]));
                    }
                };
                for (int b = 0; b < nblk_c; ++b) {
                    float sr[T], si[T];
                    clen_block<T, L>(m4 + b * (L / 2), clen, c2, zr, zi, sr, si);
                    anchor(sr, si, LSH - 5);
                }
                const int rem = ns - nblk_c * L;
                const float4 *mr4 = m4 + nblk_c * (L / 2);
                if (rem > 0) {
                    float sr[T], si[T];
                    clen_partial<T>(reinterpret_cast<const float2 *>(mr4), rem, clen, c2, zr, zi,
                                    sr, si);
                    anchor(sr, si, 0);
                }
            } else if constexpr (FORM == kFormMixedClenEO) {
                // 64-sample blocks, each as even and odd chains in w = z^2 (clen_block_eo),
                // used for a warp's antenna when every lane has |cos 2 phi| <= kClenMaxCos;
                // otherwise, and for a row's last partial block, first-order Horner.
                static_assert(T % 2 == 0, "the second-order form takes voxels in pairs");
                const int ns = p.nsmp > 0 ? min(p.nsmp, fp) : fp;
                const int nblk_c = ns / 64;
                const float4 *m4 = reinterpret_cast<const float4 *>(mstage) + (size_t)a * (fp / 2);
                unsigned long long ph[T], stp[T];
                float zr[T], zi[T], wr[T], wi[T];
                bool eo = true;
                {
                    int32_t za[T], wa[T];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        const double d = range_fp64_newton((double)vx[k], (double)vy[k],
                                                           (double)vz[k], ar, mono, p.ti);
                        const unsigned long long u = turns_fixed64(-d * p.tsmp);
                        za[k] = (int32_t)(u >> 32);
                        wa[k] = (int32_t)((u << 1) >> 32);  // 2 phi, exact in fixed point
                        stp[k] = u << 6;
                        ph[k] = turns_fixed_top(-d * p.t0);
                        cr[k] = ci[k] = 0.f;
                    }
#pragma unroll
                    for (int q = 0; q < T / 2; ++q) {
                        float2 c, s, nsn;
                        cis_turns_pair(za[2 * q], za[2 * q + 1], c, s, nsn);
                        zr[2 * q] = c.x;
                        zr[2 * q + 1] = c.y;
                        zi[2 * q] = s.x;
                        zi[2 * q + 1] = s.y;
                        cis_turns_pair(wa[2 * q], wa[2 * q + 1], c, s, nsn);
                        wr[2 * q] = c.x;
                        wr[2 * q + 1] = c.y;
                        wi[2 * q] = s.x;
                        wi[2 * q + 1] = s.y;
                    }
#pragma unroll
                    for (int k = 0; k < T; ++k) eo = eo && fabsf(wr[k]) <= kClenMaxCos;
                }
                eo = __all_sync(0xffffffffu, eo);
                const float2 none[T] = {};
                auto anchor = [&](const float (&sr)[T], const float (&si)[T]) {
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        float anr, ani;
                        fixed_cis(ph[k], anr, ani);
                        ph[k] += stp[k];
                        cr[k] = fmaf(anr, sr[k], fmaf(-ani, si[k], cr[k]));
                        ci[k] = fmaf(anr, si[k], fmaf(ani, sr[k], ci[k]));
                    }
                };
                for (int b = 0; b < nblk_c; ++b) {
                    float sr[T], si[T];
                    if (eo)
                        clen_block_eo<T>(m4 + b * 32, zr, zi, wr, wi, sr, si);
                    else
                        clen_block<T, 64>(m4 + b * 32, false, none, zr, zi, sr, si);
                    anchor(sr, si);
                }
                const int rem = ns - nblk_c * 64;
                if (rem > 0) {
                    float sr[T], si[T];
                    clen_partial<T>(reinterpret_cast<const float2 *>(m4 + nblk_c * 32), rem,
                                    false, none, zr, zi, sr, si);
                    anchor(sr, si);
                }
            } else if constexpr (FORM == kFormMixedScalar) {
                const float4 *m4 = reinterpret_cast<const float4 *>(mstage) + (size_t)a * (fp / 2);
                double d[T];
                float zr[T], zi[T], nzi[T];
#pragma unroll
                for (int k = 0; k < T; ++k) {
                    d[k] = range_fp64((double)vx[k], (double)vy[k], (double)vz[k], ar, mono, p.ti);
                    const float2 z = cis_fp64_phase(-d[k] * p.kd);
                    zr[k] = z.x;
                    zi[k] = z.y;
                    nzi[k] = -z.y;
                    cr[k] = ci[k] = 0.f;
                }
                for (int b = 0; b < nblk; ++b) {
                    const float4 *mb = m4 + b * (kBlockF / 2);
                    float hr[T], hi[T];
                    const float4 top = mb[kBlockF / 2 - 1];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        hr[k] = top.z;
                        hi[k] = top.w;
                        const float u = fmaf(hr[k], zr[k], top.x);
                        const float w = fmaf(hr[k], zi[k], top.y);
                        hr[k] = fmaf(hi[k], nzi[k], u);
                        hi[k] = fmaf(hi[k], zr[k], w);
                    }
#pragma unroll
                    for (int q = kBlockF / 2 - 2; q >= 0; --q) {
                        const float4 mm = mb[q];
#pragma unroll
                        for (int k = 0; k < T; ++k) {
                            float u = fmaf(hr[k], zr[k], mm.z);
                            float w = fmaf(hr[k], zi[k], mm.w);
                            hr[k] = fmaf(hi[k], nzi[k], u);
                            hi[k] = fmaf(hi[k], zr[k], w);
                            u = fmaf(hr[k], zr[k], mm.x);
                            w = fmaf(hr[k], zi[k], mm.y);
                            hr[k] = fmaf(hi[k], nzi[k], u);
                            hi[k] = fmaf(hi[k], zr[k], w);
                        }
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
                const float4 *m4 = reinterpret_cast<const float4 *>(mstage) + (size_t)a * (fp / 2);
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
                    cr[k] = ci[k] = 0.f;
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
        if (threadIdx.x == 0 && c + 2 < n_chunks) st.issue(p, c + 2, (int)((g0 + (uint32_t)c) & 1), a_begin, a_end);
    }
    if (c_failed >= 0)
        return 2 * (int)(g0 + (uint32_t)c_failed) + (c_failed + 1 < n_chunks ? 1 : 0);
    if (PERSISTENT) gchunk = g0 + (uint32_t)n_chunks;

#pragma unroll
    for (int k = 0; k < T; ++k) store_voxel(p, split, rbase + (int64_t)k * NT, acc[k]);
    return -1;
}

__device__ __forceinline__ void init_stage_barriers(unsigned char *smem) {
    if (threadIdx.x == 0) {
        uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// One launch, grid = tiles x splits (one work item per CTA).
template <int T, int NT, int FORM, int ANCHOR = kAnchorPoly>
__global__ void __launch_bounds__(NT) bp_fwd_kernel(const FwdParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint32_t gchunk = 0;
    const int failed = fwd_item<T, NT, FORM, ANCHOR, false>(p, blockIdx.x % p.num_tiles,
                                                             blockIdx.x / p.num_tiles, smem,
                                                             gchunk);
    if (failed >= 0)
        drain_stages(reinterpret_cast<uint64_t *>(smem), (uint32_t)failed >> 1, failed & 1,
                     p.status);
}

// Persistent launch over a work list of (object, voxel tile, antenna split) items: every
// CTA pops the next item from a global counter until the list is exhausted.  Items are
// sorted by cost, largest first, so the tail is made of the smallest items.
template <int T, int NT, int FORM, int ANCHOR = kAnchorPoly>
__global__ void __launch_bounds__(NT) bp_fwd_persistent(const BatchParams bp) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_item;
    init_stage_barriers(smem);
    uint32_t gchunk = 0;
    int failed = -1;
    int32_t *status = nullptr;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(bp.counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= bp.num_items) break;
        const int4 w = bp.items[item];
        // the item's object parameters as a local copy: read once, then kept in registers
        // (a reference into global memory would be re-read inside the loops)
        const FwdParams obj = bp.objs[w.x];
        failed = fwd_item<T, NT, FORM, ANCHOR, true>(obj, w.y, w.z, smem, gchunk);
        if (failed >= 0) {
            status = obj.status;
            break;
        }
    }
    if (failed >= 0)
        drain_stages(reinterpret_cast<uint64_t *>(smem), (uint32_t)failed >> 1, failed & 1,
                     status);
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
// does (surface_normal_est.cu:128-130).  Thread 0 also records whether every RX offset
// is zero (the forward kernels then reuse the outgoing leg for the return leg).
__global__ void prep_antennas(const float *__restrict__ ant, const float *__restrict__ rxo,
                              int R, const float *__restrict__ pos_off, int A, int A_pad,
                              AntRec *__restrict__ out, int32_t *__restrict__ mono_flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        int mono = 1;
        for (int q = 0; q < 3 * R; ++q) mono &= (rxo[q] == 0.f);
        *mono_flag = mono;
    }
    if (i >= A_pad) return;
    // records past A (padding to an even count) repeat the last antenna; their staged
    // samples are zero, so they contribute exactly nothing
    const int src = i < A ? i : A - 1;
    AntRec r;
    const int q = src % R;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float a = ant[3 * src + k];
        double ad = a;
        if (pos_off) {
            ad += (double)pos_off[3 * src + k];
            a = a + pos_off[3 * src + k];
        }
        const float o = rxo[3 * q + k];
        r.tx[k] = ad;
        r.rx[k] = ad + (double)o;
        r.virt[k] = a + o / 2;
    }
    r.pad = 0.f;
    out[i] = r;
}

// Measurement rows [A, F] (complex64, or SoA planes re/im when `im` is non-null) into
// the shared-memory layout of a kernel form: rows of Fp = roundup(F, 32) samples,
// zero-padded (zero samples at the top of a Horner block add exactly nothing), each
// sample either
//   layout 0: (re, im)                       8 B per antenna-sample
//   layout 1: (re, re, im, im)              16 B per antenna-sample (voxel pairs)
//   layout 2: (re_a, re_a', im_a, im_a')    16 B per antenna PAIR-sample (antenna pairs
//             a = 2p, a' = 2p+1; an antenna index >= A is zero)
__device__ __forceinline__ float2 load_sample(const float *src, const float *im, int A, int F,
                                              int64_t a, int j) {
    if (a >= A || j >= F) return make_float2(0.f, 0.f);
    if (im) return make_float2(src[a * F + j], im[a * F + j]);
    return reinterpret_cast<const float2 *>(src)[a * F + j];
}

__global__ void stage_meas(const float *__restrict__ src, const float *__restrict__ im, int A,
                           int F, int Fp, int layout, int rows, void *__restrict__ dst) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)rows * Fp) return;
    const int64_t r = idx / Fp;
    const int j = (int)(idx - r * Fp);
    if (layout == 2) {
        const float2 m0 = load_sample(src, im, A, F, 2 * r, j);
        const float2 m1 = load_sample(src, im, A, F, 2 * r + 1, j);
        reinterpret_cast<float4 *>(dst)[idx] = make_float4(m0.x, m1.x, m0.y, m1.y);
    } else if (layout == 1) {
        const float2 m = load_sample(src, im, A, F, r, j);
        reinterpret_cast<float4 *>(dst)[idx] = make_float4(m.x, m.x, m.y, m.y);
    } else {
        reinterpret_cast<float2 *>(dst)[idx] = load_sample(src, im, A, F, r, j);
    }
}

// ------------------------------------------------------------------ instantiations
template <int T, int NT, int FORM, int ANCHOR = kAnchorPoly>
static const void *fwd_ptr() {
    return reinterpret_cast<const void *>(&bp_fwd_kernel<T, NT, FORM, ANCHOR>);
}
template <int T, int NT, int FORM, int ANCHOR = kAnchorPoly>
static const void *pers_ptr() {
    return reinterpret_cast<const void *>(&bp_fwd_persistent<T, NT, FORM, ANCHOR>);
}

const FwdVariant *fwd_variants(int *count) {
    // index order: the MIXED variants first (default first), then the PLAIN ones
    static const FwdVariant v[] = {
        // default: 64-sample blocks as two second-order chains in z^2 (near the Horner
        // form's accuracy at close to the fastest form's speed)
        {2, 256, false, 8, fwd_ptr<2, 256, kFormMixedClenEO, kAnchorFixed2>(), "mixed_clen64eo_fx2_t2_n256", 0, pers_ptr<2, 256, kFormMixedClenEO, kAnchorFixed2>()},
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedClen, kAnchorFixed2>(), "mixed_clen_fx2_t4_n128_s24", 0, pers_ptr<4, 128, kFormMixedClen, kAnchorFixed2>(), 24 * 1024},
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPair, kAnchorFixed>(), "mixed_ffma2_fx_t2_n256", 1, pers_ptr<2, 256, kFormMixedPair, kAnchorFixed>()},
        // each block as two 16-step chains joined by z^16 (kFormMixedPairSplit)
        {2, 128, false, 16, fwd_ptr<2, 128, kFormMixedPairSplit, kAnchorFixed2>(), "mixed_split_fx2_t2_n128_s24", 1, pers_ptr<2, 128, kFormMixedPairSplit, kAnchorFixed2>(), 24 * 1024},
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPairSplit, kAnchorFixed2>(), "mixed_split_fx2_t2_n256", 1, pers_ptr<2, 256, kFormMixedPairSplit, kAnchorFixed2>()},
        {2, 128, false, 16, fwd_ptr<2, 128, kFormMixedPairSplit, kAnchorFixed2>(), "mixed_split_fx2_t2_n128_s16", 1, pers_ptr<2, 128, kFormMixedPairSplit, kAnchorFixed2>(), 16 * 1024},
        // the cheaper prologue (kAnchorFixed2)
        {2, 128, false, 16, fwd_ptr<2, 128, kFormMixedPair, kAnchorFixed2>(), "mixed_ffma2_fx2_t2_n128_s24", 1, pers_ptr<2, 128, kFormMixedPair, kAnchorFixed2>(), 24 * 1024},
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPair, kAnchorFixed2>(), "mixed_ffma2_fx2_t2_n256", 1, pers_ptr<2, 256, kFormMixedPair, kAnchorFixed2>()},
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPair, kAnchorFixed2>(), "mixed_ffma2_fx2_t2_n256_s24", 1, pers_ptr<2, 256, kFormMixedPair, kAnchorFixed2>(), 24 * 1024},
        {1, 256, false, 8, fwd_ptr<1, 256, kFormMixedAntPair, kAnchorFixed2>(), "mixed_antpair_fx2_t1_n256", 2, pers_ptr<1, 256, kFormMixedAntPair, kAnchorFixed2>()},
        {2, 256, false, 8, fwd_ptr<2, 256, kFormMixedAntPair, kAnchorFixed2>(), "mixed_antpair_fx2_t2_n256", 2, pers_ptr<2, 256, kFormMixedAntPair, kAnchorFixed2>()},
        // smaller stages: more resident CTAs (shared memory limits occupancy otherwise)
        {2, 128, false, 16, fwd_ptr<2, 128, kFormMixedPair, kAnchorFixed2>(), "mixed_ffma2_fx2_t2_n128_s16", 1, pers_ptr<2, 128, kFormMixedPair, kAnchorFixed2>(), 16 * 1024},
        {2, 128, false, 16, fwd_ptr<2, 128, kFormMixedPair, kAnchorFixed2>(), "mixed_ffma2_fx2_t2_n128_s12", 1, pers_ptr<2, 128, kFormMixedPair, kAnchorFixed2>(), 12 * 1024},
        {1, 256, false, 8, fwd_ptr<1, 256, kFormMixedAntPair, kAnchorFixed2>(), "mixed_antpair_fx2_t1_n256_s24", 2, pers_ptr<1, 256, kFormMixedAntPair, kAnchorFixed2>(), 24 * 1024},
        {1, 128, false, 8, fwd_ptr<1, 128, kFormMixedAntPair, kAnchorFixed2>(), "mixed_antpair_fx2_t1_n128_s24", 2, pers_ptr<1, 128, kFormMixedAntPair, kAnchorFixed2>(), 24 * 1024},
        {1, 128, false, 8, fwd_ptr<1, 128, kFormMixedAntPair, kAnchorFixed2>(), "mixed_antpair_fx2_t1_n128_s16", 2, pers_ptr<1, 128, kFormMixedAntPair, kAnchorFixed2>(), 16 * 1024},
        {2, 256, false, 8, fwd_ptr<2, 256, kFormMixedAntPair, kAnchorFixed>(), "mixed_antpair_fx_t2_n256", 2, pers_ptr<2, 256, kFormMixedAntPair, kAnchorFixed>()},
        {1, 256, false, 8, fwd_ptr<1, 256, kFormMixedAntPair, kAnchorFixed>(), "mixed_antpair_fx_t1_n256", 2, pers_ptr<1, 256, kFormMixedAntPair, kAnchorFixed>()},
        {4, 128, false, 16, fwd_ptr<4, 128, kFormMixedPair, kAnchorFixed>(), "mixed_ffma2_fx_t4_n128", 1, pers_ptr<4, 128, kFormMixedPair, kAnchorFixed>()},
        {2, 256, false, 8, fwd_ptr<2, 256, kFormMixedAntPair>(), "mixed_antpair_t2_n256", 2, pers_ptr<2, 256, kFormMixedAntPair>()},
        {2, 128, false, 8, fwd_ptr<2, 128, kFormMixedAntPair>(), "mixed_antpair_t2_n128", 2, pers_ptr<2, 128, kFormMixedAntPair>()},
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedAntPair>(), "mixed_antpair_t4_n128", 2, pers_ptr<4, 128, kFormMixedAntPair>()},
        {1, 256, false, 8, fwd_ptr<1, 256, kFormMixedAntPair>(), "mixed_antpair_t1_n256", 2, pers_ptr<1, 256, kFormMixedAntPair>()},
        {4, 128, false, 16, fwd_ptr<4, 128, kFormMixedPair>(), "mixed_ffma2_t4_n128", 1, pers_ptr<4, 128, kFormMixedPair>()},
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPair>(), "mixed_ffma2_t2_n256", 1, pers_ptr<2, 256, kFormMixedPair>()},
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedScalar>(), "mixed_ffma_t4_n128", 0, pers_ptr<4, 128, kFormMixedScalar>()},
        // the default form with smaller stages: more CTAs per SM (occupancy is limited by
        // two 48 KB stages otherwise), at the cost of more stage hand-overs
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPair, kAnchorFixed>(), "mixed_ffma2_fx_t2_n256_s24", 1, pers_ptr<2, 256, kFormMixedPair, kAnchorFixed>(), 24 * 1024},
        {2, 256, false, 16, fwd_ptr<2, 256, kFormMixedPair, kAnchorFixed>(), "mixed_ffma2_fx_t2_n256_s16", 1, pers_ptr<2, 256, kFormMixedPair, kAnchorFixed>(), 16 * 1024},
        {2, 128, false, 16, fwd_ptr<2, 128, kFormMixedPair, kAnchorFixed>(), "mixed_ffma2_fx_t2_n128_s24", 1, pers_ptr<2, 128, kFormMixedPair, kAnchorFixed>(), 24 * 1024},
        // two voxel pairs per thread: one shared load feeds 8 FFMA2 (the stages limit
        // occupancy to two CTAs per SM either way, which leaves 128 registers a thread)
        {4, 256, false, 16, fwd_ptr<4, 256, kFormMixedPair, kAnchorFixed>(), "mixed_ffma2_fx_t4_n256", 1, pers_ptr<4, 256, kFormMixedPair, kAnchorFixed>()},
        // second-order (Clenshaw) block sums over (re, im) samples, one FADD2 + FFMA2 per
        // sample and chain
        {2, 256, false, 8, fwd_ptr<2, 256, kFormMixedClen, kAnchorFixed2>(), "mixed_clen_fx2_t2_n256", 0, pers_ptr<2, 256, kFormMixedClen, kAnchorFixed2>()},
        {2, 128, false, 8, fwd_ptr<2, 128, kFormMixedClen, kAnchorFixed2>(), "mixed_clen_fx2_t2_n128_s24", 0, pers_ptr<2, 128, kFormMixedClen, kAnchorFixed2>(), 24 * 1024},
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedClen, kAnchorFixed2>(), "mixed_clen_fx2_t4_n128", 0, pers_ptr<4, 128, kFormMixedClen, kAnchorFixed2>()},
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedClen64, kAnchorFixed2>(), "mixed_clen64_fx2_t4_n128_s24", 0, pers_ptr<4, 128, kFormMixedClen64, kAnchorFixed2>(), 24 * 1024},
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedClen64, kAnchorFixed2>(), "mixed_clen64_fx2_t4_n128", 0, pers_ptr<4, 128, kFormMixedClen64, kAnchorFixed2>()},
        {2, 256, false, 8, fwd_ptr<2, 256, kFormMixedClen64, kAnchorFixed2>(), "mixed_clen64_fx2_t2_n256", 0, pers_ptr<2, 256, kFormMixedClen64, kAnchorFixed2>()},
        // 64-sample blocks as two chains in z^2: closer to the Horner form's accuracy
        {4, 128, false, 8, fwd_ptr<4, 128, kFormMixedClenEO, kAnchorFixed2>(), "mixed_clen64eo_fx2_t4_n128_s24", 0, pers_ptr<4, 128, kFormMixedClenEO, kAnchorFixed2>(), 24 * 1024},
        {2, 256, true, 8, fwd_ptr<2, 256, kFormPlain>(), "plain_t2_n256", 0, nullptr},
        {2, 128, true, 8, fwd_ptr<2, 128, kFormPlain>(), "plain_t2_n128", 0, nullptr},
        {1, 128, true, 8, fwd_ptr<1, 128, kFormPlain>(), "plain_t1_n128", 0, nullptr},
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
                                 int A, int A_pad, AntRec *out, int32_t *mono_flag,
                                 cudaStream_t stream) {
    const int nt = 256;
    prep_antennas<<<(A_pad + nt) / nt, nt, 0, stream>>>(ant, rxo, R, pos_off, A, A_pad, out,
                                                         mono_flag);
    return cudaGetLastError();
}

cudaError_t launch_stage_meas(const float *src, const float *im, int A, int F, int Fp,
                              int layout, void *dst, cudaStream_t stream) {
    const int nt = 256;
    const int rows = layout == 2 ? (A + 1) / 2 : A;
    const int64_t n = (int64_t)rows * Fp;
    stage_meas<<<(unsigned)((n + nt - 1) / nt), nt, 0, stream>>>(src, im, A, F, Fp, layout, rows,
                                                                 dst);
    return cudaGetLastError();
}

}  // namespace mmn

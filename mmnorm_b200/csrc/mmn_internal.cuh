// mmn_internal.cuh -- shared device helpers for the sm_100a backprojection kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mmnorm_b200.h"

namespace mmn {

constexpr double kC = 2.99792458e8;  // imaging_gpu.cu:3
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int kBlockF = 32;          // samples per re-anchored block
constexpr size_t kStatusBytes = 256; // workspace header holding the status word

// One virtual antenna, prepared once per call (64 bytes, 16-byte aligned so a chunk
// of records moves with one bulk copy).
struct __align__(16) AntRec {
    double tx[3];   // TX position (plus the optional per-antenna offset)
    double rx[3];   // RX position = TX + rx_offsets[i % R]
    float virt[3];  // TX + rx_offset/2 in float32, the vote anchor (surface_normal_est.cu:128-130)
    float pad;
};
static_assert(sizeof(AntRec) == 64, "AntRec must be 64 bytes");

// ---------------------------------------------------------------------------------
// exp(i*phi) for an FP64 phase of any practical magnitude.
// The phase is reduced in FP64 to r = phi - n*pi/2 with n = rint(phi*2/pi) (the
// 1.5*2^52 rounding constant leaves n in the low mantissa bits), then sin and cos of
// r in [-pi/4, pi/4] are evaluated in FP32 from their Taylor series (terms through
// r^9 and r^10: truncation below 2e-9), and rotated by n quarter turns.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float2 cis_fp64_phase(double phi) {
    const double kTwoOverPi = 0.636619772367581343075535053490057448;
    const double kPiOver2 = 1.570796326794896619231321691639751442;
    const double kRound = 6755399441055744.0;  // 1.5 * 2^52
    double t = fma(phi, kTwoOverPi, kRound);
    int q = __double2loint(t);
    double n = t - kRound;
    float x = (float)fma(-n, kPiOver2, phi);
    float x2 = x * x;
    // sin: x - x^3/3! + x^5/5! - x^7/7! + x^9/9!
    float s = fmaf(x2, 2.75573192239858906526e-6f, -1.98412698412698412698e-4f);
    s = fmaf(x2, s, 8.33333333333333333333e-3f);
    s = fmaf(x2, s, -1.66666666666666666667e-1f);
    s = fmaf(x2 * x, s, x);
    // cos: 1 - x^2/2! + x^4/4! - x^6/6! + x^8/8! - x^10/10!
    float c = fmaf(x2, -2.75573192239858906526e-7f, 2.48015873015873015873e-5f);
    c = fmaf(x2, c, -1.38888888888888888889e-3f);
    c = fmaf(x2, c, 4.16666666666666666667e-2f);
    c = fmaf(x2, c, -0.5f);
    c = fmaf(x2, c, 1.0f);
    float sr = (q & 1) ? c : s;
    float cr = (q & 1) ? -s : c;
    if (q & 2) {
        sr = -sr;
        cr = -cr;
    }
    return make_float2(cr, sr);
}

// Two phases at once: the FP64 reduction per element as in cis_fp64_phase, the FP32
// Taylor polynomials as packed FFMA2/FMUL2 on (element 0, element 1).  Returns
// c = (cos phi0, cos phi1), s = (sin phi0, sin phi1), ns = -s.
__device__ __forceinline__ void cis_fp64_phase_pair(double phi0, double phi1, float2 &c,
                                                    float2 &s, float2 &ns) {
    const double kTwoOverPi = 0.636619772367581343075535053490057448;
    const double kPiOver2 = 1.570796326794896619231321691639751442;
    const double kRound = 6755399441055744.0;  // 1.5 * 2^52
    const double t0 = fma(phi0, kTwoOverPi, kRound);
    const double t1 = fma(phi1, kTwoOverPi, kRound);
    const int q0 = __double2loint(t0);
    const int q1 = __double2loint(t1);
    const double n0 = t0 - kRound, n1 = t1 - kRound;
    const float2 x = make_float2((float)fma(-n0, kPiOver2, phi0), (float)fma(-n1, kPiOver2, phi1));
    const float2 x2 = __fmul2_rn(x, x);
    const float2 x3 = __fmul2_rn(x2, x);
    float2 sp = __ffma2_rn(x2, make_float2(2.75573192239858906526e-6f, 2.75573192239858906526e-6f),
                           make_float2(-1.98412698412698412698e-4f, -1.98412698412698412698e-4f));
    sp = __ffma2_rn(x2, sp, make_float2(8.33333333333333333333e-3f, 8.33333333333333333333e-3f));
    sp = __ffma2_rn(x2, sp, make_float2(-1.66666666666666666667e-1f, -1.66666666666666666667e-1f));
    sp = __ffma2_rn(x3, sp, x);
    float2 cp = __ffma2_rn(x2, make_float2(-2.75573192239858906526e-7f, -2.75573192239858906526e-7f),
                           make_float2(2.48015873015873015873e-5f, 2.48015873015873015873e-5f));
    cp = __ffma2_rn(x2, cp, make_float2(-1.38888888888888888889e-3f, -1.38888888888888888889e-3f));
    cp = __ffma2_rn(x2, cp, make_float2(4.16666666666666666667e-2f, 4.16666666666666666667e-2f));
    cp = __ffma2_rn(x2, cp, make_float2(-0.5f, -0.5f));
    cp = __ffma2_rn(x2, cp, make_float2(1.0f, 1.0f));
    float s0 = (q0 & 1) ? cp.x : sp.x, c0 = (q0 & 1) ? -sp.x : cp.x;
    float s1 = (q1 & 1) ? cp.y : sp.y, c1 = (q1 & 1) ? -sp.y : cp.y;
    if (q0 & 2) { s0 = -s0; c0 = -c0; }
    if (q1 & 2) { s1 = -s1; c1 = -c1; }
    c = make_float2(c0, c1);
    s = make_float2(s0, s1);
    ns = make_float2(-s0, -s1);
}

// ---------------------------------------------------------------------------------
// Block-anchor phases as 64-bit fixed-point turns (a phase accumulator): the start
// phase -d/lambda and the per-block increment -d*32*slope/c (both in turns) are reduced
// to their fractional part in FP64 and scaled by 2^64, after which every block phase is
// one exact modular 64-bit addition.  The angle handed to the hardware sine/cosine is the
// accumulator's top 32 bits, i.e. a wrapped angle in [-pi, pi) with 2^-32-turn steps.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long turns_to_fixed(double t) {
    const double kRound = 6755399441055744.0;  // 1.5 * 2^52: rint for |t| < 2^51
    const double n = (t + kRound) - kRound;
    const double f = t - n;                     // [-0.5, 0.5]
    return (unsigned long long)__double2ll_rn(f * 18446744073709551616.0);
}

__device__ __forceinline__ void fixed_cis(unsigned long long ph, float &c, float &s) {
    const float theta = (float)(int)(ph >> 32) * 1.46291807926715968e-9f;  // 2*pi / 2^32
    __sincosf(theta, &s, &c);
}

// FP64 round-trip distance TX -> v -> RX.  `mono` (all RX offsets zero) reuses the
// forward leg for the return leg, which is bit-identical to computing it again.
__device__ __forceinline__ double range_fp64(double vx, double vy, double vz,
                                             const AntRec &a, bool mono, double ti) {
    double dx = vx - a.tx[0], dy = vy - a.tx[1], dz = vz - a.tx[2];
    double f = sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
    double d;
    if (mono) {
        d = f + f;
    } else {
        double bx = vx - a.rx[0], by = vy - a.rx[1], bz = vz - a.rx[2];
        d = f + sqrt(fma(bx, bx, fma(by, by, bz * bz)));
    }
    return d + ti;
}

// ---------------------------------------------------------------------------------
// Cheaper forms of the per-(voxel, antenna) prologue (the "fx2" anchor family).
// ---------------------------------------------------------------------------------

// sqrt(r2) in FP64 from an FP32 reciprocal-square-root seed and one Newton step
// s' = s + (r2 - s^2) / (2 s), s = r2 * y: the seed's ~2^-22 relative error squares to
// ~1e-13 (a femtometre at a metre of range).  r2 below 1e-30 (a voxel on the antenna)
// gives a value below 2e-15 instead of 0.
__device__ __forceinline__ double sqrt_newton(double r2) {
    const double y = (double)rsqrtf(fmaxf((float)r2, 1e-30f));
    const double s = r2 * y;
    return fma(fma(-s, s, r2), 0.5 * y, s);
}

__device__ __forceinline__ double range_fp64_newton(double vx, double vy, double vz,
                                                    const AntRec &a, bool mono, double ti) {
    const double dx = vx - a.tx[0], dy = vy - a.tx[1], dz = vz - a.tx[2];
    const double f = sqrt_newton(fma(dx, dx, fma(dy, dy, dz * dz)));
    double d;
    if (mono) {
        d = f + f;
    } else {
        const double bx = vx - a.rx[0], by = vy - a.rx[1], bz = vz - a.rx[2];
        d = f + sqrt_newton(fma(bx, bx, fma(by, by, bz * bz)));
    }
    return d + ti;
}

// w turns as 32.32 fixed point (the top word = the wrapped turn count in 2^-32 steps),
// from the 1.5*2^52 rounding constant instead of a 64-bit conversion: a = w*2^32 is
// exact, (a + M) - M = rint(a) whose low word IS the top word, and the exact remainder
// a - rint(a), scaled by 2^32 and rounded the same way, is the low word (signed).
// Valid for |w| < 2^19 turns.
__device__ __forceinline__ unsigned long long turns_fixed64(double w) {
    const double kM = 6755399441055744.0;  // 1.5 * 2^52
    const double a = w * 4294967296.0;
    const double t1 = a + kM;
    const double r = a - (t1 - kM);
    const double t2 = fma(r, 4294967296.0, kM);
    const unsigned long long hi = (unsigned int)__double2loint(t1);
    const long long lo = __double2loint(t2);
    return (hi << 32) + (unsigned long long)lo;
}

// The same with the low word zero (a start phase rounded to 2^-33 turns).
__device__ __forceinline__ unsigned long long turns_fixed_top(double w) {
    const double kM = 6755399441055744.0;
    return (unsigned long long)(unsigned int)__double2loint(fma(w, 4294967296.0, kM)) << 32;
}

// (cos, sin) of two angles given as wrapped 2^-32-turn integers: the nearest quarter turn
// q from the top bits, the remainder r in [-2^29, 2^29) (an angle in [-pi/4, pi/4)) in
// FP32, the Taylor polynomials of cis_fp64_phase_pair, rotated by q quarter turns.
__device__ __forceinline__ void cis_turns_pair(int32_t a0, int32_t a1, float2 &c, float2 &s,
                                               float2 &ns) {
    const uint32_t q0 = ((uint32_t)a0 + 0x20000000u) >> 30;
    const uint32_t q1 = ((uint32_t)a1 + 0x20000000u) >> 30;
    const int32_t r0 = (int32_t)((uint32_t)a0 - (q0 << 30));
    const int32_t r1 = (int32_t)((uint32_t)a1 - (q1 << 30));
    const float kTurn = 1.46291807926715968e-9f;  // 2*pi / 2^32
    const float2 x = make_float2((float)r0 * kTurn, (float)r1 * kTurn);
    const float2 x2 = __fmul2_rn(x, x);
    const float2 x3 = __fmul2_rn(x2, x);
    float2 sp = __ffma2_rn(x2, make_float2(2.75573192239858906526e-6f, 2.75573192239858906526e-6f),
                           make_float2(-1.98412698412698412698e-4f, -1.98412698412698412698e-4f));
    sp = __ffma2_rn(x2, sp, make_float2(8.33333333333333333333e-3f, 8.33333333333333333333e-3f));
    sp = __ffma2_rn(x2, sp, make_float2(-1.66666666666666666667e-1f, -1.66666666666666666667e-1f));
    sp = __ffma2_rn(x3, sp, x);
    float2 cp = __ffma2_rn(x2, make_float2(-2.75573192239858906526e-7f, -2.75573192239858906526e-7f),
                           make_float2(2.48015873015873015873e-5f, 2.48015873015873015873e-5f));
    cp = __ffma2_rn(x2, cp, make_float2(-1.38888888888888888889e-3f, -1.38888888888888888889e-3f));
    cp = __ffma2_rn(x2, cp, make_float2(4.16666666666666666667e-2f, 4.16666666666666666667e-2f));
    cp = __ffma2_rn(x2, cp, make_float2(-0.5f, -0.5f));
    cp = __ffma2_rn(x2, cp, make_float2(1.0f, 1.0f));
    float s0 = (q0 & 1) ? cp.x : sp.x, c0 = (q0 & 1) ? -sp.x : cp.x;
    float s1 = (q1 & 1) ? cp.y : sp.y, c1 = (q1 & 1) ? -sp.y : cp.y;
    if (q0 & 2) { s0 = -s0; c0 = -c0; }
    if (q1 & 2) { s1 = -s1; c1 = -c1; }
    c = make_float2(c0, c1);
    s = make_float2(s0, s1);
    ns = make_float2(-s0, -s1);
}

// ---------------------------------------------------------------- status / errors
__device__ __forceinline__ void set_status(int32_t *status, int32_t code) {
    if (status) atomicCAS(status, 0, code);
}

// ----------------------------------------------------------- mbarrier + bulk copy
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bulk (non-tensor) TMA copy global -> shared, completion counted on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase.  An unsatisfied try_wait suspends the thread for a
// hardware-defined interval (about 4 us on B200), so the bound is set in time: after
// kWaitLimitNs of %globaltimer (a second, far beyond any legitimate copy) the wait gives up,
// records MMN_ERR_TIMEOUT and returns false.  kMaxPolls caps the polls as well, in case the
// timer does not advance.  The first poll reads no timer, so a completed phase costs one
// try_wait.
constexpr uint64_t kWaitLimitNs = 1000000000ull;
constexpr uint32_t kMaxPolls = 1u << 24;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  int32_t *status,
                                                  uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < kMaxPolls; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) break;
    }
    set_status(status, MMN_ERR_TIMEOUT);
    return false;
}

}  // namespace mmn
